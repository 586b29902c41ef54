// gpk_topology.cu — topology-preserving label update on the device.
//
// Reference semantics (albert-hzbn/GPK):
//   crossings          src/gpk_transitions.cpp:273-313
//   certificates       src/gpk_connectivity.cpp:10-195
//   balanced remap     src/gpk_transitions.cpp:38-178
//   extinction         src/gpk_transitions.cpp:180-249
//
// The reference decides crossings one at a time in increasing flat index,
// each against the state left by the previous commits, and the remap
// exchanges one at a time in (label pair, rank) order.  Here both run as
// waves of a persistent kernel.  An item (crossing or exchange) is decided in
// a wave only when no earlier, still undecided item can change what it
// reads, and no later item it could be affected by has been applied before
// it.  For a crossing the reads are the 3^d box of its cell (topological
// numbers) and, only when its certificate needs them, the region or the
// count of its old/new label (global flood fill, extinction).  For a remap
// exchange the reads are the 5^d boxes of its two cells.  Items whose reads
// are disjoint from every earlier pending item's writes commute with them,
// so every decision equals the serial one and labels stay bit-identical.
#include <cub/cub.cuh>

#include "gpk_grid.h"

namespace gpk_dev {

static constexpr int32_t INT_BIG = 0x7fffffff;

// ---------------------------------------------------------------------------
// 3^d topological number with 27-bit occupancy masks
// (src/gpk_connectivity.cpp:23-77: face-connected components of `label`
// inside the 3^d box, centre removed, that touch a face of the centre)
// ---------------------------------------------------------------------------
struct Box3 {
    // bit b = lz*9 + ly*3 + lx
    static constexpr uint32_t LX0 = 0x1249249u;   // lx == 0
    static constexpr uint32_t LX2 = 0x4924924u;   // lx == 2
    static constexpr uint32_t LY0 = 0x01C0E07u;   // ly == 0
    static constexpr uint32_t LY2 = 0x70381C0u;   // ly == 2
    static constexpr uint32_t ALL = 0x7FFFFFFu;
};

__device__ __forceinline__ uint32_t dilate3(uint32_t m, bool is3d) {
    uint32_t r = m;
    r |= (m << 1) & ~Box3::LX0;
    r |= (m >> 1) & ~Box3::LX2;
    r |= (m << 3) & ~Box3::LY0;
    r |= (m >> 3) & ~Box3::LY2;
    if (is3d) { r |= (m << 9); r |= (m >> 9); }
    return r & (is3d ? Box3::ALL : 0x1FFu);
}

// Components of `occ` that contain a face neighbour of the centre.
__device__ __forceinline__ int count_face_components(uint32_t occ, bool is3d) {
    const uint32_t faces = is3d ? ((1u << 12) | (1u << 14) | (1u << 10) | (1u << 16) | (1u << 4) | (1u << 22))
                                : ((1u << 3) | (1u << 5) | (1u << 1) | (1u << 7));
    int count = 0;
    uint32_t rem = occ;
    while (rem & faces) {
        uint32_t comp = (rem & faces) & (0u - (rem & faces));  // lowest face bit
        for (;;) {
            uint32_t nxt = dilate3(comp, is3d) & occ;
            if (nxt == comp) break;
            comp = nxt;
        }
        ++count;
        rem &= ~comp;
    }
    return count;
}

// Occupancy of `label` in the 3^d box around `cell` (centre cleared), with
// an optional override of one cell's label (ov_cell < 0: none).
__device__ __forceinline__ uint32_t box3_occupancy(const Dims& D, const int32_t* __restrict__ phi, int cell,
                                                   int32_t label, int ov_cell, int32_t ov_label) {
    int z0, y0, x0;
    D.decode(cell, z0, y0, x0);
    const bool is3d = D.is3d();
    const int lzn = is3d ? 3 : 1;
    uint32_t occ = 0;
    for (int lz = 0; lz < lzn; ++lz) {
        const int z = is3d ? wrap1(z0 + lz - 1, D.Nz) : z0;
        for (int ly = 0; ly < 3; ++ly) {
            const int y = wrap1(y0 + ly - 1, D.Ny);
            for (int lx = 0; lx < 3; ++lx) {
                const int x = wrap1(x0 + lx - 1, D.Nx);
                const int j = D.idx(z, y, x);
                const int32_t v = (j == ov_cell) ? ov_label : phi[j];
                occ |= (uint32_t)(v == label) << (lz * 9 + ly * 3 + lx);
            }
        }
    }
    const int centre = is3d ? 13 : 4;
    return occ & ~(1u << centre);
}

__device__ __forceinline__ int topological_number(const Dims& D, const int32_t* __restrict__ phi, int cell,
                                                  int32_t label, int ov_cell = -1, int32_t ov_label = 0) {
    return count_face_components(box3_occupancy(D, phi, cell, label, ov_cell, ov_label), D.is3d());
}

// ---------------------------------------------------------------------------
// 5^d bounded branch connectivity (src/gpk_connectivity.cpp:124-173)
// ---------------------------------------------------------------------------
typedef unsigned __int128 u128;

__device__ __forceinline__ u128 bit128(int b) { return ((u128)1) << b; }

__device__ __forceinline__ bool bounded_branches_connected(const Dims& D, const int32_t* __restrict__ phi, int cell,
                                                           int32_t label, bool exclude_centre, int ov_cell,
                                                           int32_t ov_label) {
    int z0, y0, x0;
    D.decode(cell, z0, y0, x0);
    const bool is3d = D.is3d();
    const int zcount = is3d ? 5 : 1, zc = is3d ? 2 : 0;
    const int centre = zc * 25 + 12;
    u128 occ = 0;
    u128 lx0 = 0, lx4 = 0, ly0 = 0, ly4 = 0;
    for (int lz = 0; lz < zcount; ++lz) {
        const int z = is3d ? wrap_any(z0 + lz - 2, D.Nz) : z0;
        for (int ly = 0; ly < 5; ++ly) {
            const int y = wrap_any(y0 + ly - 2, D.Ny);
            for (int lx = 0; lx < 5; ++lx) {
                const int x = wrap_any(x0 + lx - 2, D.Nx);
                const int j = D.idx(z, y, x);
                const int32_t v = (j == ov_cell) ? ov_label : phi[j];
                const int b = lz * 25 + ly * 5 + lx;
                if (v == label) occ |= bit128(b);
                if (lx == 0) lx0 |= bit128(b);
                if (lx == 4) lx4 |= bit128(b);
                if (ly == 0) ly0 |= bit128(b);
                if (ly == 4) ly4 |= bit128(b);
            }
        }
    }
    if (exclude_centre) occ &= ~bit128(centre);
    const int branch_bit[6] = {centre - 1, centre + 1, centre - 5, centre + 5, centre - 25, centre + 25};
    const int nf = D.nface();
    int branches[6], nb = 0;
    for (int k = 0; k < nf; ++k)
        if (occ & bit128(branch_bit[k])) branches[nb++] = branch_bit[k];
    if (nb <= 1) return true;
    const u128 all = is3d ? ((((u128)1) << 125) - 1) : ((((u128)1) << 25) - 1);
    u128 comp = bit128(branches[0]);
    for (;;) {
        u128 r = comp;
        r |= (comp << 1) & ~lx0;
        r |= (comp >> 1) & ~lx4;
        r |= (comp << 5) & ~ly0;
        r |= (comp >> 5) & ~ly4;
        if (is3d) { r |= (comp << 25); r |= (comp >> 25); }
        r &= all & occ;
        if (r == comp) break;
        comp = r;
    }
    for (int k = 1; k < nb; ++k)
        if (!(comp & bit128(branches[k]))) return false;
    return true;
}

// ---------------------------------------------------------------------------
// global flood fill (src/gpk_connectivity.cpp:79-115)
// ---------------------------------------------------------------------------
// `cap` bounds the stack; overflowing it (only possible if the label counts
// were wrong) records GPK_ERR_INTERNAL instead of writing out of bounds.
__device__ bool global_branches_connected(const Dims& D, const int32_t* __restrict__ phi, int cell, int32_t label,
                                          bool exclude_centre, uint32_t* __restrict__ stamp, int32_t* __restrict__ stack,
                                          uint32_t my_stamp, int cap, unsigned* err) {
    int nb6[6];
    D.faces(cell, nb6);
    const int nf = D.nface();
    int branches[6], nbr = 0;
    for (int k = 0; k < nf; ++k)
        if (phi[nb6[k]] == label) branches[nbr++] = nb6[k];
    if (nbr <= 1) return true;
    int targets[6], nt = 0;
    for (int k = 1; k < nbr; ++k) {
        bool dup = false;
        for (int t = 0; t < nt; ++t) dup |= targets[t] == branches[k];
        if (!dup) targets[nt++] = branches[k];
    }
    int sp = 0;
    stack[sp++] = branches[0];
    stamp[branches[0]] = my_stamp;
    while (sp > 0) {
        const int cur = stack[--sp];
        int nx[6];
        D.faces(cur, nx);
        for (int k = 0; k < nf; ++k) {
            const int next = nx[k];
            if (phi[next] != label || (exclude_centre && next == cell) || stamp[next] == my_stamp) continue;
            stamp[next] = my_stamp;
            for (int t = 0; t < nt; ++t)
                if (targets[t] == next) { targets[t] = targets[--nt]; break; }
            if (nt == 0) return true;
            if (sp >= cap) { atomicCAS(err, 0u, (unsigned)GPK_ERR_INTERNAL); return false; }
            stack[sp++] = next;
        }
    }
    return nt == 0;
}

// ---------------------------------------------------------------------------
// crossing sweep
// ---------------------------------------------------------------------------
// candidate state bits
enum : int32_t {
    CS_PENDING = 1, CS_LOCAL = 2, CS_FO = 4, CS_FN = 8, CS_READY = 16, CS_ACCEPT = 32,
    CS_TO_SHIFT = 8, CS_TN_SHIFT = 12  // 2-bit capped topological numbers
};

struct CrossArgs {
    Dims D;
    int32_t* phi; int32_t* pmap; int32_t* minF; int32_t* minL; int32_t* count;
    int4* cinfo;             // cell, old label, new label, state
    const int32_t* cpos;     // active position of the candidate
    const void* alpha_new_a; void* alpha; void* g; const void* g_comp; void* rho;
    uint32_t* stamp; int32_t* ff_stack; long long pool_size;
    StepScalars* s;
    int sweep_rho; float rho_rex_f; double rho_rex_d;
  };

template <typename real>
__device__ __forceinline__ void cross_commit(const CrossArgs& a, int k, int4 ci, bool accept) {
    real* alpha = (real*)a.alpha;
    if (accept) {
        a.phi[ci.x] = ci.z;
        ((real*)a.g)[ci.x] = ((const real*)a.g_comp)[ci.x];
        alpha[ci.x] = (real)1;
        atomicSub(&a.count[ci.y], 1);
        atomicAdd(&a.count[ci.z], 1);
        atomicAdd(&a.s->accepted, 1ull);
        if (a.sweep_rho) ((real*)a.rho)[ci.x] = sizeof(real) == 4 ? (real)a.rho_rex_f : (real)a.rho_rex_d;
    } else {
        const real an = ((const real*)a.alpha_new_a)[a.cpos[k]];
        alpha[ci.x] = dmax(an, (real)1e-6);
        atomicAdd(&a.s->deferred, 1ull);
    }
}

template <typename real>
__global__ void __launch_bounds__(256) k_crossing_sweep(CrossArgs a, int m, int max_waves) {
    const int nblocks = gridDim.x;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int nthr = nblocks * blockDim.x;
    const Dims D = a.D;
    const bool is3d = D.is3d();
    unsigned* rem = a.s->wave_rem;  // three rotating counters
    unsigned prev_left = (unsigned)m;
    for (int w = 0; w < max_waves; ++w) {
        // ---- phase A: locality test, topological numbers, global-read flags
        if (tid == 0) { rem[(w + 1) % 3] = 0; a.s->ff_pool = 0; }
        for (int k = tid; k < m; k += nthr) {
            int4 ci = a.cinfo[k];
            if (!(ci.w & CS_PENDING)) continue;
            int z0, y0, x0;
            D.decode(ci.x, z0, y0, x0);
            bool local = true;
            for (int dz = (is3d ? -1 : 0); dz <= (is3d ? 1 : 0) && local; ++dz)
                for (int dy = -1; dy <= 1 && local; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        if (!dz && !dy && !dx) continue;
                        const int j = D.idx(is3d ? wrap1(z0 + dz, D.Nz) : z0, wrap1(y0 + dy, D.Ny), wrap1(x0 + dx, D.Nx));
                        const int q = a.pmap[j];
                        if (q >= 0 && q < k) {
                            const int4 cq = a.cinfo[q];
                            if (cq.y == ci.y || cq.y == ci.z || cq.z == ci.y || cq.z == ci.z) { local = false; break; }
                        }
                    }
            int st = ci.w & CS_PENDING;
            if (local) {
                const int to = topological_number(D, a.phi, ci.x, ci.y);
                const int tn = topological_number(D, a.phi, ci.x, ci.z);
                st |= CS_LOCAL | (min(to, 2) << CS_TO_SHIFT) | (min(tn, 2) << CS_TN_SHIFT);
                if (to != 1) st |= CS_FO;
                if (tn > 1) st |= CS_FN;
            } else {
                st |= CS_FO | CS_FN;
            }
            a.cinfo[k].w = st;
        }
        if (!grid_barrier(a.s, nblocks)) return;
        // ---- phase B: earliest pending item per label (global reads / any touch)
        for (int k = tid; k < m; k += nthr) {
            const int4 ci = a.cinfo[k];
            if (!(ci.w & CS_PENDING)) continue;
            if (ci.w & CS_FO) atomicMin(&a.minF[ci.y], k);
            if (ci.w & CS_FN) atomicMin(&a.minF[ci.z], k);
            atomicMin(&a.minL[ci.y], k);
            atomicMin(&a.minL[ci.z], k);
        }
        if (!grid_barrier(a.s, nblocks)) return;
        // ---- phase C: readiness and decision on the current state
        for (int k = tid; k < m; k += nthr) {
            int4 ci = a.cinfo[k];
            if (!(ci.w & CS_PENDING) || !(ci.w & CS_LOCAL)) continue;
            const bool fo = ci.w & CS_FO, fn = ci.w & CS_FN;
            if (a.minF[ci.y] < k || a.minF[ci.z] < k) continue;
            if (fo && a.minL[ci.y] < k) continue;
            if (fn && a.minL[ci.z] < k) continue;
            const int to = (ci.w >> CS_TO_SHIFT) & 3, tn = (ci.w >> CS_TN_SHIFT) & 3;
            bool acc = true;
            uint32_t base = 0, my_stamp = 0;
            int cap = 0;
            if (to > 1 || tn > 1) {
                cap = max(to > 1 ? a.count[ci.y] : 0, tn > 1 ? a.count[ci.z] : 0) + 1;
                base = atomicAdd(&a.s->ff_pool, (unsigned)cap);
                my_stamp = atomicAdd(&a.s->stamp, 2u) + 1u;
                if ((long long)base + cap > (long long)a.pool_size) {
                    atomicCAS(&a.s->error, 0u, (unsigned)GPK_ERR_INTERNAL);
                    cap = 0;
                    base = 0;
                }
            }
            if (to == 0) acc = a.count[ci.y] <= 1;
            else if (to > 1)
                acc = global_branches_connected(D, a.phi, ci.x, ci.y, true, a.stamp, a.ff_stack + base, my_stamp, cap,
                                                &a.s->error);
            if (acc) {
                if (tn == 0) acc = false;
                else if (tn > 1)
                    acc = global_branches_connected(D, a.phi, ci.x, ci.z, false, a.stamp, a.ff_stack + base,
                                                    my_stamp + 1u, cap, &a.s->error);
            }
            a.cinfo[k].w = ci.w | CS_READY | (acc ? CS_ACCEPT : 0);
        }
        if (!grid_barrier(a.s, nblocks)) return;
        // ---- phase D: commit ready items, reset per-label minima
        for (int k = tid; k < m; k += nthr) {
            const int4 ci = a.cinfo[k];
            if (!(ci.w & CS_PENDING)) continue;
            a.minF[ci.y] = INT_BIG; a.minF[ci.z] = INT_BIG;
            a.minL[ci.y] = INT_BIG; a.minL[ci.z] = INT_BIG;
            if (ci.w & CS_READY) {
                cross_commit<real>(a, k, ci, (ci.w & CS_ACCEPT) != 0);
                a.pmap[ci.x] = -1;
                a.cinfo[k].w = 0;
            } else {
                atomicAdd(&rem[w % 3], 1u);
            }
        }
        if (!grid_barrier(a.s, nblocks)) return;
        const unsigned left = *((volatile unsigned*)&rem[w % 3]);
        if (left == 0) {
            if (tid == 0) a.s->waves = w + 1;
            return;
        }
        // the earliest pending item is always ready, so every wave applies
        // at least one; every thread holds the previous count in a register
        // (the shared counter of wave w-1 is recycled by wave w+1)
        if (left >= prev_left) {
            if (threadIdx.x == 0) atomicCAS(&a.s->error, 0u, (unsigned)GPK_ERR_INTERNAL);
            return;
        }
        prev_left = left;
    }
    if (tid == 0) atomicCAS(&a.s->error, 0u, (unsigned)GPK_ERR_INTERNAL);
}

// Gathers the candidates (in active order) and arms the pending map.
template <typename real>
__global__ void k_cross_setup(Dims D, const int32_t* __restrict__ active, const int32_t* __restrict__ cpos, int m,
                              const int32_t* __restrict__ phi, const int32_t* __restrict__ phi_comp, int4* cinfo,
                              int32_t* pmap) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    const int cell = active[cpos[k]];
    cinfo[k] = make_int4(cell, phi[cell], phi_comp[cell], CS_PENDING);
    pmap[cell] = k;
}

// ---------------------------------------------------------------------------
// balanced Gaussian remap
// ---------------------------------------------------------------------------
// Scores: resident and best candidate label Gaussian support
// (src/gpk_transitions.cpp:53-91).  Writes phi_comp at interface cells.
template <typename real>
__global__ void k_bgr_scores(Dims D, const int32_t* __restrict__ active, const unsigned* __restrict__ n_active,
                             const int32_t* __restrict__ phi, int32_t* __restrict__ phi_comp, real* __restrict__ res_a,
                             real* __restrict__ best_a, const double* __restrict__ wtab, int radius) {
    const int na = (int)*n_active;
    const bool is3d = D.is3d();
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < na; a += gridDim.x * blockDim.x) {
        const int i = active[a];
        int z0, y0, x0;
        D.decode(i, z0, y0, x0);
        int face[6];
        D.faces(i, face);
        const int nf = D.nface();
        const int32_t pi = phi[i];
        int32_t cand[6];
        int nc = 0;
        for (int k = 0; k < nf; ++k) {
            const int32_t v = phi[face[k]];
            if (v == pi) continue;
            bool known = false;
            for (int q = 0; q < nc; ++q) known |= cand[q] == v;
            if (!known) cand[nc++] = v;
        }
        double resident = 0.0, sup[6] = {0, 0, 0, 0, 0, 0};
        const int dz0 = is3d ? -radius : 0, dz1 = is3d ? radius : 0;
        for (int dz = dz0; dz <= dz1; ++dz) {
            const int z = wrap_any(z0 + dz, D.Nz);
            for (int dy = -radius; dy <= radius; ++dy) {
                const int y = wrap_any(y0 + dy, D.Ny);
                for (int dx = -radius; dx <= radius; ++dx) {
                    const int x = wrap_any(x0 + dx, D.Nx);
                    const int32_t v = phi[D.idx(z, y, x)];
                    const double w = wtab[dx * dx + dy * dy + dz * dz];
                    if (v == pi) resident += w;
                    for (int q = 0; q < nc; ++q)
                        if (v == cand[q]) sup[q] += w;
                }
            }
        }
        double best = -1.0;
        int32_t best_label = pi;
        for (int q = 0; q < nc; ++q)
            if (sup[q] > best) { best = sup[q]; best_label = cand[q]; }
        res_a[a] = (real)resident;
        best_a[a] = (real)best;
        phi_comp[i] = best_label;
    }
}

// Proposals (src/gpk_transitions.cpp:93-104) keyed for two stable radix
// sorts: secondary (gain descending, cell ascending) then primary
// (low, high, direction).
template <typename real>
__global__ void k_bgr_proposals(const int32_t* __restrict__ active, const unsigned* __restrict__ n_active,
                                const int32_t* __restrict__ phi, const int32_t* __restrict__ phi_comp,
                                const real* __restrict__ res_a, const real* __restrict__ best_a,
                                unsigned long long* __restrict__ key2, int32_t* __restrict__ val, StepScalars* s) {
    const int na = (int)*n_active;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < na; a += gridDim.x * blockDim.x) {
        const int i = active[a];
        const int32_t p = phi[i], q = phi_comp[i];
        const real gain = best_a[a] - res_a[a];
        if (p == q || !(gain > (real)1e-7)) continue;
        const unsigned slot = atomicAdd(&s->n_prop, 1u);
        unsigned long long gbits;
        if (sizeof(real) == 4) {
            // positive floats order like their bit patterns
            const float gf = (float)gain;
            gbits = (unsigned long long)(~__float_as_uint(gf));
            key2[slot] = (gbits << 32) | (unsigned)i;
        } else {
            const double gd = (double)gain;
            gbits = ~(unsigned long long)__double_as_longlong(gd);
            // 64-bit gain key; the cell tie-break is applied by a first sort on cell
            key2[slot] = gbits;
        }
        val[slot] = i;
    }
}

template <typename real>
__global__ void k_bgr_primary_keys(int n, const int32_t* __restrict__ val, const int32_t* __restrict__ phi,
                                   const int32_t* __restrict__ phi_comp, unsigned long long* __restrict__ key1) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int i = val[t];
    const int32_t p = phi[i], q = phi_comp[i];
    const unsigned long long low = (unsigned long long)min(p, q), high = (unsigned long long)max(p, q);
    const unsigned long long dir = (p == min(p, q)) ? 0ull : 1ull;
    key1[t] = (low << 37) | (high << 11) | (dir << 10);
}

__device__ __forceinline__ int lower_bound_u64(const unsigned long long* a, int n, unsigned long long v) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] < v) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// Pairs the k-th forward proposal with the k-th reverse proposal of the same
// label pair (src/gpk_transitions.cpp:147-155).  Slot t (a forward element)
// becomes exchange t; unmatched slots get a = -1.
__global__ void k_bgr_match(int n, const unsigned long long* __restrict__ key1, const int32_t* __restrict__ val,
                            int4* __restrict__ exch, int32_t* __restrict__ estate, int32_t* __restrict__ pmap) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const unsigned long long k = key1[t];
    int4 e = make_int4(-1, -1, 0, 0);
    int32_t st = 0;
    if (((k >> 10) & 1ull) == 0ull) {
        const unsigned long long fwd0 = k & ~((1ull << 11) - 1);
        const unsigned long long rev0 = fwd0 | (1ull << 10);
        const int fstart = lower_bound_u64(key1, n, fwd0);
        const int rstart = lower_bound_u64(key1, n, rev0);
        const int rend = lower_bound_u64(key1, n, rev0 + (1ull << 10));
        const int r = t - fstart;
        if (r < rend - rstart) {
            e.x = val[t];
            e.y = val[rstart + r];
            e.z = (int)(k >> 37);
            e.w = (int)((k >> 11) & ((1ull << 26) - 1));
            st = CS_PENDING;
            pmap[e.x] = t;
            pmap[e.y] = t;
        }
    }
    exch[t] = e;
    estate[t] = st;
}

template <typename real>
__device__ __forceinline__ real target_orientation(const Dims& D, const int32_t* phi, const real* g, int cell,
                                                   int32_t target) {
    int nb[6];
    D.faces(cell, nb);
    const int nf = D.nface();
    for (int k = 0; k < nf; ++k)
        if (phi[nb[k]] == target) return g[nb[k]];
    return g[cell];
}

__device__ __forceinline__ int mismatch_count(const Dims& D, const int32_t* phi, int cell, int32_t proposed,
                                              int paired, int32_t paired_proposed) {
    int nb[6];
    D.faces(cell, nb);
    const int nf = D.nface();
    int m = 0;
    for (int k = 0; k < nf; ++k) {
        const int32_t q = (nb[k] == paired) ? paired_proposed : phi[nb[k]];
        m += q != proposed;
    }
    return m;
}

// Bounded certificate (local_only = true) with one overridden cell.
__device__ __forceinline__ bool certificate_local(const Dims& D, const int32_t* phi, int cell, int32_t old_label,
                                                  int32_t new_label, int old_count, int ov_cell, int32_t ov_label) {
    if (old_label == new_label) return false;
    const int old_object = topological_number(D, phi, cell, old_label, ov_cell, ov_label);
    const bool old_ext = old_count <= 1;
    if (old_object == 0 && !old_ext) return false;
    if (old_object > 1 && !bounded_branches_connected(D, phi, cell, old_label, true, ov_cell, ov_label)) return false;
    const int new_object = topological_number(D, phi, cell, new_label, ov_cell, ov_label);
    if (new_object == 0) return false;
    if (new_object > 1 && !bounded_branches_connected(D, phi, cell, new_label, false, ov_cell, ov_label)) return false;
    return true;
}

struct ExchArgs {
    Dims D;
    int32_t* phi; int32_t* pmap; const int32_t* count;
    const int4* exch; int32_t* estate;
    void* g; void* alpha; void* rho;
    StepScalars* s;
    int sweep_rho; float rho_rex_f; double rho_rex_d;
};

enum : int32_t { ES_PENDING = 1, ES_READY = 2, ES_ACCEPT = 4 };

template <typename real>
__global__ void __launch_bounds__(256) k_bgr_exchange_waves(ExchArgs a, int n, int max_waves) {
    const int nblocks = gridDim.x;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int nthr = nblocks * blockDim.x;
    const Dims D = a.D;
    const bool is3d = D.is3d();
    real* g = (real*)a.g;
    unsigned* rem = a.s->wave_rem;
    unsigned prev_left = 0xffffffffu;  // slots without an exchange are never pending
    for (int w = 0; w < max_waves; ++w) {
        if (tid == 0) rem[(w + 1) % 3] = 0;
        // ---- phase 1: readiness (no earlier pending exchange of an
        //      intersecting label pair within Chebyshev distance 2) + decision
        for (int t = tid; t < n; t += nthr) {
            const int32_t st = a.estate[t];
            if (!(st & ES_PENDING)) continue;
            const int4 e = a.exch[t];
            bool ready = true;
            for (int side = 0; side < 2 && ready; ++side) {
                int z0, y0, x0;
                D.decode(side ? e.y : e.x, z0, y0, x0);
                for (int dz = (is3d ? -2 : 0); dz <= (is3d ? 2 : 0) && ready; ++dz)
                    for (int dy = -2; dy <= 2 && ready; ++dy)
                        for (int dx = -2; dx <= 2; ++dx) {
                            const int j = D.idx(is3d ? wrap_any(z0 + dz, D.Nz) : z0, wrap_any(y0 + dy, D.Ny),
                                                wrap_any(x0 + dx, D.Nx));
                            const int q = a.pmap[j];
                            if (q >= 0 && q < t) {
                                const int4 o = a.exch[q];
                                if (o.z == e.z || o.z == e.w || o.w == e.z || o.w == e.w) { ready = false; break; }
                            }
                        }
            }
            if (!ready) continue;
            const int A = e.x, B = e.y;
            const int32_t low = e.z, high = e.w;
            bool acc = false;
            if (a.phi[A] == low && a.phi[B] == high) {
                const int before = mismatch_count(D, a.phi, A, low, B, high) + mismatch_count(D, a.phi, B, high, A, low);
                const int after = mismatch_count(D, a.phi, A, high, B, low) + mismatch_count(D, a.phi, B, low, A, high);
                if (after < before) {
                    const int cl = a.count[low], ch = a.count[high];
                    if (certificate_local(D, a.phi, A, low, high, cl, -1, 0) &&
                        certificate_local(D, a.phi, B, high, low, ch + 1, A, high))
                        acc = true;
                }
            }
            a.estate[t] = st | ES_READY | (acc ? ES_ACCEPT : 0);
        }
        if (!grid_barrier(a.s, nblocks)) return;
        // ---- phase 2: commit
        for (int t = tid; t < n; t += nthr) {
            const int32_t st = a.estate[t];
            if (!(st & ES_PENDING)) continue;
            if (st & ES_READY) {
                const int4 e = a.exch[t];
                if (st & ES_ACCEPT) {
                    const real ga = target_orientation<real>(D, a.phi, g, e.x, e.w);
                    const real gb = target_orientation<real>(D, a.phi, g, e.y, e.z);
                    // ga/gb are read before any write of this exchange; other
                    // exchanges committing now never touch these labels' cells
                    a.phi[e.x] = e.w;
                    a.phi[e.y] = e.z;
                    g[e.x] = ga;
                    g[e.y] = gb;
                    ((real*)a.alpha)[e.x] = (real)1;
                    ((real*)a.alpha)[e.y] = (real)1;
                    if (a.sweep_rho) {
                        const real r = sizeof(real) == 4 ? (real)a.rho_rex_f : (real)a.rho_rex_d;
                        ((real*)a.rho)[e.x] = r;
                        ((real*)a.rho)[e.y] = r;
                    }
                    atomicAdd(&a.s->exch_pass, 2ull);
                }
                a.pmap[e.x] = -1;
                a.pmap[e.y] = -1;
                a.estate[t] = 0;
            } else {
                atomicAdd(&rem[w % 3], 1u);
            }
        }
        if (!grid_barrier(a.s, nblocks)) return;
        const unsigned left = *((volatile unsigned*)&rem[w % 3]);
        if (left == 0) {
            if (tid == 0) a.s->waves = w + 1;
            return;
        }
        if (left >= prev_left) {
            if (threadIdx.x == 0) atomicCAS(&a.s->error, 0u, (unsigned)GPK_ERR_INTERNAL);
            return;
        }
        prev_left = left;
    }
    if (tid == 0) atomicCAS(&a.s->error, 0u, (unsigned)GPK_ERR_INTERNAL);
}

// ---------------------------------------------------------------------------
// unresolved-grain extinction (src/gpk_transitions.cpp:180-249)
// ---------------------------------------------------------------------------
__global__ void k_mark_unresolved(const int32_t* __restrict__ count, int cap, int min_resolved,
                                  uint8_t* __restrict__ unres, StepScalars* s) {
    for (int L = blockIdx.x * blockDim.x + threadIdx.x; L < cap; L += gridDim.x * blockDim.x) {
        const int c = count[L];
        const uint8_t u = (c > 0 && c < min_resolved) ? 1 : 0;
        unres[L] = u;
        if (u) atomicAdd(&s->unresolved, 1u);
        if (c > 0) atomicAdd(&s->present_labels, 1u);
    }
}

template <typename real>
__global__ void k_erosion_select(Dims D, const int32_t* __restrict__ phi, const real* __restrict__ g,
                                 const uint8_t* __restrict__ unres, int32_t* __restrict__ target,
                                 real* __restrict__ target_g, StepScalars* s) {
    const bool is3d = D.is3d();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < D.N; i += gridDim.x * blockDim.x) {
        target[i] = -1;
        if (!unres[phi[i]]) continue;
        int z, y, x;
        D.decode(i, z, y, x);
        int face[6];
        D.faces(i, face);
        const int nf = D.nface();
        int best = -1, best_support = -1;
        for (int k = 0; k < nf; ++k) {
            const int32_t q = phi[face[k]];
            if (unres[q]) continue;
            int support = 0;
            for (int dz = (is3d ? -1 : 0); dz <= (is3d ? 1 : 0); ++dz)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        const int zz = (z + dz + D.Nz) % D.Nz, yy = (y + dy + D.Ny) % D.Ny, xx = (x + dx + D.Nx) % D.Nx;
                        support += phi[D.idx(zz, yy, xx)] == q;
                    }
            if (support > best_support) { best = k; best_support = support; }
        }
        if (best >= 0) {
            target[i] = phi[face[best]];
            target_g[i] = g[face[best]];
            atomicAdd(&s->erosion_cells, 1u);
        }
    }
}

template <typename real>
__global__ void k_erosion_commit(int N, int32_t* __restrict__ phi, real* __restrict__ g, real* __restrict__ alpha,
                                 real* __restrict__ rho, const int32_t* __restrict__ target,
                                 const real* __restrict__ target_g, int32_t* __restrict__ count, int sweep_rho,
                                 real rho_rex) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const int32_t t = target[i];
        if (t < 0) continue;
        atomicSub(&count[phi[i]], 1);
        atomicAdd(&count[t], 1);
        phi[i] = t;
        g[i] = target_g[i];
        alpha[i] = (real)1;
        if (sweep_rho) rho[i] = rho_rex;
    }
}

// topology_simple_move diagnostic (src/gpk_connectivity.cpp:198-208)
__global__ void k_topology_simple_move(Dims D, const int32_t* __restrict__ phi, const int32_t* __restrict__ count,
                                       int cell, int32_t new_label, uint32_t* stamp, int32_t* stack,
                                       uint32_t my_stamp, int* out, unsigned* err) {
    const int32_t old_label = phi[cell];
    bool r = true;
    if (old_label == new_label) r = false;
    else {
        const int to = topological_number(D, phi, cell, old_label);
        const bool ext = count[old_label] <= 1;
        if (to == 0 && !ext) r = false;
        else if (to > 1 && !global_branches_connected(D, phi, cell, old_label, true, stamp, stack, my_stamp, D.N, err))
            r = false;
        else {
            const int tn = topological_number(D, phi, cell, new_label);
            if (tn == 0) r = false;
            else if (tn > 1 &&
                     !global_branches_connected(D, phi, cell, new_label, false, stamp, stack, my_stamp + 1, D.N, err))
                r = false;
        }
    }
    *out = r ? 1 : 0;
}

__global__ void k_fill_i32(int32_t* p, int n, int32_t v) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = v;
}

}  // namespace gpk_dev

using namespace gpk_dev;

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
static int coop_grid(gpk_grid* G, const void* kernel, int block, int want_items) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0);
    if (per_sm < 1) per_sm = 1;
    int maxb = per_sm * G->num_sms;
    int need = (want_items + block - 1) / block;
    if (need < 1) need = 1;
    return need < maxb ? need : maxb;
}

static int launch_coop(gpk_grid* G, const void* kernel, int grid, int block, void** args) {
    GPK_CUDA_TRY(cudaMemsetAsync(&G->scal->bar_count, 0, sizeof(unsigned), G->stream));
    GPK_CUDA_TRY(cudaMemsetAsync(G->scal->wave_rem, 0, sizeof(G->scal->wave_rem), G->stream));
    GPK_CUDA_TRY(cudaLaunchCooperativeKernel(kernel, dim3(grid), dim3(block), args, 0, G->stream));
    G->launches++;
    return GPK_OK;
}

// Crossing sweep over the m candidates gathered by the alpha kernel.
template <typename real>
int gpk_crossings(gpk_grid* G, int m) {
    if (m == 0) return GPK_OK;
    const int B = 256;
    k_cross_setup<real><<<(m + B - 1) / B, B, 0, G->stream>>>(G->d, G->active, G->cand, m, G->phi, G->phi_comp,
                                                             (int4*)G->cand_info, G->pmap);
    G->launches++;
    GPK_CUDA_TRY(cudaGetLastError());
    CrossArgs a;
    a.D = G->d;
    a.phi = G->phi; a.pmap = G->pmap; a.minF = G->minF; a.minL = G->minL; a.count = G->count;
    a.cinfo = (int4*)G->cand_info; a.cpos = G->cand;
    a.alpha_new_a = G->alpha_new_a; a.alpha = G->f[GPK_FIELD_ALPHA]; a.g = G->f[GPK_FIELD_G];
    a.g_comp = G->f[GPK_FIELD_G_COMP]; a.rho = G->f[GPK_FIELD_RHO];
    a.stamp = G->stamp; a.ff_stack = G->ff_stack; a.pool_size = 2LL * G->d.N + 64; a.s = G->scal;
    a.sweep_rho = G->th.dislocation_enabled; a.rho_rex_f = G->th.rho_rex; a.rho_rex_d = (double)G->th.rho_rex;
    int max_waves = m + 1;
    void* args[] = {&a, &m, &max_waves};
    const void* kern = (const void*)k_crossing_sweep<real>;
    const int grid = coop_grid(G, kern, 256, m);
    return launch_coop(G, kern, grid, 256, args);
}

// One balanced-remap pass.  Precondition: the interface mask and the active
// list have just been rebuilt from the current labels.
template <typename real>
int gpk_remap_pass(gpk_grid* G) {
    const Dims D = G->d;
    HostKernels<real>* hk = (HostKernels<real>*)G->host_kernels;
    const int B = 256;
    const int grid = 4 * G->num_sms;
    // phi_comp <- phi everywhere, then the best candidate at interface cells
    GPK_CUDA_TRY(cudaMemcpyAsync(G->phi_comp, G->phi, sizeof(int32_t) * D.N, cudaMemcpyDeviceToDevice, G->stream));
    k_bgr_scores<real><<<grid, B, 0, G->stream>>>(D, G->active, &G->scal->n_active, G->phi, G->phi_comp,
                                                  (real*)G->bgr_res, (real*)G->bgr_best, G->d_remap_w,
                                                  hk->remap_radius);
    GPK_CUDA_TRY(cudaMemsetAsync(&G->scal->n_prop, 0, sizeof(unsigned), G->stream));
    k_bgr_proposals<real><<<grid, B, 0, G->stream>>>(G->active, &G->scal->n_active, G->phi, G->phi_comp,
                                                     (const real*)G->bgr_res, (const real*)G->bgr_best, G->key_b,
                                                     G->val_b, G->scal);
    G->launches += 2;
    GPK_CUDA_TRY(cudaGetLastError());
    GPK_TRY(gpk_sync_scalars(G));
    const int n = (int)G->h_scal->n_prop;
    if (n == 0) return GPK_OK;
    // secondary order: (gain desc, cell asc); in f64 the cell order comes from
    // the proposal generation being re-sorted by cell first
    size_t bytes = G->cub_tmp_bytes;
    if (sizeof(real) == 8) {
        // sort by cell first (val as key), then stable by gain
        GPK_CUDA_TRY(cub::DeviceRadixSort::SortPairs(G->cub_tmp, bytes, (const int32_t*)G->val_b, (int32_t*)G->val_a,
                                                     (const unsigned long long*)G->key_b, G->key_a, n, 0, 32,
                                                     G->stream));
        bytes = G->cub_tmp_bytes;
        GPK_CUDA_TRY(cub::DeviceRadixSort::SortPairs(G->cub_tmp, bytes, (const unsigned long long*)G->key_a, G->key_b,
                                                     (const int32_t*)G->val_a, G->val_b, n, 0, 64, G->stream));
    } else {
        GPK_CUDA_TRY(cub::DeviceRadixSort::SortPairs(G->cub_tmp, bytes, (const unsigned long long*)G->key_b, G->key_a,
                                                     (const int32_t*)G->val_b, G->val_a, n, 0, 64, G->stream));
        std::swap(G->val_a, G->val_b);  // val_b holds secondary-sorted values
    }
    // primary order: (low, high, direction), stable
    k_bgr_primary_keys<real><<<(n + B - 1) / B, B, 0, G->stream>>>(n, G->val_b, G->phi, G->phi_comp, G->key_b);
    G->launches++;
    bytes = G->cub_tmp_bytes;
    GPK_CUDA_TRY(cub::DeviceRadixSort::SortPairs(G->cub_tmp, bytes, (const unsigned long long*)G->key_b, G->key_a,
                                                 (const int32_t*)G->val_b, G->val_a, n, 0, 64, G->stream));
    k_bgr_match<<<(n + B - 1) / B, B, 0, G->stream>>>(n, G->key_a, G->val_a, (int4*)G->exch, G->val_b, G->pmap);
    G->launches++;
    GPK_CUDA_TRY(cudaGetLastError());
    ExchArgs a;
    a.D = D;
    a.phi = G->phi; a.pmap = G->pmap; a.count = G->count;
    a.exch = (const int4*)G->exch; a.estate = G->val_b;
    a.g = G->f[GPK_FIELD_G]; a.alpha = G->f[GPK_FIELD_ALPHA]; a.rho = G->f[GPK_FIELD_RHO];
    a.s = G->scal;
    a.sweep_rho = G->th.dislocation_enabled; a.rho_rex_f = G->th.rho_rex; a.rho_rex_d = (double)G->th.rho_rex;
    int max_waves = n + 1;
    int nn = n;
    void* args[] = {&a, &nn, &max_waves};
    const void* kern = (const void*)k_bgr_exchange_waves<real>;
    return launch_coop(G, kern, coop_grid(G, kern, 256, n), 256, args);
}

template <typename real>
int gpk_extinction(gpk_grid* G) {
    HostKernels<real>* hk = (HostKernels<real>*)G->host_kernels;
    const Dims D = G->d;
    const double sigma = (double)dmax(hk->gauss_sigma, (real)1);
    const double pi = 3.14159265358979323846;
    const double support_volume = D.is3d() ? (4.0 * pi * sigma * sigma * sigma / 3.0) : (pi * sigma * sigma);
    int min_resolved = (int)ceil(support_volume);
    if (min_resolved < 2) min_resolved = 2;
    GPK_CUDA_TRY(cudaMemsetAsync(&G->scal->unresolved, 0, sizeof(unsigned), G->stream));
    GPK_CUDA_TRY(cudaMemsetAsync(&G->scal->present_labels, 0, sizeof(unsigned), G->stream));
    k_mark_unresolved<<<(G->label_cap + 255) / 256, 256, 0, G->stream>>>(G->count, G->label_cap, min_resolved,
                                                                         G->unres, G->scal);
    G->launches++;
    GPK_TRY(gpk_sync_scalars(G));
    const unsigned nu = G->h_scal->unresolved, present = G->h_scal->present_labels;
    if (nu == 0 || nu == present) return GPK_OK;
    const int grid = 4 * G->num_sms;
    for (int layer = 0; layer <= D.N; ++layer) {
        GPK_CUDA_TRY(cudaMemsetAsync(&G->scal->erosion_cells, 0, sizeof(unsigned), G->stream));
        k_erosion_select<real><<<grid, 256, 0, G->stream>>>(D, G->phi, (const real*)G->f[GPK_FIELD_G], G->unres,
                                                           G->ero_target, (real*)G->ero_g, G->scal);
        G->launches++;
        GPK_TRY(gpk_sync_scalars(G));
        if (G->h_scal->erosion_cells == 0) break;
        const real rr = (real)G->th.rho_rex;
        k_erosion_commit<real><<<grid, 256, 0, G->stream>>>(D.N, G->phi, (real*)G->f[GPK_FIELD_G],
                                                           (real*)G->f[GPK_FIELD_ALPHA], (real*)G->f[GPK_FIELD_RHO],
                                                           G->ero_target, (const real*)G->ero_g, G->count,
                                                           G->th.dislocation_enabled, rr);
        G->launches++;
    }
    return gpk_interface_mask<real>(G);
}

int gpk_topology_simple_move_impl(gpk_grid* G, int cell, int32_t new_label, int* result) {
    if (new_label < 0 || new_label >= G->label_cap) {
        // a label absent from the grid has count 0 and no cells
        new_label = -1;
    }
    int* d_out = (int*)G->ff_stack;  // scratch word, stack starts after it
    GPK_TRY(gpk_sync_scalars(G));
    uint32_t st = G->h_scal->stamp + 1;
    G->h_scal->stamp += 2;
    GPK_CUDA_TRY(cudaMemcpyAsync(&G->scal->stamp, &G->h_scal->stamp, sizeof(unsigned), cudaMemcpyHostToDevice,
                                 G->stream));
    k_topology_simple_move<<<1, 1, 0, G->stream>>>(G->d, G->phi, G->count, cell, new_label, G->stamp,
                                                   G->ff_stack + 1, st, d_out, &G->scal->error);
    G->launches++;
    GPK_CUDA_TRY(cudaGetLastError());
    GPK_CUDA_TRY(cudaMemcpyAsync(result, d_out, sizeof(int), cudaMemcpyDeviceToHost, G->stream));
    GPK_CUDA_TRY(cudaStreamSynchronize(G->stream));
    return GPK_OK;
}

template int gpk_crossings<float>(gpk_grid*, int);
template int gpk_crossings<double>(gpk_grid*, int);
template int gpk_remap_pass<float>(gpk_grid*);
template int gpk_remap_pass<double>(gpk_grid*);
template int gpk_extinction<float>(gpk_grid*);
template int gpk_extinction<double>(gpk_grid*);
