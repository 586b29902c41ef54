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
// waves of a persistent kernel.
//
// Crossings: every decision reads a "serial-time view" of the labels, in
// which a cell committed by a later candidate (higher index) shows its old
// label again.  Later commits therefore never change an earlier decision,
// and a candidate only has to wait for the earlier candidates it actually
// reads: those within Chebyshev distance 2 that share one of its labels
// (topological numbers read the 3^d box, bounded proofs the 5^d box), and,
// only when its certificate needs a label-wide read (a global flood fill that
// the bounded 5^d proof could not replace, or an exact label count near
// extinction), every earlier candidate that touches that label.  A bounded
// proof that succeeds implies the global flood fill succeeds, so using it
// first changes no decision.
//
// Remap exchanges read the 5^d boxes of their two cells; an exchange waits
// for earlier pending exchanges with an intersecting label pair within
// Chebyshev distance 2 (in both directions, since exchanges commit in place).
#include <cub/cub.cuh>

#include "gpk_grid.h"

namespace gpk_dev {

static constexpr int32_t INT_BIG = 0x7fffffff;

// ---- label readers ---------------------------------------------------------------
struct PhiReader {  // the current labels, with at most one overridden cell
    const int32_t* phi;
    int ov_cell;
    int32_t ov_label;
    __device__ __forceinline__ int32_t operator()(int j) const { return j == ov_cell ? ov_label : phi[j]; }
    __device__ __forceinline__ int32_t get(int j, bool& reverted) const {
        reverted = false;
        return (*this)(j);
    }
};
// labels as the serial sweep saw them when it reached candidate k: cells
// accepted by a later candidate read back their old label ("reverted")
struct SerialView {
    const int32_t* phi;
    const int32_t* cmap;   // cell -> candidate index, -1 elsewhere
    const int8_t* cres;    // 0 pending, 1 deferred, 2 accepted
    const int4* cinfo;     // cell, old label, new label, state
    int k;
    __device__ __forceinline__ int32_t get(int j, bool& reverted) const {
        const int c = cmap[j];
        reverted = c > k && cres[c] == 2;
        return reverted ? cinfo[c].y : phi[j];
    }
    __device__ __forceinline__ int32_t operator()(int j) const {
        bool r;
        return get(j, r);
    }
    // the first n of six cells at once: each round of loads is issued together
    __device__ __forceinline__ void get6(const int j[6], int n, int32_t out[6], bool rev[6]) const {
        int c[6];
        int32_t p[6];
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            c[q] = q < n ? cmap[j[q]] : -1;
            p[q] = q < n ? phi[j[q]] : -1;
        }
        int8_t r[6];
#pragma unroll
        for (int q = 0; q < 6; ++q) r[q] = c[q] > k ? cres[c[q]] : (int8_t)0;
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            rev[q] = r[q] == 2;
            out[q] = rev[q] ? cinfo[c[q]].y : p[q];
        }
    }
};

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
            const uint32_t nxt = dilate3(comp, is3d) & occ;
            if (nxt == comp) break;
            comp = nxt;
        }
        ++count;
        rem &= ~comp;
    }
    return count;
}

template <class Lab>
__device__ __forceinline__ int topological_number(const Dims& D, const Lab& lab, int cell, int32_t label) {
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
                occ |= (uint32_t)(lab(D.idx(z, y, x)) == label) << (lz * 9 + ly * 3 + lx);
            }
        }
    }
    occ &= ~(1u << (is3d ? 13 : 4));
    return count_face_components(occ, is3d);
}

// ---------------------------------------------------------------------------
// 5^d bounded branch connectivity (src/gpk_connectivity.cpp:124-173)
// ---------------------------------------------------------------------------
typedef unsigned __int128 u128;

__device__ __forceinline__ u128 bit128(int b) { return ((u128)1) << b; }

template <class Lab>
__device__ __forceinline__ bool bounded_branches_connected(const Dims& D, const Lab& lab, int cell, int32_t label,
                                                           bool exclude_centre) {
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
                const int b = lz * 25 + ly * 5 + lx;
                if (lab(D.idx(z, y, x)) == label) occ |= bit128(b);
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

// The same two tests from a 5^d occupancy mask already gathered (bit
// b = lz*25 + ly*5 + lx, lz = 0 in 2-D): the topological number of the inner
// 3^d box (centre removed) and the bounded branch connectivity.
__device__ __forceinline__ int topological_number_mask(u128 occ5, bool is3d) {
    uint32_t occ = 0;
    const int lzn = is3d ? 3 : 1;
    for (int lz = 0; lz < lzn; ++lz)
        for (int ly = 0; ly < 3; ++ly)
            for (int lx = 0; lx < 3; ++lx) {
                const int b5 = (is3d ? (lz + 1) * 25 : 0) + (ly + 1) * 5 + lx + 1;
                occ |= (uint32_t)((occ5 >> b5) & 1) << (lz * 9 + ly * 3 + lx);
            }
    occ &= ~(1u << (is3d ? 13 : 4));
    return count_face_components(occ, is3d);
}

__device__ __forceinline__ bool bounded_branches_connected_mask(u128 occ, bool is3d, bool exclude_centre) {
    const int centre = (is3d ? 2 * 25 : 0) + 12;
    u128 lx0 = 0, lx4 = 0, ly0 = 0, ly4 = 0;
    const int zcount = is3d ? 5 : 1;
    for (int lz = 0; lz < zcount; ++lz)
        for (int l = 0; l < 5; ++l) {
            lx0 |= bit128(lz * 25 + l * 5);
            lx4 |= bit128(lz * 25 + l * 5 + 4);
            ly0 |= bit128(lz * 25 + l);
            ly4 |= bit128(lz * 25 + 20 + l);
        }
    if (exclude_centre) occ &= ~bit128(centre);
    const int branch_bit[6] = {centre - 1, centre + 1, centre - 5, centre + 5, centre - 25, centre + 25};
    const int nf = is3d ? 6 : 4;
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
// global flood fill (src/gpk_connectivity.cpp:79-115).  `cap` bounds the
// stack; overflowing it (only possible if the label counts were wrong)
// records GPK_ERR_INTERNAL instead of writing out of bounds.
// ---------------------------------------------------------------------------
template <class Lab>
__device__ bool global_branches_connected(const Dims& D, const Lab& lab, int cell, int32_t label, bool exclude_centre,
                                          uint32_t* __restrict__ stamp, int32_t* __restrict__ stack, uint32_t my_stamp,
                                          int cap, unsigned* err) {
    int nb6[6];
    D.faces(cell, nb6);
    const int nf = D.nface();
    int branches[6], nbr = 0;
    for (int k = 0; k < nf; ++k)
        if (lab(nb6[k]) == label) branches[nbr++] = nb6[k];
    if (nbr <= 1) return true;
    int targets[6], nt = 0;
    for (int k = 1; k < nbr; ++k) {
        bool dup = false;
        for (int t = 0; t < nt; ++t) dup |= targets[t] == branches[k];
        if (!dup) targets[nt++] = branches[k];
    }
    if (cap < 1) { atomicCAS(err, 0u, (unsigned)GPK_ERR_INTERNAL); return false; }
    int sp = 0;
    stack[sp++] = branches[0];
    stamp[branches[0]] = my_stamp;
    while (sp > 0) {
        const int cur = stack[--sp];
        int nx[6];
        D.faces(cur, nx);
        for (int k = 0; k < nf; ++k) {
            const int next = nx[k];
            if ((exclude_centre && next == cell) || stamp[next] == my_stamp || lab(next) != label) continue;
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
enum : int32_t {
    CS_LOCAL = 1,      // no earlier pending candidate among its local reads
    CS_GO = 2,         // needs the global flood fill of the old label
    CS_GN = 4,         // needs the global flood fill of the new label
    CS_GC = 8,         // needs the exact count of the old label
    CS_CNT_REJECT = 16,  // old label isolated and provably not its last cell
    CS_OLD_LOCAL = 32, // old-label branches proven connected inside 5^d
    CS_NEW_LOCAL = 64, // new-label branches proven connected inside 5^d
    CS_READY = 128, CS_ACCEPT = 256,
    CS_TO_SHIFT = 12, CS_TN_SHIFT = 16  // 2-bit capped topological numbers
};

struct CrossArgs {
    Dims D;
    int32_t* phi; int32_t* cmap; int8_t* cres; int32_t* count; const int32_t* count0;
    int32_t* minL[2];      // earliest pending candidate per label, by wave parity (both INT_BIG between sweeps)
    const int32_t* n_old;  // candidates per old label
    int4* cinfo;           // cell, old label, new label, state
    const int32_t* cpos;   // active position of the candidate
    const void* alpha_new_a; void* alpha; void* g; const void* g_comp; void* rho;
    uint32_t* stamp; uint32_t* stamp_rev; int32_t* ff_stack; long long pool_size;
    int32_t* tasks;        // candidates whose decision needs label-wide reads
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
    a.cres[k] = accept ? 2 : 1;
}

// Exact count of `label` at candidate k's serial time; every earlier
// candidate touching the label has been decided.
__device__ int serial_count(const CrossArgs& a, int k, int32_t label) {
    int c = a.count0[label];
    for (int j = 0; j < k; ++j) {
        if (a.cres[j] != 2) continue;
        const int4 cj = a.cinfo[j];
        c += (cj.z == label) - (cj.y == label);
    }
    return c;
}

// The same count with the 32 lanes of a warp splitting the earlier candidates.
__device__ int warp_serial_count(const CrossArgs& a, int k, int32_t label) {
    const int lane = threadIdx.x & 31;
    int c = 0;
    for (int j = lane; j < k; j += 32) {
        if (a.cres[j] != 2) continue;
        const int4 cj = a.cinfo[j];
        c += (cj.z == label) - (cj.y == label);
    }
    c = __reduce_add_sync(0xffffffffu, c);
    return a.count0[label] + c;
}

// Warp-cooperative breadth-first form of global_branches_connected: are all
// face branches of `label` around `cell` connected within the label's region
// (minus the centre when exclude_centre)?  The answer does not depend on the
// visiting order.  All 32 lanes call it with the same arguments; `queue`
// holds `cap` cells.
//
// Visit marks: flood fills running in the same wave cover distinct labels,
// but in the serial-time view a cell accepted by candidate m shows its old
// label to candidates before m and its new label to candidates after m, so
// it can lie in two regions at once — never in two regions as the same kind
// of cell.  Reverted cells therefore carry their marks in a second array.
template <class Lab>
__device__ bool warp_branches_connected(const Dims& D, const Lab& lab, int cell, int32_t label, bool exclude_centre,
                                        uint32_t* __restrict__ stamp, uint32_t* __restrict__ stamp_rev,
                                        int32_t* __restrict__ queue, int cap, uint32_t my_stamp, unsigned* err,
                                        int& visited) {
    visited = 0;
    const int lane = threadIdx.x & 31;
    int nb6[6];
    D.faces(cell, nb6);
    const int nf = D.nface();
    int branches[6], nbr = 0;
    for (int k = 0; k < nf; ++k)
        if (lab(nb6[k]) == label) branches[nbr++] = nb6[k];
    if (nbr <= 1) return true;
    int targets[6], nt = 0;
    for (int k = 1; k < nbr; ++k) {
        bool dup = false;
        for (int t = 0; t < nt; ++t) dup |= targets[t] == branches[k];
        if (!dup) targets[nt++] = branches[k];
    }
    if (cap < 1) {
        if (lane == 0) atomicCAS(err, 0u, (unsigned)GPK_ERR_INTERNAL);
        return false;
    }
    const unsigned all = (1u << nt) - 1u;
    unsigned found = 0;
    if (lane == 0) {
        bool rev;
        lab.get(branches[0], rev);
        queue[0] = branches[0];
        (rev ? stamp_rev : stamp)[branches[0]] = my_stamp;
    }
    __syncwarp();
    int head = 0, tail = 1;
    while (head < tail) {
        const int n = min(32, tail - head);
        int fresh[6];
        int nfresh = 0;
        if (lane < n) {
            const int cur = queue[head + lane];
            int nx[6];
            D.faces(cur, nx);
            for (int k = 0; k < nf; ++k) {
                const int next = nx[k];
                if (exclude_centre && next == cell) continue;
                bool rev;
                if (lab.get(next, rev) != label) continue;
                uint32_t* mark = rev ? &stamp_rev[next] : &stamp[next];
                if (*mark == my_stamp || atomicExch(mark, my_stamp) == my_stamp) continue;  // seen / taken by a lane
                fresh[nfresh++] = next;
            }
        }
        head += n;
        unsigned hit = 0;
        for (int q = 0; q < nfresh; ++q)
            for (int t = 0; t < nt; ++t) hit |= (fresh[q] == targets[t]) ? (1u << t) : 0u;
        found |= __reduce_or_sync(0xffffffffu, hit);
        visited = tail;
        if (found == all) return true;
        int incl = nfresh;
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        if (tail + total > cap) {
            if (lane == 0) atomicCAS(err, 0u, (unsigned)GPK_ERR_INTERNAL);
            return false;
        }
        const int off = tail + incl - nfresh;
        for (int q = 0; q < nfresh; ++q) queue[off + q] = fresh[q];
        tail += total;
        __syncwarp();
    }
    visited = tail;
    return found == all;
}

// Multi-source form of the same test: one breadth-first search grows from
// every branch at once (search i marks its cells with my_stamp + i); when a
// search reaches a cell of another search the two are united.  All branches
// connected <=> all searches end up united; a group of united searches whose
// frontier empties before that proves the branches disconnected.  A failed
// test therefore costs about the smaller side instead of the whole region.
// Needs distinct branch cells (always so unless a grid side is shorter than
// three cells; callers fall back to warp_branches_connected then).  `queue`
// holds 2*cap entries (cells, then search ids); stamps my_stamp..my_stamp+7.
template <class Lab>
__device__ bool warp_branches_connected_ms(const Dims& D, const Lab& lab, int cell, int32_t label, bool exclude_centre,
                                           uint32_t* __restrict__ stamp, uint32_t* __restrict__ stamp_rev,
                                           int32_t* __restrict__ queue, int cap, uint32_t my_stamp, unsigned* err,
                                           int& visited) {
    const int lane = threadIdx.x & 31;
    visited = 0;
    int nb6[6];
    D.faces(cell, nb6);
    const int nf = D.nface();
    int br[6], nbr = 0;
    for (int k = 0; k < nf; ++k)
        if (lab(nb6[k]) == label) br[nbr++] = nb6[k];
    if (nbr <= 1) return true;
    for (int i = 0; i < nbr; ++i)
        for (int j = i + 1; j < nbr; ++j)
            if (br[i] == br[j])
                return warp_branches_connected(D, lab, cell, label, exclude_centre, stamp, stamp_rev, queue, cap,
                                               my_stamp, err, visited);
    if (cap < nbr) {
        if (lane == 0) atomicCAS(err, 0u, (unsigned)GPK_ERR_INTERNAL);
        return false;
    }
    int32_t* qcell = queue;
    int32_t* qsid = queue + cap;
    int root[6], pend[6];
    for (int i = 0; i < 6; ++i) { root[i] = i; pend[i] = i < nbr ? 1 : 0; }
    if (lane < nbr) {
        bool rev;
        lab.get(br[lane], rev);
        (rev ? stamp_rev : stamp)[br[lane]] = my_stamp + (uint32_t)lane;
        qcell[lane] = br[lane];
        qsid[lane] = lane;
    }
    __syncwarp();
    int head = 0, tail = nbr;
    while (head < tail) {
        const int n = min(32, tail - head);
        int fresh[6];
        int nfresh = 0, sid = -1;
        uint64_t unions = 0;  // bit 6*i + j: search i touched search j
        if (lane < n) {
            const int cur = qcell[head + lane];
            sid = qsid[head + lane];
            int nx[6];
            D.faces(cur, nx);
            // the six neighbours' labels, then their stamps, each round of
            // loads issued together; the claims follow in face order
            int32_t lv[6];
            bool rv[6];
            lab.get6(nx, nf, lv, rv);
            bool want[6];
            uint32_t sv[6];
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                want[k] = k < nf && !(exclude_centre && nx[k] == cell) && lv[k] == label;
                sv[k] = want[k] ? (rv[k] ? stamp_rev[nx[k]] : stamp[nx[k]]) : 0u;
            }
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                if (!want[k]) continue;
                const int next = nx[k];
                const uint32_t seen = sv[k] - my_stamp;
                if (seen < 8u) {  // already claimed by a search of this test
                    if ((int)seen != sid) unions |= 1ull << (6 * sid + (int)seen);
                    continue;
                }
                uint32_t* mark = rv[k] ? &stamp_rev[next] : &stamp[next];
                const uint32_t old = atomicExch(mark, my_stamp + (uint32_t)sid) - my_stamp;
                if (old < 8u) {  // another lane (or an earlier face of this one) claimed it first
                    if ((int)old != sid) unions |= 1ull << (6 * sid + (int)old);
                    continue;
                }
                fresh[nfresh++] = next;
            }
        }
        head += n;
        // processed entries leave their search's frontier, fresh ones join it
        for (int i = 0; i < nbr; ++i) {
            pend[i] -= __reduce_add_sync(0xffffffffu, (sid == i) ? 1 : 0);
            pend[i] += __reduce_add_sync(0xffffffffu, (sid == i) ? nfresh : 0);
        }
        const uint32_t ulo = __reduce_or_sync(0xffffffffu, (uint32_t)unions);
        const uint32_t uhi = __reduce_or_sync(0xffffffffu, (uint32_t)(unions >> 32));
        uint64_t u = ((uint64_t)uhi << 32) | ulo;
        while (u) {
            const int b = __ffsll((long long)u) - 1;
            u &= u - 1;
            int ri = root[b / 6], rj = root[b % 6];
            if (ri != rj) {
                const int lo = min(ri, rj), hi = max(ri, rj);
                for (int i = 0; i < 6; ++i)
                    if (root[i] == hi) root[i] = lo;
            }
        }
        // one group left: connected; a group with an empty frontier: not
        bool single = true, closed = false;
        for (int i = 0; i < nbr; ++i) single &= root[i] == root[0];
        for (int r = 0; r < nbr && !single; ++r) {
            if (root[r] != r) continue;
            int p = 0;
            for (int i = 0; i < nbr; ++i) p += (root[i] == r) ? pend[i] : 0;
            closed |= p == 0;
        }
        int incl = nfresh;
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        visited = tail + total;
        if (single) return true;
        if (closed) return false;
        if (tail + total > cap) {
            if (lane == 0) atomicCAS(err, 0u, (unsigned)GPK_ERR_INTERNAL);
            return false;
        }
        const int off = tail + incl - nfresh;
        for (int q = 0; q < nfresh; ++q) {
            qcell[off + q] = fresh[q];
            qsid[off + q] = sid;
        }
        tail += total;
        __syncwarp();
    }
    // every frontier empty without one group: not connected
    bool single = true;
    for (int i = 0; i < nbr; ++i) single &= root[i] == root[0];
    return single;
}

template <typename real>
__global__ void __launch_bounds__(256) k_crossing_sweep(CrossArgs a, int m, int max_waves) {
    const int nblocks = gridDim.x;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int nthr = nblocks * blockDim.x;
    const Dims D = a.D;
    const bool is3d = D.is3d();
    unsigned* rem = a.s->wave_rem;  // three rotating counters
    unsigned prev_left = (unsigned)m + 1u;  // pending counts at wave starts: m, then strictly fewer
    for (int w = 0; w < max_waves; ++w) {
        // ---- phase A: locality, local certificate parts, label-wide needs;
        //      earliest pending candidate touching each label.  One warp per
        //      pending candidate: the lanes read the 5^d box around its cell
        //      at once (labels in the serial-time view, and the earlier
        //      pending candidates there), and ballots give the occupancy
        //      masks of its old and new label.
        int32_t* minA = a.minL[w & 1];        // this wave's per-label minima
        int32_t* minN = a.minL[(w + 1) & 1];  // the next wave's, cleared here
        if (tid == 0) a.s->ff_pool = 0;
        __shared__ unsigned s_pending;
        if (threadIdx.x == 0) s_pending = 0;
        __syncthreads();
        {
            const int lane = threadIdx.x & 31;
            const int gwarp = tid >> 5, nwarps = nthr >> 5;
            const int nbox = is3d ? 125 : 25, centre = is3d ? 62 : 12;
            unsigned pending = 0;
            // warp w takes candidates w, w + nwarps, ...; its lanes read the
            // states of 32 of them at once, then it walks the pending ones
            for (int k0 = gwarp; k0 < m; k0 += 32 * nwarps) {
                const int kl = k0 + lane * nwarps;
                unsigned todo = __ballot_sync(0xffffffffu, kl < m && a.cres[kl] == 0);
            while (todo) {
                const int k = k0 + (__ffs(todo) - 1) * nwarps;
                todo &= todo - 1;
                const int4 ci = a.cinfo[k];
                ++pending;
                if (lane == 0) {
                    atomicMin(&minA[ci.y], k);
                    atomicMin(&minA[ci.z], k);
                    minN[ci.y] = INT_BIG;
                    minN[ci.z] = INT_BIG;
                }
                int z0, y0, x0;
                D.decode(ci.x, z0, y0, x0);
                // the box in three rounds of loads: cell indices, then labels
                // and candidate slots, then the candidates' states
                int jq[4], cq4[4];
                int32_t lq[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int e = q * 32 + lane;
                    jq[q] = -1;
                    if (e < nbox && (q == 0 || nbox > 32)) {
                        const int lz = e / 25, ly = (e / 5) % 5, lx = e % 5;
                        // offsets of at most 2: one period at extents of 3 or more
                        const int zz = !is3d ? z0 : (D.Nz >= 3 ? wrap1(z0 + lz - 2, D.Nz) : wrap_any(z0 + lz - 2, D.Nz));
                        const int yy = D.Ny >= 3 ? wrap1(y0 + ly - 2, D.Ny) : wrap_any(y0 + ly - 2, D.Ny);
                        const int xx = D.Nx >= 3 ? wrap1(x0 + lx - 2, D.Nx) : wrap_any(x0 + lx - 2, D.Nx);
                        jq[q] = D.idx(zz, yy, xx);
                    }
                }
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    cq4[q] = jq[q] >= 0 ? a.cmap[jq[q]] : -1;
                    lq[q] = jq[q] >= 0 ? a.phi[jq[q]] : -1;
                }
                bool conflict = false;
                uint32_t wo[4] = {0u, 0u, 0u, 0u}, wn[4] = {0u, 0u, 0u, 0u};
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int e = q * 32 + lane;
                    const int c = cq4[q];
                    int32_t lbl = lq[q];
                    if (c > k) {
                        if (a.cres[c] == 2) lbl = a.cinfo[c].y;  // accepted later: the old label
                    } else if (c >= 0 && c < k && e != centre && a.cres[c] == 0) {
                        const int4 cq = a.cinfo[c];
                        conflict |= cq.y == ci.y || cq.y == ci.z || cq.z == ci.y || cq.z == ci.z;
                    }
                    wo[q] = __ballot_sync(0xffffffffu, lbl == ci.y);
                    wn[q] = __ballot_sync(0xffffffffu, lbl == ci.z);
                    if (nbox <= 32) break;
                }
                const bool local = !__any_sync(0xffffffffu, conflict);
                // lane 0 takes the old label's topology, lane 1 the new one's
                // (the same code on two masks runs side by side)
                int part = 0;
                if (local && lane < 2) {
                    const uint32_t* wv = lane == 0 ? wo : wn;
                    const u128 occ = (u128)wv[0] | ((u128)wv[1] << 32) | ((u128)wv[2] << 64) | ((u128)wv[3] << 96);
                    const int tv = topological_number_mask(occ, is3d);
                    part = min(tv, 2);
                    if (tv > 1) part |= bounded_branches_connected_mask(occ, is3d, lane == 0) ? 4 : 8;
                }
                const int part_n = __shfl_sync(0xffffffffu, part, 1);
                if (lane == 0) {
                    int st = 0;
                    if (local) {
                        const int to = part & 3, tn = part_n & 3;
                        st = CS_LOCAL | (to << CS_TO_SHIFT) | (tn << CS_TN_SHIFT);
                        if (to == 0) {
                            // at k's serial time the label holds at least count0 - (its other candidates) cells
                            if (a.count0[ci.y] - (a.n_old[ci.y] - 1) >= 2) st |= CS_CNT_REJECT;
                            else st |= CS_GC;
                        } else if (to > 1) {
                            st |= (part & 4) ? CS_OLD_LOCAL : CS_GO;
                        }
                        if (tn > 1) st |= (part_n & 4) ? CS_NEW_LOCAL : CS_GN;
                    }
                    a.cinfo[k].w = st;
                }
            }
            }
            if (lane == 0 && pending) atomicAdd(&s_pending, pending);
        }
        __syncthreads();
        if (threadIdx.x == 0 && s_pending) atomicAdd(&rem[w % 3], s_pending);
        if (!grid_barrier(a.s, nblocks)) return;
        const unsigned left = *((volatile unsigned*)&rem[w % 3]);
        if (left == 0) {
            if (tid == 0) a.s->waves = w;
            return;
        }
        // the earliest pending candidate is always decided, so every wave
        // decides at least one; every thread holds the previous count in a
        // register (the shared counter of wave w-1 is recycled by wave w+2)
        if (left >= prev_left) {
            if (threadIdx.x == 0) atomicCAS(&a.s->error, 0u, (unsigned)GPK_ERR_INTERNAL);
            return;
        }
        prev_left = left;
        if (tid == 0) rem[(w + 1) % 3] = 0;
        // ---- phase B: readiness; decisions that need only local reads are
        //      committed at once (they depend on nothing another decision of
        //      this wave writes: their local reads hold no earlier pending
        //      candidate, and later ones read back through the serial view)
        for (int k = tid; k < m; k += nthr) {
            if (a.cres[k] != 0) continue;
            const int4 ci = a.cinfo[k];
            const int st = ci.w;
            if (!(st & CS_LOCAL)) continue;
            if ((st & (CS_GO | CS_GC)) && minA[ci.y] < k) continue;
            if ((st & CS_GN) && minA[ci.z] < k) continue;
            if (st & (CS_GO | CS_GN | CS_GC)) {
                // label-wide work: one warp per candidate in phase B2
                a.tasks[atomicAdd(&a.s->n_tasks, 1u)] = k;
                continue;
            }
            const int to = (st >> CS_TO_SHIFT) & 3, tn = (st >> CS_TN_SHIFT) & 3;
            // to == 0 without GC is CS_CNT_REJECT; to > 1 without GO passed the 5^d proof
            bool acc = to != 0;
            if (acc && tn == 0) acc = false;
            cross_commit<real>(a, k, ci, acc);
        }
        if (!grid_barrier(a.s, nblocks)) return;
        const unsigned ntask = *((volatile unsigned*)&a.s->n_tasks);
        if (ntask == 0) continue;  // no label-wide work: the next wave reads these commits
        // ---- phase B2: global flood fills and exact counts, a warp per candidate
        {
            const int lane = threadIdx.x & 31;
            const int gwarp = tid >> 5, nwarps = nthr >> 5;
            for (unsigned t = gwarp; t < ntask; t += nwarps) {
                const int k = a.tasks[t];
                const int4 ci = a.cinfo[k];
                const int st = ci.w;
                const SerialView view{a.phi, a.cmap, a.cres, a.cinfo, k};
                const int to = (st >> CS_TO_SHIFT) & 3, tn = (st >> CS_TN_SHIFT) & 3;
                int base = 0, cap = 0;
                uint32_t my_stamp = 0;
                if (st & (CS_GO | CS_GN)) {
                    // the view of a label holds at most its count plus its later candidates' cells
                    cap = max((st & CS_GO) ? a.count[ci.y] + a.n_old[ci.y] : 0,
                              (st & CS_GN) ? a.count[ci.z] + a.n_old[ci.z] : 0) + 1;
                    if (lane == 0) {
                        // queue of cap cells plus cap search ids; 8 stamps per flood fill
                        base = (int)atomicAdd(&a.s->ff_pool, (unsigned)(2 * cap));
                        my_stamp = atomicAdd(&a.s->stamp, 16u) + 1u;
                    }
                    base = __shfl_sync(0xffffffffu, base, 0);
                    my_stamp = __shfl_sync(0xffffffffu, my_stamp, 0);
                    if ((long long)base + 2 * cap > a.pool_size) {
                        if (lane == 0) atomicCAS(&a.s->error, 0u, (unsigned)GPK_ERR_INTERNAL);
                        cap = 0;
                        base = 0;
                    }
                }
                bool acc = true;
                int visited = 0, vis = 0;
                if (to == 0) {
                    if (st & CS_CNT_REJECT) acc = false;
                    else {
                        acc = warp_serial_count(a, k, ci.y) <= 1;
                        if (lane == 0) {
                            atomicAdd(&a.s->count_tasks, 1ull);
                            atomicAdd(&a.s->count_scanned, (unsigned long long)k);
                        }
                    }
                } else if (to > 1 && !(st & CS_OLD_LOCAL)) {
                    acc = warp_branches_connected_ms(D, view, ci.x, ci.y, true, a.stamp, a.stamp_rev,
                                                     a.ff_stack + base, cap, my_stamp, &a.s->error, vis);
                    visited += vis;
                }
                if (acc) {
                    if (tn == 0) acc = false;
                    else if (tn > 1 && !(st & CS_NEW_LOCAL))
                        acc = warp_branches_connected_ms(D, view, ci.x, ci.z, false, a.stamp, a.stamp_rev,
                                                         a.ff_stack + base, cap, my_stamp + 8u, &a.s->error, vis);
                    visited += vis;
                }
                if (lane == 0) {
                    a.cinfo[k].w = st | CS_READY | (acc ? CS_ACCEPT : 0);
                    if (st & (CS_GO | CS_GN)) {
                        atomicAdd(&a.s->flood_tasks, 1ull);
                        atomicAdd(&a.s->flood_cells, (unsigned long long)visited);
                    }
                }
            }
        }
        if (!grid_barrier(a.s, nblocks)) return;
        // ---- phase C: commit the label-wide decisions (after all of them
        //      were taken, on the labels as they stood)
        for (unsigned t = tid; t < ntask; t += nthr) {
            const int k = a.tasks[t];
            const int4 ci = a.cinfo[k];
            cross_commit<real>(a, k, ci, (ci.w & CS_ACCEPT) != 0);
        }
        if (!grid_barrier(a.s, nblocks)) return;
        if (tid == 0) a.s->n_tasks = 0;
    }
    if (tid == 0) atomicCAS(&a.s->error, 0u, (unsigned)GPK_ERR_INTERNAL);
}

// Gathers the candidates (in active order), maps their cells and counts
// the candidates per old label.
__global__ void k_cross_setup(const int32_t* __restrict__ active, const int32_t* __restrict__ cpos, int m,
                              const int32_t* __restrict__ phi, const int32_t* __restrict__ phi_comp, int4* cinfo,
                              int32_t* cmap, int8_t* cres, int32_t* n_old) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    const int cell = active[cpos[k]];
    const int32_t o = phi[cell];
    cinfo[k] = make_int4(cell, o, phi_comp[cell], 0);
    cmap[cell] = k;
    cres[k] = 0;
    atomicAdd(&n_old[o], 1);
}

// Clears the cell map and the per-label candidate counts after the sweep.
__global__ void k_cross_cleanup(int m, const int4* __restrict__ cinfo, int32_t* cmap, int32_t* n_old, int32_t* minL,
                                int32_t* minF) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    const int4 ci = cinfo[k];
    cmap[ci.x] = -1;
    n_old[ci.y] = 0;
    minL[ci.y] = INT_BIG; minL[ci.z] = INT_BIG;
    minF[ci.y] = INT_BIG; minF[ci.z] = INT_BIG;
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
        res_a[i] = (real)resident;
        best_a[i] = (real)best;
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
                                unsigned long long* __restrict__ key2, int32_t* __restrict__ val, StepScalars* s,
                                const unsigned long long* gate = nullptr) {
    if (gate && *gate == 0ull) return;
    const int na = (int)*n_active;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < na; a += gridDim.x * blockDim.x) {
        const int i = active[a];
        const int32_t p = phi[i], q = phi_comp[i];
        const real gain = best_a[i] - res_a[i];  // scores are stored by cell
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
                            int4* __restrict__ exch, int32_t* __restrict__ estate, int32_t* __restrict__ pmap,
                            const unsigned* n_dev = nullptr) {
    if (n_dev) n = (int)*n_dev;  // count read on the device (captured step); grid-stride below
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
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
            st = 1;  // pending (ES_PENDING)
            pmap[e.x] = t;
            pmap[e.y] = t;
        }
    }
    exch[t] = e;
    estate[t] = st;
    }
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
    const PhiReader lab{phi, ov_cell, ov_label};
    const int old_object = topological_number(D, lab, cell, old_label);
    const bool old_ext = old_count <= 1;
    if (old_object == 0 && !old_ext) return false;
    if (old_object > 1 && !bounded_branches_connected(D, lab, cell, old_label, true)) return false;
    const int new_object = topological_number(D, lab, cell, new_label);
    if (new_object == 0) return false;
    if (new_object > 1 && !bounded_branches_connected(D, lab, cell, new_label, false)) return false;
    return true;
}

// certificate_local from the 5^d occupancy masks of the old and new label
__device__ __forceinline__ bool certificate_mask(u128 occ_old, u128 occ_new, int old_count, bool is3d) {
    const int old_object = topological_number_mask(occ_old, is3d);
    if (old_object == 0 && !(old_count <= 1)) return false;
    if (old_object > 1 && !bounded_branches_connected_mask(occ_old, is3d, true)) return false;
    const int new_object = topological_number_mask(occ_new, is3d);
    if (new_object == 0) return false;
    if (new_object > 1 && !bounded_branches_connected_mask(occ_new, is3d, false)) return false;
    return true;
}

__device__ __forceinline__ u128 mask128(const uint32_t w[4]) {
    return (u128)w[0] | ((u128)w[1] << 32) | ((u128)w[2] << 64) | ((u128)w[3] << 96);
}

struct ExchArgs {
    const unsigned* n_dev;  // exchange slots read on the device (captured step), else null
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
    if (a.n_dev) {
        n = (int)*a.n_dev;
        max_waves = n + 1;
        if (n == 0) return;
    }
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
        //      intersecting label pair within Chebyshev distance 2) + decision.
        //      One warp per pending exchange: the lanes read the 5^d boxes
        //      around both cells at once; ballots give the occupancy masks
        //      of the two labels that the certificates test.
        {
            const int lane = threadIdx.x & 31;
            const int gwarp = tid >> 5, nwarps = nthr >> 5;
            const int nbox = is3d ? 125 : 25;
            // warp w takes exchanges w, w + nwarps, ...; its lanes read the
            // states of 32 of them at once, then it walks the pending ones
            for (int t0 = gwarp; t0 < n; t0 += 32 * nwarps) {
                const int tl = t0 + lane * nwarps;
                const int32_t stl = tl < n ? a.estate[tl] : 0;
                unsigned todo = __ballot_sync(0xffffffffu, (stl & ES_PENDING) != 0);
            while (todo) {
                const int j0 = __ffs(todo) - 1;
                todo &= todo - 1;
                const int t = t0 + j0 * nwarps;
                const int32_t st = __shfl_sync(0xffffffffu, stl, j0);
                const int4 e = a.exch[t];
                const int A = e.x, B = e.y;
                const int32_t low = e.z, high = e.w;
                bool blocked = false;
                uint32_t aLow[4] = {0u, 0u, 0u, 0u}, aHigh[4] = {0u, 0u, 0u, 0u};
                uint32_t bLow[4] = {0u, 0u, 0u, 0u}, bHigh[4] = {0u, 0u, 0u, 0u};
#pragma unroll
                for (int side = 0; side < 2; ++side) {
                    int z0, y0, x0;
                    D.decode(side ? B : A, z0, y0, x0);
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int b = q * 32 + lane;
                        int32_t lbl = -1;
                        if (b < nbox) {
                            const int lz = b / 25, ly = (b / 5) % 5, lx = b % 5;
                            // offsets of at most 2: one period at extents of 3 or more
                            const int zz = !is3d ? z0
                                                 : (D.Nz >= 3 ? wrap1(z0 + lz - 2, D.Nz) : wrap_any(z0 + lz - 2, D.Nz));
                            const int yy = D.Ny >= 3 ? wrap1(y0 + ly - 2, D.Ny) : wrap_any(y0 + ly - 2, D.Ny);
                            const int xx = D.Nx >= 3 ? wrap1(x0 + lx - 2, D.Nx) : wrap_any(x0 + lx - 2, D.Nx);
                            const int j = D.idx(zz, yy, xx);
                            const int pq = a.pmap[j];
                            if (pq >= 0 && pq < t) {
                                const int4 o = a.exch[pq];
                                blocked |= o.z == e.z || o.z == e.w || o.w == e.z || o.w == e.w;
                            }
                            lbl = a.phi[j];
                            if (side == 1 && j == A) lbl = high;  // B's certificate sees A already exchanged
                        }
                        const uint32_t ml = __ballot_sync(0xffffffffu, lbl == low);
                        const uint32_t mh = __ballot_sync(0xffffffffu, lbl == high);
                        if (side) { bLow[q] = ml; bHigh[q] = mh; } else { aLow[q] = ml; aHigh[q] = mh; }
                        if (nbox <= 32) break;
                    }
                }
                if (__any_sync(0xffffffffu, blocked)) continue;
                if (lane == 0) {
                    bool acc = false;
                    if (a.phi[A] == low && a.phi[B] == high) {
                        const int before =
                            mismatch_count(D, a.phi, A, low, B, high) + mismatch_count(D, a.phi, B, high, A, low);
                        const int after =
                            mismatch_count(D, a.phi, A, high, B, low) + mismatch_count(D, a.phi, B, low, A, high);
                        if (after < before) {
                            const int cl = a.count[low], ch = a.count[high];
                            if (certificate_mask(mask128(aLow), mask128(aHigh), cl, is3d) &&
                                certificate_mask(mask128(bHigh), mask128(bLow), ch + 1, is3d))
                                acc = true;
                        }
                    }
                    a.estate[t] = st | ES_READY | (acc ? ES_ACCEPT : 0);
                }
            }
            }
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
    const PhiReader lab{phi, -1, 0};
    bool r = true;
    if (old_label == new_label) r = false;
    else {
        const int to = topological_number(D, lab, cell, old_label);
        const bool ext = count[old_label] <= 1;
        if (to == 0 && !ext) r = false;
        else if (to > 1 && !global_branches_connected(D, lab, cell, old_label, true, stamp, stack, my_stamp, D.N, err))
            r = false;
        else {
            const int tn = topological_number(D, lab, cell, new_label);
            if (tn == 0) r = false;
            else if (tn > 1 &&
                     !global_branches_connected(D, lab, cell, new_label, false, stamp, stack, my_stamp + 1, D.N, err))
                r = false;
        }
    }
    *out = r ? 1 : 0;
}

__global__ void k_fill_i32(int32_t* p, int n, int32_t v) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = v;
}

// ---------------------------------------------------------------------------
// captured-step form of the remap ordering
// ---------------------------------------------------------------------------
// The proposals in the reference's order — pair (low, high), direction,
// gain descending, cell ascending; the cell makes every key distinct — by
// one block: a merge sort whose run width doubles each pass, each element
// placed by a binary search in the neighbouring run.  The count is read on
// the device, so the launch can sit in a captured step.  Input: gain keys in
// k2[0], cells in v[0] (as k_bgr_proposals writes them).  Output: primary
// keys in k1[0] and cells in v[0], what k_bgr_match reads.
struct SortItem {
    unsigned long long k1, k2;
    int32_t v;
};
__device__ __forceinline__ bool item_less(const SortItem& a, const SortItem& b) {
    if (a.k1 != b.k1) return a.k1 < b.k1;
    if (a.k2 != b.k2) return a.k2 < b.k2;
    return a.v < b.v;
}

__global__ void __launch_bounds__(1024) k_sort_proposals(const unsigned* __restrict__ n_dev,
                                                         const unsigned long long* __restrict__ gate,
                                                         const int32_t* __restrict__ phi,
                                                         const int32_t* __restrict__ phi_comp,
                                                         unsigned long long* k1a, unsigned long long* k2a, int32_t* va,
                                                         unsigned long long* k1b, unsigned long long* k2b, int32_t* vb) {
    if (gate && *gate == 0ull) return;
    const int n = (int)*n_dev;
    if (n <= 1) {
        if (n == 1) {
            const int i = va[0];
            const int32_t p = phi[i], q = phi_comp[i];
            k1a[0] = ((unsigned long long)min(p, q) << 37) | ((unsigned long long)max(p, q) << 11) |
                     ((p == min(p, q) ? 0ull : 1ull) << 10);
        }
        return;
    }
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        const int i = va[t];
        const int32_t p = phi[i], q = phi_comp[i];
        const unsigned long long low = (unsigned long long)min(p, q), high = (unsigned long long)max(p, q);
        k1a[t] = (low << 37) | (high << 11) | ((p == min(p, q) ? 0ull : 1ull) << 10);
    }
    __syncthreads();
    unsigned long long *s1 = k1a, *s2 = k2a, *d1 = k1b, *d2 = k2b;
    int32_t *sv = va, *dv = vb;
    for (int width = 1; width < n; width *= 2) {
        for (int t = threadIdx.x; t < n; t += blockDim.x) {
            const SortItem it{s1[t], s2[t], sv[t]};
            const int run = t / width;
            const int lo_self = run * width;
            // the neighbouring run
            const int other = (run & 1) ? lo_self - width : lo_self + width;
            int pos;
            if (other >= n) {
                pos = t;  // an odd run at the end stays in place
            } else {
                const int olo = other, ohi = min(other + width, n);
                int a = olo, b = ohi;  // elements of the other run smaller than it
                while (a < b) {
                    const int mid = (a + b) >> 1;
                    const SortItem o{s1[mid], s2[mid], sv[mid]};
                    if (item_less(o, it)) a = mid + 1;
                    else b = mid;
                }
                const int base = min(lo_self, olo);
                pos = base + (t - lo_self) + (a - olo);
            }
            d1[pos] = it.k1;
            d2[pos] = it.k2;
            dv[pos] = it.v;
        }
        __syncthreads();
        unsigned long long* x = s1; s1 = d1; d1 = x;
        x = s2; s2 = d2; d2 = x;
        int32_t* y = sv; sv = dv; dv = y;
    }
    if (s1 != k1a) {
        for (int t = threadIdx.x; t < n; t += blockDim.x) {
            k1a[t] = s1[t];
            va[t] = sv[t];
        }
    }
}

// Second remap pass of a 3-D step inside a captured step: it runs when the
// first pass (gated on accepted crossings) exchanged cells; the two passes'
// exchanges are summed into the step's counter afterwards.
__global__ void k_remap_second_gate(StepScalars* s) {
    s->remap_waves_sum += s->waves;
    s->remap_props_sum += s->n_prop;
    s->exch_first = s->exch_pass;
    s->gate2 = (s->accepted > 0 && s->exch_pass > 0) ? 1ull : 0ull;
    s->exch_pass = 0;
    s->waves = 0;
}
__global__ void k_remap_total(StepScalars* s, int is3d) {
    s->remap_waves_sum += s->waves;  // the last pass (a skipped pass left 0 in both)
    s->remap_props_sum += s->n_prop;
    if (is3d) s->exchanges = s->exch_first + (s->gate2 ? s->exch_pass : 0ull);
    else s->exchanges = s->exch_pass;
}
__global__ void k_copy_i32_gated(int n, const int32_t* __restrict__ src, int32_t* __restrict__ dst,
                                 const unsigned long long* __restrict__ gate) {
    if (gate && *gate == 0ull) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = src[i];
}

}  // namespace gpk_dev

using namespace gpk_dev;

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
// Blocks of a persistent wave kernel: enough for want_items threads, at most
// two per SM (a grid barrier costs more the more blocks arrive at it) and
// never more than can be resident at once.
static int coop_grid(gpk_grid* G, const void* kernel, int block, int want_items) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0);
    if (per_sm < 1) per_sm = 1;
    if (per_sm > 2) per_sm = 2;
    int maxb = per_sm * G->num_sms;
    int need = (want_items + block - 1) / block;
    if (need < 1) need = 1;
    return need < maxb ? need : maxb;
}

static int launch_coop(gpk_grid* G, const void* kernel, int grid, int block, void** args) {
    GPK_CUDA_TRY(cudaMemsetAsync(&G->scal->bar_count, 0, sizeof(unsigned), G->stream));
    GPK_CUDA_TRY(cudaMemsetAsync(G->scal->wave_rem, 0, sizeof(G->scal->wave_rem), G->stream));
    const bool inject = G->inject_spin_limit > 0;
    if (inject) {
        // failure injection (gpk_grid_inject_wait_timeout): the first grid
        // barrier waits for one block more than launched and gives up after
        // the given number of spins, so the kernel returns GPK_ERR_TIMEOUT
        const long long lim = G->inject_spin_limit;
        const unsigned extra = 1;
        GPK_CUDA_TRY(cudaMemcpyAsync(&G->scal->spin_limit, &lim, sizeof(lim), cudaMemcpyHostToDevice, G->stream));
        GPK_CUDA_TRY(cudaMemcpyAsync(&G->scal->bar_extra, &extra, sizeof(extra), cudaMemcpyHostToDevice, G->stream));
        GPK_CUDA_TRY(cudaStreamSynchronize(G->stream));  // the host values above are locals
        G->inject_spin_limit = 0;
    }
    GPK_CUDA_TRY(cudaLaunchCooperativeKernel(kernel, dim3(grid), dim3(block), args, 0, G->stream));
    G->launches++;
    if (inject) {
        GPK_CUDA_TRY(cudaMemsetAsync(&G->scal->spin_limit, 0, sizeof(long long), G->stream));
        GPK_CUDA_TRY(cudaMemsetAsync(&G->scal->bar_extra, 0, sizeof(unsigned), G->stream));
    }
    return GPK_OK;
}

// Crossing sweep over the m candidates gathered by the alpha kernel.
template <typename real>
int gpk_crossings(gpk_grid* G, int m) {
    if (m == 0) return GPK_OK;
    const int B = 256;
    // label counts at the start of the sweep (exact counts near extinction)
    GPK_CUDA_TRY(cudaMemcpyAsync(G->count0, G->count, sizeof(int32_t) * G->label_cap, cudaMemcpyDeviceToDevice,
                                 G->stream));
    int8_t* cres = (int8_t*)G->val_a;  // candidate results, scratch until the remap
    k_cross_setup<<<(m + B - 1) / B, B, 0, G->stream>>>(G->active, G->cand, m, G->phi, G->phi_comp,
                                                        (int4*)G->cand_info, G->pmap, cres, G->n_old);
    G->launches++;
    GPK_CUDA_TRY(cudaGetLastError());
    CrossArgs a;
    a.D = G->d;
    a.phi = G->phi; a.cmap = G->pmap; a.cres = cres; a.count = G->count; a.count0 = G->count0;
    a.minL[0] = G->minL; a.minL[1] = G->minF;
    a.n_old = G->n_old;
    a.cinfo = (int4*)G->cand_info; a.cpos = G->cand;
    a.alpha_new_a = G->alpha_new_a; a.alpha = G->f[GPK_FIELD_ALPHA]; a.g = G->f[GPK_FIELD_G];
    a.g_comp = G->f[GPK_FIELD_G_COMP]; a.rho = G->f[GPK_FIELD_RHO];
    a.stamp = G->stamp; a.stamp_rev = G->stamp_rev; a.ff_stack = G->ff_stack; a.pool_size = 5LL * G->d.N + 64;
    a.s = G->scal;
    a.tasks = (int32_t*)G->key_a;  // free until the remap
    GPK_CUDA_TRY(cudaMemsetAsync(&G->scal->n_tasks, 0, sizeof(unsigned), G->stream));
    a.sweep_rho = G->th.dislocation_enabled; a.rho_rex_f = G->th.rho_rex; a.rho_rex_d = (double)G->th.rho_rex;
    int max_waves = m + 1;
    void* args[] = {&a, &m, &max_waves};
    const void* kern = (const void*)k_crossing_sweep<real>;
    // phase A runs one warp per pending candidate
    const int grid = coop_grid(G, kern, 256, (int)std::min<long long>(32LL * m, 1LL << 30));
    GPK_TRY(launch_coop(G, kern, grid, 256, args));
    k_cross_cleanup<<<(m + B - 1) / B, B, 0, G->stream>>>(m, (const int4*)G->cand_info, G->pmap, G->n_old, G->minL,
                                                        G->minF);
    G->launches++;
    GPK_CUDA_TRY(cudaGetLastError());
    return GPK_OK;
}

// One balanced-remap pass.  Precondition: the interface mask and the active
// list have just been rebuilt from the current labels.
template <typename real>
int gpk_remap_pass(gpk_grid* G, const unsigned long long* gate) {
    const Dims D = G->d;
    HostKernels<real>* hk = (HostKernels<real>*)G->host_kernels;
    const int B = 256;
    const int grid = 4 * G->num_sms;
    // phi_comp <- phi everywhere, then the best candidate at interface cells;
    // under a device-side gate (the second 3-D pass) every kernel up to the
    // proposals checks it, and a closed gate leaves no proposal
    if (gate) {
        k_copy_i32_gated<<<grid, B, 0, G->stream>>>(D.N, G->phi, G->phi_comp, gate);
        G->launches++;
    } else {
        GPK_CUDA_TRY(cudaMemcpyAsync(G->phi_comp, G->phi, sizeof(int32_t) * D.N, cudaMemcpyDeviceToDevice, G->stream));
    }
    const int rc = G->geometry_kernel != 1
                       ? gpk_bgr_scores_tiled<real>(G, hk->remap_radius, (real*)G->bgr_res, (real*)G->bgr_best, gate)
                       : -1;
    if (rc == -1) {
        if (gate) return GPK_ERR_INTERNAL;  // callers gate only where a tiled score kernel exists
        k_bgr_scores<real><<<grid, B, 0, G->stream>>>(D, G->active, &G->scal->n_active, G->phi, G->phi_comp,
                                                      (real*)G->bgr_res, (real*)G->bgr_best, G->d_remap_w,
                                                      hk->remap_radius);
    } else if (rc != GPK_OK) {
        return rc;
    }
    GPK_CUDA_TRY(cudaMemsetAsync(&G->scal->n_prop, 0, sizeof(unsigned), G->stream));
    k_bgr_proposals<real><<<grid, B, 0, G->stream>>>(G->active, &G->scal->n_active, G->phi, G->phi_comp,
                                                     (const real*)G->bgr_res, (const real*)G->bgr_best, G->key_b,
                                                     G->val_b, G->scal, gate);
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
    // the keys' set bits lie in [10, 37 + bits of the largest label): sorting
    // those bits alone gives the same order with fewer digit passes
    int lbits = 1;
    while (lbits < 27 && (1LL << lbits) < (long long)G->label_cap) ++lbits;
    GPK_CUDA_TRY(cub::DeviceRadixSort::SortPairs(G->cub_tmp, bytes, (const unsigned long long*)G->key_b, G->key_a,
                                                 (const int32_t*)G->val_b, G->val_a, n, 10, 37 + lbits, G->stream));
    k_bgr_match<<<(n + B - 1) / B, B, 0, G->stream>>>(n, G->key_a, G->val_a, (int4*)G->exch, G->val_b, G->pmap);
    G->launches++;
    GPK_CUDA_TRY(cudaGetLastError());
    ExchArgs a;
    a.n_dev = nullptr;
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
    // phase 1 runs one warp per pending exchange
    return launch_coop(G, kern, coop_grid(G, kern, 256, (int)std::min<long long>(32LL * n, 1LL << 30)), 256, args);
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
// One balanced-remap pass inside a captured step: every launch is sized for
// the worst case and reads its counts on the device, and nothing runs when
// *gate is zero.  Same kernels and order as gpk_remap_pass (the proposals
// ordered by k_sort_proposals instead of the radix sorts).
template <typename real>
int gpk_remap_pass_graph(gpk_grid* G, const unsigned long long* gate) {
    const Dims D = G->d;
    HostKernels<real>* hk = (HostKernels<real>*)G->host_kernels;
    const int B = 256;
    const int grid = 4 * G->num_sms;
    k_copy_i32_gated<<<grid, B, 0, G->stream>>>(D.N, G->phi, G->phi_comp, gate);
    const int rc = G->geometry_kernel != 1
                       ? gpk_bgr_scores_tiled<real>(G, hk->remap_radius, (real*)G->bgr_res, (real*)G->bgr_best, gate)
                       : -1;
    if (rc == -1) {
        gpk_set_error("captured step: the remap radius has no tiled score kernel");
        return GPK_ERR_UNSUPPORTED_MODEL;
    }
    if (rc != GPK_OK) return rc;
    GPK_CUDA_TRY(cudaMemsetAsync(&G->scal->n_prop, 0, sizeof(unsigned), G->stream));
    k_bgr_proposals<real><<<grid, B, 0, G->stream>>>(G->active, &G->scal->n_active, G->phi, G->phi_comp,
                                                     (const real*)G->bgr_res, (const real*)G->bgr_best, G->key_b,
                                                     G->val_b, G->scal, gate);
    // k_sort_proposals reads gain keys in key_b, cells in val_b; ping-pong
    // through the candidate record buffer (free while no crossing sweep runs)
    unsigned long long* k1b = (unsigned long long*)G->cand_info;
    unsigned long long* k2b = k1b + D.N;
    k_sort_proposals<<<1, 1024, 0, G->stream>>>(&G->scal->n_prop, gate, G->phi, G->phi_comp, G->key_a, G->key_b,
                                                G->val_b, k1b, k2b, G->val_a);
    // sorted: primary keys in key_a, cells in val_b
    k_bgr_match<<<grid, B, 0, G->stream>>>(0, G->key_a, G->val_b, (int4*)G->exch, G->val_a, G->pmap,
                                           &G->scal->n_prop);
    G->launches += 4;
    GPK_CUDA_TRY(cudaGetLastError());
    ExchArgs a;
    a.n_dev = &G->scal->n_prop;
    a.D = D;
    a.phi = G->phi; a.pmap = G->pmap; a.count = G->count;
    a.exch = (const int4*)G->exch; a.estate = G->val_a;
    a.g = G->f[GPK_FIELD_G]; a.alpha = G->f[GPK_FIELD_ALPHA]; a.rho = G->f[GPK_FIELD_RHO];
    a.s = G->scal;
    a.sweep_rho = G->th.dislocation_enabled; a.rho_rex_f = G->th.rho_rex; a.rho_rex_d = (double)G->th.rho_rex;
    int max_waves = 1, nn = 0;
    void* args[] = {&a, &nn, &max_waves};
    const void* kern = (const void*)k_bgr_exchange_waves<real>;
    // the slot count is known only on the device: one block per 8192 cells
    // (at most the usual cap), so that the exchange loops of many small grids
    // captured side by side fit on the GPU together
    const long long want = std::max(1LL, ((long long)D.N + 8191) / 8192) * 256;
    return launch_coop(G, kern, coop_grid(G, kern, 256, (int)std::min<long long>(want, 1LL << 30)), 256, args);
}

template int gpk_remap_pass<float>(gpk_grid*, const unsigned long long*);
template int gpk_remap_pass<double>(gpk_grid*, const unsigned long long*);
template int gpk_remap_pass_graph<float>(gpk_grid*, const unsigned long long*);
template int gpk_remap_pass_graph<double>(gpk_grid*, const unsigned long long*);

int gpk_remap_gates(gpk_grid* G, int stage) {
    if (stage == 0) k_remap_second_gate<<<1, 1, 0, G->stream>>>(G->scal);
    else k_remap_total<<<1, 1, 0, G->stream>>>(G->scal, G->d.is3d() ? 1 : 0);
    G->launches++;
    GPK_CUDA_TRY(cudaGetLastError());
    return GPK_OK;
}
template int gpk_extinction<float>(gpk_grid*);
template int gpk_extinction<double>(gpk_grid*);
