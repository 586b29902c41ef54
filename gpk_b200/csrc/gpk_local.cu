// gpk_local.cu — tiled kernels for the small-radius Gaussian boxes of a step:
// the pair velocity projection (src/gpk_physics.cpp:152-193) and the
// balanced-remap scores (src/gpk_transitions.cpp:53-91).
//
// Both visit a (2R+1)^d box (R = 3 at the configured sigmas) around every
// interface cell and accumulate, in double and in the reference's z -> y -> x
// tap order, the weights (double)expf(-r2/(2 s^2)) of the taps that satisfy a
// label condition.  One CTA stages its tile's labels (and, for the
// projection, each cell's label pair and signed velocity) with an R-cell
// periodic halo in shared memory and walks the tile's interface cells.  The
// pair-compare and tap-by-tap kernels write the conditional additions as
// fma(w, m, acc) with m in {0, 1}; the bitmap kernels add only the taps whose
// bit is set.  A sum that starts at +0 is never -0 in round-to-nearest, so
// adding a signed zero changes nothing and both forms are bit-identical to
// `if (cond) acc += w`.
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include "gpk_grid.h"

namespace gpk_dev {

template <bool IS3D> struct LocTile;
template <> struct LocTile<true> { static constexpr int TX = 16, TY = 8, TZ = 8; };
template <> struct LocTile<false> { static constexpr int TX = 32, TY = 32, TZ = 1; };

template <int R, bool IS3D>
struct LocShape {
    static constexpr int TX = LocTile<IS3D>::TX, TY = LocTile<IS3D>::TY, TZ = LocTile<IS3D>::TZ;
    static constexpr int HX = TX + 2 * R, HY = TY + 2 * R, HZ = IS3D ? TZ + 2 * R : 1;
    static constexpr int NH = HX * HY * HZ;
    static constexpr int NCELL = TX * TY * TZ;
    static constexpr int R2MAX = (IS3D ? 3 : 2) * R * R;
};

// Compacts the tile's interface cells (flat tile order) into `cells`; returns
// their number.  All threads of the 256-thread block call it.
template <int R, bool IS3D>
__device__ __forceinline__ int tile_interface_cells(const Dims& D, const uint8_t* __restrict__ mask, int x0, int y0,
                                                    int z0, int16_t* cells) {
    typedef LocShape<R, IS3D> S;
    typedef cub::BlockScan<int, 256> BS;
    __shared__ typename BS::TempStorage scan;
    __shared__ int s_total;
    constexpr int PER = (S::NCELL + 255) / 256;
    int flags[PER];
    int cnt = 0;
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int c = threadIdx.x * PER + k;
        int f = 0;
        if (c < S::NCELL) {
            const int lx = c % S::TX, ly = (c / S::TX) % S::TY, lz = c / (S::TX * S::TY);
            const int x = x0 + lx, y = y0 + ly, z = z0 + lz;
            if (x < D.Nx && y < D.Ny && z < D.Nz) f = mask[D.idx(z, y, x)];
        }
        flags[k] = f;
        cnt += f;
    }
    int ex, total;
    BS(scan).ExclusiveSum(cnt, ex, total);
#pragma unroll
    for (int k = 0; k < PER; ++k)
        if (flags[k]) cells[ex++] = (int16_t)(threadIdx.x * PER + k);
    if (threadIdx.x == 0) s_total = total;
    __syncthreads();
    return s_total;
}

// ---------------------------------------------------------------------------
// balanced-remap scores
// ---------------------------------------------------------------------------
// Weighted support of the resident label and of the first NC candidates over
// the box (tap order z -> y -> x).  Unused candidate slots hold -1 and match
// nothing, so running fewer slots than 6 changes no sum.
template <int R, bool IS3D, int NC, int HX, int HY>
__device__ __forceinline__ void score_box_impl(const int32_t* __restrict__ lab, int base, const double* __restrict__ w,
                                               int32_t pi, const int32_t cand[6], double& resident, double sup[6]) {
#pragma unroll 1
    for (int dz = (IS3D ? -R : 0); dz <= (IS3D ? R : 0); ++dz)
#pragma unroll 1
        for (int dy = -R; dy <= R; ++dy) {
            const int rowb = base + ((IS3D ? dz + R : 0) * HY + dy + R) * HX + R;
            const int r2yz = dy * dy + dz * dz;
#pragma unroll
            for (int dx = -R; dx <= R; ++dx) {
                const int32_t v = lab[rowb + dx];
                const double wt = w[r2yz + dx * dx];
                resident = __fma_rn(wt, v == pi ? 1.0 : 0.0, resident);
#pragma unroll
                for (int q = 0; q < NC; ++q) sup[q] = __fma_rn(wt, v == cand[q] ? 1.0 : 0.0, sup[q]);
            }
        }
}
template <int R, bool IS3D, int NC>
__device__ __forceinline__ void score_box(const int32_t* __restrict__ lab, int base, const double* __restrict__ w,
                                          int32_t pi, const int32_t cand[6], double& resident, double sup[6]) {
    typedef LocShape<R, IS3D> S;
    score_box_impl<R, IS3D, NC, S::HX, S::HY>(lab, base, w, pi, cand, resident, sup);
}
template <typename real, int R, bool IS3D>
__global__ void __launch_bounds__(256) k_bgr_scores_tiled(Dims D, const int32_t* __restrict__ phi,
                                                          const uint8_t* __restrict__ mask, int ntx, int nty,
                                                          const double* __restrict__ wtab, int32_t* __restrict__ phi_comp,
                                                          real* __restrict__ res_out, real* __restrict__ best_out,
                                                          const unsigned long long* __restrict__ gate) {
    if (gate && *gate == 0ull) return;  // device-side skip inside a captured step
    typedef LocShape<R, IS3D> S;
    __shared__ int32_t lab[S::NH];
    __shared__ int16_t cells[S::NCELL];
    __shared__ double w[S::R2MAX + 1];
    const int t = blockIdx.x;
    const int tx = t % ntx, ty = (t / ntx) % nty, tz = t / (ntx * nty);
    const int x0 = tx * S::TX, y0 = ty * S::TY, z0 = tz * S::TZ;
    const int ncell = tile_interface_cells<R, IS3D>(D, mask, x0, y0, z0, cells);
    if (ncell == 0) return;
    for (int e = threadIdx.x; e < S::NH; e += 256) {
        const int hx = e % S::HX, hy = (e / S::HX) % S::HY, hz = e / (S::HX * S::HY);
        const int x = wrap_any(x0 + hx - R, D.Nx), y = wrap_any(y0 + hy - R, D.Ny);
        const int z = IS3D ? wrap_any(z0 + hz - R, D.Nz) : 0;
        lab[e] = phi[D.idx(z, y, x)];
    }
    for (int e = threadIdx.x; e <= S::R2MAX; e += 256) w[e] = wtab[e];
    __syncthreads();
    const int plane = S::HX * S::HY;
    for (int c = threadIdx.x; c < ncell; c += 256) {
        const int lc = cells[c];
        const int lx = lc % S::TX, ly = (lc / S::TX) % S::TY, lz = lc / (S::TX * S::TY);
        const int cb = ((IS3D ? lz + R : 0) * S::HY + ly + R) * S::HX + lx + R;
        const int32_t pi = lab[cb];
        // distinct unlike face-neighbour labels in face order; -1 pads
        const int fo[6] = {-1, +1, -S::HX, +S::HX, -plane, +plane};
        int32_t cand[6] = {-1, -1, -1, -1, -1, -1};
        int nc = 0;
        for (int k = 0; k < (IS3D ? 6 : 4); ++k) {
            const int32_t v = lab[cb + fo[k]];
            if (v == pi) continue;
            bool known = false;
            for (int q = 0; q < nc; ++q) known |= cand[q] == v;
            if (!known) cand[nc++] = v;
        }
        double resident = 0.0, sup[6] = {0, 0, 0, 0, 0, 0};
        const int base = cb - (IS3D ? R * plane : 0) - R * S::HX - R;
        // candidate slots beyond the warp's largest count are skipped
        const int ncw = __reduce_max_sync(__activemask(), nc);
        switch (ncw) {
        case 0: score_box<R, IS3D, 0>(lab, base, w, pi, cand, resident, sup); break;
        case 1: score_box<R, IS3D, 1>(lab, base, w, pi, cand, resident, sup); break;
        case 2: score_box<R, IS3D, 2>(lab, base, w, pi, cand, resident, sup); break;
        case 3: score_box<R, IS3D, 3>(lab, base, w, pi, cand, resident, sup); break;
        default: score_box<R, IS3D, 6>(lab, base, w, pi, cand, resident, sup); break;
        }
        double best = -1.0;
        int32_t best_label = pi;
        for (int q = 0; q < nc; ++q)
            if (sup[q] > best) { best = sup[q]; best_label = cand[q]; }
        const int i = D.idx(z0 + lz, y0 + ly, x0 + lx);
        res_out[i] = (real)resident;
        best_out[i] = (real)best;
        phi_comp[i] = best_label;
    }
}

// ---------------------------------------------------------------------------
// pair projection
// ---------------------------------------------------------------------------
// Staged per halo cell: its unordered label pair (low, high), or (-1, -1) when
// it is not an interface cell or has no competitor, and orientation*vn.
template <typename real, int R, bool IS3D>
__global__ void __launch_bounds__(256) k_projection_tiled(Dims D, const int32_t* __restrict__ phi,
                                                          const int32_t* __restrict__ phi_comp,
                                                          const uint8_t* __restrict__ mask, const real* __restrict__ vn,
                                                          real* __restrict__ vn_out, int ntx, int nty,
                                                          const double* __restrict__ wtab) {
    typedef LocShape<R, IS3D> S;
    extern __shared__ __align__(16) unsigned char dyn[];
    int2* pair = reinterpret_cast<int2*>(dyn);          // S::NH entries
    real* svn = reinterpret_cast<real*>(pair + S::NH);  // S::NH entries
    __shared__ int16_t cells[S::NCELL];
    __shared__ double w[S::R2MAX + 1];
    const int t = blockIdx.x;
    const int tx = t % ntx, ty = (t / ntx) % nty, tz = t / (ntx * nty);
    const int x0 = tx * S::TX, y0 = ty * S::TY, z0 = tz * S::TZ;
    const int ncell = tile_interface_cells<R, IS3D>(D, mask, x0, y0, z0, cells);
    if (ncell == 0) return;
    for (int e = threadIdx.x; e < S::NH; e += 256) {
        const int hx = e % S::HX, hy = (e / S::HX) % S::HY, hz = e / (S::HX * S::HY);
        const int x = wrap_any(x0 + hx - R, D.Nx), y = wrap_any(y0 + hy - R, D.Ny);
        const int z = IS3D ? wrap_any(z0 + hz - R, D.Nz) : 0;
        const int j = D.idx(z, y, x);
        const int32_t pj = phi[j], qj = phi_comp[j];
        if (mask[j] && pj != qj) {
            const int32_t lo = min(pj, qj);
            pair[e] = make_int2(lo, max(pj, qj));
            svn[e] = (pj == lo) ? vn[j] : -vn[j];
        } else {
            pair[e] = make_int2(-1, -1);
            svn[e] = (real)0;
        }
    }
    for (int e = threadIdx.x; e <= S::R2MAX; e += 256) w[e] = wtab[e];
    __syncthreads();
    const int plane = S::HX * S::HY;
    for (int c = threadIdx.x; c < ncell; c += 256) {
        const int lc = cells[c];
        const int lx = lc % S::TX, ly = (lc / S::TX) % S::TY, lz = lc / (S::TX * S::TY);
        const int cb = ((IS3D ? lz + R : 0) * S::HY + ly + R) * S::HX + lx + R;
        const int i = D.idx(z0 + lz, y0 + ly, x0 + lx);
        const int2 pr = pair[cb];
        real out = vn[i];
        if (pr.x >= 0) {
            // interface cell with a competitor: average over the same pair
            const real orient_i = (phi[i] == pr.x) ? (real)1 : (real)-1;
            double num = 0.0, den = 0.0;
            const int base = cb - (IS3D ? R * plane : 0) - R * S::HX - R;
#pragma unroll 1
            for (int dz = (IS3D ? -R : 0); dz <= (IS3D ? R : 0); ++dz)
#pragma unroll 1
                for (int dy = -R; dy <= R; ++dy) {
                    const int rowb = base + ((IS3D ? dz + R : 0) * S::HY + dy + R) * S::HX + R;
                    const int r2yz = dy * dy + dz * dz;
#pragma unroll
                    for (int dx = -R; dx <= R; ++dx) {
                        const int e = rowb + dx;
                        const int2 pj = pair[e];
                        const double m = (pj.x == pr.x && pj.y == pr.y) ? 1.0 : 0.0;
                        const double wt = w[r2yz + dx * dx];
                        // reference: (w * orientation_j) * vn_j == w * (orientation_j * vn_j), exactly
                        num = __fma_rn(wt * (double)svn[e], m, num);
                        den = __fma_rn(wt, m, den);
                    }
                }
            if (den > 0.0) out = orient_i * (real)(num / den);
        }
        vn_out[i] = out;
    }
}

// ---------------------------------------------------------------------------
// balanced-remap scores: screening on label bitmaps, exact sums where needed
// ---------------------------------------------------------------------------
// The scores only matter through three outcomes: the best candidate label
// (phi_comp, public), whether gain = best - resident exceeds 1e-7 (a
// proposal) and, for proposals, the gain itself (their order).  A tile of
// 26 x TY x TZ cells has halo rows of exactly 32 cells (R = 3), so for one
// label a halo row is one 32-bit word; a 7-tap window of a row is a 7-bit
// pattern, and a table of the weight sums of all 128 patterns per (dy, dz)
// gives every score in 49 lookups.  Those sums are added in another order
// than the reference's, so they differ from its sums by far less than
// 1e-9.  A cell whose screened gain is below -1e-5 and whose best candidate
// leads the others by more than 1e-9 cannot make a proposal nor pick
// another candidate, whatever the rounding: it keeps the screened values
// (read only by the proposal test).  Every other cell is queued and summed
// exactly, tap by tap in z -> y -> x order as the reference adds them
// (src/gpk_transitions.cpp:67-85), by all threads of the CTA together.
template <bool IS3D> struct BitTile;
template <> struct BitTile<true> { static constexpr int TY = 8, TZ = 8; };
template <> struct BitTile<false> { static constexpr int TY = 32, TZ = 1; };

template <bool IS3D>
struct BitShape {
    static constexpr int R = 3;
    static constexpr int TX = 32 - 2 * R, HX = 32;
    static constexpr int TY = BitTile<IS3D>::TY, TZ = BitTile<IS3D>::TZ;
    static constexpr int HY = TY + 2 * R, HZ = IS3D ? TZ + 2 * R : 1;
    static constexpr int NROW = HY * HZ;
    static constexpr int NROWP = NROW | 1;
    static constexpr int NCELL = TX * TY * TZ;
    static constexpr int NH = NROW * HX;
    static constexpr int R2MAX = (IS3D ? 3 : 2) * R * R;
    static constexpr int NL = 16;       // bitmaps per tile
    static constexpr int HSLOT = 64;    // label hash slots
    static constexpr int NRS = 10;      // distinct dy^2 + dz^2 of a 7 x 7 row block
};

// index of dy^2 + dz^2 in {0, 1, 2, 4, 5, 8, 9, 10, 13, 18}
__device__ __forceinline__ int rsum_index(int r2) {
    switch (r2) {
    case 0: return 0; case 1: return 1; case 2: return 2; case 4: return 3; case 5: return 4;
    case 8: return 5; case 9: return 6; case 10: return 7; case 13: return 8; default: return 9;
    }
}
__host__ __device__ constexpr int rsum_value(int k) {
    return k == 0 ? 0 : k == 1 ? 1 : k == 2 ? 2 : k == 3 ? 4 : k == 4 ? 5 : k == 5 ? 8 : k == 6 ? 9 : k == 7 ? 10
           : k == 8 ? 13 : 18;
}

// the hash slot of label v, inserting it when absent (-1: table full)
__device__ __forceinline__ int label_slot_insert(int32_t* keys, int32_t v, int nslot) {
    unsigned h = ((unsigned)v * 2654435761u) >> 26;  // 6 bits
    for (int k = 0; k < nslot; ++k) {
        const int sl = (int)((h + k) & (nslot - 1));
        const int32_t old = atomicCAS(&keys[sl], -1, v);
        if (old == -1 || old == v) return sl;
    }
    return -1;
}
__device__ __forceinline__ int label_slot_find(const int32_t* keys, int32_t v, int nslot) {
    unsigned h = ((unsigned)v * 2654435761u) >> 26;
    for (int k = 0; k < nslot; ++k) {
        const int sl = (int)((h + k) & (nslot - 1));
        const int32_t key = keys[sl];
        if (key == v) return sl;
        if (key == -1) return -1;
    }
    return -1;
}

// screened sums of the resident label and NC candidates: one table lookup
// per row of 7 taps; li[k] is the bitmap base of label k (0: resident)
template <bool IS3D, int NC, bool RES = true>
__device__ __forceinline__ void screen_rows(const uint32_t* __restrict__ bm, const double* __restrict__ rtab,
                                            const int li[7], int lx, int ly, int lz, double& resident,
                                            double sup[6]) {
    typedef BitShape<IS3D> S;
    constexpr int R = S::R;
    const int row0 = (IS3D ? lz * S::HY : 0) + ly;  // halo row of tap (-R, -R) (2-D: (0, -R))
    // the dz loop stays rolled (code size); the table row of (dy, dz) is
    // rsum_index(dy^2 + dz^2), with dz^2 in {0, 1, 4, 9}
#pragma unroll 1
    for (int dz = (IS3D ? -R : 0); dz <= (IS3D ? R : 0); ++dz) {
        const int az = dz < 0 ? -dz : dz;
        // rsum_index(ay^2 + az^2) for ay = 0..3: four bits each, az's 16-bit row of
        // 0x9876'8543'7421'6310
        const unsigned idx4 = (unsigned)(0x9876854374216310ull >> (16 * az)) & 0xFFFFu;
#pragma unroll
        for (int dy = -R; dy <= R; ++dy) {
            const int row = row0 + (IS3D ? (dz + R) * S::HY : 0) + dy + R;
            const int ay = dy < 0 ? -dy : dy;
            const double* t = rtab + ((idx4 >> (4 * ay)) & 0xFu) * 128;
            if (RES) resident += t[(bm[li[0] + row] >> lx) & 0x7Fu];
#pragma unroll
            for (int q = 0; q < NC; ++q) sup[q] += t[(bm[li[q + 1] + row] >> lx) & 0x7Fu];
        }
    }
}

// Distinct face-neighbour labels other than pi, in face order, kept in
// registers (no indexed arrays): c[q] for q < n, -1 beyond.
template <bool IS3D>
__device__ __forceinline__ int face_candidates(const int32_t* __restrict__ lab, int cb, int32_t pi, int32_t c[6]) {
    typedef BitShape<IS3D> S;
    constexpr int NF = IS3D ? 6 : 4;
    const int fo[6] = {-1, +1, -S::HX, +S::HX, -S::HX * S::HY, +S::HX * S::HY};
    int32_t v[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) { v[k] = k < NF ? lab[cb + fo[k]] : pi; c[k] = -1; }
    int n = 0;
#pragma unroll
    for (int k = 0; k < NF; ++k) {
        bool fresh = v[k] != pi;
#pragma unroll
        for (int j = 0; j < k; ++j) fresh &= v[j] != v[k];
        if (fresh) {
#pragma unroll
            for (int q = 0; q <= k; ++q)
                if (q == n) c[q] = v[k];
            ++n;
        }
    }
    return n;
}

template <typename real, bool IS3D>
__global__ void __launch_bounds__(256) k_bgr_scores_screen(Dims D, const int32_t* __restrict__ phi,
                                                           const uint8_t* __restrict__ mask, int ntx, int nty,
                                                           const double* __restrict__ wtab,
                                                           const double* __restrict__ rtab_g, int nl_cap,
                                                           int32_t* __restrict__ phi_comp, real* __restrict__ res_out,
                                                           real* __restrict__ best_out,
                                                           const unsigned long long* __restrict__ gate,
                                                           StepScalars* stats) {
    if (gate && *gate == 0ull) return;  // device-side skip inside a captured step
    typedef BitShape<IS3D> S;
    constexpr int R = S::R;
    extern __shared__ __align__(16) int32_t lab[];  // S::NH halo labels (dynamic: the rest is static)
    __shared__ uint32_t bm[S::NL * S::NROWP];
    __shared__ int16_t cells[S::NCELL];
    __shared__ int16_t exact[S::NCELL];
    __shared__ double w[S::R2MAX + 1];
    __shared__ double rtab[S::NRS * 128];
    __shared__ int32_t keys[S::HSLOT];
    __shared__ int8_t dense[S::HSLOT];   // bitmap index of a slot, -1 when unused
    __shared__ int s_ncell, s_nl, s_full, s_nexact;
    __shared__ double s_wtot;  // weight of the whole box
    typedef cub::BlockScan<int, 256> BS;
    __shared__ typename BS::TempStorage scan;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    __shared__ int rowbase[S::NROW];  // flat index of halo row r's periodic (z, y) row
    const int t = blockIdx.x;
    const int tx = t % ntx, ty = (t / ntx) % nty, tz = t / (ntx * nty);
    const int x0 = tx * S::TX, y0 = ty * S::TY, z0 = tz * S::TZ;
    const int xw = wrap_any(x0 + lane - R, D.Nx);  // periodic x of halo column `lane`
    for (int r = tid; r < S::NROW; r += 256) {
        const int hy = r % S::HY, hz = r / S::HY;
        rowbase[r] = D.idx(IS3D ? wrap_any(z0 + hz - R, D.Nz) : 0, wrap_any(y0 + hy - R, D.Ny), 0);
    }
    // 1. interface cells of the tile, in flat tile order
    {
        constexpr int PER = (S::NCELL + 255) / 256;
        int flags[PER];
        int cnt = 0;
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const int c = tid * PER + k;
            int f = 0;
            if (c < S::NCELL) {
                const int lx = c % S::TX, ly = (c / S::TX) % S::TY, lz = c / (S::TX * S::TY);
                const int x = x0 + lx, y = y0 + ly, z = z0 + lz;
                if (x < D.Nx && y < D.Ny && z < D.Nz) f = mask[D.idx(z, y, x)];
            }
            flags[k] = f;
            cnt += f;
        }
        int ex, total;
        BS(scan).ExclusiveSum(cnt, ex, total);
#pragma unroll
        for (int k = 0; k < PER; ++k)
            if (flags[k]) cells[ex++] = (int16_t)(tid * PER + k);
        if (tid == 0) { s_ncell = total; s_full = 0; s_nexact = 0; }
    }
    if (tid < S::HSLOT) keys[tid] = -1;
    __syncthreads();
    const int ncell = s_ncell;
    if (ncell == 0) return;
    // 2. halo labels (one warp per row of 32 consecutive cells), weights, and
    //    the row table: rtab[k][p] = sum of the weights of pattern p's taps
    for (int r0 = warp; r0 < S::NROW; r0 += 64) {  // eight rows per warp at a time, loads issued together
        int32_t v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u)
            if (r0 + 8 * u < S::NROW) v[u] = phi[rowbase[r0 + 8 * u] + xw];
#pragma unroll
        for (int u = 0; u < 8; ++u)
            if (r0 + 8 * u < S::NROW) lab[(r0 + 8 * u) * S::HX + lane] = v[u];
    }
    for (int e = tid; e <= S::R2MAX; e += 256) w[e] = wtab[e];
    __syncthreads();
    for (int e = tid; e < S::NRS * 128; e += 256) rtab[e] = rtab_g[e];  // built on the host
    const int plane = S::HX * S::HY;
    const int fo[6] = {-1, +1, -S::HX, +S::HX, -plane, +plane};
    // 3. labels the scores need: a cell's label and its distinct other face
    //    labels; of the lanes of a warp holding one label, one inserts it
    for (int c0 = 0; c0 < ncell; c0 += 256) {
        const int c = c0 + tid;
        int32_t own = -1, cn[6] = {-1, -1, -1, -1, -1, -1};
        if (c < ncell) {
            const int lc = cells[c];
            const int lx = lc % S::TX, ly = (lc / S::TX) % S::TY, lz = lc / (S::TX * S::TY);
            const int cb = ((IS3D ? lz + R : 0) * S::HY + ly + R) * S::HX + lx + R;
            own = lab[cb];
            face_candidates<IS3D>(lab, cb, own, cn);
        }
#pragma unroll
        for (int q = 0; q < 7; ++q) {
            const int32_t v = q == 0 ? own : cn[q - 1];
            const unsigned grp = __match_any_sync(0xffffffffu, v);
            if (v >= 0 && lane == __ffs(grp) - 1 && label_slot_insert(keys, v, S::HSLOT) < 0) s_full = 1;
        }
    }
    __syncthreads();
    if (warp == 0) {
        // dense bitmap index per used slot, in slot order
        int total = 0;
        for (int base = 0; base < S::HSLOT; base += 32) {
            const bool used = keys[base + lane] != -1;
            const unsigned bal = __ballot_sync(0xffffffffu, used);
            dense[base + lane] = (int8_t)(used ? total + __popc(bal & ((1u << lane) - 1u)) : -1);
            total += __popc(bal);
        }
        if (lane == 0) {
            s_nl = total;
            double wt = 0.0;
            for (int dz = (IS3D ? -R : 0); dz <= (IS3D ? R : 0); ++dz)
                for (int dy = -R; dy <= R; ++dy) wt += rtab[rsum_index(dy * dy + dz * dz) * 128 + 127];
            s_wtot = wt;
        }
    }
    __syncthreads();
    const int nl = s_nl;
    const double wtot = s_wtot;
    const bool screen = !s_full && nl <= (nl_cap < S::NL ? nl_cap : S::NL);
    if (screen) {
        // 4. one word per halo row and listed label (words of absent labels stay 0)
        for (int e = tid; e < nl * S::NROWP; e += 256) bm[e] = 0u;
        __syncthreads();
        for (int r = warp; r < S::NROW; r += 8) {
            const int32_t v = lab[r * S::HX + lane];
            const unsigned grp = __match_any_sync(0xffffffffu, v);
            if (lane == __ffs(grp) - 1) {
                const int sl = label_slot_find(keys, v, S::HSLOT);
                if (sl >= 0 && dense[sl] >= 0) bm[dense[sl] * S::NROWP + r] = grp;
            }
        }
        __syncthreads();
    }
    // 5. screening; cells it cannot settle are queued
    for (int c = tid; c < ncell; c += 256) {
        bool settled = false;
        if (screen) {
            const int lc = cells[c];
            const int lx = lc % S::TX, ly = (lc / S::TX) % S::TY, lz = lc / (S::TX * S::TY);
            const int cb = ((IS3D ? lz + R : 0) * S::HY + ly + R) * S::HX + lx + R;
            const int32_t pi = lab[cb];
            int32_t cand[6];
            const int nc = face_candidates<IS3D>(lab, cb, pi, cand);
            int li[7];
            li[0] = dense[label_slot_find(keys, pi, S::HSLOT)] * S::NROWP;
#pragma unroll
            for (int q = 0; q < 6; ++q)
                li[q + 1] = q < nc ? dense[label_slot_find(keys, cand[q], S::HSLOT)] * S::NROWP : li[0];
            double resident = 0.0, sup[6] = {0, 0, 0, 0, 0, 0};
            screen_rows<IS3D, 0>(bm, rtab, li, lx, ly, lz, resident, sup);
            // One candidate: it is the best, and its score is at most the
            // weight of the box outside the resident label, wtot - resident;
            // when that bound already puts the gain below -1e-5 (with 1e-9 to
            // spare for the other summation order) its sum is not needed.
            const bool bounded = nc == 1 && wtot - resident - resident < -1e-5 - 1e-9;
            const int ncw = __reduce_max_sync(__activemask(), bounded ? 0 : nc);
            switch (ncw) {
            case 0: break;
            case 1: screen_rows<IS3D, 1, false>(bm, rtab, li, lx, ly, lz, resident, sup); break;
            case 2: screen_rows<IS3D, 2, false>(bm, rtab, li, lx, ly, lz, resident, sup); break;
            case 3: screen_rows<IS3D, 3, false>(bm, rtab, li, lx, ly, lz, resident, sup); break;
            default: screen_rows<IS3D, 6, false>(bm, rtab, li, lx, ly, lz, resident, sup); break;
            }
            if (bounded) sup[0] = wtot - resident;
            double best = -1.0, second = -1.0;
            int32_t best_label = pi;
#pragma unroll
            for (int q = 0; q < 6; ++q) {
                if (q >= nc) break;
                if (sup[q] > best) { second = best; best = sup[q]; best_label = cand[q]; }
                else if (sup[q] > second) second = sup[q];
            }
            if (best - resident < -1e-5 && (nc < 2 || best - second > 1e-9)) {
                settled = true;
                const int i = D.idx(z0 + lz, y0 + ly, x0 + lx);
                res_out[i] = (real)resident;
                best_out[i] = (real)best;
                phi_comp[i] = best_label;
            }
        }
        if (!settled) exact[atomicAdd(&s_nexact, 1)] = (int16_t)c;
    }
    __syncthreads();
    // 6. exact sums of the queued cells, all threads together
    const int nexact = s_nexact;
    if (tid == 0 && stats) {
        atomicAdd(&stats->score_cells, (unsigned long long)ncell);
        atomicAdd(&stats->score_exact, (unsigned long long)nexact);
    }
    for (int e = tid; e < nexact; e += 256) {
        const int lc = cells[exact[e]];
        const int lx = lc % S::TX, ly = (lc / S::TX) % S::TY, lz = lc / (S::TX * S::TY);
        const int cb = ((IS3D ? lz + R : 0) * S::HY + ly + R) * S::HX + lx + R;
        const int32_t pi = lab[cb];
        int32_t cand[6] = {-1, -1, -1, -1, -1, -1};
        int nc = 0;
        for (int k = 0; k < (IS3D ? 6 : 4); ++k) {
            const int32_t v = lab[cb + fo[k]];
            if (v == pi) continue;
            bool known = false;
            for (int q = 0; q < nc; ++q) known |= cand[q] == v;
            if (!known) cand[nc++] = v;
        }
        double resident = 0.0, sup[6] = {0, 0, 0, 0, 0, 0};
        const int base = cb - (IS3D ? R * plane : 0) - R * S::HX - R;
        const int ncw = __reduce_max_sync(__activemask(), nc);
        switch (ncw) {
        case 0: score_box_impl<R, IS3D, 0, S::HX, S::HY>(lab, base, w, pi, cand, resident, sup); break;
        case 1: score_box_impl<R, IS3D, 1, S::HX, S::HY>(lab, base, w, pi, cand, resident, sup); break;
        case 2: score_box_impl<R, IS3D, 2, S::HX, S::HY>(lab, base, w, pi, cand, resident, sup); break;
        case 3: score_box_impl<R, IS3D, 3, S::HX, S::HY>(lab, base, w, pi, cand, resident, sup); break;
        default: score_box_impl<R, IS3D, 6, S::HX, S::HY>(lab, base, w, pi, cand, resident, sup); break;
        }
        double best = -1.0;
        int32_t best_label = pi;
        for (int q = 0; q < nc; ++q)
            if (sup[q] > best) { best = sup[q]; best_label = cand[q]; }
        const int i = D.idx(z0 + lz, y0 + ly, x0 + lx);
        res_out[i] = (real)resident;
        best_out[i] = (real)best;
        phi_comp[i] = best_label;
    }
}

// ---------------------------------------------------------------------------
// pair projection on pair bitmaps (radius 3)
// ---------------------------------------------------------------------------
// A tap of the projection counts when its cell is an interface cell with the
// centre's unordered label pair (src/gpk_physics.cpp:152-193).  A tile of
// 26 x TY x TZ cells lists the distinct pairs of its interface cells; per
// pair, one 32-bit word per halo row marks the halo cells holding that pair
// (a halo row is 32 cells), so a row of 7 taps is a 7-bit pattern and only
// its set bits add: num += w * (orientation_j * vn_j), den += w, in double,
// z -> y -> x, as the reference adds them.  The 28 weights by squared
// distance are kernel parameters (constant-bank operands of the products).
// Tiles with more than 64 distinct pairs sum their cells straight from global
// memory in the same order.
struct ProjW {
    double w[28];  // (double)expf(-r2 / (2 s^2)) for r2 = 0..27
};

__device__ __forceinline__ unsigned long long pair_key(int32_t p, int32_t q) {
    const int32_t lo = p < q ? p : q, hi = p < q ? q : p;
    return ((unsigned long long)(uint32_t)lo << 32) | (uint32_t)hi;
}
__device__ __forceinline__ int pair_slot_insert(unsigned long long* keys, unsigned long long v) {
    const unsigned h = (unsigned)((v * 0x9E3779B97F4A7C15ull) >> 58);  // 6 bits: 64 slots
    for (int k = 0; k < 64; ++k) {
        const int sl = (int)((h + k) & 63u);
        const unsigned long long old = atomicCAS(&keys[sl], ~0ull, v);
        if (old == ~0ull || old == v) return sl;
    }
    return -1;
}
__device__ __forceinline__ int pair_slot_find(const unsigned long long* keys, unsigned long long v) {
    const unsigned h = (unsigned)((v * 0x9E3779B97F4A7C15ull) >> 58);
    for (int k = 0; k < 64; ++k) {
        const int sl = (int)((h + k) & 63u);
        const unsigned long long key = keys[sl];
        if (key == v) return sl;
        if (key == ~0ull) return -1;
    }
    return -1;
}

// One cell's sums read from global memory (tiles whose pairs overflow the
// slot table): the same taps, order and operations as the bitmap path.
template <typename real, bool IS3D>
__device__ void proj_cell_global(const Dims& D, const int32_t* __restrict__ phi, const int32_t* __restrict__ phi_comp,
                                 const uint8_t* __restrict__ mask, const real* __restrict__ vn, const ProjW& pw,
                                 int x, int y, int z, unsigned long long key, double& num, double& den) {
    constexpr int R = 3, RZ = IS3D ? 3 : 0;
#pragma unroll 1
    for (int dz = -RZ; dz <= RZ; ++dz)
#pragma unroll 1
        for (int dy = -R; dy <= R; ++dy)
#pragma unroll
            for (int dx = -R; dx <= R; ++dx) {
                const int j = D.idx(IS3D ? wrap_any(z + dz, D.Nz) : 0, wrap_any(y + dy, D.Ny), wrap_any(x + dx, D.Nx));
                const int32_t pj = phi[j], qj = phi_comp[j];
                if (mask[j] && pj != qj && pair_key(pj, qj) == key) {
                    const double wt = pw.w[dz * dz + dy * dy + dx * dx];
                    const double sv = pj < qj ? (double)vn[j] : -(double)vn[j];
                    num = num + wt * sv;
                    den = den + wt;
                }
            }
}

template <typename real, bool IS3D>
__global__ void __launch_bounds__(256) k_projection_bits(Dims D, const int32_t* __restrict__ phi,
                                                         const int32_t* __restrict__ phi_comp,
                                                         const uint8_t* __restrict__ mask, const real* __restrict__ vn,
                                                         real* __restrict__ vn_out, int ntx, int nty, int nl_cap,
                                                         ProjW pw) {
    typedef BitShape<IS3D> S;
    constexpr int R = S::R, RZ = IS3D ? R : 0;
    constexpr unsigned long long NONE = ~0ull;
    extern __shared__ __align__(16) double svn[];  // S::NH signed velocities of the halo
    __shared__ uint32_t bm[S::NL * S::NROWP];
    __shared__ int16_t cells[S::NCELL];
    __shared__ int8_t cslot[S::NCELL];  // pair slot of a listed cell; -1: no competitor, -2: slots full
    __shared__ unsigned long long keys[64];
    __shared__ int8_t dense[64];
    __shared__ int rowbase[S::NROW];  // flat index of halo row r's periodic (z, y) row
    __shared__ int s_ncell, s_np, s_full;
    typedef cub::BlockScan<int, 256> BS;
    __shared__ typename BS::TempStorage scan;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int t = blockIdx.x;
    const int tx = t % ntx, ty = (t / ntx) % nty, tz = t / (ntx * nty);
    const int x0 = tx * S::TX, y0 = ty * S::TY, z0 = tz * S::TZ;
    const int xw = wrap_any(x0 + lane - R, D.Nx);  // periodic x of halo column `lane`
    for (int r = tid; r < S::NROW; r += 256) {
        const int hy = r % S::HY, hz = r / S::HY;
        rowbase[r] = D.idx(IS3D ? wrap_any(z0 + hz - R, D.Nz) : 0, wrap_any(y0 + hy - R, D.Ny), 0);
    }
    // 1. interface cells of the tile, in flat tile order
    {
        constexpr int PER = (S::NCELL + 255) / 256;
        int flags[PER];
        int cnt = 0;
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const int c = tid * PER + k;
            int f = 0;
            if (c < S::NCELL) {
                const int lx = c % S::TX, ly = (c / S::TX) % S::TY, lz = c / (S::TX * S::TY);
                const int x = x0 + lx, y = y0 + ly, z = z0 + lz;
                if (x < D.Nx && y < D.Ny && z < D.Nz) f = mask[D.idx(z, y, x)];
            }
            flags[k] = f;
            cnt += f;
        }
        int ex, total;
        BS(scan).ExclusiveSum(cnt, ex, total);
#pragma unroll
        for (int k = 0; k < PER; ++k)
            if (flags[k]) cells[ex++] = (int16_t)(tid * PER + k);
        if (tid == 0) { s_ncell = total; s_full = 0; }
    }
    if (tid < 64) keys[tid] = NONE;
    __syncthreads();
    const int ncell = s_ncell;
    if (ncell == 0) return;
    // 2. the pair of every listed cell (of the lanes of a warp holding one
    //    pair, one inserts it); cells without a competitor keep vn
    for (int c0 = 0; c0 < ncell; c0 += 256) {
        const int c = c0 + tid;
        unsigned long long key = NONE;
        if (c < ncell) {
            const int lc = cells[c];
            const int lx = lc % S::TX, ly = (lc / S::TX) % S::TY, lz = lc / (S::TX * S::TY);
            const int i = D.idx(z0 + lz, y0 + ly, x0 + lx);
            const int32_t p = phi[i], q = phi_comp[i];
            if (p != q) key = pair_key(p, q);
            else vn_out[i] = vn[i];
        }
        const unsigned grp = __match_any_sync(0xffffffffu, key);
        const int leader = __ffs(grp) - 1;
        int sl = -1;
        if (key != NONE && lane == leader) {
            sl = pair_slot_insert(keys, key);
            if (sl < 0) s_full = 1;
        }
        sl = __shfl_sync(0xffffffffu, sl, leader);
        if (c < ncell) cslot[c] = (int8_t)(key == NONE ? -1 : (sl < 0 ? -2 : sl));
    }
    __syncthreads();
    if (s_full) {
        for (int c = tid; c < ncell; c += 256) {
            if (cslot[c] == -1) continue;
            const int lc = cells[c];
            const int lx = lc % S::TX, ly = (lc / S::TX) % S::TY, lz = lc / (S::TX * S::TY);
            const int i = D.idx(z0 + lz, y0 + ly, x0 + lx);
            const int32_t p = phi[i], q = phi_comp[i];
            double num = 0.0, den = 0.0;
            proj_cell_global<real, IS3D>(D, phi, phi_comp, mask, vn, pw, x0 + lx, y0 + ly, z0 + lz, pair_key(p, q),
                                         num, den);
            real out = vn[i];
            if (den > 0.0) out = (p < q ? (real)1 : (real)-1) * (real)(num / den);
            vn_out[i] = out;
        }
        return;
    }
    if (warp == 0) {
        // dense pair index per used slot, in slot order
        int total = 0;
        for (int base = 0; base < 64; base += 32) {
            const bool used = keys[base + lane] != NONE;
            const unsigned bal = __ballot_sync(0xffffffffu, used);
            dense[base + lane] = (int8_t)(used ? total + __popc(bal & ((1u << lane) - 1u)) : -1);
            total += __popc(bal);
        }
        if (lane == 0) s_np = total;
    }
    __syncthreads();
    const int np = s_np;
    const int nlb = nl_cap < S::NL ? nl_cap : S::NL;
    // 3. per batch of pairs: halo bitmaps (the first batch also stages the
    //    signed velocities), then the batch's cells
    for (int b0 = 0; b0 < np; b0 += nlb) {
        const int nb = np - b0 < nlb ? np - b0 : nlb;
        for (int e = tid; e < nb * S::NROWP; e += 256) bm[e] = 0u;
        __syncthreads();
        // a warp takes four rows at a time, their loads issued together
        for (int r0 = warp; r0 < S::NROW; r0 += 32) {
            int32_t pj[4], qj[4];
            uint8_t mj[4];
            real vj[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int r = r0 + 8 * u;
                if (r < S::NROW) {
                    const int j = rowbase[r] + xw;
                    pj[u] = phi[j];
                    qj[u] = phi_comp[j];
                    mj[u] = mask[j];
                    vj[u] = vn[j];
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int r = r0 + 8 * u;
                if (r >= S::NROW) break;
                const bool valid = mj[u] && pj[u] != qj[u];
                const unsigned long long key = valid ? pair_key(pj[u], qj[u]) : NONE;
                if (b0 == 0) svn[r * S::HX + lane] = valid ? (pj[u] < qj[u] ? (double)vj[u] : -(double)vj[u]) : 0.0;
                const unsigned grp = __match_any_sync(0xffffffffu, key);
                if (key != NONE && lane == __ffs(grp) - 1) {
                    const int sl = pair_slot_find(keys, key);
                    if (sl >= 0) {
                        const int d = dense[sl] - b0;
                        if (d >= 0 && d < nb) bm[d * S::NROWP + r] = grp;
                    }
                }
            }
        }
        __syncthreads();
        for (int c = tid; c < ncell; c += 256) {
            const int sl = cslot[c];
            if (sl < 0) continue;
            const int d = dense[sl] - b0;
            if (d < 0 || d >= nb) continue;
            const int lc = cells[c];
            const int lx = lc % S::TX, ly = (lc / S::TX) % S::TY, lz = lc / (S::TX * S::TY);
            const int rc = (IS3D ? lz * S::HY : 0) + ly;  // halo row of tap (-RZ, -R)
            const uint32_t* bmb = bm + d * S::NROWP + rc;
            const double* sv = svn + rc * S::HX + lx;
            double num = 0.0, den = 0.0;
#pragma unroll
            for (int dz = -RZ; dz <= RZ; ++dz)
#pragma unroll
                for (int dy = -R; dy <= R; ++dy) {
                    const int ro = (dz + RZ) * S::HY + dy + R;
                    const uint32_t bits = (bmb[ro] >> lx) & 0x7Fu;
                    if (!bits) continue;
                    const double* s = sv + ro * S::HX;
#pragma unroll
                    for (int k = 0; k < 2 * R + 1; ++k)
                        if (bits & (1u << k)) {
                            const double wt = pw.w[dz * dz + dy * dy + (k - R) * (k - R)];
                            num = num + wt * s[k];
                            den = den + wt;
                        }
                }
            const int i = D.idx(z0 + lz, y0 + ly, x0 + lx);
            const int32_t p = phi[i], q = phi_comp[i];
            real out = vn[i];
            if (den > 0.0) out = (p < q ? (real)1 : (real)-1) * (real)(num / den);
            vn_out[i] = out;
        }
        __syncthreads();  // the next batch rewrites the bitmaps
    }
}

template <typename real, bool IS3D>
static int launch_projection_bits(gpk_grid* G) {
    typedef BitShape<IS3D> S;
    const HostKernels<real>* hk = (const HostKernels<real>*)G->host_kernels;
    if (hk->proj_w.size() > 28) return -1;
    ProjW pw{};
    for (size_t k = 0; k < hk->proj_w.size(); ++k) pw.w[k] = hk->proj_w[k];
    const Dims D = G->d;
    const int ntx = (D.Nx + S::TX - 1) / S::TX, nty = (D.Ny + S::TY - 1) / S::TY, ntz = (D.Nz + S::TZ - 1) / S::TZ;
    const size_t smem = sizeof(double) * S::NH;
    // set once per process (thread-safe initialisation of a function-local static)
    static const cudaError_t attr_rc = cudaFuncSetAttribute(
        k_projection_bits<real, IS3D>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    GPK_CUDA_TRY(attr_rc);
    k_projection_bits<real, IS3D><<<ntx * nty * ntz, 256, smem, G->stream>>>(
        D, G->phi, G->phi_comp, G->mask, (const real*)G->f[GPK_FIELD_VN], (real*)G->vn2, ntx, nty,
        G->geometry_kernel == 2 ? 1 : S::NL, pw);
    G->launches++;
    GPK_CUDA_TRY(cudaGetLastError());
    return GPK_OK;
}

template <typename real, bool IS3D>
static int launch_scores_screen(gpk_grid* G, real* res, real* best, const unsigned long long* gate) {
    typedef BitShape<IS3D> S;
    const Dims D = G->d;
    const int ntx = (D.Nx + S::TX - 1) / S::TX, nty = (D.Ny + S::TY - 1) / S::TY, ntz = (D.Nz + S::TZ - 1) / S::TZ;
    const size_t smem = sizeof(int32_t) * S::NH;
    // set once per process (thread-safe initialisation of a function-local static)
    static const cudaError_t attr_rc = cudaFuncSetAttribute(
        k_bgr_scores_screen<real, IS3D>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    GPK_CUDA_TRY(attr_rc);
    k_bgr_scores_screen<real, IS3D><<<ntx * nty * ntz, 256, smem, G->stream>>>(
        D, G->phi, G->mask, ntx, nty, G->d_remap_w, G->d_remap_rtab, G->geometry_kernel == 2 ? 1 : S::NL,
        G->phi_comp, res, best,
        gate, G->scal);
    G->launches++;
    GPK_CUDA_TRY(cudaGetLastError());
    return GPK_OK;
}

template <typename real, int R, bool IS3D>
static int launch_scores(gpk_grid* G, real* res, real* best, const unsigned long long* gate) {
    typedef LocShape<R, IS3D> S;
    const Dims D = G->d;
    const int ntx = (D.Nx + S::TX - 1) / S::TX, nty = (D.Ny + S::TY - 1) / S::TY, ntz = (D.Nz + S::TZ - 1) / S::TZ;
    k_bgr_scores_tiled<real, R, IS3D><<<ntx * nty * ntz, 256, 0, G->stream>>>(D, G->phi, G->mask, ntx, nty,
                                                                               G->d_remap_w, G->phi_comp, res, best,
                                                                               gate);
    G->launches++;
    GPK_CUDA_TRY(cudaGetLastError());
    return GPK_OK;
}

template <typename real, int R, bool IS3D>
static int launch_projection(gpk_grid* G) {
    typedef LocShape<R, IS3D> S;
    const Dims D = G->d;
    const int ntx = (D.Nx + S::TX - 1) / S::TX, nty = (D.Ny + S::TY - 1) / S::TY, ntz = (D.Nz + S::TZ - 1) / S::TZ;
    const size_t smem = (size_t)S::NH * (sizeof(int2) + sizeof(real));
    // set once per process (thread-safe initialisation of a function-local static)
    static const cudaError_t attr_rc = cudaFuncSetAttribute(
        k_projection_tiled<real, R, IS3D>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    GPK_CUDA_TRY(attr_rc);
    k_projection_tiled<real, R, IS3D><<<ntx * nty * ntz, 256, smem, G->stream>>>(
        D, G->phi, G->phi_comp, G->mask, (const real*)G->f[GPK_FIELD_VN], (real*)G->vn2, ntx, nty, G->d_proj_w);
    G->launches++;
    GPK_CUDA_TRY(cudaGetLastError());
    return GPK_OK;
}

}  // namespace gpk_dev

using namespace gpk_dev;

// Tiled remap scores for radius 3 (the remap radius ceil(3 s) at every sigma:
// s = clamp(sigma / 8, 0.7, 1)); -1 when no tiled instantiation applies.
template <typename real>
int gpk_bgr_scores_tiled(gpk_grid* G, int radius, real* res, real* best, const unsigned long long* gate) {
    if (radius != 3) return -1;
    if (G->geometry_kernel == 3)  // the all-exact tiled kernel (comparison runs)
        return G->d.is3d() ? launch_scores<real, 3, true>(G, res, best, gate)
                           : launch_scores<real, 3, false>(G, res, best, gate);
    return G->d.is3d() ? launch_scores_screen<real, true>(G, res, best, gate)
                       : launch_scores_screen<real, false>(G, res, best, gate);
}

// Tiled projection for the radii ceil(3 s) of the velocity kernel (s =
// clamp(0.375 sigma, 0.85, 3) in 3-D: radii 3 to 9) whose 3-D halo tile fits
// in the 227 KB of shared memory: 3 to 8 in FP32, 3 to 6 in FP64 (2-D: 3 to
// 9).  -1 otherwise (the per-cell kernel runs).
template <typename real, int R>
static constexpr bool proj_fits() {
    // dynamic halo arrays plus 8 KB for the static cell list, weights and scan
    return (size_t)LocShape<R, true>::NH * (sizeof(int2) + sizeof(real)) + 8 * 1024 <= 227 * 1024;
}

template <typename real, int R>
static int projection_r(gpk_grid* G) {
    if (!G->d.is3d()) return launch_projection<real, R, false>(G);
    if constexpr (proj_fits<real, R>()) return launch_projection<real, R, true>(G);
    return -1;
}

template <typename real>
int gpk_projection_tiled(gpk_grid* G, int radius) {
    switch (radius) {
        case 3:
            // pair bitmaps; kind 3 keeps the pair-compare tiles (comparison runs)
            if (G->geometry_kernel != 3)
                return G->d.is3d() ? launch_projection_bits<real, true>(G) : launch_projection_bits<real, false>(G);
            return projection_r<real, 3>(G);
        case 4: return projection_r<real, 4>(G);
        case 5: return projection_r<real, 5>(G);
        case 6: return projection_r<real, 6>(G);
        case 7: return projection_r<real, 7>(G);
        case 8: return projection_r<real, 8>(G);
        case 9: return projection_r<real, 9>(G);
        default: return -1;
    }
}

template int gpk_bgr_scores_tiled<float>(gpk_grid*, int, float*, float*, const unsigned long long*);
template int gpk_bgr_scores_tiled<double>(gpk_grid*, int, double*, double*, const unsigned long long*);
template int gpk_projection_tiled<float>(gpk_grid*, int);
template int gpk_projection_tiled<double>(gpk_grid*, int);
