// gpk_geometry.cu — tiled, branch-free Gaussian-Hessian geometry for sm_100a.
//
// Same result, bit for bit, as the direct masked tensor stencil of the
// reference (src/gpk_geometry.cpp:88-152): for every interface cell the nine
// sums Ix..Iyz run over the (2R+1)^d taps in z -> y -> x order, each tap
// adding its precomputed product (formed on the host exactly as (a*b)*c)
// when the tap's label equals the cell's label.
//
// Exactness of the branch-free form: each sum starts at +0 and in round-to-
// nearest a sum that starts at +0 can never become -0 (x + (-x) = +0, and
// +0 + -0 = +0).  Adding a signed zero to such a sum is therefore an exact
// no-op, so fma(w, m, acc) with m in {0, 1} rounds exactly like the
// reference's `if (match) acc += w`: for m = 1 it is one correctly rounded
// addition of w, for m = 0 it adds +-0.
//
// Layout: one CTA per TX x TY x TZ tile of cells.  The CTA stages the tile's
// labels with an R-cell periodic halo in shared memory (row pitch padded by
// one word so that rows start in different banks), compacts the tile's
// interface cells, and gives each thread 1..4 of them.  The product table is
// streamed one z-plane at a time (W*W taps x 12 reals) into a double buffer
// by TMA bulk copies (cp.async.bulk + mbarrier), overlapping the next
// plane's copy with the current plane's arithmetic.  All warps read the
// same table entry at the same time (broadcast), and each thread's label
// reads are one LDS per cell and tap.
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include "gpk_grid.h"

namespace gpk_dev {

// ---- mbarrier / bulk-copy helpers (bounded waits) ---------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
// true when the phase with the given parity has completed; gives up (false)
// after a bounded number of polls
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    for (int it = 0; it < (1 << 22); ++it) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

template <typename real> __device__ __forceinline__ real fma_rn(real a, real b, real c);
template <> __device__ __forceinline__ float fma_rn<float>(float a, float b, float c) { return __fmaf_rn(a, b, c); }
template <> __device__ __forceinline__ double fma_rn<double>(double a, double b, double c) { return __fma_rn(a, b, c); }

template <bool IS3D> struct GeoTile;
template <> struct GeoTile<true> { static constexpr int TX = 16, TY = 8, TZ = 8; };
template <> struct GeoTile<false> { static constexpr int TX = 32, TY = 32, TZ = 1; };

template <typename real>
struct GeoArgs {
    Dims D;
    const int32_t* phi;
    const uint8_t* mask;
    const real* table;  // W^dz planes of W*W taps x 12 reals
    int ntx, nty, ntz;
    real inv_dx, inv_dx2, dx, kappa_limit;
    real *nx, *ny, *nz, *kappa;
    int32_t* phi_comp;
    StepScalars* s;
};

template <int R, bool IS3D>
struct GeoShape {
    static constexpr int W = 2 * R + 1;
    static constexpr int TX = GeoTile<IS3D>::TX, TY = GeoTile<IS3D>::TY, TZ = GeoTile<IS3D>::TZ;
    static constexpr int HX = TX + 2 * R, HXP = HX + 1, HY = TY + 2 * R, HZ = IS3D ? TZ + 2 * R : 1;
    static constexpr int NLAB = HZ * HY * HXP;
    static constexpr int NCELL = TX * TY * TZ;
    static constexpr int PLANE = W * W * 12;  // reals per table plane
    static constexpr int NPLANES = IS3D ? W : 1;
};

template <typename real, int R, bool IS3D>
constexpr size_t geo_smem_bytes() {
    typedef GeoShape<R, IS3D> S;
    // table planes (16-byte aligned) | labels | cell list | 2 mbarriers
    return (size_t)2 * S::PLANE * sizeof(real) + (size_t)S::NLAB * 4 + (size_t)S::NCELL * 2 + 64;
}

// One row of W taps (fixed dz, dy).  The Gaussian factor w0(o) is exactly 0
// for |o| in {R-1, R} (the Gaussian has radius R-2), so a product with such
// a factor is +-0 and adding it is an exact no-op (see the file comment):
//   x factor zero (|dx| >= R-1): Iy, Iyy, Iz, Izz, Iyz have no contribution
//   y factor zero (ZY0):         Ix, Ixx, Iz, Izz, Ixz
//   z factor zero (ZZ0):         Ix, Iy, Ixx, Iyy, Ixy
// Components: 0 Ix, 1 Iy, 2 Ixx, 3 Iyy, 4 Ixy, 5 Iz, 6 Izz, 7 Ixz, 8 Iyz.
template <typename real, int R, bool IS3D, int SLOTS, bool ZY0, bool ZZ0>
__device__ __forceinline__ void geo_row(const int32_t* __restrict__ lab, const real* __restrict__ trow, int yoff,
                                        real acc[SLOTS][9], const int base[SLOTS], const int32_t res[SLOTS]) {
    constexpr int W = 2 * R + 1;
#pragma unroll
    for (int dxs = 0; dxs < W; ++dxs) {
        const bool zx0 = dxs <= 1 || dxs >= W - 2;  // compile-time after unrolling
        bool live[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) live[k] = IS3D || k < 5;
        if (zx0) live[1] = live[3] = live[5] = live[6] = live[8] = false;
        if (ZY0) live[0] = live[2] = live[5] = live[6] = live[7] = false;
        if (ZZ0) live[0] = live[1] = live[2] = live[3] = live[4] = false;
        bool any = false;
#pragma unroll
        for (int k = 0; k < 9; ++k) any |= live[k];
        if (!any) continue;
        const real* t = trow + dxs * 12;
        real w[9];
        if (sizeof(real) == 4) {
            const float4 t0 = *reinterpret_cast<const float4*>(t);
            const float4 t1 = *reinterpret_cast<const float4*>(t + 4);
            w[0] = t0.x; w[1] = t0.y; w[2] = t0.z; w[3] = t0.w;
            w[4] = t1.x; w[5] = t1.y; w[6] = t1.z; w[7] = t1.w;
            w[8] = live[8] ? t[8] : (real)0;
        } else {
#pragma unroll
            for (int k = 0; k < 9; ++k) w[k] = live[k] ? t[k] : (real)0;
        }
#pragma unroll
        for (int s = 0; s < SLOTS; ++s) {
            const real m = (lab[base[s] + yoff + dxs] == res[s]) ? (real)1 : (real)0;
#pragma unroll
            for (int k = 0; k < 9; ++k)
                if (live[k]) acc[s][k] = fma_rn<real>(w[k], m, acc[s][k]);
        }
    }
}

template <typename real, int R, bool IS3D, int SLOTS>
__device__ __forceinline__ void geo_accumulate(const GeoArgs<real>& a, const int32_t* __restrict__ lab,
                                               const real* __restrict__ tab0, const real* __restrict__ tab1,
                                               uint64_t* bars, const int16_t* cells, int nact, int tid,
                                               real acc[SLOTS][9], int base[SLOTS], int32_t res[SLOTS], bool& ok) {
    typedef GeoShape<R, IS3D> S;
    constexpr int W = S::W;
#pragma unroll
    for (int s = 0; s < SLOTS; ++s)
#pragma unroll
        for (int k = 0; k < 9; ++k) acc[s][k] = (real)0;
    for (int p = 0; p < S::NPLANES; ++p) {
        const real* tab = (p & 1) ? tab1 : tab0;
        if (!mbar_wait(&bars[p & 1], (uint32_t)((p >> 1) & 1))) {
            ok = false;
            atomicCAS(&a.s->error, 0u, (unsigned)GPK_ERR_TIMEOUT);
        }
        if (tid == 0 && p + 1 < S::NPLANES) {
            // the other buffer was last read in plane p-1, which every thread
            // finished before the barrier at the end of that plane
            fence_proxy_async();
            real* dst = ((p + 1) & 1) ? (real*)tab1 : (real*)tab0;
            mbar_expect_tx(&bars[(p + 1) & 1], S::PLANE * sizeof(real));
            bulk_g2s(dst, a.table + (size_t)(p + 1) * S::PLANE, S::PLANE * sizeof(real), &bars[(p + 1) & 1]);
        }
        if (ok && tid < nact) {
            const int zoff = p * S::HY * S::HXP;
            // rows whose y or z Gaussian factor is exactly zero run
            // specialised bodies without the corresponding products
            const bool zz0 = IS3D && (p <= 1 || p >= W - 2);
#pragma unroll 1
            for (int dy = 0; dy < W; ++dy) {
                const real* trow = tab + dy * W * 12;
                const int yoff = zoff + dy * S::HXP;
                const bool yy0 = dy <= 1 || dy >= W - 2;
                if (zz0) {
                    if (yy0) geo_row<real, R, IS3D, SLOTS, true, true>(lab, trow, yoff, acc, base, res);
                    else geo_row<real, R, IS3D, SLOTS, false, true>(lab, trow, yoff, acc, base, res);
                } else {
                    if (yy0) geo_row<real, R, IS3D, SLOTS, true, false>(lab, trow, yoff, acc, base, res);
                    else geo_row<real, R, IS3D, SLOTS, false, false>(lab, trow, yoff, acc, base, res);
                }
            }
        }
        __syncthreads();
    }
}

template <typename real>
__device__ __forceinline__ void geo_finish(const GeoArgs<real>& a, int i, const real* acc, const int32_t* __restrict__ lab,
                                           int cbase, int HXP, int HY, bool is3d) {
    real Ix = acc[0] * a.inv_dx, Iy = acc[1] * a.inv_dx, Iz = acc[5] * a.inv_dx;
    real Ixx = acc[2] * a.inv_dx2, Iyy = acc[3] * a.inv_dx2, Izz = acc[6] * a.inv_dx2;
    real Ixy = acc[4] * a.inv_dx2, Ixz = acc[7] * a.inv_dx2, Iyz = acc[8] * a.inv_dx2;
    const real dx = a.dx;
    const real grad_sq = Ix * Ix + Iy * Iy + Iz * Iz;
    real nxv = 0, nyv = 0, nzv = 0;
    if (grad_sq * dx * dx > (real)1e-8) {
        const real grad = sqrt(grad_sq);
        nxv = -Ix / grad;
        nyv = -Iy / grad;
        nzv = -Iz / grad;
        const real trace_H = Ixx + Iyy + Izz;
        const real gHg = Ix * Ix * Ixx + Iy * Iy * Iyy + Iz * Iz * Izz + (real)2 * (Ix * Iy * Ixy + Ix * Iz * Ixz + Iy * Iz * Iyz);
        real curvature = (gHg - grad_sq * trace_H) / (grad_sq * grad);
        if (fabs(curvature * dx) < (real)1e-6) curvature = (real)0;
        a.nx[i] = nxv; a.ny[i] = nyv; a.nz[i] = nzv;
        a.kappa[i] = dclamp(curvature, -a.kappa_limit, a.kappa_limit);
    }
    // competitor choice (src/gpk_geometry.cpp:154-182) from the staged labels
    const int32_t pi = lab[cbase];
    const int plane = HY * HXP;
    const int fo[6] = {-1, +1, -HXP, +HXP, -plane, +plane};
    const real score[6] = {-nxv, nxv, -nyv, nyv, -nzv, nzv};
    const int nf = is3d ? 6 : 4;
    int best = -1, best_support = -1;
    real best_score = (real)-2;
    for (int k = 0; k < nf; ++k) {
        const int32_t q = lab[cbase + fo[k]];
        if (q == pi) continue;
        int support = 0;
        for (int dz = (is3d ? -1 : 0); dz <= (is3d ? 1 : 0); ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dxs = -1; dxs <= 1; ++dxs) {
                    if (!dxs && !dy && !dz) continue;
                    support += lab[cbase + dz * plane + dy * HXP + dxs] == q;
                }
        if (support > best_support || (support == best_support && score[k] > best_score)) {
            best = k; best_support = support; best_score = score[k];
        }
    }
    a.phi_comp[i] = (best >= 0) ? lab[cbase + fo[best]] : pi;
}

template <typename real, int R, bool IS3D>
__global__ void __launch_bounds__(256) k_geometry_tiled(GeoArgs<real> a) {
    typedef GeoShape<R, IS3D> S;
    extern __shared__ __align__(128) unsigned char smem[];
    real* tab0 = reinterpret_cast<real*>(smem);
    real* tab1 = tab0 + S::PLANE;
    int32_t* lab = reinterpret_cast<int32_t*>(tab1 + S::PLANE);
    int16_t* cells = reinterpret_cast<int16_t*>(lab + S::NLAB);
    uint64_t* bars = reinterpret_cast<uint64_t*>((reinterpret_cast<uintptr_t>(cells + S::NCELL) + 15) & ~(uintptr_t)15);
    __shared__ int s_count;
    const int tid = threadIdx.x;
    const Dims D = a.D;

    const int t = blockIdx.x;
    const int tx = t % a.ntx, ty = (t / a.ntx) % a.nty, tz = t / (a.ntx * a.nty);
    const int x0 = tx * S::TX, y0 = ty * S::TY, z0 = tz * S::TZ;

    // interface cells of the tile, in flat order
    if (tid == 0) s_count = 0;
    __syncthreads();
    {
        typedef cub::BlockScan<int, 256> BS;
        __shared__ typename BS::TempStorage scan;
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
                if (x < D.Nx && y < D.Ny && z < D.Nz) f = a.mask[D.idx(z, y, x)];
            }
            flags[k] = f;
            cnt += f;
        }
        int ex, total;
        BS(scan).ExclusiveSum(cnt, ex, total);
#pragma unroll
        for (int k = 0; k < PER; ++k)
            if (flags[k]) cells[ex++] = (int16_t)(tid * PER + k);
        if (tid == 0) s_count = total;
    }
    __syncthreads();
    const int ncell = s_count;
    if (ncell == 0) return;  // nothing staged or in flight yet

    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        fence_proxy_async();
        mbar_expect_tx(&bars[0], S::PLANE * sizeof(real));
        bulk_g2s(tab0, a.table, S::PLANE * sizeof(real), &bars[0]);
    }
    // labels with a periodic halo of R cells
    for (int e = tid; e < S::HZ * S::HY * S::HX; e += 256) {
        const int hx = e % S::HX, hy = (e / S::HX) % S::HY, hz = e / (S::HX * S::HY);
        const int x = wrap_any(x0 + hx - R, D.Nx), y = wrap_any(y0 + hy - R, D.Ny);
        const int z = IS3D ? wrap_any(z0 + hz - R, D.Nz) : 0;
        lab[(hz * S::HY + hy) * S::HXP + hx] = a.phi[D.idx(z, y, x)];
    }
    __syncthreads();

    // The tile's cells go to the fewest threads that hold them at `slots`
    // cells each: thread t < nact takes cells t, t + nact, ...  Warps whose
    // threads all lie beyond nact skip the arithmetic, leaving their issue
    // slots to the other resident CTA instead of computing dummy cells.
    const int slots = (ncell + 255) / 256;
    const int nact = (ncell + slots - 1) / slots;
    bool ok = true;
    int base[4], myc[4];
    int32_t res[4];
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        const int k = tid + nact * s;
        myc[s] = (tid < nact && k < ncell) ? cells[k] : -1;
        const int c = myc[s] < 0 ? cells[0] : myc[s];
        const int lx = c % S::TX, ly = (c / S::TX) % S::TY, lz = c / (S::TX * S::TY);
        // label of tap (dz,dy,dx) at lab[base + (dz+R)*plane + (dy+R)*HXP + (dx+R)]
        base[s] = (lz * S::HY + ly) * S::HXP + lx;
        res[s] = lab[base[s] + ((IS3D ? R : 0) * S::HY + R) * S::HXP + R];
    }

    real acc[4][9];
    switch (slots) {
    case 1: geo_accumulate<real, R, IS3D, 1>(a, lab, tab0, tab1, bars, cells, nact, tid, (real(*)[9])acc, base, res, ok); break;
    case 2: geo_accumulate<real, R, IS3D, 2>(a, lab, tab0, tab1, bars, cells, nact, tid, (real(*)[9])acc, base, res, ok); break;
    case 3: geo_accumulate<real, R, IS3D, 3>(a, lab, tab0, tab1, bars, cells, nact, tid, (real(*)[9])acc, base, res, ok); break;
    default: geo_accumulate<real, R, IS3D, 4>(a, lab, tab0, tab1, bars, cells, nact, tid, (real(*)[9])acc, base, res, ok); break;
    }
    if (!ok) return;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        if (s >= slots || myc[s] < 0) continue;
        const int c = myc[s];
        const int lx = c % S::TX, ly = (c / S::TX) % S::TY, lz = c / (S::TX * S::TY);
        const int i = D.idx(z0 + lz, y0 + ly, x0 + lx);
        const int cbase = base[s] + ((IS3D ? R : 0) * S::HY + R) * S::HXP + R;
        geo_finish<real>(a, i, acc[s], lab, cbase, S::HXP, S::HY, IS3D);
    }
}

template <typename real, int R, bool IS3D>
static int launch_tiled(gpk_grid* G, const GeoArgs<real>& a0) {
    typedef GeoShape<R, IS3D> S;
    GeoArgs<real> a = a0;
    a.ntx = (G->d.Nx + S::TX - 1) / S::TX;
    a.nty = (G->d.Ny + S::TY - 1) / S::TY;
    a.ntz = (G->d.Nz + S::TZ - 1) / S::TZ;
    const size_t smem = geo_smem_bytes<real, R, IS3D>();
    static bool attr_set = false;
    if (!attr_set) {
        GPK_CUDA_TRY(cudaFuncSetAttribute(k_geometry_tiled<real, R, IS3D>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem));
        attr_set = true;
    }
    const int ntiles = a.ntx * a.nty * a.ntz;
    k_geometry_tiled<real, R, IS3D><<<ntiles, 256, smem, G->stream>>>(a);
    G->launches++;
    GPK_CUDA_TRY(cudaGetLastError());
    return GPK_OK;
}

}  // namespace gpk_dev

using namespace gpk_dev;

// Tiled geometry for the common kernel radii; returns -1 when the radius or
// the shared-memory footprint has no tiled instantiation (the caller then uses
// the per-cell kernel).
template <typename real>
int gpk_geometry_tiled(gpk_grid* G, int R, real inv_dx, real inv_dx2, real dx, real kappa_limit) {
    GeoArgs<real> a;
    a.D = G->d;
    a.phi = G->phi;
    a.mask = G->mask;
    a.table = (const real*)G->d_geom_table;
    a.inv_dx = inv_dx; a.inv_dx2 = inv_dx2; a.dx = dx; a.kappa_limit = kappa_limit;
    a.nx = (real*)G->f[GPK_FIELD_NX]; a.ny = (real*)G->f[GPK_FIELD_NY]; a.nz = (real*)G->f[GPK_FIELD_NZ];
    a.kappa = (real*)G->f[GPK_FIELD_KAPPA];
    a.phi_comp = G->phi_comp;
    a.s = G->scal;
    const bool is3d = G->d.is3d();
    if (is3d) {
        switch (R) {
        case 6: return launch_tiled<real, 6, true>(G, a);
        case 7: return launch_tiled<real, 7, true>(G, a);
        case 8: return launch_tiled<real, 8, true>(G, a);
        case 9: return sizeof(real) == 4 ? launch_tiled<real, 9, true>(G, a) : -1;
        default: return -1;
        }
    }
    switch (R) {
    case 6: return launch_tiled<real, 6, false>(G, a);
    case 7: return launch_tiled<real, 7, false>(G, a);
    case 8: return launch_tiled<real, 8, false>(G, a);
    case 9: return launch_tiled<real, 9, false>(G, a);
    case 10: return launch_tiled<real, 10, false>(G, a);
    default: return -1;
    }
}

template int gpk_geometry_tiled<float>(gpk_grid*, int, float, float, float, float);
template int gpk_geometry_tiled<double>(gpk_grid*, int, double, double, double, double);
