// gpk_geometry.cu — tiled Gaussian-Hessian geometry on label bitmaps, sm_100a.
//
// Same result, bit for bit, as the direct masked tensor stencil of the
// reference (src/gpk_geometry.cpp:88-152): for every interface cell the nine
// sums Ix..Iyz run over the (2R+1)^d taps in z -> y -> x order, each tap
// adding its precomputed product (formed on the host exactly as (a*b)*c)
// when the tap's label equals the cell's label.  Here that test is one bit
// of a per-label bitmap, and the additions are predicated on it, so every
// sum is the reference's sequence of correctly rounded additions.
//
// Zero products: the Gaussian factor w0(o) is exactly 0 for |o| in
// {R-1, R} (the Gaussian has radius R-2), so some products of those taps
// are +-0.  Each sum starts at +0, and in round-to-nearest a sum that starts
// at +0 never becomes -0 (x + (-x) = +0 and +0 + -0 = +0), so adding +-0 to
// it is an exact no-op and such products are skipped.
//
// Layout: one CTA per tile of TX x TY x TZ cells with TX = 32 - 2R, so a row
// of the tile's halo (x from x0-R to x0+TX+R-1) is exactly 32 cells and, for
// one label, one 32-bit word.  The CTA
//   1. compacts the tile's interface cells and lists their distinct labels;
//   2. for each batch of labels, builds one word per halo row and label
//      (warp-per-row ballots over the labels read from global memory);
//   3. streams the product table one z-plane (W*W taps x 12 reals) at a time
//      into a double buffer with TMA bulk copies (cp.async.bulk + mbarrier),
//      overlapping the next plane's copy with the current plane's arithmetic;
//   4. gives each thread 2..4 of the batch's cells: per tap row it loads one
//      bitmap word per cell, and per tap it tests a bit and adds the live
//      products.  All warps read the same table entry at the same time
//      (broadcast), so the shared-memory traffic per tap is 1-3 LDS.128 for
//      all of a thread's cells.
// Table entry of a tap (12 reals, three quads):
//   A = (Ix, Ixx, Ixy, Ixz)   B = (Iy, Iyy, Ixy, Iyz)   C = (Iz, Izz, Ixz, Iyz)
// so a tap with a zero x (y, z) Gaussian factor needs quad A (B, C) alone.
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

// ---- predicated additions: acc_k += w_k when bit != 0 -----------------------
// One setp per tap and cell; the additions are plain IEEE round-to-nearest
// adds (no flush to zero), exactly the reference's `if (match) acc += w`.
// acc operands are %0..%n-1, the bit %n, the weights follow
__device__ __forceinline__ void padd(uint32_t b, float& a0, float w0) {
    asm("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %1, 0;\n\t" "@p add.rn.f32 %0, %0, %2;\n\t" "}"
        : "+f"(a0)
        : "r"(b), "f"(w0));
}
__device__ __forceinline__ void padd(uint32_t b, float& a0, float& a1, float w0, float w1) {
    asm("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %2, 0;\n\t" "@p add.rn.f32 %0, %0, %3;\n\t""@p add.rn.f32 %1, %1, %4;\n\t" "}"
        : "+f"(a0), "+f"(a1)
        : "r"(b), "f"(w0), "f"(w1));
}
__device__ __forceinline__ void padd(uint32_t b, float& a0, float& a1, float& a2, float w0, float w1, float w2) {
    asm("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %3, 0;\n\t" "@p add.rn.f32 %0, %0, %4;\n\t""@p add.rn.f32 %1, %1, %5;\n\t""@p add.rn.f32 %2, %2, %6;\n\t" "}"
        : "+f"(a0), "+f"(a1), "+f"(a2)
        : "r"(b), "f"(w0), "f"(w1), "f"(w2));
}
__device__ __forceinline__ void padd(uint32_t b, float& a0, float& a1, float& a2, float& a3, float w0, float w1, float w2, float w3) {
    asm("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t" "@p add.rn.f32 %0, %0, %5;\n\t""@p add.rn.f32 %1, %1, %6;\n\t""@p add.rn.f32 %2, %2, %7;\n\t""@p add.rn.f32 %3, %3, %8;\n\t" "}"
        : "+f"(a0), "+f"(a1), "+f"(a2), "+f"(a3)
        : "r"(b), "f"(w0), "f"(w1), "f"(w2), "f"(w3));
}
__device__ __forceinline__ void padd(uint32_t b, double& a0, double w0) {
    asm("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %1, 0;\n\t" "@p add.rn.f64 %0, %0, %2;\n\t" "}"
        : "+d"(a0)
        : "r"(b), "d"(w0));
}
__device__ __forceinline__ void padd(uint32_t b, double& a0, double& a1, double w0, double w1) {
    asm("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %2, 0;\n\t" "@p add.rn.f64 %0, %0, %3;\n\t""@p add.rn.f64 %1, %1, %4;\n\t" "}"
        : "+d"(a0), "+d"(a1)
        : "r"(b), "d"(w0), "d"(w1));
}
__device__ __forceinline__ void padd(uint32_t b, double& a0, double& a1, double& a2, double w0, double w1, double w2) {
    asm("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %3, 0;\n\t" "@p add.rn.f64 %0, %0, %4;\n\t""@p add.rn.f64 %1, %1, %5;\n\t""@p add.rn.f64 %2, %2, %6;\n\t" "}"
        : "+d"(a0), "+d"(a1), "+d"(a2)
        : "r"(b), "d"(w0), "d"(w1), "d"(w2));
}
__device__ __forceinline__ void padd(uint32_t b, double& a0, double& a1, double& a2, double& a3, double w0, double w1, double w2, double w3) {
    asm("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t" "@p add.rn.f64 %0, %0, %5;\n\t""@p add.rn.f64 %1, %1, %6;\n\t""@p add.rn.f64 %2, %2, %7;\n\t""@p add.rn.f64 %3, %3, %8;\n\t" "}"
        : "+d"(a0), "+d"(a1), "+d"(a2), "+d"(a3)
        : "r"(b), "d"(w0), "d"(w1), "d"(w2), "d"(w3));
}

// One predicate for all additions of a tap: nine (3-D, no zero factor) or
// five (2-D) accumulators.
__device__ __forceinline__ void padd9(uint32_t b, float& a0, float& a1, float& a2, float& a3, float& a4, float& a5,
                                      float& a6, float& a7, float& a8, float w0, float w1, float w2, float w3,
                                      float w4, float w5, float w6, float w7, float w8) {
    asm("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %9, 0;\n\t"
        "@p add.rn.f32 %0, %0, %10;\n\t@p add.rn.f32 %1, %1, %11;\n\t@p add.rn.f32 %2, %2, %12;\n\t"
        "@p add.rn.f32 %3, %3, %13;\n\t@p add.rn.f32 %4, %4, %14;\n\t@p add.rn.f32 %5, %5, %15;\n\t"
        "@p add.rn.f32 %6, %6, %16;\n\t@p add.rn.f32 %7, %7, %17;\n\t@p add.rn.f32 %8, %8, %18;\n\t}"
        : "+f"(a0), "+f"(a1), "+f"(a2), "+f"(a3), "+f"(a4), "+f"(a5), "+f"(a6), "+f"(a7), "+f"(a8)
        : "r"(b), "f"(w0), "f"(w1), "f"(w2), "f"(w3), "f"(w4), "f"(w5), "f"(w6), "f"(w7), "f"(w8));
}
__device__ __forceinline__ void padd9(uint32_t b, double& a0, double& a1, double& a2, double& a3, double& a4,
                                      double& a5, double& a6, double& a7, double& a8, double w0, double w1,
                                      double w2, double w3, double w4, double w5, double w6, double w7, double w8) {
    asm("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %9, 0;\n\t"
        "@p add.rn.f64 %0, %0, %10;\n\t@p add.rn.f64 %1, %1, %11;\n\t@p add.rn.f64 %2, %2, %12;\n\t"
        "@p add.rn.f64 %3, %3, %13;\n\t@p add.rn.f64 %4, %4, %14;\n\t@p add.rn.f64 %5, %5, %15;\n\t"
        "@p add.rn.f64 %6, %6, %16;\n\t@p add.rn.f64 %7, %7, %17;\n\t@p add.rn.f64 %8, %8, %18;\n\t}"
        : "+d"(a0), "+d"(a1), "+d"(a2), "+d"(a3), "+d"(a4), "+d"(a5), "+d"(a6), "+d"(a7), "+d"(a8)
        : "r"(b), "d"(w0), "d"(w1), "d"(w2), "d"(w3), "d"(w4), "d"(w5), "d"(w6), "d"(w7), "d"(w8));
}
__device__ __forceinline__ void padd5(uint32_t b, float& a0, float& a1, float& a2, float& a3, float& a4, float w0,
                                      float w1, float w2, float w3, float w4) {
    asm("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %5, 0;\n\t"
        "@p add.rn.f32 %0, %0, %6;\n\t@p add.rn.f32 %1, %1, %7;\n\t@p add.rn.f32 %2, %2, %8;\n\t"
        "@p add.rn.f32 %3, %3, %9;\n\t@p add.rn.f32 %4, %4, %10;\n\t}"
        : "+f"(a0), "+f"(a1), "+f"(a2), "+f"(a3), "+f"(a4)
        : "r"(b), "f"(w0), "f"(w1), "f"(w2), "f"(w3), "f"(w4));
}
__device__ __forceinline__ void padd5(uint32_t b, double& a0, double& a1, double& a2, double& a3, double& a4,
                                      double w0, double w1, double w2, double w3, double w4) {
    asm("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %5, 0;\n\t"
        "@p add.rn.f64 %0, %0, %6;\n\t@p add.rn.f64 %1, %1, %7;\n\t@p add.rn.f64 %2, %2, %8;\n\t"
        "@p add.rn.f64 %3, %3, %9;\n\t@p add.rn.f64 %4, %4, %10;\n\t}"
        : "+d"(a0), "+d"(a1), "+d"(a2), "+d"(a3), "+d"(a4)
        : "r"(b), "d"(w0), "d"(w1), "d"(w2), "d"(w3), "d"(w4));
}

template <typename real> struct Quad;
template <> struct Quad<float> {
    float x, y, z, w;
    __device__ __forceinline__ static Quad load(const float* p) {
        const float4 v = *reinterpret_cast<const float4*>(p);
        return {v.x, v.y, v.z, v.w};
    }
};
template <> struct Quad<double> {
    double x, y, z, w;
    __device__ __forceinline__ static Quad load(const double* p) {
        const double2 u = reinterpret_cast<const double2*>(p)[0];
        const double2 v = reinterpret_cast<const double2*>(p)[1];
        return {u.x, u.y, v.x, v.y};
    }
};

template <typename real>
struct GeoArgs {
    Dims D;
    const int32_t* phi;
    const uint8_t* mask;
    const real* table;  // W^dz planes of W*W taps x 12 reals
    int ntx, nty, ntz;
    int nl_cap;         // labels per bitmap batch at most (tests force small batches)
    real inv_dx, inv_dx2, dx, kappa_limit;
    real *nx, *ny, *nz, *kappa;
    int32_t* phi_comp;
    StepScalars* s;
};

// TD divides the rows of a 2-D tile (1: 1024 cells, 2: 512, 4: 256); smaller
// tiles give small grids more CTAs (chosen per grid, gpk_grid_set_tile_rows)
template <int R, bool IS3D, int TD = 1>
struct GeoShape {
    static constexpr int W = 2 * R + 1;
    static constexpr int TX = 32 - 2 * R;  // halo row = 32 cells = one bitmap word
    static constexpr int TY = IS3D ? 8 : 1024 / TX / TD;
    static constexpr int TZ = IS3D ? 1024 / (TX * 8) : 1;
    static constexpr int HY = TY + 2 * R, HZ = IS3D ? TZ + 2 * R : 1;
    static constexpr int NROW = HZ * HY;
    static constexpr int NROWP = NROW | 1;  // odd pitch: one row's words for several labels hit distinct banks
    static constexpr int NCELL = TX * TY * TZ;
    static constexpr int CX = TX + 2, CY = TY + 2, CZ = IS3D ? TZ + 2 : 1;  // tile labels with a 1-cell halo
    static constexpr int NCORE = CX * CY * CZ;
    static constexpr int PLANE = W * W * 12;  // reals per table plane
    static constexpr int NPLANES = IS3D ? W : 1;
    static constexpr int BM_WORDS = 6912;
    static constexpr int NLB = BM_WORDS / NROWP;  // labels per bitmap batch
    static_assert(NCELL <= 1024 && NLB >= 1, "tile shape");
};

template <typename real, int R, bool IS3D, int TD>
constexpr size_t geo_smem_bytes() {
    typedef GeoShape<R, IS3D, TD> S;
    // table planes | bitmaps | core labels | distinct labels | cells | cell label
    // index | batch cells | 2 mbarriers
    return (size_t)2 * S::PLANE * sizeof(real) + (size_t)S::BM_WORDS * 4 + (size_t)S::NCORE * 4 + (size_t)S::NCELL * 4 +
           (size_t)S::NCELL * 2 * 3 + 64;
}

// One row of W taps (fixed dz, dy) for SLOTS cells; wd[s] holds bit j set
// when tap x-offset j - R of cell s matches its label.
//   x factor zero (|dx| >= R-1): only Ix, Ixx, Ixy, Ixz live   (quad A)
//   y factor zero (ZY0):         only Iy, Iyy, Ixy, Iyz live   (quad B)
//   z factor zero (ZZ0):         only Iz, Izz, Ixz, Iyz live   (quad C)
// Components: 0 Ix, 1 Iy, 2 Ixx, 3 Iyy, 4 Ixy, 5 Iz, 6 Izz, 7 Ixz, 8 Iyz.
template <typename real, int R, bool IS3D, int SLOTS, bool ZY0, bool ZZ0>
__device__ __forceinline__ void geo_row(const real* __restrict__ trow, const uint32_t wd[SLOTS], real acc[SLOTS][9]) {
    constexpr int W = 2 * R + 1;
#pragma unroll
    for (int j = 0; j < W; ++j) {
        const bool zx0 = j <= 1 || j >= W - 2;  // compile-time after unrolling
        const real* t = trow + j * 12;
        const uint32_t bit = 1u << j;
        if (!IS3D) {
            if (!zx0 && !ZY0) {
                const Quad<real> A = Quad<real>::load(t), B = Quad<real>::load(t + 4);
#pragma unroll
                for (int s = 0; s < SLOTS; ++s)
                    padd5(wd[s] & bit, acc[s][0], acc[s][2], acc[s][4], acc[s][1], acc[s][3], A.x, A.y, A.z, B.x,
                          B.y);
            } else if (zx0 && !ZY0) {
                const Quad<real> A = Quad<real>::load(t);
#pragma unroll
                for (int s = 0; s < SLOTS; ++s) padd(wd[s] & bit, acc[s][0], acc[s][2], acc[s][4], A.x, A.y, A.z);
            } else if (!zx0 && ZY0) {
                const Quad<real> B = Quad<real>::load(t + 4);
#pragma unroll
                for (int s = 0; s < SLOTS; ++s) padd(wd[s] & bit, acc[s][1], acc[s][3], acc[s][4], B.x, B.y, B.z);
            } else {
                const real wxy = t[2];
#pragma unroll
                for (int s = 0; s < SLOTS; ++s) padd(wd[s] & bit, acc[s][4], wxy);
            }
            continue;
        }
        if (!zx0 && !ZY0 && !ZZ0) {
            const Quad<real> A = Quad<real>::load(t), B = Quad<real>::load(t + 4), C = Quad<real>::load(t + 8);
#pragma unroll
            for (int s = 0; s < SLOTS; ++s)
                padd9(wd[s] & bit, acc[s][0], acc[s][2], acc[s][4], acc[s][7], acc[s][1], acc[s][3], acc[s][8],
                      acc[s][5], acc[s][6], A.x, A.y, A.z, A.w, B.x, B.y, B.w, C.x, C.y);
        } else if (zx0 && !ZY0 && !ZZ0) {
            const Quad<real> A = Quad<real>::load(t);
#pragma unroll
            for (int s = 0; s < SLOTS; ++s)
                padd(wd[s] & bit, acc[s][0], acc[s][2], acc[s][4], acc[s][7], A.x, A.y, A.z, A.w);
        } else if (!zx0 && ZY0 && !ZZ0) {
            const Quad<real> B = Quad<real>::load(t + 4);
#pragma unroll
            for (int s = 0; s < SLOTS; ++s)
                padd(wd[s] & bit, acc[s][1], acc[s][3], acc[s][4], acc[s][8], B.x, B.y, B.z, B.w);
        } else if (!zx0 && !ZY0 && ZZ0) {
            const Quad<real> C = Quad<real>::load(t + 8);
#pragma unroll
            for (int s = 0; s < SLOTS; ++s)
                padd(wd[s] & bit, acc[s][5], acc[s][6], acc[s][7], acc[s][8], C.x, C.y, C.z, C.w);
        } else if (zx0 && ZY0 && !ZZ0) {
            const real wxy = t[2];
#pragma unroll
            for (int s = 0; s < SLOTS; ++s) padd(wd[s] & bit, acc[s][4], wxy);
        } else if (zx0 && !ZY0 && ZZ0) {
            const real wxz = t[3];
#pragma unroll
            for (int s = 0; s < SLOTS; ++s) padd(wd[s] & bit, acc[s][7], wxz);
        } else if (!zx0 && ZY0 && ZZ0) {
            const real wyz = t[7];
#pragma unroll
            for (int s = 0; s < SLOTS; ++s) padd(wd[s] & bit, acc[s][8], wyz);
        }
    }
}

// The tap planes of one label batch.  gp0 = planes streamed before this
// batch (buffer of global plane g: g & 1, its phase parity: (g >> 1) & 1);
// gp_total = planes of all batches (the last plane prefetches nothing).
template <typename real, int R, bool IS3D, int TD, int SLOTS>
__device__ __forceinline__ void geo_accumulate(const GeoArgs<real>& a, const uint32_t* __restrict__ bm,
                                               const real* __restrict__ tab0, const real* __restrict__ tab1,
                                               uint64_t* bars, int gp0, int gp_total, int nact, int tid,
                                               real acc[SLOTS][9], const int bmrow[SLOTS], const int lx[SLOTS],
                                               const uint32_t vmask[SLOTS], bool& ok) {
    typedef GeoShape<R, IS3D, TD> S;
    constexpr int W = S::W;
#pragma unroll
    for (int s = 0; s < SLOTS; ++s)
#pragma unroll
        for (int k = 0; k < 9; ++k) acc[s][k] = (real)0;
    for (int p = 0; p < S::NPLANES; ++p) {
        const int g = gp0 + p;
        const real* tab = (g & 1) ? tab1 : tab0;
        if (!mbar_wait(&bars[g & 1], (uint32_t)((g >> 1) & 1))) {
            ok = false;
            atomicCAS(&a.s->error, 0u, (unsigned)GPK_ERR_TIMEOUT);
        }
        if (tid == 0 && g + 1 < gp_total) {
            // the other buffer was last read in plane g-1, which every thread
            // finished before the barrier at the end of that plane
            fence_proxy_async();
            real* dst = ((g + 1) & 1) ? (real*)tab1 : (real*)tab0;
            const int pn = (g + 1) % S::NPLANES;
            mbar_expect_tx(&bars[(g + 1) & 1], S::PLANE * sizeof(real));
            bulk_g2s(dst, a.table + (size_t)pn * S::PLANE, S::PLANE * sizeof(real), &bars[(g + 1) & 1]);
        }
        if (ok && tid < nact) {
            // rows whose y or z Gaussian factor is exactly zero run
            // specialised bodies without the corresponding products
            const bool zz0 = IS3D && (p <= 1 || p >= W - 2);
#pragma unroll 1
            for (int dy = 0; dy < W; ++dy) {
                uint32_t wd[SLOTS];
                uint32_t any = 0;
#pragma unroll
                for (int s = 0; s < SLOTS; ++s) {
                    wd[s] = (bm[bmrow[s] + p * S::HY + dy] >> lx[s]) & vmask[s];
                    any |= wd[s];
                }
                if (!any) continue;
                const real* trow = tab + dy * W * 12;
                const bool yy0 = dy <= 1 || dy >= W - 2;
                if (zz0) {
                    if (yy0) geo_row<real, R, IS3D, SLOTS, true, true>(trow, wd, acc);
                    else geo_row<real, R, IS3D, SLOTS, false, true>(trow, wd, acc);
                } else {
                    if (yy0) geo_row<real, R, IS3D, SLOTS, true, false>(trow, wd, acc);
                    else geo_row<real, R, IS3D, SLOTS, false, false>(trow, wd, acc);
                }
            }
        }
        __syncthreads();
    }
}

template <typename real>
__device__ __forceinline__ void geo_competitor(int32_t* __restrict__ phi_comp, int i, real nxv, real nyv, real nzv,
                                               const int32_t* __restrict__ lab, int cbase, int pitch, int rows,
                                               bool is3d);

template <typename real>
__device__ __forceinline__ void geo_finish(const GeoArgs<real>& a, int i, const real* acc, const int32_t* __restrict__ lab,
                                           int cbase, int pitch, int rows, bool is3d) {
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
    geo_competitor<real>(a.phi_comp, i, nxv, nyv, nzv, lab, cbase, pitch, rows, is3d);
}

// competitor choice (src/gpk_geometry.cpp:154-182) from the staged labels
template <typename real>
__device__ __forceinline__ void geo_competitor(int32_t* __restrict__ phi_comp, int i, real nxv, real nyv, real nzv,
                                               const int32_t* __restrict__ lab, int cbase, int pitch, int rows,
                                               bool is3d) {
    const int32_t pi = lab[cbase];
    const int plane = rows * pitch;
    const int fo[6] = {-1, +1, -pitch, +pitch, -plane, +plane};
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
                    support += lab[cbase + dz * plane + dy * pitch + dxs] == q;
                }
        if (support > best_support || (support == best_support && score[k] > best_score)) {
            best = k; best_support = support; best_score = score[k];
        }
    }
    phi_comp[i] = (best >= 0) ? lab[cbase + fo[best]] : pi;
}

// Fewest cells per thread; with one cell per thread the three table loads of
// a tap would be shared by a single cell's additions.
constexpr int GEO_MIN_SLOTS = 2;

// three CTAs per SM in float (80 registers); two in double, whose 36
// accumulators of a 4-cell thread take 72 registers
template <typename real, int R, bool IS3D, int TD>
__global__ void __launch_bounds__(256, sizeof(real) == 4 ? 3 : 2) k_geometry_tiled(GeoArgs<real> a) {
    typedef GeoShape<R, IS3D, TD> S;
    extern __shared__ __align__(128) unsigned char smem[];
    real* tab0 = reinterpret_cast<real*>(smem);
    real* tab1 = tab0 + S::PLANE;
    uint32_t* bm = reinterpret_cast<uint32_t*>(tab1 + S::PLANE);
    int32_t* core = reinterpret_cast<int32_t*>(bm + S::BM_WORDS);
    int32_t* dl = core + S::NCORE;                      // distinct labels of the tile's interface cells
    int16_t* cells = reinterpret_cast<int16_t*>(dl + S::NCELL);
    uint16_t* cli = reinterpret_cast<uint16_t*>(cells + S::NCELL);  // index into dl per cell
    int16_t* bcell = reinterpret_cast<int16_t*>(cli + S::NCELL);    // cells of the current batch
    uint64_t* bars = reinterpret_cast<uint64_t*>((reinterpret_cast<uintptr_t>(bcell + S::NCELL) + 15) & ~(uintptr_t)15);
    int32_t* cand = reinterpret_cast<int32_t*>(bm);      // label candidates, before the first bitmap
    __shared__ int s_count, s_ncand, s_nl;
    typedef cub::BlockScan<int, 256> BS;
    __shared__ typename BS::TempStorage scan;
    constexpr int PER = (S::NCELL + 255) / 256;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const Dims D = a.D;

    const int t = blockIdx.x;
    const int tx = t % a.ntx, ty = (t / a.ntx) % a.nty, tz = t / (a.ntx * a.nty);
    const int x0 = tx * S::TX, y0 = ty * S::TY, z0 = tz * S::TZ;

    // 1. interface cells of the tile, in flat order
    {
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
        if (tid == 0) {
            s_count = total;
            s_ncand = 0;
            s_nl = 0;
        }
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
    // tile labels with a periodic halo of one cell (competitor choice)
    for (int e = tid; e < S::NCORE; e += 256) {
        const int cx = e % S::CX, cy = (e / S::CX) % S::CY, cz = e / (S::CX * S::CY);
        const int x = wrap_any(x0 + cx - 1, D.Nx), y = wrap_any(y0 + cy - 1, D.Ny);
        const int z = IS3D ? wrap_any(z0 + cz - 1, D.Nz) : 0;
        core[e] = a.phi[D.idx(z, y, x)];
    }
    __syncthreads();

    // 2. distinct labels of the interface cells: one candidate per label and
    //    warp (match_any leaders), then the first occurrence of each candidate
    auto core_of = [&](int c) {
        const int lx = c % S::TX, ly = (c / S::TX) % S::TY, lz = c / (S::TX * S::TY);
        return ((IS3D ? lz + 1 : 0) * S::CY + ly + 1) * S::CX + lx + 1;
    };
    for (int k0 = 0; k0 < ncell; k0 += 256) {
        const int k = k0 + tid;
        const bool v = k < ncell;
        const unsigned am = __ballot_sync(0xffffffffu, v);
        if (v) {
            const int32_t lab = core[core_of(cells[k])];
            const unsigned grp = __match_any_sync(am, lab);
            if (lane == __ffs(grp) - 1) cand[atomicAdd(&s_ncand, 1)] = lab;
        }
    }
    __syncthreads();
    const int ncand = s_ncand;
    for (int e = tid; e < ncand; e += 256) {
        const int32_t lab = cand[e];
        bool first = true;
        for (int j = 0; j < e && first; ++j) first = cand[j] != lab;
        if (first) dl[atomicAdd(&s_nl, 1)] = lab;
    }
    __syncthreads();
    const int nl = s_nl;
    for (int k = tid; k < ncell; k += 256) {
        const int32_t lab = core[core_of(cells[k])];
        int li = 0;
        while (li < nl - 1 && dl[li] != lab) ++li;  // every cell label is listed
        cli[k] = (uint16_t)li;
    }
    const int nlb = a.nl_cap < S::NLB ? a.nl_cap : S::NLB;
    const int nbatch = (nl + nlb - 1) / nlb;
    const int gp_total = nbatch * S::NPLANES;
    bool ok = true;

    for (int b = 0; b < nbatch; ++b) {
        const int lb0 = b * nlb;
        const int nb = nl - lb0 < nlb ? nl - lb0 : nlb;
        __syncthreads();  // bitmaps, candidates and batch cells of the previous pass are free

        // 3. one word per halo row and label of the batch; a warp takes two
        //    rows at a time, their label loads issued together
        for (int r0 = warp; r0 < S::NROW; r0 += 16) {
            int32_t gv[2];
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const int r = r0 + 8 * u;
                const int hz = r / S::HY, hy = r % S::HY;
                const int x = wrap_any(x0 - R + lane, D.Nx), y = wrap_any(y0 + hy - R, D.Ny);
                const int z = IS3D ? wrap_any(z0 + hz - R, D.Nz) : 0;
                gv[u] = r < S::NROW ? a.phi[D.idx(z, y, x)] : -1;
            }
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const int r = r0 + 8 * u;
                if (r >= S::NROW) break;
                for (int L0 = 0; L0 < nb; L0 += 32) {
                    const int cnt = nb - L0 < 32 ? nb - L0 : 32;
                    uint32_t mine = 0;
                    for (int L = 0; L < cnt; ++L) {
                        const uint32_t bits = __ballot_sync(0xffffffffu, gv[u] == dl[lb0 + L0 + L]);
                        if (lane == L) mine = bits;
                    }
                    if (lane < cnt) bm[(L0 + lane) * S::NROWP + r] = mine;
                }
            }
        }
        // cells of the batch, grouped by label (flat order within a label), so
        // that a warp's cells share a label and skip the same empty rows
        int nbc = 0;
        {
            for (int L = lb0; L < lb0 + nb; ++L) {
                int flags[PER];
                int cnt = 0;
#pragma unroll
                for (int k = 0; k < PER; ++k) {
                    const int e = tid * PER + k;
                    flags[k] = e < ncell && (int)cli[e] == L;
                    cnt += flags[k];
                }
                int ex, total;
                BS(scan).ExclusiveSum(cnt, ex, total);
#pragma unroll
                for (int k = 0; k < PER; ++k)
                    if (flags[k]) bcell[nbc + ex++] = (int16_t)(tid * PER + k);
                nbc += total;
                __syncthreads();
            }
        }
        __syncthreads();

        // 4. each thread takes `slots` of the batch's cells: thread t < nact
        //    takes cells t, t + nact, ...; warps beyond nact leave their issue
        //    slots to the other resident CTAs
        int slots = (nbc + 255) / 256;
        if (slots < GEO_MIN_SLOTS) slots = GEO_MIN_SLOTS;
        const int nact = (nbc + slots - 1) / slots;
        int bmrow[4], lx[4], kc[4];
        uint32_t vmask[4];
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const int kk = tid + nact * s;
            const bool valid = s < slots && tid < nact && kk < nbc;
            const int k = valid ? bcell[kk] : bcell[0];
            const int c = cells[k];
            const int cx = c % S::TX, cy = (c / S::TX) % S::TY, cz = c / (S::TX * S::TY);
            // bitmap word of halo row (cz + dz + R, cy + dy + R): bmrow + (dz+R)*HY + (dy+R)
            bmrow[s] = ((int)cli[k] - lb0) * S::NROWP + (IS3D ? cz : 0) * S::HY + cy;
            lx[s] = cx;
            kc[s] = valid ? c : -1;
            vmask[s] = valid ? 0xffffffffu : 0u;
        }
        real acc[4][9];
        const int gp0 = b * S::NPLANES;
        switch (slots) {
        case 2: geo_accumulate<real, R, IS3D, TD, 2>(a, bm, tab0, tab1, bars, gp0, gp_total, nact, tid, acc, bmrow, lx, vmask, ok); break;
        case 3: geo_accumulate<real, R, IS3D, TD, 3>(a, bm, tab0, tab1, bars, gp0, gp_total, nact, tid, acc, bmrow, lx, vmask, ok); break;
        default: geo_accumulate<real, R, IS3D, TD, 4>(a, bm, tab0, tab1, bars, gp0, gp_total, nact, tid, acc, bmrow, lx, vmask, ok); break;
        }
        if (ok) {
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                if (kc[s] < 0) continue;
                const int c = kc[s];
                const int cx = c % S::TX, cy = (c / S::TX) % S::TY, cz = c / (S::TX * S::TY);
                const int i = D.idx(z0 + cz, y0 + cy, x0 + cx);
                geo_finish<real>(a, i, acc[s], core, core_of(c), S::CX, S::CY, IS3D);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Separable tiles (FP64 throughput mode)
// ---------------------------------------------------------------------------
// The reference's separable geometry (src/gpk_geometry.cpp:185-347: Gaussian
// smoothing of one label's indicator, then fourth-order differences at that
// label's interface cells) evaluated per tile instead of per label over the
// whole grid.  The direct stencil's tap products are exactly these filters
// composed (w1 = d1 * G, w2 = d2 * G), so both give the same fields up to
// rounding; in FP64 the two agree far below 1e-10.  Per tile and label:
//   x: a 2K+1-tap window of a halo row is 2K+1 bits of its bitmap word; its
//      smoothed value is two or three table lookups (7-bit chunks);
//   y: each thread owns a column (x, y) of the smoothed region and sums the
//      2K+1 x-values above and below it for every halo plane, in registers;
//   z: the same column's planes give the smoothed indicator S on the tile
//      plus two cells each side, stored in shared memory;
//   then the differences at the label's interface cells.
struct SepArgs {
    Dims D;
    const int32_t* phi;
    const uint8_t* mask;
    int ntx, nty;
    double g[17];  // Gaussian taps (radius K = R - 2 <= 8)
    double dx, idx12, idx12_sq, idx144_sq, kappa_limit;
    double *nx, *ny, *nz, *kappa;
    int32_t* phi_comp;
};

template <int R, bool IS3D>
struct SepShape {
    typedef GeoShape<R, IS3D, 1> G;
    static constexpr int K = R - 2, NT = 2 * K + 1, NCH = (NT + 6) / 7;
    static constexpr int SX = G::TX + 4, SY = G::TY + 4, SZ = IS3D ? G::TZ + 4 : 1;
    static constexpr int NS = SX * SY * SZ;
    static constexpr int NY = IS3D ? SX * SY * G::HZ : 0;  // y-smoothed values of every halo plane
    static constexpr int NLB = 4;                            // labels per bitmap batch
    // the bitmaps' words first hold up to one label candidate per interface cell
    static constexpr int BM_WORDS = NLB * G::NROWP > G::NCELL ? NLB * G::NROWP : G::NCELL;
};

template <int R, bool IS3D>
constexpr size_t sep_smem_bytes() {
    typedef GeoShape<R, IS3D, 1> S;
    typedef SepShape<R, IS3D> P;
    // smoothed indicator | y-smoothed planes | chunk tables | bitmaps | core labels | distinct labels |
    // cells | cell label index
    return (size_t)(P::NS + P::NY) * 8 + (size_t)P::NCH * 128 * 8 + (size_t)P::BM_WORDS * 4 +
           (size_t)S::NCORE * 4 + (size_t)S::NCELL * 4 + (size_t)S::NCELL * 2 * 2;
}

template <int R, bool IS3D>
__global__ void __launch_bounds__(256) k_geometry_sep_tiles(SepArgs a) {
    typedef GeoShape<R, IS3D, 1> S;
    typedef SepShape<R, IS3D> P;
    extern __shared__ __align__(128) unsigned char smem[];
    double* Sm = reinterpret_cast<double*>(smem);  // P::NS
    double* Ym = Sm + P::NS;                        // P::NY
    double* lut = Ym + P::NY;                       // P::NCH x 128
    uint32_t* bm = reinterpret_cast<uint32_t*>(lut + P::NCH * 128);
    int32_t* core = reinterpret_cast<int32_t*>(bm + P::BM_WORDS);
    int32_t* dl = core + S::NCORE;
    int16_t* cells = reinterpret_cast<int16_t*>(dl + S::NCELL);
    uint16_t* cli = reinterpret_cast<uint16_t*>(cells + S::NCELL);
    int32_t* cand = reinterpret_cast<int32_t*>(bm);  // label candidates, before the first bitmap
    __shared__ int s_count, s_ncand, s_nl;
    __shared__ int sbox[6 * P::NLB];  // per label of the batch: min x, y, z, max x, y, z of its cells
    typedef cub::BlockScan<int, 256> BS;
    __shared__ typename BS::TempStorage scan;
    constexpr int PER = (S::NCELL + 255) / 256;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const Dims D = a.D;
    const int t = blockIdx.x;
    const int tx = t % a.ntx, ty = (t / a.ntx) % a.nty, tz = t / (a.ntx * a.nty);
    const int x0 = tx * S::TX, y0 = ty * S::TY, z0 = tz * S::TZ;

    // interface cells of the tile, in flat order
    {
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
        if (tid == 0) { s_count = total; s_ncand = 0; s_nl = 0; }
    }
    __syncthreads();
    const int ncell = s_count;
    if (ncell == 0) return;
    // tile labels with a one-cell periodic halo (competitor choice); chunk tables
    for (int e = tid; e < S::NCORE; e += 256) {
        const int cx = e % S::CX, cy = (e / S::CX) % S::CY, cz = e / (S::CX * S::CY);
        const int x = wrap_any(x0 + cx - 1, D.Nx), y = wrap_any(y0 + cy - 1, D.Ny);
        const int z = IS3D ? wrap_any(z0 + cz - 1, D.Nz) : 0;
        core[e] = a.phi[D.idx(z, y, x)];
    }
    for (int e = tid; e < P::NCH * 128; e += 256) {
        const int ch = e >> 7, pat = e & 127;
        double v = 0.0;
        for (int j = 0; j < 7; ++j)
            if ((pat >> j) & 1) {
                const int tap = 7 * ch + j;
                if (tap < P::NT) v += a.g[tap];
            }
        lut[e] = v;
    }
    __syncthreads();
    // distinct labels of the interface cells
    auto core_of = [&](int c) {
        const int lx = c % S::TX, ly = (c / S::TX) % S::TY, lz = c / (S::TX * S::TY);
        return ((IS3D ? lz + 1 : 0) * S::CY + ly + 1) * S::CX + lx + 1;
    };
    for (int k0 = 0; k0 < ncell; k0 += 256) {
        const int k = k0 + tid;
        const bool v = k < ncell;
        const unsigned am = __ballot_sync(0xffffffffu, v);
        if (v) {
            const int32_t lab = core[core_of(cells[k])];
            const unsigned grp = __match_any_sync(am, lab);
            if (lane == __ffs(grp) - 1) cand[atomicAdd(&s_ncand, 1)] = lab;
        }
    }
    __syncthreads();
    const int ncand = s_ncand;
    for (int e = tid; e < ncand; e += 256) {
        const int32_t lab = cand[e];
        bool first = true;
        for (int j = 0; j < e && first; ++j) first = cand[j] != lab;
        if (first) dl[atomicAdd(&s_nl, 1)] = lab;
    }
    __syncthreads();
    const int nl = s_nl;
    for (int k = tid; k < ncell; k += 256) {
        const int32_t lab = core[core_of(cells[k])];
        int li = 0;
        while (li < nl - 1 && dl[li] != lab) ++li;
        cli[k] = (uint16_t)li;
    }
    const double dx = a.dx;
    for (int lb0 = 0; lb0 < nl; lb0 += P::NLB) {
        const int nb = nl - lb0 < P::NLB ? nl - lb0 : P::NLB;
        __syncthreads();  // the previous batch's bitmaps and smoothed values are free
        // a warp takes four halo rows at a time, their label loads issued together
        const int xw = wrap_any(x0 - R + lane, D.Nx);
        for (int r0 = warp; r0 < S::NROW; r0 += 32) {
            int32_t gv[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int r = r0 + 8 * u;
                const int hz = r / S::HY, hy = r % S::HY;
                const int y = wrap_any(y0 + hy - R, D.Ny);
                const int z = IS3D ? wrap_any(z0 + hz - R, D.Nz) : 0;
                gv[u] = r < S::NROW ? a.phi[D.idx(z, y, xw)] : -1;
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int r = r0 + 8 * u;
                if (r >= S::NROW) break;
                for (int L = 0; L < nb; ++L) {
                    const uint32_t bits = __ballot_sync(0xffffffffu, gv[u] == dl[lb0 + L]);
                    if (lane == 0) bm[L * S::NROWP + r] = bits;
                }
            }
        }
        // each label's interface cells span a box of the tile; its smoothed
        // values are needed there plus two cells each side (the differences)
        if (tid < 6 * P::NLB) sbox[tid] = (tid % 6) < 3 ? 1 << 20 : -1;
        __syncthreads();
        for (int k = tid; k < ncell; k += 256) {
            const int L = (int)cli[k] - lb0;
            if (L < 0 || L >= nb) continue;
            const int c = cells[k];
            atomicMin(&sbox[6 * L + 0], c % S::TX);
            atomicMin(&sbox[6 * L + 1], (c / S::TX) % S::TY);
            atomicMin(&sbox[6 * L + 2], c / (S::TX * S::TY));
            atomicMax(&sbox[6 * L + 3], c % S::TX);
            atomicMax(&sbox[6 * L + 4], (c / S::TX) % S::TY);
            atomicMax(&sbox[6 * L + 5], c / (S::TX * S::TY));
        }
        for (int L = 0; L < nb; ++L) {
            __syncthreads();  // bitmaps and boxes written / the previous label's S read
            const uint32_t* bml = bm + L * S::NROWP;
            // the label's box in smoothed-value coordinates: x in [bx, bx + nsx)
            const int bx = sbox[6 * L + 0], by = sbox[6 * L + 1], bz = IS3D ? sbox[6 * L + 2] : 0;
            const int nsx = sbox[6 * L + 3] - bx + 5, nsy = sbox[6 * L + 4] - by + 5;
            const int nhz = IS3D ? sbox[6 * L + 5] - bz + 5 + 2 * P::K : 1;
            // smoothed x value of the window starting at bit xs of halo row `row`
            auto xval = [&](int row, int xs) -> double {
                const uint32_t w = bml[row] >> xs;
                double v = lut[w & 0x7Fu];
                if (P::NCH > 1) v += lut[128 + ((w >> 7) & 0x7Fu)];
                if (P::NCH > 2) v += lut[256 + ((w >> 14) & 0x7Fu)];
                return v;
            };
            if (IS3D) {
                // a strip (x, halo plane): its x values down all halo rows, then
                // the y sums of the tile's rows plus two each side
                // (the strips and columns outside the label's box are skipped;
                // their stale values are never read)
                for (int st = tid; st < nsx * nhz; st += 256) {
                    const int xs = bx + st % nsx, hz = bz + st / nsx;
                    double X[S::HY];
#pragma unroll
                    for (int r = 0; r < S::HY; ++r) X[r] = xval(hz * S::HY + r, xs);
#pragma unroll
                    for (int ys = 0; ys < P::SY; ++ys) {
                        double acc = 0.0;
#pragma unroll
                        for (int j = 0; j < P::NT; ++j) acc = __fma_rn(a.g[j], X[ys + j], acc);
                        Ym[(hz * P::SY + ys) * P::SX + xs] = acc;
                    }
                }
                __syncthreads();
                // a column (x, y): the z sums from its y-smoothed planes
                for (int cc = tid; cc < nsx * nsy; cc += 256) {
                    const int col = (by + cc / nsx) * P::SX + bx + cc % nsx;
                    double Y[S::HZ];
#pragma unroll
                    for (int hz = 0; hz < S::HZ; ++hz) Y[hz] = Ym[hz * P::SX * P::SY + col];
#pragma unroll
                    for (int zs = 0; zs < P::SZ; ++zs) {
                        double acc = 0.0;
#pragma unroll
                        for (int j = 0; j < P::NT; ++j) acc = __fma_rn(a.g[j], Y[zs + j], acc);
                        Sm[zs * P::SX * P::SY + col] = acc;
                    }
                }
            } else {
                for (int pt = tid; pt < nsx * nsy; pt += 256) {
                    const int xs = bx + pt % nsx, ys = by + pt / nsx;
                    double acc = 0.0;
#pragma unroll
                    for (int j = 0; j < P::NT; ++j) acc = __fma_rn(a.g[j], xval(ys + j, xs), acc);
                    Sm[ys * P::SX + xs] = acc;
                }
            }
            __syncthreads();
            // fourth-order differences at this label's interface cells
            for (int k = tid; k < ncell; k += 256) {
                if ((int)cli[k] != lb0 + L) continue;
                const int c = cells[k];
                const int lx = c % S::TX, ly = (c / S::TX) % S::TY, lz = c / (S::TX * S::TY);
                const int PY = P::SX, PZ = P::SX * P::SY;
                const int c0 = ((IS3D ? lz + 2 : 0) * P::SY + ly + 2) * P::SX + lx + 2;
                const double I0 = Sm[c0];
                const double Ix = (Sm[c0 - 2] - 8.0 * Sm[c0 - 1] + 8.0 * Sm[c0 + 1] - Sm[c0 + 2]) * a.idx12;
                const double Iy = (Sm[c0 - 2 * PY] - 8.0 * Sm[c0 - PY] + 8.0 * Sm[c0 + PY] - Sm[c0 + 2 * PY]) * a.idx12;
                const double Iz = IS3D ? (Sm[c0 - 2 * PZ] - 8.0 * Sm[c0 - PZ] + 8.0 * Sm[c0 + PZ] - Sm[c0 + 2 * PZ]) *
                                             a.idx12
                                       : 0.0;
                const double Ixx =
                    (-Sm[c0 + 2] + 16.0 * Sm[c0 + 1] - 30.0 * I0 + 16.0 * Sm[c0 - 1] - Sm[c0 - 2]) * a.idx12_sq;
                const double Iyy = (-Sm[c0 + 2 * PY] + 16.0 * Sm[c0 + PY] - 30.0 * I0 + 16.0 * Sm[c0 - PY] -
                                    Sm[c0 - 2 * PY]) *
                                   a.idx12_sq;
                const double Izz = IS3D ? (-Sm[c0 + 2 * PZ] + 16.0 * Sm[c0 + PZ] - 30.0 * I0 + 16.0 * Sm[c0 - PZ] -
                                           Sm[c0 - 2 * PZ]) *
                                              a.idx12_sq
                                        : 0.0;
                const int off[4] = {-2, -1, 1, 2};
                const double dc[4] = {1.0, -8.0, 8.0, -1.0};
                double sxy = 0.0, sxz = 0.0, syz = 0.0;
#pragma unroll
                for (int p = 0; p < 4; ++p)
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const double w = dc[p] * dc[q];
                        sxy += w * Sm[c0 + off[q] * PY + off[p]];
                        if (IS3D) {
                            sxz += w * Sm[c0 + off[q] * PZ + off[p]];
                            syz += w * Sm[c0 + off[q] * PZ + off[p] * PY];
                        }
                    }
                const double Ixy = sxy * a.idx144_sq, Ixz = IS3D ? sxz * a.idx144_sq : 0.0;
                const double Iyz = IS3D ? syz * a.idx144_sq : 0.0;
                const double grad_sq = Ix * Ix + Iy * Iy + Iz * Iz;
                double nxv = 0.0, nyv = 0.0, nzv = 0.0;
                const int i = D.idx(z0 + lz, y0 + ly, x0 + lx);
                if (grad_sq * dx * dx > 1e-8) {
                    const double inv_grad = 1.0 / sqrt(grad_sq);
                    nxv = -Ix * inv_grad;
                    nyv = -Iy * inv_grad;
                    nzv = -Iz * inv_grad;
                    const double trace_H = Ixx + Iyy + Izz;
                    const double gHg =
                        Ix * Ix * Ixx + Iy * Iy * Iyy + Iz * Iz * Izz + 2.0 * (Ix * Iy * Ixy + Ix * Iz * Ixz + Iy * Iz * Iyz);
                    double kap = (gHg - grad_sq * trace_H) / (grad_sq * sqrt(grad_sq));
                    if (fabs(kap * dx) < 1e-6) kap = 0.0;
                    a.nx[i] = nxv; a.ny[i] = nyv; a.nz[i] = nzv;
                    a.kappa[i] = dclamp(kap, -a.kappa_limit, a.kappa_limit);
                }
                geo_competitor<double>(a.phi_comp, i, nxv, nyv, nzv, core, core_of(c), S::CX, S::CY, IS3D);
            }
        }
    }
}

template <int R, bool IS3D>
static int launch_sep_tiles(gpk_grid* G, SepArgs a) {
    typedef GeoShape<R, IS3D, 1> S;
    a.ntx = (G->d.Nx + S::TX - 1) / S::TX;
    a.nty = (G->d.Ny + S::TY - 1) / S::TY;
    const int ntz = (G->d.Nz + S::TZ - 1) / S::TZ;
    const size_t smem = sep_smem_bytes<R, IS3D>();
    // set once per process (thread-safe initialisation of a function-local static)
    static const cudaError_t attr_rc =
        cudaFuncSetAttribute(k_geometry_sep_tiles<R, IS3D>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    GPK_CUDA_TRY(attr_rc);
    k_geometry_sep_tiles<R, IS3D><<<a.ntx * a.nty * ntz, 256, smem, G->stream>>>(a);
    G->launches++;
    GPK_CUDA_TRY(cudaGetLastError());
    return GPK_OK;
}

template <typename real, int R, bool IS3D, int TD = 1>
static int launch_tiled(gpk_grid* G, const GeoArgs<real>& a0) {
    typedef GeoShape<R, IS3D, TD> S;
    GeoArgs<real> a = a0;
    a.ntx = (G->d.Nx + S::TX - 1) / S::TX;
    a.nty = (G->d.Ny + S::TY - 1) / S::TY;
    a.ntz = (G->d.Nz + S::TZ - 1) / S::TZ;
    const size_t smem = geo_smem_bytes<real, R, IS3D, TD>();
    // set once per process (thread-safe initialisation of a function-local static)
    static const cudaError_t attr_rc = cudaFuncSetAttribute(
        k_geometry_tiled<real, R, IS3D, TD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    GPK_CUDA_TRY(attr_rc);
    const int ntiles = a.ntx * a.nty * a.ntz;
    k_geometry_tiled<real, R, IS3D, TD><<<ntiles, 256, smem, G->stream>>>(a);
    G->launches++;
    GPK_CUDA_TRY(cudaGetLastError());
    return GPK_OK;
}

}  // namespace gpk_dev

using namespace gpk_dev;

// Tiled geometry for kernel radii 4..10 (Gaussian radius 2..8); returns -1
// for other radii (the caller then uses the per-cell kernel).
template <typename real>
int gpk_geometry_tiled(gpk_grid* G, int R, real inv_dx, real inv_dx2, real dx, real kappa_limit) {
    GeoArgs<real> a;
    a.D = G->d;
    a.phi = G->phi;
    a.mask = G->mask;
    a.table = (const real*)G->d_geom_table;
    a.nl_cap = G->geometry_kernel == 2 ? 1 : (1 << 30);
    a.inv_dx = inv_dx; a.inv_dx2 = inv_dx2; a.dx = dx; a.kappa_limit = kappa_limit;
    a.nx = (real*)G->f[GPK_FIELD_NX]; a.ny = (real*)G->f[GPK_FIELD_NY]; a.nz = (real*)G->f[GPK_FIELD_NZ];
    a.kappa = (real*)G->f[GPK_FIELD_KAPPA];
    a.phi_comp = G->phi_comp;
    a.s = G->scal;
    if (G->d.is3d()) {
        switch (R) {
        case 4: return launch_tiled<real, 4, true>(G, a);
        case 5: return launch_tiled<real, 5, true>(G, a);
        case 6: return launch_tiled<real, 6, true>(G, a);
        case 7: return launch_tiled<real, 7, true>(G, a);
        case 8: return launch_tiled<real, 8, true>(G, a);
        case 9: return launch_tiled<real, 9, true>(G, a);
        case 10: return launch_tiled<real, 10, true>(G, a);
        default: return -1;
        }
    }
    switch (R) {
    case 4: return launch_tiled<real, 4, false>(G, a);
    case 5: return launch_tiled<real, 5, false>(G, a);
    case 6: return launch_tiled<real, 6, false>(G, a);
    case 7: return launch_tiled<real, 7, false>(G, a);
    case 8:
        // the sweep's sigma 1.5: tile height per grid
        if (G->tile_rows_div == 4) return launch_tiled<real, 8, false, 4>(G, a);
        if (G->tile_rows_div == 2) return launch_tiled<real, 8, false, 2>(G, a);
        return launch_tiled<real, 8, false>(G, a);
    case 9: return launch_tiled<real, 9, false>(G, a);
    case 10: return launch_tiled<real, 10, false>(G, a);
    default: return -1;
    }
}

// Separable tiles (FP64 grids, kernel radii 4..10); -1 when they do not apply.
int gpk_geometry_sep_tiles(gpk_grid* G, int R, const double* gauss, int gauss_radius, double dx,
                           double kappa_limit) {
    if (G->precision != GPK_PREC_F64 || gauss_radius != R - 2 || R < 4 || R > 10) return -1;
    SepArgs a{};
    a.D = G->d;
    a.phi = G->phi;
    a.mask = G->mask;
    for (int j = 0; j < 2 * gauss_radius + 1; ++j) a.g[j] = gauss[j];
    a.dx = dx;
    a.idx12 = 1.0 / (12.0 * dx);
    const double idx_sq = 1.0 / (dx * dx);
    a.idx12_sq = idx_sq / 12.0;
    a.idx144_sq = idx_sq / 144.0;
    a.kappa_limit = kappa_limit;
    a.nx = (double*)G->f[GPK_FIELD_NX]; a.ny = (double*)G->f[GPK_FIELD_NY]; a.nz = (double*)G->f[GPK_FIELD_NZ];
    a.kappa = (double*)G->f[GPK_FIELD_KAPPA];
    a.phi_comp = G->phi_comp;
    if (G->d.is3d()) {
        switch (R) {
        case 4: return launch_sep_tiles<4, true>(G, a);
        case 5: return launch_sep_tiles<5, true>(G, a);
        case 6: return launch_sep_tiles<6, true>(G, a);
        case 7: return launch_sep_tiles<7, true>(G, a);
        case 8: return launch_sep_tiles<8, true>(G, a);
        case 9: return launch_sep_tiles<9, true>(G, a);
        default: return launch_sep_tiles<10, true>(G, a);
        }
    }
    switch (R) {
    case 4: return launch_sep_tiles<4, false>(G, a);
    case 5: return launch_sep_tiles<5, false>(G, a);
    case 6: return launch_sep_tiles<6, false>(G, a);
    case 7: return launch_sep_tiles<7, false>(G, a);
    case 8: return launch_sep_tiles<8, false>(G, a);
    case 9: return launch_sep_tiles<9, false>(G, a);
    default: return launch_sep_tiles<10, false>(G, a);
    }
}

template int gpk_geometry_tiled<float>(gpk_grid*, int, float, float, float, float);
template int gpk_geometry_tiled<double>(gpk_grid*, int, double, double, double, double);
