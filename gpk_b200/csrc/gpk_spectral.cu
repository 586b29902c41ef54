// gpk_spectral.cu — FP64 spectral micro-elasticity for a cubic solid (sm_100a).
//
// Restates `spectral_elasticity` of the reference's Al-Cu material module
// (scripts/run_alcu_gpk_microstructure.py:99-190).  One solve is
//
//   k_eigenstrain   eps*_j = sum_v eig[v][j] f_v (3 real fields)
//   cuFFT D2Z       3 transforms to half spectra (one batched plan)
//   k_green         per half-spectrum wave vector: cubic acoustic tensor
//                   A(k), b(k), the 3x3 SPD solve A x = b (LDL^T), u = -i x,
//                   the strain transform e(k) (free mean expansion at k = 0),
//                   its Hermitian part, and the equilibrium residual
//                   |k . C:(e - e*)|^2 and |b|^2 over the full spectrum,
//                   summed per block (fixed order: deterministic)
//   cuFFT Z2D       6 transforms back to real fields (one batched plan)
//   k_epilogue      strain = field / N; eps* recomputed from the fractions
//                   (not stored); stress, energy, driving, hydrostatic stress
//   k_residual_sum  one block sums the block partials in a fixed order
//
// Algorithmic bytes per cell and solve: eigenstrain 24 read + 24 written,
// forward transforms 24 + 24, green 24 + 48, inverse transforms 48 + 48,
// epilogue 48 + 24 read and 40 written: 376.  Every stage is HBM-bound; none
// is a contraction.
#include <cuda_runtime.h>
#include <cufft.h>

#include <string>

#include "../../include/gpk_spectral.h"
#include "gpk_grid.h"

namespace {

struct SpecConst {
    int e0, e1, e2;     // extents along the reference's axes (e2 = 1 in 2-D)
    int h0, h1, h2;     // half-spectrum extents (the last transformed axis halved)
    int hax;            // that axis (2 in 3-D, 1 in 2-D)
    long long N, Nh;    // cells, half-spectrum bins
    double v0, v1, v2;  // 1 / (n_a * dx), the fftfreq scale of each axis (0 beyond ndim)
    double c11, c12, c44;
    double eig[9];
};

#define SPEC_CUDA_TRY(expr)                                                            \
    do {                                                                               \
        cudaError_t _e = (expr);                                                       \
        if (_e != cudaSuccess) {                                                       \
            gpk_set_error(std::string(#expr " failed: ") + cudaGetErrorString(_e));    \
            return GPK_ERR_CUDA;                                                       \
        }                                                                              \
    } while (0)
#define SPEC_FFT_TRY(expr)                                                             \
    do {                                                                               \
        cufftResult _r = (expr);                                                       \
        if (_r != CUFFT_SUCCESS) {                                                     \
            gpk_set_error(std::string(#expr " failed: cufft status ") + std::to_string((int)_r)); \
            return GPK_ERR_CUDA;                                                       \
        }                                                                              \
    } while (0)

// wave number of FFT index i on an axis of n points: 2 pi * fftfreq(n, dx)[i]
__device__ __forceinline__ double wave_number(long long i, int n, double scale) {
    const long long m = (i <= (n - 1) / 2) ? i : i - n;
    return 6.283185307179586 * ((double)m * scale);
}

__global__ void k_eigenstrain(SpecConst c, const double* __restrict__ f, double* __restrict__ e0) {
    const long long N = c.N;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        const double f0 = f[i], f1 = f[N + i], f2 = f[2 * N + i];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            double e = c.eig[j] * f0;
            e = e + c.eig[3 + j] * f1;
            e = e + c.eig[6 + j] * f2;
            e0[j * N + i] = e;
        }
    }
}

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cscale(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
__device__ __forceinline__ double cabs2(double2 a) { return a.x * a.x + a.y * a.y; }
__device__ __forceinline__ double2 conj2(double2 a) { return make_double2(a.x, -a.y); }
// i * a
__device__ __forceinline__ double2 cmul_i(double2 a) { return make_double2(-a.y, a.x); }

template <int NT>
__device__ __forceinline__ void block_sum2(double& a, double& b, double* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) { sh[2 * w] = a; sh[2 * w + 1] = b; }
    __syncthreads();
    if (w == 0) {
        a = lane < NT / 32 ? sh[2 * lane] : 0.0;
        b = lane < NT / 32 ? sh[2 * lane + 1] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            b += __shfl_down_sync(0xffffffffu, b, o);
        }
    }
}

// The reference's strain transform at one wave vector (lines 123-153): the
// cubic acoustic tensor A, b = k.C:e*, an LDL^T solve of A x = b, u = -i x,
// e = sym(i k u), free mean normal expansion at k = 0.  Also |k . C:(e - e*)|^2
// and |b|^2, the terms of the equilibrium residual (lines 170-184).
__device__ __forceinline__ void strain_at(const SpecConst& c, double kx, double ky, double kz, double2 e0, double2 e1,
                                          double2 e2, double2 e[6], double& r2, double& b2) {
    const bool origin = kx == 0.0 && ky == 0.0 && kz == 0.0;
    const double c11 = c.c11, c12 = c.c12, c44 = c.c44, cs = c12 + c44;
    double a00 = c11 * kx * kx + c44 * (ky * ky + kz * kz);
    double a11 = c11 * ky * ky + c44 * (kx * kx + kz * kz);
    double a22 = c11 * kz * kz + c44 * (kx * kx + ky * ky);
    double a01 = cs * kx * ky, a02 = cs * kx * kz, a12 = cs * ky * kz;
    double2 b[3];
    b[0] = cscale(kx, cadd(cscale(c11, e0), cscale(c12, cadd(e1, e2))));
    b[1] = cscale(ky, cadd(cscale(c11, e1), cscale(c12, cadd(e0, e2))));
    b[2] = cscale(kz, cadd(cscale(c11, e2), cscale(c12, cadd(e0, e1))));
    if (origin) {
        a00 = a11 = a22 = 1.0;
        a01 = a02 = a12 = 0.0;
        b[0] = b[1] = b[2] = make_double2(0.0, 0.0);
    }
    // A = L D L^T (A is symmetric positive definite for a stable cubic solid)
    const double d0 = a00, l10 = a01 / d0, l20 = a02 / d0;
    const double d1 = a11 - l10 * a01;
    const double l21 = (a12 - l20 * a01) / d1;
    const double d2 = a22 - l20 * a02 - l21 * l21 * d1;
    const double2 y0 = b[0];
    const double2 y1 = csub(b[1], cscale(l10, y0));
    const double2 y2 = csub(csub(b[2], cscale(l20, y0)), cscale(l21, y1));
    const double2 x2 = cscale(1.0 / d2, y2);
    const double2 x1 = csub(cscale(1.0 / d1, y1), cscale(l21, x2));
    const double2 x0 = csub(csub(cscale(1.0 / d0, y0), cscale(l10, x1)), cscale(l20, x2));
    // u = -i x
    const double2 u0 = make_double2(x0.y, -x0.x), u1 = make_double2(x1.y, -x1.x), u2 = make_double2(x2.y, -x2.x);
    e[0] = cmul_i(cscale(kx, u0));
    e[1] = cmul_i(cscale(ky, u1));
    e[2] = cmul_i(cscale(kz, u2));
    e[3] = cscale(0.5, cmul_i(cadd(cscale(kx, u1), cscale(ky, u0))));
    e[4] = cscale(0.5, cmul_i(cadd(cscale(kx, u2), cscale(kz, u0))));
    e[5] = cscale(0.5, cmul_i(cadd(cscale(ky, u2), cscale(kz, u1))));
    if (origin) { e[0] = e0; e[1] = e1; e[2] = e2; }
    const double2 dh0 = csub(e[0], e0), dh1 = csub(e[1], e1), dh2 = csub(e[2], e2);
    const double2 s0 = cadd(cscale(c11, dh0), cscale(c12, cadd(dh1, dh2)));
    const double2 s1 = cadd(cscale(c11, dh1), cscale(c12, cadd(dh0, dh2)));
    const double2 s2 = cadd(cscale(c11, dh2), cscale(c12, cadd(dh0, dh1)));
    const double2 s3 = cscale(2.0 * c44, e[3]), s4 = cscale(2.0 * c44, e[4]), s5 = cscale(2.0 * c44, e[5]);
    const double2 rx = cadd(cadd(cscale(kx, s0), cscale(ky, s3)), cscale(kz, s4));
    const double2 ry = cadd(cadd(cscale(kx, s3), cscale(ky, s1)), cscale(kz, s5));
    const double2 rz = cadd(cadd(cscale(kx, s4), cscale(ky, s5)), cscale(kz, s2));
    r2 = cabs2(rx) + cabs2(ry) + cabs2(rz);
    b2 = cabs2(b[0]) + cabs2(b[1]) + cabs2(b[2]);
}

// Green's-function / eigenstrain kernel on the half spectrum: e0h (3 half
// spectra of the real eigenstrain fields) -> eh (6 half spectra).
// The reference takes Re(ifftn(Y)) of the full-spectrum strain transform Y,
// which is the inverse transform of the Hermitian part
// H(k) = (Y(k) + conj(Y(m(k)))) / 2, m(k) the mirror bin.  Away from the
// Nyquist planes of even extents Y(m(k)) = conj(Y(k)) exactly (A(-k) = A(k),
// b(-k) = -conj(b(k)) term by term), so H = Y; on those planes the mirror bin
// carries the same Nyquist wave number as the bin, Y(m(k)) is evaluated
// there explicitly, and H is formed.  The residual sums run over the full
// spectrum: a stored bin whose mirror is not stored also counts the mirror.
__global__ void __launch_bounds__(256) k_green(SpecConst c, const double2* __restrict__ e0h, double2* __restrict__ eh,
                                               double* __restrict__ partial) {
    __shared__ double sh[16];
    const long long Nh = c.Nh;
    double r2s = 0.0, b2s = 0.0;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < Nh;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long i2 = idx % c.h2, t = idx / c.h2;
        const long long i1 = t % c.h1, i0 = t / c.h1;
        const double kx = wave_number(i0, c.e0, c.v0);
        const double ky = wave_number(i1, c.e1, c.v1);
        const double kz = wave_number(i2, c.e2, c.v2);
        const double2 a0 = e0h[idx], a1 = e0h[Nh + idx], a2 = e0h[2 * Nh + idx];
        double2 e[6];
        double r2, b2;
        strain_at(c, kx, ky, kz, a0, a1, a2, e, r2, b2);
        const bool ny0 = (c.e0 % 2 == 0) && i0 == c.e0 / 2;
        const bool ny1 = (c.e1 % 2 == 0) && i1 == c.e1 / 2;
        const bool ny2 = (c.e2 % 2 == 0) && i2 == c.e2 / 2;
        const long long ih = c.hax == 2 ? i2 : i1;
        const int eh_n = c.hax == 2 ? c.e2 : c.e1;
        const bool self_mirror = ih == 0 || ((eh_n % 2 == 0) && ih == eh_n / 2);
        double mr2 = r2, mb2 = b2;
        if (ny0 || ny1 || ny2) {
            const long long m0 = (c.e0 - i0) % c.e0, m1 = (c.e1 - i1) % c.e1, m2 = (c.e2 - i2) % c.e2;
            double2 em[6];
            strain_at(c, wave_number(m0, c.e0, c.v0), wave_number(m1, c.e1, c.v1), wave_number(m2, c.e2, c.v2),
                      conj2(a0), conj2(a1), conj2(a2), em, mr2, mb2);
#pragma unroll
            for (int k = 0; k < 6; ++k) e[k] = cscale(0.5, cadd(e[k], conj2(em[k])));
        }
#pragma unroll
        for (int m = 0; m < 6; ++m) eh[m * Nh + idx] = e[m];
        r2s += r2;
        b2s += b2;
        if (!self_mirror) { r2s += mr2; b2s += mb2; }
    }
    block_sum2<256>(r2s, b2s, sh);
    if (threadIdx.x == 0) {
        partial[2 * blockIdx.x] = r2s;
        partial[2 * blockIdx.x + 1] = b2s;
    }
}

__global__ void __launch_bounds__(256) k_residual_sum(const double* __restrict__ partial, int nblocks,
                                                      double* __restrict__ out) {
    __shared__ double sh[16];
    double a = 0.0, b = 0.0;
    for (int i = threadIdx.x; i < nblocks; i += 256) {
        a += partial[2 * i];
        b += partial[2 * i + 1];
    }
    block_sum2<256>(a, b, sh);
    if (threadIdx.x == 0) { out[0] = a; out[1] = b; }
}

// st: the six real strain fields (unnormalised inverse transforms)
__global__ void k_epilogue(SpecConst c, const double* __restrict__ f, const double* __restrict__ st,
                           double* __restrict__ driving, double* __restrict__ energy, double* __restrict__ hydro) {
    const long long N = c.N;
    const double inv_n = 1.0 / (double)N;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        const double f0 = f[i], f1 = f[N + i], f2 = f[2 * N + i];
        double de[6];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            double e = c.eig[j] * f0;
            e = e + c.eig[3 + j] * f1;
            e = e + c.eig[6 + j] * f2;
            de[j] = st[j * N + i] * inv_n - e;
        }
#pragma unroll
        for (int m = 3; m < 6; ++m) de[m] = st[m * N + i] * inv_n;
        const double c11 = c.c11, c12 = c.c12, c44x2 = 2.0 * c.c44;
        const double s0 = c11 * de[0] + c12 * (de[1] + de[2]);
        const double s1 = c11 * de[1] + c12 * (de[0] + de[2]);
        const double s2 = c11 * de[2] + c12 * (de[0] + de[1]);
        const double s3 = c44x2 * de[3], s4 = c44x2 * de[4], s5 = c44x2 * de[5];
        if (energy)
            energy[i] = 0.5 * (s0 * de[0] + s1 * de[1] + s2 * de[2] + 2.0 * (s3 * de[3] + s4 * de[4] + s5 * de[5]));
        if (driving) {
#pragma unroll
            for (int v = 0; v < 3; ++v)
                driving[v * N + i] = -(s0 * c.eig[3 * v] + s1 * c.eig[3 * v + 1] + s2 * c.eig[3 * v + 2]);
        }
        if (hydro) hydro[i] = (s0 + s1 + s2) / 3.0;
    }
}

// variant fractions of a label map: variant 0 = every non-matrix label
__global__ void k_label_fractions(long long N, const int32_t* __restrict__ phi, int32_t matrix, double* __restrict__ f) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        f[i] = phi[i] != matrix ? 1.0 : 0.0;
        f[N + i] = 0.0;
        f[2 * N + i] = 0.0;
    }
}
__global__ void k_to_float(long long N, const double* __restrict__ a, float* __restrict__ b) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

}  // namespace

struct gpk_spectral {
    int ndim = 0;
    int n[3] = {1, 1, 1};
    long long N = 0;
    SpecConst c{};
    int device = 0;
    int num_sms = 148;
    cudaStream_t own = nullptr;
    cudaStream_t stream = nullptr;
    cufftHandle fwd = 0, inv = 0;
    bool have_fwd = false, have_inv = false;
    double* er = nullptr;     // 3 N real eigenstrain fields
    double2* e0h = nullptr;   // 3 Nh half spectra
    double2* eh = nullptr;    // 6 Nh half spectra
    double* st = nullptr;     // 6 N real strain fields
    double* partial = nullptr;
    double* red = nullptr;   // 2 doubles
    int nblocks = 0;
    double* stage = nullptr;  // host-path staging: 3N fractions, 3N driving, N energy, N hydro
    long long bytes = 0;
};

static int spec_set_constants(gpk_spectral* s, double dx, double c11, double c12, double c44, const double eig[9]) {
    if (!(dx > 0.0) || !eig) {
        gpk_set_error("spectral: dx must be positive and eig non-null");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    SpecConst& c = s->c;
    c.e0 = s->n[0]; c.e1 = s->n[1]; c.e2 = s->ndim == 3 ? s->n[2] : 1;
    c.hax = s->ndim == 3 ? 2 : 1;
    c.h0 = c.e0;
    c.h1 = c.hax == 1 ? c.e1 / 2 + 1 : c.e1;
    c.h2 = c.hax == 2 ? c.e2 / 2 + 1 : 1;
    c.N = s->N;
    c.Nh = (long long)c.h0 * c.h1 * c.h2;
    // numpy's fftfreq scale 1 / (n * d) of each array axis; axes beyond ndim have k = 0
    c.v0 = 1.0 / (s->n[0] * dx);
    c.v1 = 1.0 / (s->n[1] * dx);
    c.v2 = s->ndim == 3 ? 1.0 / (s->n[2] * dx) : 0.0;
    c.c11 = c11; c.c12 = c12; c.c44 = c44;
    for (int k = 0; k < 9; ++k) c.eig[k] = eig[k];
    return GPK_OK;
}

static void spec_free(gpk_spectral* s) {
    if (s->have_fwd) cufftDestroy(s->fwd);
    if (s->have_inv) cufftDestroy(s->inv);
    cudaFree(s->er); cudaFree(s->e0h); cudaFree(s->eh); cudaFree(s->st);
    cudaFree(s->partial); cudaFree(s->red); cudaFree(s->stage);
    if (s->own) cudaStreamDestroy(s->own);
}

extern "C" int gpk_spectral_create(int ndim, const int* shape, double dx, double c11, double c12, double c44,
                                   const double eig[9], gpk_spectral** out) {
    if (!out || !shape || (ndim != 2 && ndim != 3)) {
        gpk_set_error("spectral: ndim must be 2 or 3 with a shape array and an output pointer");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    long long N = 1;
    for (int a = 0; a < ndim; ++a) {
        if (shape[a] < 1 || shape[a] > (1 << 20)) {
            gpk_set_error("spectral: extents must lie in [1, 2^20]");
            return GPK_ERR_INVALID_ARGUMENT;
        }
        N *= shape[a];
    }
    if (N >= (1ll << 31)) {
        gpk_set_error("spectral: fewer than 2^31 cells");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        gpk_set_error("no CUDA device available");
        return GPK_ERR_NO_DEVICE;
    }
    gpk_spectral* s = new gpk_spectral();
    s->ndim = ndim;
    for (int a = 0; a < ndim; ++a) s->n[a] = shape[a];
    s->N = N;
    int rc = spec_set_constants(s, dx, c11, c12, c44, eig);
    if (rc != GPK_OK) { delete s; return rc; }
    auto fail = [&](int code) { spec_free(s); delete s; return code; };
    if (cudaGetDevice(&s->device) != cudaSuccess) return fail(GPK_ERR_CUDA);
    cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, s->device);
    if (cudaStreamCreateWithFlags(&s->own, cudaStreamNonBlocking) != cudaSuccess) {
        gpk_set_error("spectral: cudaStreamCreate failed");
        return fail(GPK_ERR_CUDA);
    }
    s->stream = s->own;
    long long blocks = (N + 255) / 256;
    if (blocks > (long long)s->num_sms * 8) blocks = (long long)s->num_sms * 8;
    s->nblocks = (int)blocks;
    const long long Nh = s->c.Nh;
    const size_t want[6] = {sizeof(double) * 3 * N, sizeof(double2) * 3 * Nh, sizeof(double2) * 6 * Nh,
                            sizeof(double) * 6 * N, sizeof(double) * 2 * s->nblocks, sizeof(double) * 2};
    void** dst[6] = {(void**)&s->er, (void**)&s->e0h, (void**)&s->eh, (void**)&s->st, (void**)&s->partial,
                     (void**)&s->red};
    for (int k = 0; k < 6; ++k) {
        if (cudaMalloc(dst[k], want[k]) != cudaSuccess) {
            cudaGetLastError();
            gpk_set_error("spectral: cudaMalloc of " + std::to_string(want[k]) + " bytes failed");
            return fail(GPK_ERR_OUT_OF_MEMORY);
        }
        s->bytes += (long long)want[k];
    }
    // real-to-complex forward (3 fields), complex-to-real inverse (6 fields),
    // out of place, default layouts: the last axis is halved to n/2 + 1
    int dims[3] = {s->n[0], s->n[1], s->n[2]};
    if (cufftPlanMany(&s->fwd, ndim, dims, nullptr, 1, (int)N, nullptr, 1, (int)Nh, CUFFT_D2Z, 3) != CUFFT_SUCCESS) {
        gpk_set_error("spectral: cufftPlanMany (D2Z, batch 3) failed");
        return fail(GPK_ERR_CUDA);
    }
    s->have_fwd = true;
    if (cufftPlanMany(&s->inv, ndim, dims, nullptr, 1, (int)Nh, nullptr, 1, (int)N, CUFFT_Z2D, 6) != CUFFT_SUCCESS) {
        gpk_set_error("spectral: cufftPlanMany (Z2D, batch 6) failed");
        return fail(GPK_ERR_CUDA);
    }
    s->have_inv = true;
    *out = s;
    return GPK_OK;
}

extern "C" int gpk_spectral_destroy(gpk_spectral* s) {
    if (!s) return GPK_OK;
    cudaStreamSynchronize(s->stream);
    spec_free(s);
    delete s;
    return GPK_OK;
}

extern "C" int gpk_spectral_set_constants(gpk_spectral* s, double dx, double c11, double c12, double c44,
                                          const double eig[9]) {
    if (!s) { gpk_set_error("spectral: null handle"); return GPK_ERR_INVALID_ARGUMENT; }
    return spec_set_constants(s, dx, c11, c12, c44, eig);
}

extern "C" int gpk_spectral_set_stream(gpk_spectral* s, void* stream) {
    if (!s) { gpk_set_error("spectral: null handle"); return GPK_ERR_INVALID_ARGUMENT; }
    s->stream = (cudaStream_t)stream;
    return GPK_OK;
}

extern "C" int gpk_spectral_solve(gpk_spectral* s, const double* fractions, double* driving, double* energy,
                                  double* hydro, double* residual) {
    if (!s || !fractions) { gpk_set_error("spectral: null handle or fractions"); return GPK_ERR_INVALID_ARGUMENT; }
    const long long N = s->N;
    const int grid = s->nblocks;
    k_eigenstrain<<<grid, 256, 0, s->stream>>>(s->c, fractions, s->er);
    SPEC_CUDA_TRY(cudaGetLastError());
    SPEC_FFT_TRY(cufftSetStream(s->fwd, s->stream));
    SPEC_FFT_TRY(cufftExecD2Z(s->fwd, (cufftDoubleReal*)s->er, (cufftDoubleComplex*)s->e0h));
    k_green<<<grid, 256, 0, s->stream>>>(s->c, s->e0h, s->eh, s->partial);
    SPEC_CUDA_TRY(cudaGetLastError());
    k_residual_sum<<<1, 256, 0, s->stream>>>(s->partial, grid, s->red);
    SPEC_CUDA_TRY(cudaGetLastError());
    SPEC_FFT_TRY(cufftSetStream(s->inv, s->stream));
    SPEC_FFT_TRY(cufftExecZ2D(s->inv, (cufftDoubleComplex*)s->eh, (cufftDoubleReal*)s->st));
    if (driving || energy || hydro) {
        k_epilogue<<<grid, 256, 0, s->stream>>>(s->c, fractions, s->st, driving, energy, hydro);
        SPEC_CUDA_TRY(cudaGetLastError());
    }
    if (residual) {
        double h[2];
        SPEC_CUDA_TRY(cudaMemcpyAsync(h, s->red, sizeof(h), cudaMemcpyDeviceToHost, s->stream));
        SPEC_CUDA_TRY(cudaStreamSynchronize(s->stream));
        // rms over all N wave vectors, as np.sqrt(np.mean(...)) of the reference
        const double num = sqrt(h[0] / (double)N), den = sqrt(h[1] / (double)N);
        *residual = num / (den > 1e-30 ? den : 1e-30);
    }
    return GPK_OK;
}

extern "C" int gpk_spectral_solve_host(gpk_spectral* s, const double* fractions, double* driving, double* energy,
                                       double* hydro, double* residual) {
    if (!s || !fractions) { gpk_set_error("spectral: null handle or fractions"); return GPK_ERR_INVALID_ARGUMENT; }
    const long long N = s->N;
    if (!s->stage) {
        const size_t b = sizeof(double) * 8 * N;
        if (cudaMalloc((void**)&s->stage, b) != cudaSuccess) {
            cudaGetLastError();
            gpk_set_error("spectral: cudaMalloc of host-path staging failed");
            return GPK_ERR_OUT_OF_MEMORY;
        }
        s->bytes += (long long)b;
    }
    double* f = s->stage;
    double* d = f + 3 * N;
    double* e = d + 3 * N;
    double* h = e + N;
    SPEC_CUDA_TRY(cudaMemcpyAsync(f, fractions, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, s->stream));
    int rc = gpk_spectral_solve(s, f, driving ? d : nullptr, energy ? e : nullptr, hydro ? h : nullptr, residual);
    if (rc != GPK_OK) return rc;
    if (driving) SPEC_CUDA_TRY(cudaMemcpyAsync(driving, d, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, s->stream));
    if (energy) SPEC_CUDA_TRY(cudaMemcpyAsync(energy, e, sizeof(double) * N, cudaMemcpyDeviceToHost, s->stream));
    if (hydro) SPEC_CUDA_TRY(cudaMemcpyAsync(hydro, h, sizeof(double) * N, cudaMemcpyDeviceToHost, s->stream));
    SPEC_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return GPK_OK;
}

extern "C" int gpk_spectral_couple_grid(gpk_spectral* s, gpk_grid* G, int32_t matrix_label, double* residual) {
    if (!s || !G) { gpk_set_error("spectral: null handle"); return GPK_ERR_INVALID_ARGUMENT; }
    const bool same = s->ndim == 3 ? (s->n[0] == G->d.Nz && s->n[1] == G->d.Ny && s->n[2] == G->d.Nx)
                                   : (G->d.Nz == 1 && s->n[0] == G->d.Ny && s->n[1] == G->d.Nx);
    if (!same) {
        gpk_set_error("spectral: the solve's shape differs from the grid's");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    const long long N = s->N;
    if (!s->stage) {
        const size_t b = sizeof(double) * 8 * N;
        if (cudaMalloc((void**)&s->stage, b) != cudaSuccess) {
            cudaGetLastError();
            gpk_set_error("spectral: cudaMalloc of the coupling buffers failed");
            return GPK_ERR_OUT_OF_MEMORY;
        }
        s->bytes += (long long)b;
    }
    double* f = s->stage;
    double* e = f + 7 * N;  // energy when the grid holds floats
    cudaStream_t saved = s->stream;
    s->stream = G->stream;
    k_label_fractions<<<s->nblocks, 256, 0, s->stream>>>(N, G->phi, matrix_label, f);
    G->launches++;
    double* E = G->precision == GPK_PREC_F64 ? (double*)G->f[GPK_FIELD_E_EL] : e;
    int rc = gpk_spectral_solve(s, f, nullptr, E, nullptr, residual);
    if (rc == GPK_OK && G->precision != GPK_PREC_F64) {
        k_to_float<<<s->nblocks, 256, 0, s->stream>>>(N, e, (float*)G->f[GPK_FIELD_E_EL]);
        G->launches++;
        if (cudaGetLastError() != cudaSuccess) rc = GPK_ERR_CUDA;
    }
    G->launches += 4;
    s->stream = saved;
    return rc;
}

extern "C" int gpk_spectral_info(const gpk_spectral* s, int64_t* cells, int64_t* device_bytes) {
    if (!s) { gpk_set_error("spectral: null handle"); return GPK_ERR_INVALID_ARGUMENT; }
    if (cells) *cells = s->N;
    if (device_bytes) *device_bytes = s->bytes;
    return GPK_OK;
}
