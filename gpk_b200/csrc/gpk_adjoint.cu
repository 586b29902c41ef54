// gpk_adjoint.cu — FP64 forward model and exact discrete adjoint of an
// interface-velocity loss at a fixed label map (2-D, plane strain).
//
// Forward (theta = E_xx, E_yy, E_xy, a_1..a_4, M_0..M_{n-1}):
//   k_adj_eig(0)   eigenstrain field eta(x) E (3 real fields)
//   cuFFT D2Z      3 transforms to half spectra
//   k_adj_green    per half-spectrum wave vector: 2x2 acoustic solve, strain
//                  transform (mean normal strain = mean eigenstrain, mean
//                  shear 0), its Hermitian part on Nyquist rows/columns
//   cuFFT Z2D      3 transforms back to real fields
//   k_adj_stress(0) elastic strain de, energy density e(x), sum of e
//   k_adj_velocity v_raw = M (e(q) - e(i) - sigma_a kappa) per interface cell
//   k_adj_project  pair-restricted Gaussian average (FP64, one warp per
//                  interface cell), residual r
// Adjoint:
//   k_adj_qfield   o r / D at projected cells
//   k_adj_project_t rho = o_j sum_i w_ij (o_i r_i / D_i)  (transposed stencil,
//                  one warp per cell), lambda = rho M, anisotropy-gradient sums
//   k_adj_mu       mu(x) = dL/de(x): gather of lambda over the cells whose
//                  product neighbour is x, plus w_E dx^2
//   k_adj_eig(1) .. k_adj_stress(1)  adjoint solve for the field mu(x) de(x);
//                  dL/dE = sum_x eta(x) sigma_adj(x) : e_k (self-adjoint operator)
//   k_adj_mobility dL/dM_l = sum over label-l cells of rho B (CSR, fixed order)
// All sums are block partials that the last block to finish reduces in a
// fixed order: results are deterministic.
#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/gpk_adjoint.h"
#include "gpk_grid.h"

using gpk_dev::Dims;

namespace {

struct AdjC {
    int Nx, Ny;
    long long N;
    int Hx;          // half-spectrum width Nx / 2 + 1
    long long Nh;    // half-spectrum bins Ny * Hx
    double vx, vy;  // fftfreq scales 1/(n dx) along x (last axis) and y
    double c11, c12, c44;
    double dx2;      // dx^2, the cell area of the energy sum
    double wE;       // energy weight
    double sigma0, m_fixed;
    int R;           // projection radius
};

__device__ __forceinline__ double wavenum(long long i, int n, double scale) {
    const long long m = (i <= (n - 1) / 2) ? i : i - n;
    return 6.283185307179586 * ((double)m * scale);
}

template <int SLOTS>
__device__ __forceinline__ void block_partials(double (&v)[SLOTS], double* partial) {
    __shared__ double sh[8][SLOTS];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int s = 0; s < SLOTS; ++s) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[s] += __shfl_down_sync(0xffffffffu, v[s], o);
        if (lane == 0) sh[w][s] = v[s];
    }
    __syncthreads();
    if (threadIdx.x < SLOTS) {
        double t = 0.0;
        for (int k = 0; k < 8; ++k) t += sh[k][threadIdx.x];
        partial[blockIdx.x * 8 + threadIdx.x] = t;
    }
}

// Block partials, then the last block to finish sums every block's partials
// in a fixed order (out[s], s < SLOTS) and re-arms the counter: the result
// does not depend on which block finishes last.
template <int SLOTS>
__device__ __forceinline__ void reduce_to(double (&v)[SLOTS], double* partial, unsigned* counter, double* out) {
    block_partials<SLOTS>(v, partial);
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    __shared__ double sh[256];
    for (int s = 0; s < SLOTS; ++s) {
        double t = 0.0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += 256) t += __ldcg(&partial[b * 8 + s]);
        sh[threadIdx.x] = t;
        __syncthreads();
        for (int h = 128; h > 0; h >>= 1) {
            if (threadIdx.x < h) sh[threadIdx.x] += sh[threadIdx.x + h];
            __syncthreads();
        }
        if (threadIdx.x == 0) out[s] = sh[0];
        __syncthreads();
    }
    if (threadIdx.x == 0) *counter = 0u;
}

// eigenstrain field: mode 0 eta(x) E; mode 1 mu(x) de(x)
// th: the parameters in device memory (E_xx, E_yy, E_xy, a_1..a_4, M...)
__global__ void k_adj_eig(AdjC c, int mode, const double* __restrict__ th, const double* __restrict__ eta,
                          const double* __restrict__ mu, const double* __restrict__ de, double* __restrict__ er) {
    const long long N = c.N;
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < N; x += (long long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int k = 0; k < 3; ++k) er[k * N + x] = mode == 0 ? eta[x] * th[k] : mu[x] * de[k * N + x];
    }
}

__device__ __forceinline__ double2 cax(double s, double2 a, double t, double2 b) {
    return make_double2(s * a.x + t * b.x, s * a.y + t * b.y);
}

// plane-strain strain transform of the eigenstrain transform at (kx, ky)
__device__ __forceinline__ void green2d(const AdjC& c, double kx, double ky, double2 exx, double2 eyy, double2 exy,
                                        double2& sxx, double2& syy, double2& sxy) {
    if (kx == 0.0 && ky == 0.0) {
        // free mean expansion: mean normal strain follows the eigenstrain, mean shear 0
        sxx = exx; syy = eyy; sxy = make_double2(0.0, 0.0);
        return;
    }
    const double c11 = c.c11, c12 = c.c12, c44 = c.c44;
    const double2 txx = cax(c11, exx, c12, eyy), tyy = cax(c12, exx, c11, eyy);
    const double2 txy = make_double2(2.0 * c44 * exy.x, 2.0 * c44 * exy.y);
    const double2 bx = cax(kx, txx, ky, txy), by = cax(kx, txy, ky, tyy);
    const double a00 = c11 * kx * kx + c44 * ky * ky, a11 = c44 * kx * kx + c11 * ky * ky;
    const double a01 = (c12 + c44) * kx * ky;
    const double det = a00 * a11 - a01 * a01;
    const double2 x0 = cax(a11 / det, bx, -a01 / det, by), x1 = cax(-a01 / det, bx, a00 / det, by);
    // u = -i x; e_xx = i kx u_x = kx x0, e_yy = ky x1, e_xy = (kx x1 + ky x0) / 2
    sxx = make_double2(kx * x0.x, kx * x0.y);
    syy = make_double2(ky * x1.x, ky * x1.y);
    sxy = cax(0.5 * kx, x1, 0.5 * ky, x0);
}

__device__ __forceinline__ double2 cj(double2 a) { return make_double2(a.x, -a.y); }

// In place on the half spectrum (x halved).  The strain is the real part of
// the full inverse transform, i.e. the inverse transform of the Hermitian
// part of the strain transform; away from the Nyquist row/column of an even
// extent the mirror bin's transform is exactly the conjugate, and on them it
// is evaluated at the mirror bin's own (Nyquist) wave numbers.
__global__ void k_adj_green(AdjC c, double2* __restrict__ eh) {
    const long long Nh = c.Nh;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < Nh;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long iy = idx / c.Hx, ix = idx % c.Hx;
        const double kx = wavenum(ix, c.Nx, c.vx), ky = wavenum(iy, c.Ny, c.vy);
        const double2 exx = eh[idx], eyy = eh[Nh + idx], exy = eh[2 * Nh + idx];
        double2 sxx, syy, sxy;
        green2d(c, kx, ky, exx, eyy, exy, sxx, syy, sxy);
        if (((c.Nx & 1) == 0 && ix == c.Nx / 2) || ((c.Ny & 1) == 0 && iy == c.Ny / 2)) {
            const long long mx = (c.Nx - ix) % c.Nx, my = (c.Ny - iy) % c.Ny;
            double2 mxx, myy, mxy;
            green2d(c, wavenum(mx, c.Nx, c.vx), wavenum(my, c.Ny, c.vy), cj(exx), cj(eyy), cj(exy), mxx, myy, mxy);
            sxx = cax(0.5, sxx, 0.5, cj(mxx));
            syy = cax(0.5, syy, 0.5, cj(myy));
            sxy = cax(0.5, sxy, 0.5, cj(mxy));
        }
        eh[idx] = sxx; eh[Nh + idx] = syy; eh[2 * Nh + idx] = sxy;
    }
}

// mode 0: de = eps - eta E, energy density e(x), slot 0 = sum e dx^2.
// mode 1: adjoint stress of the field mu de; slots 0..2 = sums of eta*sigma.
__global__ void __launch_bounds__(256) k_adj_stress(AdjC c, int mode, const double* __restrict__ th,
                                                   const double* __restrict__ st,
                                                   const double* __restrict__ eta, const double* __restrict__ mu,
                                                   double* __restrict__ de, double* __restrict__ en,
                                                   double* __restrict__ partial, unsigned* __restrict__ counter,
                                                   double* __restrict__ out) {
    const long long N = c.N;
    const double inv_n = 1.0 / (double)N;
    double acc[3] = {0.0, 0.0, 0.0};
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < N; x += (long long)gridDim.x * blockDim.x) {
        double d[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const double es = mode == 0 ? eta[x] * th[k] : mu[x] * de[k * N + x];
            d[k] = st[k * N + x] * inv_n - es;
        }
        const double sxx = c.c11 * d[0] + c.c12 * d[1];
        const double syy = c.c12 * d[0] + c.c11 * d[1];
        const double sxy = 2.0 * c.c44 * d[2];
        if (mode == 0) {
            const double e = 0.5 * (sxx * d[0] + syy * d[1] + 2.0 * sxy * d[2]);
#pragma unroll
            for (int k = 0; k < 3; ++k) de[k * N + x] = d[k];
            en[x] = e;
            acc[0] += e * c.dx2;
        } else {
            const double h = eta[x];
            acc[0] += h * sxx;
            acc[1] += h * syy;
            acc[2] += h * sxy;
        }
    }
    reduce_to<3>(acc, partial, counter, out);
}

struct Act {
    const int32_t* act;   // cell of each interface position
    const int32_t* mobp;  // mobility index or -1
    const double* kap;    // curvature
    const double* cm;     // cos(4 m theta_c), 4 x na
    const int8_t* o;      // +1 if the cell's label is the lower of its pair
    const uint8_t* proj;  // projected (phi != phi_comp)
    int na;
};

__global__ void k_adj_velocity(AdjC c, Act A, const int32_t* __restrict__ qn, const double* __restrict__ en,
                               const double* __restrict__ th, double* __restrict__ B, double* __restrict__ vr) {
    const double a0 = th[3], a1 = th[4], a2 = th[5], a3 = th[6];
    const double* __restrict__ mob = th + 7;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < A.na; a += gridDim.x * blockDim.x) {
        const int i = A.act[a];
        const int q = qn[i];
        const double dE = q >= 0 ? en[q] - en[i] : 0.0;
        const double sa = c.sigma0 * (1.0 + a0 * A.cm[a] + a1 * A.cm[A.na + a] + a2 * A.cm[2 * A.na + a] +
                                      a3 * A.cm[3 * A.na + a]);
        const double b = dE - sa * A.kap[a];
        const int p = A.mobp[a];
        B[a] = b;
        vr[i] = (p >= 0 ? mob[p] : c.m_fixed) * b;
    }
}

struct Labels {
    const int32_t* phi;
    const int32_t* comp;
    const uint8_t* mask;
    const double* w;  // weight by r^2
};

// Sum over the same-pair projected cells j within R of cell i of w * f(j)
// (oriented by o_j when ORIENT), by one warp: lane l takes taps l, l + 32, ...
// of the (2R+1)^2 box, then a fixed-order tree over the lanes; every lane
// returns lane 0's totals.
template <bool ORIENT>
__device__ __forceinline__ double warp_pair_sum(const AdjC& c, const Labels& L, int i, const double* __restrict__ f,
                                                int lane, double& den) {
    const int y0 = i / c.Nx, x0 = i % c.Nx;
    const int32_t low = min(L.phi[i], L.comp[i]), high = max(L.phi[i], L.comp[i]);
    const int W = 2 * c.R + 1;
    double num = 0.0;
    den = 0.0;
    for (int t = lane; t < W * W; t += 32) {
        const int dy = t / W - c.R, dxs = t % W - c.R;
        const int j = gpk_dev::wrap_any(y0 + dy, c.Ny) * c.Nx + gpk_dev::wrap_any(x0 + dxs, c.Nx);
        const int32_t pj = L.phi[j], qj = L.comp[j];
        if (!L.mask[j] || pj == qj || min(pj, qj) != low || max(pj, qj) != high) continue;
        const double w = L.w[dxs * dxs + dy * dy];
        num += ORIENT ? w * (pj == low ? 1.0 : -1.0) * f[j] : w * f[j];
        den += w;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        num += __shfl_down_sync(0xffffffffu, num, o);
        den += __shfl_down_sync(0xffffffffu, den, o);
    }
    den = __shfl_sync(0xffffffffu, den, 0);
    return __shfl_sync(0xffffffffu, num, 0);
}

// forward projection, one warp per interface position; r = v - target;
// out[0] = sum r^2 / 2
__global__ void __launch_bounds__(256) k_adj_project(AdjC c, Act A, Labels L, const double* __restrict__ vr,
                                                     const double* __restrict__ target, double* __restrict__ v,
                                                     double* __restrict__ Dn, double* __restrict__ r,
                                                     double* __restrict__ vout, double* __restrict__ partial,
                                                     unsigned* __restrict__ counter, double* __restrict__ out) {
    double acc[1] = {0.0};
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; a < A.na; a += nw) {
        const int i = A.act[a];
        double val = vr[i], den = 1.0;
        if (A.proj[a]) {
            const double num = warp_pair_sum<true>(c, L, i, vr, lane, den);
            val = (double)A.o[a] * (num / den);
        }
        if (lane == 0) {
            v[a] = val;
            Dn[a] = den;
            const double ri = val - target[i];
            r[a] = ri;
            if (vout) vout[i] = val;
            acc[0] += 0.5 * ri * ri;
        }
    }
    reduce_to<1>(acc, partial, counter, out);
}

__global__ void k_adj_qfield(Act A, const double* __restrict__ r, const double* __restrict__ Dn,
                             double* __restrict__ qf) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < A.na; a += gridDim.x * blockDim.x)
        qf[A.act[a]] = A.proj[a] ? (double)A.o[a] * r[a] / Dn[a] : 0.0;
}

// rho = P^T r (one warp per position); lambda = rho M; out[0..3] = dL/da_m
__global__ void __launch_bounds__(256) k_adj_project_t(AdjC c, Act A, Labels L, const double* __restrict__ qf,
                                                       const double* __restrict__ r, const double* __restrict__ mob,
                                                       double* __restrict__ rho, double* __restrict__ lam,
                                                       double* __restrict__ partial, unsigned* __restrict__ counter,
                                                       double* __restrict__ out) {
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; a < A.na; a += nw) {
        const int j = A.act[a];
        double rj = r[a];
        if (A.proj[a]) {
            double den;
            rj = (double)A.o[a] * warp_pair_sum<false>(c, L, j, qf, lane, den);
        }
        if (lane == 0) {
            rho[a] = rj;
            const int p = A.mobp[a];
            const double M = p >= 0 ? mob[p] : c.m_fixed;
            lam[j] = rj * M;
            const double g = -rj * M * c.sigma0 * A.kap[a];
#pragma unroll
            for (int m = 0; m < 4; ++m) acc[m] += g * A.cm[m * A.na + a];
        }
    }
    reduce_to<4>(acc, partial, counter, out);
}

// mu(x) = dL/de(x)
__global__ void k_adj_mu(AdjC c, const int32_t* __restrict__ qn, const double* __restrict__ lam,
                         double* __restrict__ mu) {
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < c.N; x += (long long)gridDim.x * blockDim.x) {
        double m = c.wE * c.dx2;
        if (qn[x] >= 0) m -= lam[x];
        const int y0 = (int)(x / c.Nx), x0 = (int)(x % c.Nx);
        const int nb[4] = {y0 * c.Nx + gpk_dev::wrap_any(x0 - 1, c.Nx), y0 * c.Nx + gpk_dev::wrap_any(x0 + 1, c.Nx),
                           gpk_dev::wrap_any(y0 - 1, c.Ny) * c.Nx + x0, gpk_dev::wrap_any(y0 + 1, c.Ny) * c.Nx + x0};
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (qn[nb[k]] == (int)x) m += lam[nb[k]];
        mu[x] = m;
    }
}

// one block per mobility parameter: sum of rho B over its cells (CSR order)
__global__ void k_adj_mobility(const int32_t* __restrict__ off, const int32_t* __restrict__ pos,
                               const double* __restrict__ rho, const double* __restrict__ B, double* __restrict__ g) {
    __shared__ double sh[256];
    const int p = blockIdx.x;
    double t = 0.0;
    for (int k = off[p] + threadIdx.x; k < off[p + 1]; k += 256) t += rho[pos[k]] * B[pos[k]];
    sh[threadIdx.x] = t;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if (threadIdx.x < h) sh[threadIdx.x] += sh[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) g[p] = sh[0];
}

// product neighbour (first face neighbour x-, x+, y-, y+ with the competitor
// label; -1 when none or when the competitor is the cell's own label)
__global__ void k_adj_prep(AdjC c, Act A, const int32_t* __restrict__ phi, const int32_t* __restrict__ comp,
                           const double* __restrict__ nx, const double* __restrict__ ny, const double* __restrict__ g,
                           const double* __restrict__ kappa, const int32_t* __restrict__ mob_label,
                           int32_t* __restrict__ qn, double* kap, double* cm, int8_t* o, uint8_t* proj,
                           int32_t* mobp) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < A.na; a += gridDim.x * blockDim.x) {
        const int i = A.act[a];
        const int y0 = i / c.Nx, x0 = i % c.Nx;
        const int32_t p = phi[i], q = comp[i];
        int prod = -1;
        if (q != p) {
            const int nb[4] = {y0 * c.Nx + gpk_dev::wrap_any(x0 - 1, c.Nx), y0 * c.Nx + gpk_dev::wrap_any(x0 + 1, c.Nx),
                               gpk_dev::wrap_any(y0 - 1, c.Ny) * c.Nx + x0, gpk_dev::wrap_any(y0 + 1, c.Ny) * c.Nx + x0};
            for (int k = 0; k < 4 && prod < 0; ++k)
                if (phi[nb[k]] == q) prod = nb[k];
        }
        qn[i] = prod;
        kap[a] = kappa[i];
        const double cg = cos(g[i]), sg = sin(g[i]);
        const double ncx = nx[i] * cg + ny[i] * sg, ncy = -nx[i] * sg + ny[i] * cg;
        const double th = atan2(ncy, ncx);
#pragma unroll
        for (int m = 0; m < 4; ++m) cm[m * A.na + a] = cos(4.0 * (m + 1) * th);
        o[a] = p == min(p, q) ? 1 : -1;
        proj[a] = p != q;
        mobp[a] = mob_label[p];
    }
}

__global__ void k_adj_eta(long long N, const int32_t* __restrict__ phi, const int32_t* __restrict__ mob_label,
                          double* __restrict__ eta) {
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < N; x += (long long)gridDim.x * blockDim.x)
        eta[x] = mob_label[phi[x]] < 0 ? 1.0 : 0.0;
}

#define ADJ_CUDA_TRY(expr)                                                             \
    do {                                                                               \
        cudaError_t _e = (expr);                                                       \
        if (_e != cudaSuccess) {                                                       \
            gpk_set_error(std::string(#expr " failed: ") + cudaGetErrorString(_e));    \
            return GPK_ERR_CUDA;                                                       \
        }                                                                              \
    } while (0)
#define ADJ_FFT_TRY(expr)                                                              \
    do {                                                                               \
        if ((expr) != CUFFT_SUCCESS) {                                                 \
            gpk_set_error(std::string(#expr " failed"));                               \
            return GPK_ERR_CUDA;                                                       \
        }                                                                              \
    } while (0)

}  // namespace

struct gpk_adjoint {
    gpk_grid* G = nullptr;
    AdjC c{};
    int na = 0, n_labels = 0, n_mob = 0, nblocks = 0;
    Act A{};
    Labels L{};
    cufftHandle plan = 0, iplan = 0;
    bool have_plan = false, have_iplan = false;
    std::vector<void*> mem;
    int32_t *mob_label = nullptr, *act = nullptr, *mobp = nullptr, *qn = nullptr, *csr_off = nullptr, *csr_pos = nullptr;
    double *kap = nullptr, *cm = nullptr, *eta = nullptr, *target = nullptr, *de = nullptr, *en = nullptr;
    double *vr = nullptr, *qf = nullptr, *lam = nullptr, *mu = nullptr, *B = nullptr, *v = nullptr, *Dn = nullptr;
    double *r = nullptr, *rho = nullptr, *th = nullptr, *gmob = nullptr, *partial = nullptr, *red = nullptr;
    double *h_in = nullptr, *h_out = nullptr;  // pinned: parameters in, sums and mobility gradient out
    // the forward pass and the gradient as CUDA graphs (captured at first use)
    cudaGraphExec_t g_fwd = nullptr, g_grad = nullptr;
    uint64_t fwd_launches = 0, grad_launches = 0;
    double *vout = nullptr;
    int8_t* o = nullptr;
    uint8_t* proj = nullptr;
    double* er = nullptr;    // 3 real eigenstrain fields
    double2* eh = nullptr;   // 3 half spectra
    double* st = nullptr;    // 3 real strain fields
    unsigned* cnt = nullptr; // last-block counters of the reductions
};

template <typename T>
static int adj_alloc(gpk_adjoint* a, T** p, size_t count) {
    void* q = nullptr;
    if (cudaMalloc(&q, sizeof(T) * (count ? count : 1)) != cudaSuccess) {
        cudaGetLastError();
        gpk_set_error("adjoint: cudaMalloc failed");
        return GPK_ERR_OUT_OF_MEMORY;
    }
    a->mem.push_back(q);
    *p = (T*)q;
    return GPK_OK;
}

static void adj_free(gpk_adjoint* a) {
    if (a->g_fwd) cudaGraphExecDestroy(a->g_fwd);
    if (a->g_grad) cudaGraphExecDestroy(a->g_grad);
    cudaFreeHost(a->h_in);
    cudaFreeHost(a->h_out);
    if (a->have_plan) cufftDestroy(a->plan);
    if (a->have_iplan) cufftDestroy(a->iplan);
    for (void* p : a->mem) cudaFree(p);
    a->mem.clear();
}

extern "C" int gpk_adjoint_create(gpk_grid* G, int n_labels, const int32_t* mob_index, int n_mob, double m_fixed,
                                  double sigma0, double c11, double c12, double c44, double energy_weight,
                                  gpk_adjoint** out) {
    if (!out || !G || !mob_index || n_labels < 1 || n_mob < 0) {
        gpk_set_error("adjoint: null argument or empty label table");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    if (G->d.is3d() || G->precision != GPK_PREC_F64 || G->d.Nx < 3 || G->d.Ny < 3) {
        gpk_set_error("adjoint: needs a 2-D GPK_PREC_F64 grid of at least 3 x 3 cells");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    for (int l = 0; l < n_labels; ++l)
        if (mob_index[l] < -1 || mob_index[l] >= n_mob) {
            gpk_set_error("adjoint: mob_index entries must lie in [-1, n_mob)");
            return GPK_ERR_INVALID_ARGUMENT;
        }
    const Dims D = G->d;
    std::vector<int32_t> phi(D.N);
    ADJ_CUDA_TRY(cudaMemcpy(phi.data(), G->phi, sizeof(int32_t) * D.N, cudaMemcpyDeviceToHost));
    for (int32_t l : phi)
        if (l < 0 || l >= n_labels) {
            gpk_set_error("adjoint: a label of the grid lies outside the mobility table");
            return GPK_ERR_LABEL_RANGE;
        }
    GPK_TRY(gpk_grid_geometry(G));
    GPK_TRY(gpk_sync_scalars(G));
    gpk_adjoint* a = new gpk_adjoint();
    a->G = G;
    a->n_labels = n_labels;
    a->n_mob = n_mob;
    a->na = (int)G->h_scal->n_active;
    AdjC& c = a->c;
    c.Nx = D.Nx; c.Ny = D.Ny; c.N = D.N;
    c.Hx = D.Nx / 2 + 1;
    c.Nh = (long long)D.Ny * c.Hx;
    c.vx = 1.0 / (D.Nx * G->dx);
    c.vy = 1.0 / (D.Ny * G->dx);
    c.c11 = c11; c.c12 = c12; c.c44 = c44;
    c.dx2 = G->dx * G->dx;
    c.wE = energy_weight;
    c.sigma0 = sigma0;
    c.m_fixed = m_fixed;
    c.R = ((HostKernels<double>*)G->host_kernels)->proj_radius;
    long long nb = (D.N + 255) / 256;
    a->nblocks = (int)std::min<long long>(nb, (long long)G->num_sms * 4);
    auto fail = [&](int rc) { adj_free(a); delete a; return rc; };
    const size_t N = D.N, na = a->na;
    int rc = GPK_OK;
#define ADJ_A(p, n) if ((rc = adj_alloc(a, &a->p, (n))) != GPK_OK) return fail(rc)
    ADJ_A(mob_label, n_labels); ADJ_A(act, na); ADJ_A(mobp, na); ADJ_A(qn, N); ADJ_A(csr_off, n_mob + 1);
    ADJ_A(csr_pos, na); ADJ_A(kap, na); ADJ_A(cm, 4 * na); ADJ_A(eta, N); ADJ_A(target, N); ADJ_A(de, 3 * N);
    ADJ_A(en, N); ADJ_A(vr, N); ADJ_A(qf, N); ADJ_A(lam, N); ADJ_A(mu, N); ADJ_A(B, na); ADJ_A(v, na);
    ADJ_A(Dn, na); ADJ_A(r, na); ADJ_A(rho, na); ADJ_A(th, 7 + n_mob); ADJ_A(gmob, n_mob);
    ADJ_A(partial, (size_t)a->nblocks * 8); ADJ_A(red, 32); ADJ_A(vout, N); ADJ_A(o, na); ADJ_A(proj, na);
    ADJ_A(er, 3 * N); ADJ_A(eh, 3 * (size_t)c.Nh); ADJ_A(st, 3 * N); ADJ_A(cnt, 8);
#undef ADJ_A
    if (cudaMallocHost((void**)&a->h_in, sizeof(double) * (7 + n_mob)) != cudaSuccess ||
        cudaMallocHost((void**)&a->h_out, sizeof(double) * (32 + n_mob)) != cudaSuccess) {
        cudaGetLastError();
        gpk_set_error("adjoint: pinned host buffers could not be allocated");
        return fail(GPK_ERR_OUT_OF_MEMORY);
    }
    cudaStream_t st = G->stream;
    if (cudaMemcpyAsync(a->mob_label, mob_index, sizeof(int32_t) * n_labels, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(a->act, G->active, sizeof(int32_t) * na, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
        cudaMemsetAsync(a->qn, 0xff, sizeof(int32_t) * N, st) != cudaSuccess ||
        cudaMemsetAsync(a->target, 0, sizeof(double) * N, st) != cudaSuccess ||
        cudaMemsetAsync(a->vr, 0, sizeof(double) * N, st) != cudaSuccess ||
        cudaMemsetAsync(a->cnt, 0, sizeof(unsigned) * 8, st) != cudaSuccess) {
        gpk_set_error("adjoint: set-up copies failed");
        return fail(GPK_ERR_CUDA);
    }
    a->A = Act{a->act, a->mobp, a->kap, a->cm, a->o, a->proj, a->na};
    a->L = Labels{G->phi, G->phi_comp, G->mask, G->d_proj_w};
    const int grid = a->nblocks;
    if (na > 0)
        k_adj_prep<<<grid, 256, 0, st>>>(c, a->A, G->phi, G->phi_comp, (const double*)G->f[GPK_FIELD_NX],
                                         (const double*)G->f[GPK_FIELD_NY], (const double*)G->f[GPK_FIELD_G],
                                         (const double*)G->f[GPK_FIELD_KAPPA], a->mob_label, a->qn, a->kap, a->cm,
                                         a->o, a->proj, a->mobp);
    k_adj_eta<<<grid, 256, 0, st>>>(c.N, G->phi, a->mob_label, a->eta);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess) {
        gpk_set_error("adjoint: set-up kernels failed");
        return fail(GPK_ERR_CUDA);
    }
    // interface positions grouped by mobility parameter, in position order
    std::vector<int32_t> mp(na);
    if (na && cudaMemcpy(mp.data(), a->mobp, sizeof(int32_t) * na, cudaMemcpyDeviceToHost) != cudaSuccess) {
        gpk_set_error("adjoint: copy of mobility indices failed");
        return fail(GPK_ERR_CUDA);
    }
    std::vector<int32_t> off(n_mob + 1, 0), pos;
    for (int32_t p : mp)
        if (p >= 0) off[p + 1]++;
    for (int p = 0; p < n_mob; ++p) off[p + 1] += off[p];
    pos.resize(off[n_mob]);
    std::vector<int32_t> fill(off.begin(), off.end() - 1);
    for (int k = 0; k < (int)na; ++k)
        if (mp[k] >= 0) pos[fill[mp[k]]++] = k;
    if (cudaMemcpy(a->csr_off, off.data(), sizeof(int32_t) * (n_mob + 1), cudaMemcpyHostToDevice) != cudaSuccess ||
        (!pos.empty() &&
         cudaMemcpy(a->csr_pos, pos.data(), sizeof(int32_t) * pos.size(), cudaMemcpyHostToDevice) != cudaSuccess)) {
        gpk_set_error("adjoint: copy of the mobility lists failed");
        return fail(GPK_ERR_CUDA);
    }
    int dims[2] = {D.Ny, D.Nx};
    if (cufftPlanMany(&a->plan, 2, dims, nullptr, 1, (int)N, nullptr, 1, (int)c.Nh, CUFFT_D2Z, 3) != CUFFT_SUCCESS) {
        gpk_set_error("adjoint: cufftPlanMany (D2Z) failed");
        return fail(GPK_ERR_CUDA);
    }
    a->have_plan = true;
    if (cufftPlanMany(&a->iplan, 2, dims, nullptr, 1, (int)c.Nh, nullptr, 1, (int)N, CUFFT_Z2D, 3) != CUFFT_SUCCESS) {
        gpk_set_error("adjoint: cufftPlanMany (Z2D) failed");
        return fail(GPK_ERR_CUDA);
    }
    a->have_iplan = true;
    *out = a;
    return GPK_OK;
}

extern "C" int gpk_adjoint_destroy(gpk_adjoint* a) {
    if (!a) return GPK_OK;
    cudaStreamSynchronize(a->G->stream);
    adj_free(a);
    delete a;
    return GPK_OK;
}

extern "C" int gpk_adjoint_num_params(const gpk_adjoint* a, int* n) {
    if (!a || !n) { gpk_set_error("adjoint: null argument"); return GPK_ERR_INVALID_ARGUMENT; }
    *n = 7 + a->n_mob;
    return GPK_OK;
}

extern "C" int gpk_adjoint_set_target(gpk_adjoint* a, const double* v_target) {
    if (!a || !v_target) { gpk_set_error("adjoint: null argument"); return GPK_ERR_INVALID_ARGUMENT; }
    ADJ_CUDA_TRY(cudaMemcpyAsync(a->target, v_target, sizeof(double) * a->c.N, cudaMemcpyHostToDevice, a->G->stream));
    ADJ_CUDA_TRY(cudaStreamSynchronize(a->G->stream));
    return GPK_OK;
}

// one spectral solve: mode 0 forward (eta E), mode 1 adjoint (mu de)
static int adj_solve(gpk_adjoint* a, int mode) {
    cudaStream_t st = a->G->stream;
    const int grid = a->nblocks;
    k_adj_eig<<<grid, 256, 0, st>>>(a->c, mode, a->th, a->eta, a->mu, a->de, a->er);
    ADJ_FFT_TRY(cufftSetStream(a->plan, st));
    ADJ_FFT_TRY(cufftSetStream(a->iplan, st));
    ADJ_FFT_TRY(cufftExecD2Z(a->plan, (cufftDoubleReal*)a->er, (cufftDoubleComplex*)a->eh));
    k_adj_green<<<grid, 256, 0, st>>>(a->c, a->eh);
    ADJ_FFT_TRY(cufftExecZ2D(a->iplan, (cufftDoubleComplex*)a->eh, (cufftDoubleReal*)a->st));
    k_adj_stress<<<grid, 256, 0, st>>>(a->c, mode, a->th, a->st, a->eta, a->mu, a->de, a->en, a->partial, a->cnt + mode,
                                       a->red + (mode == 0 ? 0 : 24));
    ADJ_CUDA_TRY(cudaGetLastError());
    a->G->launches += 3;
    return GPK_OK;
}

// parameters (pinned h_in) -> device, forward pass; v kept when keep_v
static int enqueue_forward(gpk_adjoint* a, bool keep_v) {
    const AdjC& c = a->c;
    cudaStream_t st = a->G->stream;
    ADJ_CUDA_TRY(cudaMemcpyAsync(a->th, a->h_in, sizeof(double) * (7 + a->n_mob), cudaMemcpyHostToDevice, st));
    GPK_TRY(adj_solve(a, 0));
    const int grid = a->nblocks;
    if (a->na > 0) {
        k_adj_velocity<<<grid, 256, 0, st>>>(c, a->A, a->qn, a->en, a->th, a->B, a->vr);
        if (keep_v) ADJ_CUDA_TRY(cudaMemsetAsync(a->vout, 0, sizeof(double) * c.N, st));
        k_adj_project<<<grid, 256, 0, st>>>(c, a->A, a->L, a->vr, a->target, a->v, a->Dn, a->r,
                                            keep_v ? a->vout : nullptr, a->partial, a->cnt + 2, a->red + 8);
        a->G->launches += 2;
    } else {
        ADJ_CUDA_TRY(cudaMemsetAsync(a->red + 8, 0, sizeof(double), st));
    }
    ADJ_CUDA_TRY(cudaGetLastError());
    return GPK_OK;
}

// the adjoint pass after a forward pass
static int enqueue_backward(gpk_adjoint* a) {
    cudaStream_t st = a->G->stream;
    const int grid = a->nblocks;
    const AdjC& c = a->c;
    ADJ_CUDA_TRY(cudaMemsetAsync(a->qf, 0, sizeof(double) * c.N, st));
    ADJ_CUDA_TRY(cudaMemsetAsync(a->lam, 0, sizeof(double) * c.N, st));
    if (a->na > 0) {
        k_adj_qfield<<<grid, 256, 0, st>>>(a->A, a->r, a->Dn, a->qf);
        k_adj_project_t<<<grid, 256, 0, st>>>(c, a->A, a->L, a->qf, a->r, a->th + 7, a->rho, a->lam, a->partial,
                                              a->cnt + 3, a->red + 16);
        a->G->launches += 2;
    } else {
        ADJ_CUDA_TRY(cudaMemsetAsync(a->red + 16, 0, 4 * sizeof(double), st));
    }
    k_adj_mu<<<grid, 256, 0, st>>>(c, a->qn, a->lam, a->mu);
    GPK_TRY(adj_solve(a, 1));
    if (a->n_mob) k_adj_mobility<<<a->n_mob, 256, 0, st>>>(a->csr_off, a->csr_pos, a->rho, a->B, a->gmob);
    ADJ_CUDA_TRY(cudaGetLastError());
    a->G->launches += 2;
    return GPK_OK;
}

// sums (and the mobility gradient) -> pinned h_out
static int enqueue_outputs(gpk_adjoint* a, bool grad) {
    cudaStream_t st = a->G->stream;
    ADJ_CUDA_TRY(cudaMemcpyAsync(a->h_out, a->red, sizeof(double) * 32, cudaMemcpyDeviceToHost, st));
    if (grad && a->n_mob)
        ADJ_CUDA_TRY(cudaMemcpyAsync(a->h_out + 32, a->gmob, sizeof(double) * a->n_mob, cudaMemcpyDeviceToHost, st));
    return GPK_OK;
}

// Captures forward (+ adjoint when grad) into a graph on the grid's stream;
// every later call is one graph launch.  The parameters are read from
// device memory that the graph's first node fills from h_in.
static int capture(gpk_adjoint* a, bool grad, cudaGraphExec_t* out, uint64_t* launches) {
    cudaStream_t st = a->G->stream;
    ADJ_CUDA_TRY(cudaStreamSynchronize(st));
    const uint64_t l0 = a->G->launches;
    ADJ_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_forward(a, false);
    if (rc == GPK_OK && grad) rc = enqueue_backward(a);
    if (rc == GPK_OK) rc = enqueue_outputs(a, grad);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(st, &g);
    if (rc != GPK_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) {
        gpk_set_error(std::string("adjoint: stream capture failed: ") + cudaGetErrorString(e));
        return GPK_ERR_CUDA;
    }
    const cudaError_t ie = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) {
        gpk_set_error(std::string("adjoint: graph instantiation failed: ") + cudaGetErrorString(ie));
        return GPK_ERR_CUDA;
    }
    *launches = a->G->launches - l0;
    return GPK_OK;
}

extern "C" int gpk_adjoint_forward(gpk_adjoint* a, const double* theta, double* loss, double* v_out) {
    if (!a || !theta) { gpk_set_error("adjoint: null argument"); return GPK_ERR_INVALID_ARGUMENT; }
    cudaStream_t st = a->G->stream;
    ADJ_CUDA_TRY(cudaStreamSynchronize(st));  // h_in / h_out are free
    std::memcpy(a->h_in, theta, sizeof(double) * (7 + a->n_mob));
    if (v_out) {
        GPK_TRY(enqueue_forward(a, true));
        GPK_TRY(enqueue_outputs(a, false));
        ADJ_CUDA_TRY(cudaMemcpyAsync(v_out, a->vout, sizeof(double) * a->c.N, cudaMemcpyDeviceToHost, st));
    } else {
        if (!a->g_fwd) GPK_TRY(capture(a, false, &a->g_fwd, &a->fwd_launches));
        ADJ_CUDA_TRY(cudaGraphLaunch(a->g_fwd, st));
        a->G->launches += a->fwd_launches;
    }
    ADJ_CUDA_TRY(cudaStreamSynchronize(st));
    if (loss) *loss = a->h_out[8] + a->c.wE * a->h_out[0];
    return GPK_OK;
}

extern "C" int gpk_adjoint_gradient(gpk_adjoint* a, const double* theta, double* loss, double* grad) {
    if (!a || !theta || !grad) { gpk_set_error("adjoint: null argument"); return GPK_ERR_INVALID_ARGUMENT; }
    cudaStream_t st = a->G->stream;
    ADJ_CUDA_TRY(cudaStreamSynchronize(st));
    std::memcpy(a->h_in, theta, sizeof(double) * (7 + a->n_mob));
    if (!a->g_grad) GPK_TRY(capture(a, true, &a->g_grad, &a->grad_launches));
    ADJ_CUDA_TRY(cudaGraphLaunch(a->g_grad, st));
    a->G->launches += a->grad_launches;
    ADJ_CUDA_TRY(cudaStreamSynchronize(st));
    const double* h = a->h_out;
    if (loss) *loss = h[8] + a->c.wE * h[0];
    grad[0] = h[24];
    grad[1] = h[25];
    grad[2] = 2.0 * h[26];
    for (int m = 0; m < 4; ++m) grad[3 + m] = h[16 + m];
    if (a->n_mob) std::memcpy(grad + 7, h + 32, sizeof(double) * a->n_mob);
    return GPK_OK;
}
