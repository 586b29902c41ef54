// gpk_capi.cu — the C ABI of include/gpk_b200.h: grid lifetime, host-built
// tap tables, state transfer and diagnostics.
#include <cuda_runtime.h>

#include <atomic>

#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "gpk_grid.h"

using namespace gpk_dev;

static thread_local std::string g_last_error;
void gpk_set_error(const std::string& msg) { g_last_error = msg; }

extern "C" const char* gpk_last_error(void) { return g_last_error.c_str(); }
extern "C" const char* gpk_version(void) { return "gpk_b200 0.1 (sm_100a)"; }

// literal in the grid's real type: the float value for the reference's FP32
// arithmetic, the double value for the FP64 variant
template <typename real> static inline real L(float f, double d);
template <> inline float L<float>(float f, double) { return f; }
template <> inline double L<double>(float, double d) { return d; }

static std::atomic<bool> g_device_ok{false};

extern "C" int gpk_device_init(int device) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        gpk_set_error("no CUDA device available");
        return GPK_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= n) {
        gpk_set_error("device index out of range");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    GPK_CUDA_TRY(cudaSetDevice(device));
    cudaDeviceProp p;
    GPK_CUDA_TRY(cudaGetDeviceProperties(&p, device));
    if (p.major != 10) {
        gpk_set_error("gpk_b200 is built for sm_100a (B200); found sm_" + std::to_string(p.major) +
                      std::to_string(p.minor));
        return GPK_ERR_NO_DEVICE;
    }
    g_device_ok = true;
    return GPK_OK;
}

extern "C" void gpk_thermo_desc_init(gpk_thermo_desc* d, int32_t model) {
    std::memset(d, 0, sizeof(*d));
    d->model = model;
    d->sigma0 = 0.5f; d->eps4 = 0.f; d->M0 = 1e-8f; d->Q = 0.f; d->Rgas = 8.314f;
    d->noise_scale = 1.0f; d->kB = 1.380649e-23f;
    d->k_partition = 1.0f;
    d->elastic_smooth_iters = 8;
}

int gpk_alloc(gpk_grid* G, void** p, size_t bytes) {
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        gpk_set_error("cudaMalloc of " + std::to_string(bytes) + " bytes failed: " + cudaGetErrorString(e));
        *p = nullptr;
        return GPK_ERR_OUT_OF_MEMORY;
    }
    G->allocations.push_back(*p);
    G->device_bytes += bytes;
    return GPK_OK;
}

static void gpk_free(gpk_grid* G, void* p) {
    if (!p) return;
    auto it = std::find(G->allocations.begin(), G->allocations.end(), p);
    if (it != G->allocations.end()) G->allocations.erase(it);
    cudaFree(p);
}

__global__ static void k_fill_u32(int32_t* p, int n, int32_t v) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = v;
}
template <typename real>
__global__ static void k_fill_real(real* p, int n, real v) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = v;
}
// cells per label; the lanes of a warp holding the same label add once
__global__ static void k_histogram(int N, const int32_t* __restrict__ phi, int32_t* __restrict__ count) {
    for (int base = blockIdx.x * blockDim.x; base < N; base += gridDim.x * blockDim.x) {
        const int i = base + threadIdx.x;
        const bool v = i < N;
        const int32_t label = v ? phi[i] : -1;
        const unsigned act = __ballot_sync(0xffffffffu, v);
        if (v) {
            const unsigned grp = __match_any_sync(act, label);
            if ((threadIdx.x & 31) == __ffs(grp) - 1) atomicAdd(&count[label], (int)__popc(grp));
        }
    }
}
// out[0] = lowest cell index whose label lies outside [0, 2^26) (or ~0u),
// out[1] = largest label in range
__global__ static void k_label_scan(int N, const int32_t* __restrict__ p, unsigned* __restrict__ out) {
    unsigned bad = 0xffffffffu, mx = 0;
    for (int base = blockIdx.x * blockDim.x; base < N; base += gridDim.x * blockDim.x) {
        const int i = base + threadIdx.x;
        if (i < N) {
            const int32_t v = p[i];
            if (v < 0 || v >= (1 << 26)) bad = min(bad, (unsigned)i);
            else mx = max(mx, (unsigned)v);
        }
    }
    bad = __reduce_min_sync(0xffffffffu, bad);
    mx = __reduce_max_sync(0xffffffffu, mx);
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&out[0], bad);
        atomicMax(&out[1], mx);
    }
}

int gpk_ensure_label_capacity(gpk_grid* G, int cap) {
    if (cap <= G->label_cap) return GPK_OK;
    int nc = std::max(cap, 64);
    gpk_free(G, G->count); gpk_free(G, G->minF); gpk_free(G, G->minL); gpk_free(G, G->unres);
    gpk_free(G, G->count0); gpk_free(G, G->n_old);
    GPK_TRY(gpk_alloc(G, (void**)&G->count, sizeof(int32_t) * nc));
    GPK_TRY(gpk_alloc(G, (void**)&G->minF, sizeof(int32_t) * nc));
    GPK_TRY(gpk_alloc(G, (void**)&G->minL, sizeof(int32_t) * nc));
    GPK_TRY(gpk_alloc(G, (void**)&G->unres, nc));
    GPK_TRY(gpk_alloc(G, (void**)&G->count0, sizeof(int32_t) * nc));
    GPK_TRY(gpk_alloc(G, (void**)&G->n_old, sizeof(int32_t) * nc));
    GPK_CUDA_TRY(cudaMemsetAsync(G->n_old, 0, sizeof(int32_t) * nc, G->stream));
    k_fill_u32<<<(nc + 255) / 256, 256, 0, G->stream>>>(G->minF, nc, 0x7fffffff);
    k_fill_u32<<<(nc + 255) / 256, 256, 0, G->stream>>>(G->minL, nc, 0x7fffffff);
    G->label_cap = nc;
    return gpk_recount_labels(G);
}

int gpk_recount_labels(gpk_grid* G) {
    GPK_CUDA_TRY(cudaMemsetAsync(G->count, 0, sizeof(int32_t) * G->label_cap, G->stream));
    k_histogram<<<G->num_sms * 8, 256, 0, G->stream>>>(G->d.N, G->phi, G->count);
    G->launches++;
    GPK_CUDA_TRY(cudaGetLastError());
    return GPK_OK;
}

// ---- host-built kernels (include/gpk_core.hpp:37-55, src/gpk_geometry.cpp:12-36) ----
template <typename real>
static void gauss_kernel(real sigma, std::vector<real>& w, int& radius, real& sigma_cells) {
    sigma_cells = std::max(sigma, L<real>(0.5f, 0.5));
    sigma = sigma_cells;
    radius = (int)std::ceil(L<real>(3.5f, 3.5) * sigma);
    const int sz = 2 * radius + 1;
    w.assign(sz, (real)0);
    real sum = 0;
    for (int i = 0; i < sz; ++i) {
        const real x = (real)(i - radius);
        w[i] = std::exp(-x * x / (L<real>(2.f, 2.0) * sigma * sigma));
        sum += w[i];
    }
    for (auto& v : w) v /= sum;
}

template <typename real>
int gpk_build_tables(gpk_grid* G) {
    HostKernels<real>* hk = new HostKernels<real>();
    G->host_kernels = hk;
    const real gs = (real)G->sigma;
    gauss_kernel<real>(gs, hk->gauss_w, hk->gauss_radius, hk->gauss_sigma);
    std::vector<real> tmp;
    int r_unused;
    const real vs_in = G->d.Nz > 1 ? std::clamp(L<real>(0.375f, 0.375) * gs, L<real>(0.85f, 0.85), L<real>(3.00f, 3.00))
                                   : L<real>(0.85f, 0.85);
    const real rs_in = G->d.Nz > 1 ? std::clamp(L<real>(0.125f, 0.125) * gs, L<real>(0.70f, 0.70), L<real>(1.00f, 1.00))
                                   : L<real>(0.70f, 0.70);
    gauss_kernel<real>(vs_in, tmp, r_unused, hk->vel_sigma);
    gauss_kernel<real>(rs_in, tmp, r_unused, hk->remap_sigma);
    // derivative-of-Gaussian taps
    const int R = hk->gauss_radius + 2;
    hk->geom_radius = R;
    const int W = 2 * R + 1;
    hk->w0.assign(W, (real)0); hk->w1.assign(W, (real)0); hk->w2.assign(W, (real)0);
    const int first_offset[4] = {-2, -1, 1, 2};
    const real first_coeff[4] = {L<real>(1.f, 1.0) / L<real>(12.f, 12.0), -L<real>(8.f, 8.0) / L<real>(12.f, 12.0),
                                 L<real>(8.f, 8.0) / L<real>(12.f, 12.0), -L<real>(1.f, 1.0) / L<real>(12.f, 12.0)};
    const int second_offset[5] = {-2, -1, 0, 1, 2};
    const real second_coeff[5] = {-L<real>(1.f, 1.0) / L<real>(12.f, 12.0), L<real>(16.f, 16.0) / L<real>(12.f, 12.0),
                                  -L<real>(30.f, 30.0) / L<real>(12.f, 12.0), L<real>(16.f, 16.0) / L<real>(12.f, 12.0),
                                  -L<real>(1.f, 1.0) / L<real>(12.f, 12.0)};
    auto gat = [&](int o) -> real {
        if (o < -hk->gauss_radius || o > hk->gauss_radius) return (real)0;
        return hk->gauss_w[o + hk->gauss_radius];
    };
    for (int o = -R; o <= R; ++o) {
        const int j = o + R;
        hk->w0[j] = gat(o);
        for (int k = 0; k < 4; ++k) hk->w1[j] += first_coeff[k] * gat(o - first_offset[k]);
        for (int k = 0; k < 5; ++k) hk->w2[j] += second_coeff[k] * gat(o - second_offset[k]);
    }
    hk->global_separable = G->d.Nz > 1 && R > 18;
    // per-tap products, formed as the reference forms them: (gx*gy)*gz
    const bool is3d = G->d.Nz > 1;
    const int nz_taps = is3d ? W : 1;
    hk->geom_table.assign((size_t)nz_taps * W * W * 12, (real)0);
    for (int jz = 0; jz < nz_taps; ++jz) {
        const real gz0 = is3d ? hk->w0[jz] : (real)1;
        const real gz1 = is3d ? hk->w1[jz] : (real)0;
        const real gz2 = is3d ? hk->w2[jz] : (real)0;
        for (int jy = 0; jy < W; ++jy) {
            const real gy0 = hk->w0[jy], gy1 = hk->w1[jy], gy2 = hk->w2[jy];
            for (int jx = 0; jx < W; ++jx) {
                const real gx0 = hk->w0[jx], gx1 = hk->w1[jx], gx2 = hk->w2[jx];
                real* t = &hk->geom_table[(((size_t)jz * W + jy) * W + jx) * 12];
                // three quads: A = (Ix, Ixx, Ixy, Ixz), B = (Iy, Iyy, Ixy, Iyz),
                // C = (Iz, Izz, Ixz, Iyz); a tap whose x (y, z) Gaussian factor is
                // zero needs quad A (B, C) alone
                volatile real p;  // keep each product a separate rounded operation
                real ix, iy, ixx, iyy, ixy, iz, izz, ixz, iyz;
                p = gx1 * gy0; ix = p * gz0;
                p = gx0 * gy1; iy = p * gz0;
                p = gx2 * gy0; ixx = p * gz0;
                p = gx0 * gy2; iyy = p * gz0;
                p = gx1 * gy1; ixy = p * gz0;
                p = gx0 * gy0; iz = p * gz1;
                p = gx0 * gy0; izz = p * gz2;
                p = gx1 * gy0; ixz = p * gz1;
                p = gx0 * gy1; iyz = p * gz1;
                t[0] = ix; t[1] = ixx; t[2] = ixy; t[3] = ixz;
                t[4] = iy; t[5] = iyy; t[6] = ixy; t[7] = iyz;
                t[8] = iz; t[9] = izz; t[10] = ixz; t[11] = iyz;
            }
        }
    }
    // projection / remap weights by squared distance
    auto weights = [&](real s, int& radius, std::vector<double>& w) {
        radius = std::max(1, (int)std::ceil(L<real>(3.f, 3.0) * s));
        const real inv_two_sigma2 = L<real>(0.5f, 0.5) / (s * s);
        const int r2max = 3 * radius * radius;
        w.assign(r2max + 1, 0.0);
        for (int r2 = 0; r2 <= r2max; ++r2) {
            const real rr = (real)r2;
            w[r2] = (double)std::exp(-rr * inv_two_sigma2);
        }
    };
    weights(hk->vel_sigma, hk->proj_radius, hk->proj_w);
    weights(hk->remap_sigma, hk->remap_radius, hk->remap_w);
    // upload
    GPK_TRY(gpk_alloc(G, &G->d_geom_table, sizeof(real) * hk->geom_table.size()));
    GPK_CUDA_TRY(cudaMemcpy(G->d_geom_table, hk->geom_table.data(), sizeof(real) * hk->geom_table.size(),
                            cudaMemcpyHostToDevice));
    GPK_TRY(gpk_alloc(G, &G->d_gauss, sizeof(real) * hk->gauss_w.size()));
    GPK_CUDA_TRY(cudaMemcpy(G->d_gauss, hk->gauss_w.data(), sizeof(real) * hk->gauss_w.size(), cudaMemcpyHostToDevice));
    GPK_TRY(gpk_alloc(G, (void**)&G->d_proj_w, sizeof(double) * hk->proj_w.size()));
    GPK_CUDA_TRY(cudaMemcpy(G->d_proj_w, hk->proj_w.data(), sizeof(double) * hk->proj_w.size(), cudaMemcpyHostToDevice));
    if (hk->remap_radius == 3) {
        // rows of the remap screening table, summed as the screening kernel
        // reads them: bit j of a pattern is tap x-offset j - 3, ascending
        const int r2s[10] = {0, 1, 2, 4, 5, 8, 9, 10, 13, 18};
        std::vector<double> rt(10 * 128);
        for (int k = 0; k < 10; ++k)
            for (int p = 0; p < 128; ++p) {
                double sum = 0.0;
                for (int j = 0; j < 7; ++j)
                    if (p & (1 << j)) sum += hk->remap_w[r2s[k] + (j - 3) * (j - 3)];
                rt[k * 128 + p] = sum;
            }
        GPK_TRY(gpk_alloc(G, (void**)&G->d_remap_rtab, sizeof(double) * rt.size()));
        GPK_CUDA_TRY(cudaMemcpy(G->d_remap_rtab, rt.data(), sizeof(double) * rt.size(), cudaMemcpyHostToDevice));
    }
    GPK_TRY(gpk_alloc(G, (void**)&G->d_remap_w, sizeof(double) * hk->remap_w.size()));
    GPK_CUDA_TRY(cudaMemcpy(G->d_remap_w, hk->remap_w.data(), sizeof(double) * hk->remap_w.size(),
                            cudaMemcpyHostToDevice));
    return GPK_OK;
}

template <typename real>
static int init_fields(gpk_grid* G) {
    const int N = G->d.N;
    const int gN = std::min((N + 255) / 256, G->num_sms * 8);
    struct Init { int f; double v; };
    const Init inits[] = {{GPK_FIELD_ALPHA, 1.0}, {GPK_FIELD_T, 800.0}};
    for (int f = 0; f < GPK_NUM_FIELDS; ++f)
        if (G->f[f]) GPK_CUDA_TRY(cudaMemsetAsync(G->f[f], 0, G->rsz * N, G->stream));
    for (const Init& in : inits) k_fill_real<real><<<gN, 256, 0, G->stream>>>((real*)G->f[in.f], N, (real)in.v);
    GPK_CUDA_TRY(cudaMemsetAsync(G->phi, 0, sizeof(int32_t) * N, G->stream));
    GPK_CUDA_TRY(cudaMemsetAsync(G->phi_comp, 0, sizeof(int32_t) * N, G->stream));
    GPK_CUDA_TRY(cudaMemsetAsync(G->mask, 0, N, G->stream));
    k_fill_u32<<<gN, 256, 0, G->stream>>>(G->pmap, N, -1);
    // flood-fill visit marks: stamps start at 1, so 0 means "never visited"
    GPK_CUDA_TRY(cudaMemsetAsync(G->stamp, 0, sizeof(uint32_t) * N, G->stream));
    GPK_CUDA_TRY(cudaMemsetAsync(G->stamp_rev, 0, sizeof(uint32_t) * N, G->stream));
    GPK_CUDA_TRY(cudaGetLastError());
    return GPK_OK;
}

static int validate_thermo(const gpk_thermo_desc* t) {
    if (!t) { gpk_set_error("thermo descriptor is null"); return GPK_ERR_INVALID_ARGUMENT; }
    if (t->model < 0 || t->model >= GPK_NUM_MODELS) {
        gpk_set_error("unknown thermodynamic model tag " + std::to_string(t->model));
        return GPK_ERR_UNSUPPORTED_MODEL;
    }
    if (t->model == GPK_MODEL_PRECIPITATION && (t->p[0] < 0 || t->p[0] > GPK_MAX_PHASES)) {
        gpk_set_error("PrecipitationThermo: at most 8 phases");
        return GPK_ERR_UNSUPPORTED_MODEL;
    }
    return GPK_OK;
}

extern "C" int gpk_grid_create(int Nz, int Ny, int Nx, double dx, const gpk_thermo_desc* thermo, double D,
                               double gaussian_sigma, int precision, gpk_grid** out) {
    if (!out) { gpk_set_error("out is null"); return GPK_ERR_INVALID_ARGUMENT; }
    *out = nullptr;
    if (Nz < 1 || Ny < 1 || Nx < 1 || (long long)Nz * Ny * Nx >= (1LL << 30)) {
        gpk_set_error("grid dimensions must be positive with fewer than 2^30 cells");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    if (precision != GPK_PREC_F32 && precision != GPK_PREC_F64) {
        gpk_set_error("precision must be GPK_PREC_F32 or GPK_PREC_F64");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    GPK_TRY(validate_thermo(thermo));
    if (!g_device_ok) GPK_TRY(gpk_device_init(0));
    gpk_grid* G = new gpk_grid();
    G->d = Dims{Nz, Ny, Nx, Nz * Ny * Nx};
    G->precision = precision;
    G->rsz = precision == GPK_PREC_F32 ? 4 : 8;
    G->dx = dx; G->D = D; G->sigma = gaussian_sigma;
    G->th = *thermo;
    cudaGetDevice(&G->device);
    cudaDeviceGetAttribute(&G->num_sms, cudaDevAttrMultiProcessorCount, G->device);
    int rc = GPK_OK;
    auto fail = [&](int code) {
        gpk_grid_destroy(G);
        return code;
    };
    if (cudaStreamCreateWithFlags(&G->stream, cudaStreamNonBlocking) != cudaSuccess) {
        gpk_set_error("cudaStreamCreate failed");
        return fail(GPK_ERR_CUDA);
    }
    const size_t N = G->d.N;
    const size_t rb = G->rsz * N;
#define ALLOC(ptr, bytes) do { if ((rc = gpk_alloc(G, (void**)&(ptr), (bytes))) != GPK_OK) return fail(rc); } while (0)
    ALLOC(G->phi, 4 * N);
    ALLOC(G->phi_comp, 4 * N);
    ALLOC(G->mask, N);
    for (int f = 0; f < GPK_NUM_FIELDS; ++f) {
        if (f == GPK_FIELD_PHI || f == GPK_FIELD_PHI_COMP || f == GPK_FIELD_MASK) continue;
        ALLOC(G->f[f], rb);
    }
    ALLOC(G->vn2, rb);
    ALLOC(G->c_new, rb);
    ALLOC(G->active, 4 * N);
    G->ntiles = (int)((N + 2047) / 2048);
    ALLOC(G->tile_off, 4 * (size_t)(2 * G->ntiles + 8));
    ALLOC(G->alpha_new_a, rb + 16);
    ALLOC(G->cand, 4 * N);
    ALLOC(G->cand_info, 16 * N);
    ALLOC(G->pmap, 4 * N);
    ALLOC(G->stamp, 4 * N);
    ALLOC(G->stamp_rev, 4 * N);
    ALLOC(G->ff_stack, 4 * (5 * N + 64));  // flood-fill queues: cells + search ids
    ALLOC(G->near_list, 4 * (size_t)N);    // near-threshold cells of the last step
    ALLOC(G->bgr_res, rb);
    ALLOC(G->bgr_best, rb);
    ALLOC(G->key_a, 8 * N);
    ALLOC(G->key_b, 8 * N);
    ALLOC(G->val_a, 4 * N);
    ALLOC(G->val_b, 4 * N);
    ALLOC(G->upload_check, 2 * sizeof(unsigned));
    ALLOC(G->exch, 16 * N);
    ALLOC(G->ero_target, 4 * N);
    ALLOC(G->ero_g, rb);
    ALLOC(G->scal, sizeof(StepScalars));
    {
        size_t b1 = 0, b2 = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, b1, (const unsigned long long*)nullptr, (unsigned long long*)nullptr,
                                        (const int32_t*)nullptr, (int32_t*)nullptr, (int)N, 0, 64);
        cub::DeviceRadixSort::SortPairs(nullptr, b2, (const int32_t*)nullptr, (int32_t*)nullptr,
                                        (const unsigned long long*)nullptr, (unsigned long long*)nullptr, (int)N, 0, 32);
        G->cub_tmp_bytes = std::max(b1, b2) + 256;
        ALLOC(G->cub_tmp, G->cub_tmp_bytes);
    }
#undef ALLOC
    if (cudaMallocHost((void**)&G->h_scal, sizeof(StepScalars)) != cudaSuccess) {
        gpk_set_error("cudaMallocHost failed");
        return fail(GPK_ERR_OUT_OF_MEMORY);
    }
    std::memset(G->h_scal, 0, sizeof(StepScalars));
    if (cudaMemsetAsync(G->scal, 0, sizeof(StepScalars), G->stream) != cudaSuccess) return fail(GPK_ERR_CUDA);
    rc = precision == GPK_PREC_F32 ? gpk_build_tables<float>(G) : gpk_build_tables<double>(G);
    if (rc != GPK_OK) return fail(rc);
    bool sep = precision == GPK_PREC_F32 ? ((HostKernels<float>*)G->host_kernels)->global_separable
                                         : ((HostKernels<double>*)G->host_kernels)->global_separable;
    if (sep) {
        if ((rc = gpk_alloc(G, &G->sep_I, rb)) || (rc = gpk_alloc(G, &G->sep_t1, rb)) ||
            (rc = gpk_alloc(G, &G->sep_t2, rb)) || (rc = gpk_alloc(G, &G->sep_S, rb)))
            return fail(rc);
    }
    rc = precision == GPK_PREC_F32 ? init_fields<float>(G) : init_fields<double>(G);
    if (rc != GPK_OK) return fail(rc);
    if ((rc = gpk_ensure_label_capacity(G, 64)) != GPK_OK) return fail(rc);
    if (cudaStreamSynchronize(G->stream) != cudaSuccess) {
        gpk_set_error(std::string("grid initialisation failed: ") + cudaGetErrorString(cudaGetLastError()));
        return fail(GPK_ERR_CUDA);
    }
    *out = G;
    return GPK_OK;
}

extern "C" int gpk_grid_destroy(gpk_grid* G) {
    if (!G) return GPK_OK;
    if (G->stream) cudaStreamSynchronize(G->stream);
    gpk_grid_graph_release(G);
    for (void* p : G->allocations) cudaFree(p);
    G->allocations.clear();
    if (G->h_scal) cudaFreeHost(G->h_scal);
    if (G->stream) cudaStreamDestroy(G->stream);
    if (G->host_kernels) {
        if (G->precision == GPK_PREC_F32) delete (HostKernels<float>*)G->host_kernels;
        else delete (HostKernels<double>*)G->host_kernels;
    }
    delete G;
    return GPK_OK;
}

extern "C" int gpk_grid_set_thermo(gpk_grid* G, const gpk_thermo_desc* thermo) {
    if (!G) return GPK_ERR_INVALID_ARGUMENT;
    GPK_TRY(validate_thermo(thermo));
    G->th = *thermo;
    return GPK_OK;
}

static int check_field(gpk_grid* G, int field, size_t count) {
    if (!G) { gpk_set_error("grid is null"); return GPK_ERR_INVALID_ARGUMENT; }
    if (field < 0 || field >= GPK_NUM_FIELDS) {
        gpk_set_error("unknown field id " + std::to_string(field));
        return GPK_ERR_INVALID_ARGUMENT;
    }
    if (count != (size_t)G->d.N) {
        gpk_set_error("field transfer of " + std::to_string(count) + " elements; the grid has " +
                      std::to_string(G->d.N));
        return GPK_ERR_INVALID_ARGUMENT;
    }
    return GPK_OK;
}

static void* field_ptr(gpk_grid* G, int field, size_t* esz) {
    switch (field) {
    case GPK_FIELD_PHI: *esz = 4; return G->phi;
    case GPK_FIELD_PHI_COMP: *esz = 4; return G->phi_comp;
    case GPK_FIELD_MASK: *esz = 1; return G->mask;
    default: *esz = G->rsz; return G->f[field];
    }
}

extern "C" int gpk_grid_upload(gpk_grid* G, int field, const void* host, size_t count) {
    GPK_TRY(check_field(G, field, count));
    if (!host) { gpk_set_error("host pointer is null"); return GPK_ERR_INVALID_ARGUMENT; }
    size_t esz;
    void* dst = field_ptr(G, field, &esz);
    if (field == GPK_FIELD_PHI || field == GPK_FIELD_PHI_COMP) {
        // labels are staged in scratch and checked on the device; the field is
        // written only when every label lies in range
        const int32_t* p = (const int32_t*)host;
        GPK_CUDA_TRY(cudaMemcpyAsync(G->val_a, host, esz * count, cudaMemcpyHostToDevice, G->stream));
        const unsigned init[2] = {0xffffffffu, 0u};
        GPK_CUDA_TRY(cudaMemcpyAsync(G->upload_check, init, sizeof(init), cudaMemcpyHostToDevice, G->stream));
        k_label_scan<<<G->num_sms * 8, 256, 0, G->stream>>>((int)count, G->val_a, G->upload_check);
        G->launches++;
        GPK_CUDA_TRY(cudaGetLastError());
        unsigned res[2];
        GPK_CUDA_TRY(cudaMemcpyAsync(res, G->upload_check, sizeof(res), cudaMemcpyDeviceToHost, G->stream));
        GPK_CUDA_TRY(cudaStreamSynchronize(G->stream));
        if (res[0] != 0xffffffffu) {
            gpk_set_error(std::string(field == GPK_FIELD_PHI ? "label " : "competitor label ") +
                          std::to_string(p[res[0]]) + " at cell " + std::to_string(res[0]) +
                          " lies outside [0, 2^26)");
            return GPK_ERR_LABEL_RANGE;
        }
        GPK_CUDA_TRY(cudaMemcpyAsync(dst, G->val_a, esz * count, cudaMemcpyDeviceToDevice, G->stream));
        if (field == GPK_FIELD_PHI) {
            GPK_TRY(gpk_ensure_label_capacity(G, (int)res[1] + 1));
            GPK_TRY(gpk_recount_labels(G));
        }
    } else {
        GPK_CUDA_TRY(cudaMemcpyAsync(dst, host, esz * count, cudaMemcpyHostToDevice, G->stream));
    }
    GPK_CUDA_TRY(cudaStreamSynchronize(G->stream));
    return GPK_OK;
}

extern "C" int gpk_grid_download(gpk_grid* G, int field, void* host, size_t count) {
    GPK_TRY(check_field(G, field, count));
    if (!host) { gpk_set_error("host pointer is null"); return GPK_ERR_INVALID_ARGUMENT; }
    size_t esz;
    void* src = field_ptr(G, field, &esz);
    GPK_CUDA_TRY(cudaMemcpyAsync(host, src, esz * count, cudaMemcpyDeviceToHost, G->stream));
    GPK_CUDA_TRY(cudaStreamSynchronize(G->stream));
    return GPK_OK;
}

extern "C" int gpk_grid_device_ptr(gpk_grid* G, int field, void** dev_ptr) {
    GPK_TRY(check_field(G, field, G ? (size_t)G->d.N : 0));
    size_t esz;
    *dev_ptr = field_ptr(G, field, &esz);
    return GPK_OK;
}

extern "C" int gpk_grid_get_time(gpk_grid* G, double* t) {
    if (!G || !t) return GPK_ERR_INVALID_ARGUMENT;
    GPK_TRY(gpk_sync_scalars(G));
    *t = G->h_scal->time;
    return GPK_OK;
}
extern "C" int gpk_grid_set_time(gpk_grid* G, double t) {
    if (!G) return GPK_ERR_INVALID_ARGUMENT;
    GPK_CUDA_TRY(cudaMemcpyAsync(&G->scal->time, &t, sizeof(double), cudaMemcpyHostToDevice, G->stream));
    GPK_CUDA_TRY(cudaStreamSynchronize(G->stream));
    return GPK_OK;
}
extern "C" int gpk_grid_get_step_id(gpk_grid* G, uint64_t* s) {
    if (!G || !s) return GPK_ERR_INVALID_ARGUMENT;
    *s = G->step_id;
    return GPK_OK;
}
extern "C" int gpk_grid_set_step_id(gpk_grid* G, uint64_t s) {
    if (!G) return GPK_ERR_INVALID_ARGUMENT;
    G->step_id = s;
    return GPK_OK;
}

static int step_once(gpk_grid* G, double dt, double cap) {
    return G->precision == GPK_PREC_F32 ? gpk_step_impl<float>(G, dt, cap) : gpk_step_impl<double>(G, dt, cap);
}

extern "C" int gpk_grid_step(gpk_grid* G, double dt, double dt_cap, double* dt_used) {
    if (!G) return GPK_ERR_INVALID_ARGUMENT;
    GPK_TRY(step_once(G, dt, dt_cap));
    if (dt_used) {
        GPK_TRY(gpk_sync_scalars(G));
        *dt_used = G->h_scal->dt;
    }
    return GPK_OK;
}

// ---- the step as a captured graph ---------------------------------------------
// What a captured step depends on besides device memory: the buffers the
// host swaps (two steps swap each pair back), the arguments frozen into its
// launches, and the model.
static std::vector<uint64_t> graph_signature(gpk_grid* G, double dt, double dt_cap) {
    std::vector<uint64_t> v;
    auto P = [&](const void* p) { v.push_back((uint64_t)(uintptr_t)p); };
    auto D = [&](double d) { uint64_t u; std::memcpy(&u, &d, 8); v.push_back(u); };
    for (int f = 0; f < GPK_NUM_FIELDS; ++f) P(G->f[f]);
    P(G->vn2); P(G->c_new); P(G->eps_star); P(G->eps_smooth); P(G->eps_tmp); P(G->solid_old); P(G->s_new);
    v.push_back((uint64_t)G->have_solid_old);
    D(dt); D(dt_cap); D(G->near_tol); D(G->solid_ratio); D(G->D); D(G->dx);
    v.push_back((uint64_t)G->external_elastic);
    v.push_back((uint64_t)G->geometry_kernel);
    v.push_back((uint64_t)G->tile_rows_div);
    v.push_back((uint64_t)G->label_cap);
    P(G->count);
    const uint64_t* th = reinterpret_cast<const uint64_t*>(&G->th);
    for (size_t k = 0; k < sizeof(gpk_thermo_desc) / 8; ++k) v.push_back(th[k]);
    return v;
}

void gpk_grid_graph_release(gpk_grid* G) {
    if (G->step_exec) cudaGraphExecDestroy(G->step_exec);
    if (G->step_graph) cudaGraphDestroy(G->step_graph);
    G->step_exec = nullptr;
    G->step_graph = nullptr;
    G->graph_sig.clear();
}

int gpk_grid_graph_prepare(gpk_grid* G, double dt, double dt_cap) {
    std::string why;
    if (!gpk_step_graph_supported(G, &why)) {
        gpk_set_error("captured step unsupported: " + why);
        return GPK_ERR_UNSUPPORTED_MODEL;
    }
    const std::vector<uint64_t> sig = graph_signature(G, dt, dt_cap);
    if (G->step_graph && sig == G->graph_sig) return GPK_OK;
    gpk_grid_graph_release(G);
    GPK_CUDA_TRY(cudaStreamSynchronize(G->stream));
    const uint64_t step0 = G->step_id, launches0 = G->launches;
    GPK_CUDA_TRY(cudaStreamBeginCapture(G->stream, cudaStreamCaptureModeThreadLocal));
    int rc = GPK_OK;
    for (int k = 0; k < 2 && rc == GPK_OK; ++k)
        rc = G->precision == GPK_PREC_F64 ? gpk_step_graph_body<double>(G, dt, dt_cap)
                                          : gpk_step_graph_body<float>(G, dt, dt_cap);
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(G->stream, &graph);
    G->step_id = step0;  // nothing ran yet
    G->graph_launches = G->launches - launches0;
    G->launches = launches0;
    if (rc != GPK_OK || ce != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        if (rc == GPK_OK) {
            gpk_set_error(std::string("step capture failed: ") + cudaGetErrorString(ce));
            rc = GPK_ERR_CUDA;
        }
        return rc;
    }
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
    if (ie != cudaSuccess) {
        cudaGraphDestroy(graph);
        gpk_set_error(std::string("step graph instantiation failed: ") + cudaGetErrorString(ie));
        return GPK_ERR_CUDA;
    }
    G->step_graph = graph;
    G->step_exec = exec;
    G->graph_sig = graph_signature(G, dt, dt_cap);  // two steps swap every buffer pair back
    return G->graph_sig == sig ? GPK_OK : (gpk_grid_graph_release(G), gpk_set_error("step capture left swapped buffers"),
                                           GPK_ERR_INTERNAL);
}

extern "C" int gpk_grid_step_graph(gpk_grid* G, int n, double dt, double dt_cap, double* time_out) {
    if (!G || n < 0) return GPK_ERR_INVALID_ARGUMENT;
    int done = 0;
    if (n > 0 && G->step_id == 0) {
        // the first ordinary step makes the buffers and settings a captured step relies on
        GPK_TRY(step_once(G, dt, dt_cap));
        ++done;
    }
    if (n - done >= 2) {
        GPK_TRY(gpk_grid_graph_prepare(G, dt, dt_cap));
        for (; n - done >= 2; done += 2) {
            GPK_CUDA_TRY(cudaGraphLaunch(G->step_exec, G->stream));
            G->step_id += 2;
            G->launches += G->graph_launches;
        }
    }
    for (; done < n; ++done) GPK_TRY(step_once(G, dt, dt_cap));
    GPK_TRY(gpk_sync_scalars(G));  // reports a device-side failure of any step
    if (time_out) *time_out = G->h_scal->time;
    return GPK_OK;
}

extern "C" int gpk_grid_graph_supported(gpk_grid* G, int* supported) {
    if (!G || !supported) return GPK_ERR_INVALID_ARGUMENT;
    std::string why;
    *supported = gpk_step_graph_supported(G, &why);
    if (!*supported) gpk_set_error(why);
    return GPK_OK;
}

extern "C" int gpk_grid_geometry(gpk_grid* G) {
    if (!G) return GPK_ERR_INVALID_ARGUMENT;
    return G->precision == GPK_PREC_F64 ? gpk_geometry_only<double>(G) : gpk_geometry_only<float>(G);
}

extern "C" int gpk_grid_step_n(gpk_grid* G, int n, double dt, double dt_cap, double* time_out) {
    if (!G || n < 0) return GPK_ERR_INVALID_ARGUMENT;
    for (int k = 0; k < n; ++k) GPK_TRY(step_once(G, dt, dt_cap));
    if (time_out) {
        GPK_TRY(gpk_sync_scalars(G));
        *time_out = G->h_scal->time;
    }
    return GPK_OK;
}

// GPKGrid::run without callback (src/gpk_simulation.cpp:60-73)
extern "C" int gpk_grid_run(gpk_grid* G, double t_end, double dt, int max_steps, int* steps_out) {
    if (!G) return GPK_ERR_INVALID_ARGUMENT;
    GPK_TRY(gpk_sync_scalars(G));
    int n = 0;
    while (G->h_scal->time < t_end && (max_steps <= 0 || n < max_steps)) {
        const float remaining = (float)(t_end - G->h_scal->time);
        GPK_TRY(step_once(G, dt, (double)remaining));
        GPK_TRY(gpk_sync_scalars(G));
        ++n;
    }
    if (steps_out) *steps_out = n;
    return GPK_OK;
}

extern "C" int gpk_grid_sync(gpk_grid* G) {
    if (!G) return GPK_ERR_INVALID_ARGUMENT;
    return gpk_sync_scalars(G);
}

extern "C" int gpk_grid_max_dt(gpk_grid* G, double* out) {
    if (!G || !out) return GPK_ERR_INVALID_ARGUMENT;
    return G->precision == GPK_PREC_F32 ? gpk_max_dt_impl<float>(G, out) : gpk_max_dt_impl<double>(G, out);
}

extern "C" int gpk_grid_counters(gpk_grid* G, uint64_t c[3]) {
    if (!G || !c) return GPK_ERR_INVALID_ARGUMENT;
    GPK_TRY(gpk_sync_scalars(G));
    c[0] = G->h_scal->accepted;
    c[1] = G->h_scal->deferred;
    c[2] = G->h_scal->exchanges;
    return GPK_OK;
}

extern "C" int gpk_grid_topology_simple_move(gpk_grid* G, int cell, int32_t new_label, int* result) {
    if (!G || !result) return GPK_ERR_INVALID_ARGUMENT;
    if (cell < 0 || cell >= G->d.N) { *result = 0; return GPK_OK; }
    return gpk_topology_simple_move_impl(G, cell, new_label, result);
}

extern "C" int gpk_grid_device_bytes(gpk_grid* G, size_t* out) {
    if (!G || !out) return GPK_ERR_INVALID_ARGUMENT;
    *out = G->device_bytes;
    return GPK_OK;
}

extern "C" int gpk_grid_launch_count(gpk_grid* G, uint64_t* out) {
    if (!G || !out) return GPK_ERR_INVALID_ARGUMENT;
    *out = G->launches;
    return GPK_OK;
}

// ---- diagnostics (src/gpk_simulation.cpp:78-124) ---------------------------
// phase_volume is a serial double sum in flat-index order in the reference;
// it is a diagnostic outside the step, so the state is read back and summed
// in that order.
template <typename real>
static int phase_volume_t(gpk_grid* G, int32_t label, double* out) {
    const int N = G->d.N;
    std::vector<int32_t> phi(N), pc(N);
    std::vector<uint8_t> m(N);
    std::vector<real> al(N);
    GPK_CUDA_TRY(cudaMemcpyAsync(phi.data(), G->phi, 4 * (size_t)N, cudaMemcpyDeviceToHost, G->stream));
    GPK_CUDA_TRY(cudaMemcpyAsync(pc.data(), G->phi_comp, 4 * (size_t)N, cudaMemcpyDeviceToHost, G->stream));
    GPK_CUDA_TRY(cudaMemcpyAsync(m.data(), G->mask, (size_t)N, cudaMemcpyDeviceToHost, G->stream));
    GPK_CUDA_TRY(cudaMemcpyAsync(al.data(), G->f[GPK_FIELD_ALPHA], sizeof(real) * N, cudaMemcpyDeviceToHost, G->stream));
    GPK_CUDA_TRY(cudaStreamSynchronize(G->stream));
    double v = 0.0;
    for (int i = 0; i < N; ++i) {
        if (phi[i] == label) v += al[i];
        if (m[i] && pc[i] == label && pc[i] != phi[i]) v += 1.0 - al[i];
    }
    *out = v;
    return GPK_OK;
}

extern "C" int gpk_grid_phase_volume(gpk_grid* G, int32_t label, double* out) {
    if (!G || !out) return GPK_ERR_INVALID_ARGUMENT;
    return G->precision == GPK_PREC_F32 ? phase_volume_t<float>(G, label, out) : phase_volume_t<double>(G, label, out);
}

extern "C" int gpk_grid_n_grains(gpk_grid* G, int* out) {
    if (!G || !out) return GPK_ERR_INVALID_ARGUMENT;
    std::vector<int32_t> c(G->label_cap);
    GPK_CUDA_TRY(cudaMemcpyAsync(c.data(), G->count, sizeof(int32_t) * G->label_cap, cudaMemcpyDeviceToHost, G->stream));
    GPK_CUDA_TRY(cudaStreamSynchronize(G->stream));
    int n = 0;
    for (int v : c) n += v > 0;
    *out = n;
    return GPK_OK;
}

extern "C" int gpk_grid_interface_fraction(gpk_grid* G, double* out) {
    if (!G || !out) return GPK_ERR_INVALID_ARGUMENT;
    std::vector<uint8_t> m(G->d.N);
    GPK_CUDA_TRY(cudaMemcpyAsync(m.data(), G->mask, G->d.N, cudaMemcpyDeviceToHost, G->stream));
    GPK_CUDA_TRY(cudaStreamSynchronize(G->stream));
    int cnt = 0;
    for (uint8_t v : m) cnt += v != 0;
    *out = (double)((float)cnt / (float)G->d.N);
    return GPK_OK;
}

template int gpk_build_tables<float>(gpk_grid*);
template int gpk_build_tables<double>(gpk_grid*);

extern "C" int gpk_grid_stream(gpk_grid* G, void** stream) {
    if (!G || !stream) return GPK_ERR_INVALID_ARGUMENT;
    *stream = (void*)G->stream;
    return GPK_OK;
}

extern "C" int gpk_grid_profile(gpk_grid* G, int enable) {
    if (!G) return GPK_ERR_INVALID_ARGUMENT;
    G->profile = enable != 0;
    return GPK_OK;
}

extern "C" int gpk_grid_stage_times(gpk_grid* G, double ms[GPK_NUM_STAGES], uint64_t calls[GPK_NUM_STAGES]) {
    if (!G || !ms || !calls) return GPK_ERR_INVALID_ARGUMENT;
    GPK_TRY(gpk_stage_collect(G));
    for (int k = 0; k < GPK_NUM_STAGES; ++k) {
        ms[k] = G->stage_ms[k];
        calls[k] = G->stage_calls[k];
        G->stage_ms[k] = 0;
        G->stage_calls[k] = 0;
    }
    return GPK_OK;
}

extern "C" int gpk_grid_wave_stats(gpk_grid* G, uint64_t out[10]) {
    if (!G || !out) return GPK_ERR_INVALID_ARGUMENT;
    for (int k = 0; k < 4; ++k) {
        out[k] = G->wave_stats[k];
        G->wave_stats[k] = 0;
    }
    GPK_TRY(gpk_sync_scalars(G));
    out[4] = G->h_scal->flood_tasks;
    out[5] = G->h_scal->flood_cells;
    out[6] = G->h_scal->count_tasks;
    out[7] = G->h_scal->count_scanned;
    out[8] = G->h_scal->score_cells;
    out[9] = G->h_scal->score_exact;
    out[1] += G->h_scal->remap_waves_sum;  // remap passes ordered on the device
    out[3] += G->h_scal->remap_props_sum;
    GPK_CUDA_TRY(cudaMemsetAsync(&G->scal->flood_tasks, 0, 8 * sizeof(unsigned long long), G->stream));
    return GPK_OK;
}

extern "C" int gpk_grid_set_external_elastic(gpk_grid* G, int on) {
    if (!G) return GPK_ERR_INVALID_ARGUMENT;
    G->external_elastic = on ? 1 : 0;
    return GPK_OK;
}

extern "C" int gpk_grid_set_near_threshold(gpk_grid* G, double tol) {
    if (!G || !(tol >= 0.0)) {
        gpk_set_error("near-threshold tolerance must be a number >= 0");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    G->near_tol = tol;
    return GPK_OK;
}

extern "C" int gpk_grid_near_threshold(gpk_grid* G, int32_t* cells, int cap, int* n) {
    if (!G || !n || cap < 0 || (cap > 0 && !cells)) return GPK_ERR_INVALID_ARGUMENT;
    GPK_TRY(gpk_sync_scalars(G));
    const unsigned total = G->h_scal->n_near;
    *n = (int)total;
    if (cap == 0 || total == 0) return GPK_OK;
    // every listed cell is stored (capacity N); restore increasing cell order
    std::vector<int32_t> all(total);
    GPK_CUDA_TRY(cudaMemcpyAsync(all.data(), G->near_list, sizeof(int32_t) * total, cudaMemcpyDeviceToHost,
                                 G->stream));
    GPK_CUDA_TRY(cudaStreamSynchronize(G->stream));
    std::sort(all.begin(), all.end());
    std::copy(all.begin(), all.begin() + std::min<size_t>((size_t)cap, all.size()), cells);
    return GPK_OK;
}

extern "C" int gpk_grid_set_solid_diffusivity_ratio(gpk_grid* G, double ratio) {
    if (!G || !(ratio >= 0.0 && ratio <= 1.0)) {
        gpk_set_error("solid/liquid diffusivity ratio must lie in [0, 1]");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    G->solid_ratio = ratio;
    return GPK_OK;
}

extern "C" int gpk_grid_inject_wait_timeout(gpk_grid* G, long long spin_limit) {
    if (!G || spin_limit < 1 || spin_limit > (1LL << 24)) {
        gpk_set_error("inject_wait_timeout: spin limit must lie in [1, 2^24]");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    G->inject_spin_limit = spin_limit;
    return GPK_OK;
}

extern "C" int gpk_grid_set_tile_rows(gpk_grid* G, int divisor) {
    if (!G || (divisor != 1 && divisor != 2 && divisor != 4)) {
        gpk_set_error("tile row divisor must be 1, 2 or 4");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    G->tile_rows_div = divisor;
    return GPK_OK;
}

extern "C" int gpk_grid_set_geometry_kernel(gpk_grid* G, int kind) {
    if (!G || kind < 0 || kind > 4) return GPK_ERR_INVALID_ARGUMENT;
    if (kind == 4) {
        // separable tiles: FP64 grids at kernel radii 4..10 (Gaussian radius 2..8)
        if (G->precision != GPK_PREC_F64) {
            gpk_set_error("separable tiles are an FP64 mode; FP32 grids keep the reference's arithmetic");
            return GPK_ERR_INVALID_ARGUMENT;
        }
        const HostKernels<double>* hk = (const HostKernels<double>*)G->host_kernels;
        if (hk->global_separable || hk->geom_radius < 4 || hk->geom_radius > 10) {
            gpk_set_error("separable tiles need a kernel radius of 4..10 (sigma 0.5..2.2)");
            return GPK_ERR_INVALID_ARGUMENT;
        }
    }
    G->geometry_kernel = kind;
    return GPK_OK;
}
