// gpk_init_dev.cu — the Voronoi initial condition built on the device.
//
// Same result, cell for cell, as gpk_voronoi_init (gpk_init.cpp), which
// follows the reference driver's voronoi_init (demos/gpk.cpp:51-189):
//   1. seeds: drawn on the host with the same generator (O(seeds));
//   2. k_nearest_seed: per cell, the seed at the smallest periodic
//      minimum-image squared distance, ties to the lowest seed index, by the
//      same bucketed ring search with the same exact stopping rule (the
//      answer, the minimum of (distance, index), does not depend on the
//      order in which seeds are visited);
//   3. face-connected components of each label by union-find that always
//      links to the smaller root, so a component's root is its lowest cell
//      index; a label keeps its largest component, ties to the lowest root
//      (the host discovers components in cell order);
//   4. the other cells are attached layer by layer: each layer reads the
//      previous layer's state (as the host collects, then applies), every
//      unattached cell with attached face neighbours takes the label with the
//      most such neighbours (ties to the lower label) and the orientation of
//      the first of them in face order.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <string>
#include <unordered_set>
#include <vector>

#include "gpk_grid.h"

namespace {

struct Split {
    uint64_t s;
    __host__ uint64_t next() {
        uint64_t z = (s += 0x9e3779b97f4a7c15ULL);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
        return z ^ (z >> 31);
    }
    __host__ uint32_t below(uint32_t n) {
        const uint64_t lim = (UINT64_MAX / n) * n;
        uint64_t v;
        do { v = next(); } while (v >= lim);
        return (uint32_t)(v % n);
    }
    __host__ float unit_float() { return (float)((next() >> 40) * (1.0 / 16777216.0)); }
};

struct VorArgs {
    int Nz, Ny, Nx, bs, bz, by, bx, maxring;
    const int* sz; const int* sy; const int* sx; const float* sg;
    const int* boff;   // bucket offsets (bz*by*bx + 1)
    const int* bseed;  // seed indices by bucket, ascending within a bucket
};

__device__ __forceinline__ long long pd(int a, int b, int n) {
    long long d = a > b ? (long long)a - b : (long long)b - a;
    return d < n - d ? d : n - d;
}

__global__ void k_nearest_seed(VorArgs v, int32_t* __restrict__ phi, float* __restrict__ g) {
    const long long N = (long long)v.Nz * v.Ny * v.Nx;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % v.Nx), y = (int)((i / v.Nx) % v.Ny), z = (int)(i / ((long long)v.Ny * v.Nx));
        const int cz = z / v.bs, cy = y / v.bs, cx = x / v.bs;
        long long best_d = LLONG_MAX;
        int best = 0;
        for (int r = 0;; ++r) {
            const int rz = min(r, v.bz / 2), ry = min(r, v.by / 2), rx = min(r, v.bx / 2);
            for (int dz = -rz; dz <= rz; ++dz)
                for (int dy = -ry; dy <= ry; ++dy)
                    for (int dx = -rx; dx <= rx; ++dx) {
                        if (max(abs(dz), max(abs(dy), abs(dx))) != r) continue;
                        const int qz = ((cz + dz) % v.bz + v.bz) % v.bz, qy = ((cy + dy) % v.by + v.by) % v.by,
                                  qx = ((cx + dx) % v.bx + v.bx) % v.bx;
                        const int b = (qz * v.by + qy) * v.bx + qx;
                        for (int e = v.boff[b]; e < v.boff[b + 1]; ++e) {
                            const int k = v.bseed[e];
                            const long long ddz = pd(z, v.sz[k], v.Nz), ddy = pd(y, v.sy[k], v.Ny), ddx = pd(x, v.sx[k], v.Nx);
                            const long long d = ddz * ddz + ddy * ddy + ddx * ddx;
                            if (d < best_d || (d == best_d && k < best)) { best_d = d; best = k; }
                        }
                    }
            const long long reach = (long long)(r - 1) * v.bs;
            if (r >= v.maxring || (r >= 1 && best_d < LLONG_MAX && best_d < reach * reach)) break;
        }
        phi[i] = best + 1;
        if (g) g[i] = v.sg[best];
    }
}

__device__ __forceinline__ void face_cells(const gpk_dev::Dims& D, long long i, long long nb[6]) {
    int z, y, x;
    D.decode((int)i, z, y, x);
    const int xm = x == 0 ? D.Nx - 1 : x - 1, xp = x == D.Nx - 1 ? 0 : x + 1;
    const int ym = y == 0 ? D.Ny - 1 : y - 1, yp = y == D.Ny - 1 ? 0 : y + 1;
    const int zm = z == 0 ? D.Nz - 1 : z - 1, zp = z == D.Nz - 1 ? 0 : z + 1;
    nb[0] = D.idx(z, y, xm); nb[1] = D.idx(z, y, xp); nb[2] = D.idx(z, ym, x);
    nb[3] = D.idx(z, yp, x); nb[4] = D.idx(zm, y, x); nb[5] = D.idx(zp, y, x);
}

// Parents only decrease, so a root walk ends within N steps and a failed
// link means another thread linked first; the loops are capped all the same
// (the cap sets *err).  Reads go to L2: other SMs change parents atomically.
constexpr int UF_CAP = 1 << 26;

__device__ __forceinline__ int find_root(int* parent, int i, unsigned* err) {
    for (int it = 0; it < UF_CAP; ++it) {
        const int p = __ldcg(&parent[i]);
        if (p == i) return i;
        const int gp = __ldcg(&parent[p]);
        if (gp != p) atomicMin(&parent[i], gp);  // path halving
        i = p;
    }
    atomicExch(err, 1u);
    return i;
}

// union of the components of a and b: the larger root is linked to the smaller
__device__ void unite(int* parent, int a, int b, unsigned* err) {
    for (int it = 0; it < UF_CAP; ++it) {
        a = find_root(parent, a, err);
        b = find_root(parent, b, err);
        if (a == b) return;
        const int lo = a < b ? a : b, hi = a < b ? b : a;
        const int old = atomicCAS(&parent[hi], hi, lo);
        if (old == hi) return;
        a = lo;
        b = old;
    }
    atomicExch(err, 1u);
}

__global__ void k_cc_init(long long N, int* __restrict__ parent) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
        parent[i] = (int)i;
}

__global__ void k_cc_union(gpk_dev::Dims D, const int32_t* __restrict__ phi, int* parent, unsigned* err) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < D.N; i += (long long)gridDim.x * blockDim.x) {
        long long nb[6];
        face_cells(D, i, nb);
        const int32_t l = phi[i];
        // +x, +y, +z faces (the others are the neighbours' + faces)
        const int pos[3] = {1, 3, 5};
        for (int q = 0; q < (D.is3d() ? 3 : 2); ++q)
            if (phi[nb[pos[q]]] == l && nb[pos[q]] != i) unite(parent, (int)i, (int)nb[pos[q]], err);
    }
}

// root of every cell; component sizes; per label the largest component
// (key = size << 32 | (2^32 - 1 - root): the larger size, then the lower root)
__global__ void k_cc_finish(long long N, int* parent, unsigned* __restrict__ size, unsigned* err) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        const int r = find_root(parent, (int)i, err);
        parent[i] = r;
        atomicAdd(&size[r], 1u);
    }
}
__global__ void k_cc_largest(long long N, const int32_t* __restrict__ phi, const int* __restrict__ root,
                             const unsigned* __restrict__ size, unsigned long long* __restrict__ best) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
        if (root[i] == (int)i) {
            const unsigned long long key = ((unsigned long long)size[i] << 32) | (0xffffffffull - (unsigned)i);
            atomicMax(&best[phi[i]], key);
        }
}
__global__ void k_cc_attached(long long N, const int32_t* __restrict__ phi, const int* __restrict__ root,
                              const unsigned long long* __restrict__ best, uint8_t* __restrict__ att,
                              unsigned* __restrict__ n_att) {
    unsigned local = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        const unsigned keep = 0xffffffffu - (unsigned)(best[phi[i]] & 0xffffffffull);
        const uint8_t a = (unsigned)root[i] == keep;
        att[i] = a;
        local += a;
    }
    local = __reduce_add_sync(0xffffffffu, local);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd(n_att, local);
}

// one attachment layer: reads (phi, g, att), writes (phi2, g2, att2)
__global__ void k_attach_layer(gpk_dev::Dims D, const int32_t* __restrict__ phi, const float* __restrict__ g,
                               const uint8_t* __restrict__ att, int32_t* __restrict__ phi2, float* __restrict__ g2,
                               uint8_t* __restrict__ att2, unsigned* __restrict__ added) {
    unsigned local = 0;
    const int nface = D.is3d() ? 6 : 4;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < D.N; i += (long long)gridDim.x * blockDim.x) {
        int32_t lab = phi[i];
        float gi = g ? g[i] : 0.f;
        uint8_t a = att[i];
        if (!a) {
            long long nb[6];
            face_cells(D, i, nb);
            int32_t cand[6];
            int support[6] = {0, 0, 0, 0, 0, 0};
            long long src[6];
            int nc = 0;
            for (int k = 0; k < nface; ++k) {
                if (!att[nb[k]]) continue;
                const int32_t v = phi[nb[k]];
                int q = 0;
                while (q < nc && cand[q] != v) ++q;
                if (q == nc) { cand[q] = v; src[q] = nb[k]; ++nc; }
                ++support[q];
            }
            if (nc > 0) {
                int best = 0;
                for (int q = 1; q < nc; ++q)
                    if (support[q] > support[best] || (support[q] == support[best] && cand[q] < cand[best])) best = q;
                lab = cand[best];
                if (g) gi = g[src[best]];
                a = 1;
                ++local;
            }
        }
        phi2[i] = lab;
        if (g2) g2[i] = gi;
        att2[i] = a;
    }
    local = __reduce_add_sync(0xffffffffu, local);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd(added, local);
}

__global__ void k_f2d(long long N, const float* __restrict__ a, double* __restrict__ b) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
        b[i] = (double)a[i];
}

}  // namespace

// The construction for a given seed list (cells distinct and in range).
static int voronoi_build(gpk_grid* G, int n_seeds, const std::vector<int>& sz, const std::vector<int>& sy,
                         const std::vector<int>& sx, const std::vector<float>& sg, int* reassigned) {
    const gpk_dev::Dims D = G->d;
    const int Nz = D.Nz, Ny = D.Ny, Nx = D.Nx;
    const long long N = D.N;
    const double cell_vol = (double)N / n_seeds;
    const int bs = std::max(1, (int)std::ceil(std::cbrt(cell_vol) * (Nz > 1 ? 1.0 : 0.0) +
                                              std::sqrt(cell_vol) * (Nz > 1 ? 0.0 : 1.0)));
    const int bz = std::max(1, (Nz + bs - 1) / bs), by = std::max(1, (Ny + bs - 1) / bs), bx = std::max(1, (Nx + bs - 1) / bs);
    const size_t nb = (size_t)bz * by * bx;
    std::vector<int> boff(nb + 1, 0), bseed(n_seeds);
    for (int k = 0; k < n_seeds; ++k) boff[((size_t)(sz[k] / bs) * by + sy[k] / bs) * bx + sx[k] / bs + 1]++;
    for (size_t b = 0; b < nb; ++b) boff[b + 1] += boff[b];
    {
        std::vector<int> fill(boff.begin(), boff.end() - 1);
        for (int k = 0; k < n_seeds; ++k) bseed[fill[((size_t)(sz[k] / bs) * by + sy[k] / bs) * bx + sx[k] / bs]++] = k;
    }
    // device scratch for the construction only, released before returning
    std::vector<void*> tmp;
    auto dalloc = [&](size_t bytes) -> void* {
        void* p = nullptr;
        if (cudaMalloc(&p, bytes) != cudaSuccess) { cudaGetLastError(); return nullptr; }
        tmp.push_back(p);
        return p;
    };
    auto cleanup = [&]() { for (void* p : tmp) cudaFree(p); };
    int* d_seed = (int*)dalloc(sizeof(int) * (3 * (size_t)n_seeds + nb + 1 + n_seeds));
    float* d_sg = (float*)dalloc(sizeof(float) * n_seeds);
    int* parent = (int*)dalloc(sizeof(int) * N);
    unsigned* csize = (unsigned*)dalloc(sizeof(unsigned) * N);
    unsigned long long* best = (unsigned long long*)dalloc(sizeof(unsigned long long) * ((size_t)n_seeds + 1));
    int32_t* phi2 = (int32_t*)dalloc(sizeof(int32_t) * N);
    float* g2 = (float*)dalloc(sizeof(float) * N);
    uint8_t* att = (uint8_t*)dalloc(N);
    uint8_t* att2 = (uint8_t*)dalloc(N);
    unsigned* counters = (unsigned*)dalloc(sizeof(unsigned) * 3);  // attached, added, union-find error
    if (!d_seed || !d_sg || !parent || !csize || !best || !phi2 || !g2 || !att || !att2 || !counters) {
        cleanup();
        gpk_set_error("voronoi: device scratch allocation failed");
        return GPK_ERR_OUT_OF_MEMORY;
    }
    cudaStream_t st = G->stream;
    int rc = GPK_OK;
    auto chk = [&](cudaError_t e) {
        if (e != cudaSuccess && rc == GPK_OK) {
            gpk_set_error(std::string("voronoi: ") + cudaGetErrorString(e));
            rc = GPK_ERR_CUDA;
        }
    };
    int* d_sz = d_seed;
    int* d_sy = d_sz + n_seeds;
    int* d_sx = d_sy + n_seeds;
    int* d_boff = d_sx + n_seeds;
    int* d_bseed = d_boff + nb + 1;
    chk(cudaMemcpyAsync(d_sz, sz.data(), sizeof(int) * n_seeds, cudaMemcpyHostToDevice, st));
    chk(cudaMemcpyAsync(d_sy, sy.data(), sizeof(int) * n_seeds, cudaMemcpyHostToDevice, st));
    chk(cudaMemcpyAsync(d_sx, sx.data(), sizeof(int) * n_seeds, cudaMemcpyHostToDevice, st));
    chk(cudaMemcpyAsync(d_boff, boff.data(), sizeof(int) * (nb + 1), cudaMemcpyHostToDevice, st));
    chk(cudaMemcpyAsync(d_bseed, bseed.data(), sizeof(int) * n_seeds, cudaMemcpyHostToDevice, st));
    chk(cudaMemcpyAsync(d_sg, sg.data(), sizeof(float) * n_seeds, cudaMemcpyHostToDevice, st));
    // 2. nearest seed (orientation as float, converted below for an FP64 grid)
    VorArgs v{Nz, Ny, Nx, bs, bz, by, bx, std::max(bz / 2, std::max(by / 2, bx / 2)), d_sz, d_sy, d_sx, d_sg, d_boff,
              d_bseed};
    const int grid = G->num_sms * 8;
    k_nearest_seed<<<grid, 256, 0, st>>>(v, G->phi, g2);
    // 3. components and the kept component of each label
    k_cc_init<<<grid, 256, 0, st>>>(N, parent);
    chk(cudaMemsetAsync(counters, 0, sizeof(unsigned) * 3, st));
    k_cc_union<<<grid, 256, 0, st>>>(D, G->phi, parent, counters + 2);
    chk(cudaMemsetAsync(csize, 0, sizeof(unsigned) * N, st));
    chk(cudaMemsetAsync(best, 0, sizeof(unsigned long long) * ((size_t)n_seeds + 1), st));
    k_cc_finish<<<grid, 256, 0, st>>>(N, parent, csize, counters + 2);
    k_cc_largest<<<grid, 256, 0, st>>>(N, G->phi, parent, csize, best);
    k_cc_attached<<<grid, 256, 0, st>>>(N, G->phi, parent, best, att, counters);
    G->launches += 6;
    chk(cudaGetLastError());
    unsigned h[3] = {0, 0, 0};
    chk(cudaMemcpyAsync(h, counters, sizeof(h), cudaMemcpyDeviceToHost, st));
    chk(cudaStreamSynchronize(st));
    if (rc == GPK_OK && h[2]) {
        gpk_set_error("voronoi: a component search exceeded its iteration cap");
        rc = GPK_ERR_INTERNAL;
    }
    const unsigned n_initial = h[0];
    unsigned n_att = h[0];
    // 4. attachment layers, double-buffered through phi2 / g2 / att2
    int32_t* pa = G->phi; int32_t* pb = phi2;
    float* ga = g2; float* gb = (float*)parent;  // parent is free now: reuse it for orientations
    uint8_t* aa = att; uint8_t* ab = att2;
    int layers = 0;
    while (rc == GPK_OK && n_att < (unsigned)N) {
        chk(cudaMemsetAsync(counters + 1, 0, sizeof(unsigned), st));
        k_attach_layer<<<grid, 256, 0, st>>>(D, pa, ga, aa, pb, gb, ab, counters + 1);
        G->launches++;
        chk(cudaGetLastError());
        chk(cudaMemcpyAsync(&h[1], counters + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
        chk(cudaStreamSynchronize(st));
        if (rc != GPK_OK) break;
        if (h[1] == 0) {
            gpk_set_error("voronoi: cells that can never be attached");
            rc = GPK_ERR_INTERNAL;
            break;
        }
        n_att += h[1];
        std::swap(pa, pb); std::swap(ga, gb); std::swap(aa, ab);
        ++layers;
    }
    if (rc == GPK_OK) {
        if (pa != G->phi) chk(cudaMemcpyAsync(G->phi, pa, sizeof(int32_t) * N, cudaMemcpyDeviceToDevice, st));
        // orientations into the grid's g field (its real type)
        if (G->precision == GPK_PREC_F64) {
            k_f2d<<<grid, 256, 0, st>>>(N, ga, (double*)G->f[GPK_FIELD_G]);
            G->launches++;
            chk(cudaGetLastError());
        } else {
            chk(cudaMemcpyAsync(G->f[GPK_FIELD_G], ga, sizeof(float) * N, cudaMemcpyDeviceToDevice, st));
        }
        chk(cudaStreamSynchronize(st));
    }
    cleanup();
    if (rc != GPK_OK) return rc;
    GPK_TRY(gpk_ensure_label_capacity(G, n_seeds + 1));
    GPK_TRY(gpk_recount_labels(G));
    GPK_CUDA_TRY(cudaStreamSynchronize(G->stream));
    if (reassigned) *reassigned = (int)((unsigned)N - n_initial);
    return GPK_OK;
}

extern "C" int gpk_grid_voronoi(gpk_grid* G, int n_seeds, uint64_t seed, int* reassigned) {
    if (!G) return GPK_ERR_INVALID_ARGUMENT;
    const int Nz = G->d.Nz, Ny = G->d.Ny, Nx = G->d.Nx;
    const long long N = G->d.N;
    if (n_seeds <= 0 || n_seeds > N || n_seeds >= (1 << 26)) {
        gpk_set_error("voronoi: need 0 < seeds <= cells and seeds < 2^26");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    // seeds, as gpk_voronoi_init draws them
    Split rng{seed};
    std::vector<int> sz(n_seeds), sy(n_seeds), sx(n_seeds);
    std::vector<float> sg(n_seeds);
    std::unordered_set<long long> used;
    used.reserve(2 * (size_t)n_seeds);
    for (int k = 0; k < n_seeds; ++k) {
        long long lin;
        do {
            sz[k] = (int)rng.below((uint32_t)Nz);
            sy[k] = (int)rng.below((uint32_t)Ny);
            sx[k] = (int)rng.below((uint32_t)Nx);
            lin = ((long long)sz[k] * Ny + sy[k]) * Nx + sx[k];
        } while (!used.insert(lin).second);
        sg[k] = rng.unit_float() * (float)(M_PI * 0.5);
    }
    return voronoi_build(G, n_seeds, sz, sy, sx, sg, reassigned);
}

extern "C" int gpk_grid_voronoi_seeds(gpk_grid* G, int n_seeds, const int* seed_z, const int* seed_y,
                                      const int* seed_x, const float* seed_g, int* reassigned) {
    if (!G || !seed_z || !seed_y || !seed_x || !seed_g) return GPK_ERR_INVALID_ARGUMENT;
    const int Nz = G->d.Nz, Ny = G->d.Ny, Nx = G->d.Nx;
    const long long N = G->d.N;
    if (n_seeds <= 0 || n_seeds > N || n_seeds >= (1 << 26)) {
        gpk_set_error("voronoi: need 0 < seeds <= cells and seeds < 2^26");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    std::vector<int> sz(seed_z, seed_z + n_seeds), sy(seed_y, seed_y + n_seeds), sx(seed_x, seed_x + n_seeds);
    std::vector<float> sg(seed_g, seed_g + n_seeds);
    std::unordered_set<long long> used;
    used.reserve(2 * (size_t)n_seeds);
    for (int k = 0; k < n_seeds; ++k) {
        if (sz[k] < 0 || sz[k] >= Nz || sy[k] < 0 || sy[k] >= Ny || sx[k] < 0 || sx[k] >= Nx) {
            gpk_set_error("voronoi: a seed lies outside the grid");
            return GPK_ERR_INVALID_ARGUMENT;
        }
        if (!used.insert(((long long)sz[k] * Ny + sy[k]) * Nx + sx[k]).second) {
            gpk_set_error("voronoi: two seeds share a cell");
            return GPK_ERR_INVALID_ARGUMENT;
        }
    }
    return voronoi_build(G, n_seeds, sz, sy, sx, sg, reassigned);
}
