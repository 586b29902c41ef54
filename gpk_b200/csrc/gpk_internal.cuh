// gpk_internal.cuh — device-side types shared by the gpk_b200 kernels.
//
// The whole library is compiled with -fmad=false (no multiply-add
// contraction), IEEE division and square root and no flush-to-zero, so that
// float expressions written in the reference's order round exactly as the
// reference's x86-64 SSE code does.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/gpk_b200.h"

namespace gpk_dev {

// ---------------------------------------------------------------------------
// grid geometry: flat index i = (z*Ny + y)*Nx + x (include/gpk_core.hpp:266-274)
// ---------------------------------------------------------------------------
struct Dims {
    int Nz, Ny, Nx, N;
    __host__ __device__ __forceinline__ int idx(int z, int y, int x) const { return (z * Ny + y) * Nx + x; }
    __host__ __device__ __forceinline__ void decode(int i, int& z, int& y, int& x) const {
        x = i % Nx;
        y = (i / Nx) % Ny;
        z = i / (Ny * Nx);
    }
    // face neighbours in the reference's order: x-, x+, y-, y+, z-, z+
    __host__ __device__ __forceinline__ void faces(int i, int nb[6]) const {
        int z, y, x;
        decode(i, z, y, x);
        const int xm = (x == 0 ? Nx - 1 : x - 1), xp = (x == Nx - 1 ? 0 : x + 1);
        const int ym = (y == 0 ? Ny - 1 : y - 1), yp = (y == Ny - 1 ? 0 : y + 1);
        const int zm = (z == 0 ? Nz - 1 : z - 1), zp = (z == Nz - 1 ? 0 : z + 1);
        nb[0] = idx(z, y, xm); nb[1] = idx(z, y, xp);
        nb[2] = idx(z, ym, x); nb[3] = idx(z, yp, x);
        nb[4] = idx(zm, y, x); nb[5] = idx(zp, y, x);
    }
    __host__ __device__ __forceinline__ int nface() const { return Nz > 1 ? 6 : 4; }
    __host__ __device__ __forceinline__ bool is3d() const { return Nz > 1; }
};

// wrap a coordinate that may lie several periods away (reference: while loops)
__host__ __device__ __forceinline__ int wrap_any(int v, int n) {
    v %= n;
    return v < 0 ? v + n : v;
}
// wrap a coordinate at most one period away
__host__ __device__ __forceinline__ int wrap1(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

template <typename T> __host__ __device__ __forceinline__ T dmax(T a, T b) { return (a < b) ? b : a; }  // std::max
template <typename T> __host__ __device__ __forceinline__ T dmin(T a, T b) { return (b < a) ? b : a; }  // std::min
template <typename T> __host__ __device__ __forceinline__ T dclamp(T v, T lo, T hi) {            // std::clamp
    return (v < lo) ? lo : (hi < v) ? hi : v;
}

// ---------------------------------------------------------------------------
// per-step device scalars (one struct per grid, in device memory)
// ---------------------------------------------------------------------------
struct StepScalars {
    double dt;              // step taken (value of the real-typed dt)
    double time;            // grid time after the step
    double vmax;            // max |vn| over interface cells
    unsigned n_active;      // interface cells
    unsigned n_cand;        // crossing candidates
    unsigned long long accepted;   // topology_accepted_last
    unsigned long long deferred;   // topology_deferred_last
    unsigned long long exchanges;  // gaussian_remap_exchanges_last
    unsigned long long exch_pass;  // exchanges of the current remap pass
    unsigned n_prop;        // remap proposals
    unsigned n_exch;        // remap exchange slots
    unsigned pending;       // pending items of the current wave loop
    unsigned waves;         // waves used by the last wave loop
    unsigned error;         // sticky device error code (GPK_ERR_*)
    unsigned unresolved;    // unresolved labels (extinction)
    unsigned erosion_cells; // cells eroded in the current extinction layer
    unsigned ff_pool;       // flood-fill stack pool cursor
    unsigned stamp;         // flood-fill stamp cursor
    unsigned bar_count;     // grid barrier arrivals
    unsigned bar_gen;       // grid barrier generation
    unsigned wave_rem[3];   // rotating "items left" counters of a wave loop
    unsigned present_labels;  // labels with at least one cell (extinction)
    unsigned n_tasks;       // crossing candidates queued for warp-wide work
    unsigned n_near;        // near-threshold cells of the step (may exceed the list)
    // wait limits of grid_barrier: spin iterations before GPK_ERR_TIMEOUT
    // (0: the default) and phantom arrivals awaited besides the real blocks
    // (0 in normal use; gpk_grid_inject_wait_timeout sets them for one launch)
    long long spin_limit;
    unsigned bar_extra;
    unsigned pad2;
    // remap passes inside a captured step: the first pass's exchanges and
    // the gate of the second (3-D) pass
    unsigned long long exch_first, gate2;
    // instrumentation of the label-wide work (summed until read)
    unsigned long long flood_tasks, flood_cells, count_tasks, count_scanned;
    // remap scores: interface cells scored, and those summed tap by tap
    unsigned long long score_cells, score_exact;
    // remap passes ordered on the device: their exchange waves and proposals
    unsigned long long remap_waves_sum, remap_props_sum;
};

// bounded grid-wide barrier for persistent kernels launched cooperatively.
// Returns false (and records GPK_ERR_TIMEOUT) when the wait exceeds the
// iteration limit; callers then leave the kernel.
__device__ __forceinline__ bool grid_barrier(StepScalars* s, unsigned nblocks) {
    __syncthreads();
    __shared__ int ok;
    if (threadIdx.x == 0) {
        ok = 1;
        volatile unsigned* gen = &s->bar_gen;
        const unsigned g = *gen;
        __threadfence();
        const long long limit = s->spin_limit > 0 ? s->spin_limit : (1LL << 24);  // ~seconds with the back-off
        if (atomicAdd(&s->bar_count, 1u) == nblocks + s->bar_extra - 1) {
            atomicExch(&s->bar_count, 0u);
            __threadfence();
            atomicAdd(&s->bar_gen, 1u);
        } else {
            long long it = 0;
            while (*gen == g) {
                if (++it > limit) {
                    atomicCAS(&s->error, 0u, (unsigned)GPK_ERR_TIMEOUT);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

}  // namespace gpk_dev
