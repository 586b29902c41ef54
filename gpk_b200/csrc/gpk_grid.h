// gpk_grid.h — host-side state of one gpk_b200 grid and the launchers that
// the C ABI (gpk_capi.cu) strings together into GPKGrid::step().
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/gpk_b200.h"
#include "gpk_internal.cuh"

// ---- error plumbing --------------------------------------------------------
void gpk_set_error(const std::string& msg);
#define GPK_CUDA_TRY(expr)                                                              \
    do {                                                                                \
        cudaError_t _e = (expr);                                                        \
        if (_e != cudaSuccess) {                                                        \
            gpk_set_error(std::string(#expr " failed: ") + cudaGetErrorString(_e));      \
            return GPK_ERR_CUDA;                                                        \
        }                                                                               \
    } while (0)
#define GPK_TRY(expr)                 \
    do {                              \
        int _s = (expr);              \
        if (_s != GPK_OK) return _s;  \
    } while (0)

// Host-computed kernels of the reference (include/gpk_core.hpp:37-55,
// src/gpk_geometry.cpp:12-36) in the grid's real type.
template <typename real>
struct HostKernels {
    std::vector<real> gauss_w;             // GaussKernel(sigma).w
    int gauss_radius = 0;
    real gauss_sigma = 0, vel_sigma = 0, remap_sigma = 0;
    std::vector<real> w0, w1, w2;          // derivative-of-Gaussian taps
    int geom_radius = 0;
    bool global_separable = false;
    int proj_radius = 0, remap_radius = 0;
    std::vector<double> proj_w;            // weight by squared distance r2
    std::vector<double> remap_w;
    std::vector<real> geom_table;          // per tap: 12 products (see build)
};

struct gpk_grid {
    gpk_dev::Dims d{};
    int precision = GPK_PREC_F32;
    size_t rsz = 4;                        // bytes per real
    double dx = 1, D = 0, sigma = 2;
    gpk_thermo_desc th{};
    cudaStream_t stream = nullptr;
    int device = 0;
    int num_sms = 148;
    uint64_t step_id = 0;
    double time = 0;                       // host mirror (device copy in scal)
    uint64_t launches = 0;

    // public fields
    int32_t* phi = nullptr;
    int32_t* phi_comp = nullptr;
    uint8_t* mask = nullptr;
    void* f[GPK_NUM_FIELDS] = {};          // real fields by field id (phi/phi_comp/mask: null)

    // scratch
    void* vn2 = nullptr;                   // projection output before swap
    void* c_new = nullptr;
    void* eps_star = nullptr; void* eps_smooth = nullptr; void* eps_tmp = nullptr;
    void* solid_old = nullptr; void* s_new = nullptr; uint8_t* grew = nullptr;
    int have_solid_old = 0;
    int32_t* active = nullptr;             // sorted interface cells
    int32_t* tile_off = nullptr;           // compaction tile offsets
    int ntiles = 0;
    void* alpha_new_a = nullptr;           // per active position
    int32_t* cand = nullptr;               // candidate active positions
    int32_t* cand_info = nullptr;          // packed per-candidate wave state
    int32_t* pmap = nullptr;               // pending map (cell -> item) or -1
    int32_t* minF = nullptr; int32_t* minL = nullptr;
    uint32_t* stamp = nullptr; uint32_t* stamp_rev = nullptr; int32_t* ff_stack = nullptr;
    // remap
    void* bgr_res = nullptr; void* bgr_best = nullptr;   // per active position (real)
    unsigned long long* key_a = nullptr; unsigned long long* key_b = nullptr;
    int32_t* val_a = nullptr; int32_t* val_b = nullptr;
    unsigned* upload_check = nullptr;      // label range check of an upload
    int32_t* exch = nullptr;               // exchange slots: a, b, low, high, state
    void* cub_tmp = nullptr; size_t cub_tmp_bytes = 0;
    // extinction
    uint8_t* unres = nullptr; int32_t* ero_target = nullptr; void* ero_g = nullptr;
    // separable geometry
    void* sep_I = nullptr; void* sep_t1 = nullptr; void* sep_t2 = nullptr; void* sep_S = nullptr;
    // labels
    int32_t* count = nullptr;              // cells per label
    int32_t* count0 = nullptr;             // cells per label when the crossing sweep started
    int32_t* n_old = nullptr;              // crossing candidates per old label (zero between sweeps)
    int label_cap = 0;                     // labels live in [0, label_cap)
    // tables
    void* d_geom_table = nullptr; void* d_w0 = nullptr; void* d_w1 = nullptr; void* d_w2 = nullptr;
    void* d_gauss = nullptr; double* d_proj_w = nullptr; double* d_remap_w = nullptr;
    // remap screening: weight sums of the 128 patterns of a 7-tap row, for the
    // ten distinct dy^2 + dz^2 of a 7 x 7 row block (radius 3 only)
    double* d_remap_rtab = nullptr;
    gpk_dev::StepScalars* scal = nullptr;  // device scalars
    gpk_dev::StepScalars* h_scal = nullptr;  // pinned host mirror
    void* host_kernels = nullptr;          // HostKernels<real>*
    std::vector<void*> allocations;
    size_t device_bytes = 0;
    // waves of the crossing sweeps, waves of the remap exchange loops,
    // crossing candidates, remap proposals (summed since last read)
    uint64_t wave_stats[4] = {};
    // rows of a 2-D geometry tile at kernel radius 8 divided by 1, 2 or 4
    // (1024, 512 or 256 cells; gpk_grid_set_tile_rows)
    int tile_rows_div = 1;
    // geometry kernel choice: 0 = tiled (per-cell kernel where no tiled
    // instantiation exists), 1 = per-cell kernel
    int geometry_kernel = 0;
    // E_el supplied by the caller (gpk_grid_set_external_elastic)
    int external_elastic = 0;
    // near-threshold listing of the last step (gpk_grid_near_threshold):
    // cells appended by k_alpha, sorted when read; capacity N
    int32_t* near_list = nullptr;
    double near_tol = 1e-12;
    // solid/liquid diffusivity ratio of the partitioned transport (0: the reference)
    double solid_ratio = 0;
    // captured two-step graph (gpk_grid_step_graph / gpk_batch_step_graph)
    // and what it was captured with; it replays only while these still hold
    cudaGraph_t step_graph = nullptr;
    cudaGraphExec_t step_exec = nullptr;
    std::vector<uint64_t> graph_sig;
    uint64_t graph_launches = 0;           // kernel launches per replay
    // gpk_grid_inject_wait_timeout: spin limit for the next cooperative
    // launch, whose grid barrier then also awaits one block that never comes
    long long inject_spin_limit = 0;
    // stage timing (gpk_grid_profile)
    int profile = 0;
    cudaEvent_t ev[GPK_NUM_STAGES][2] = {};
    double stage_ms[GPK_NUM_STAGES] = {};
    uint64_t stage_calls[GPK_NUM_STAGES] = {};
    bool stage_open[GPK_NUM_STAGES] = {};
};

// brackets a stage with events when profiling is on; the elapsed time is
// collected at the next stream synchronisation point of the step
int gpk_stage_begin(gpk_grid* G, int stage);
int gpk_stage_end(gpk_grid* G, int stage);
int gpk_stage_collect(gpk_grid* G);

// ---- launchers (templated on the grid's real type) --------------------------
template <typename real> int gpk_build_tables(gpk_grid* G);
template <typename real> int gpk_step_impl(gpk_grid* G, double dt, double dt_cap);
template <typename real> int gpk_geometry_only(gpk_grid* G);
template <typename real> int gpk_interface_mask(gpk_grid* G, const unsigned long long* gate = nullptr);
template <typename real> int gpk_max_dt_impl(gpk_grid* G, double* out);
template <typename real> int gpk_phase_volume_impl(gpk_grid* G, int32_t label, double* out);
template <typename real>
int gpk_geometry_tiled(gpk_grid* G, int R, real inv_dx, real inv_dx2, real dx, real kappa_limit);
// FP64 separable tiles (throughput geometry); -1 when they do not apply
int gpk_geometry_sep_tiles(gpk_grid* G, int R, const double* gauss, int gauss_radius, double dx,
                           double kappa_limit);
template <typename real>
int gpk_bgr_scores_tiled(gpk_grid* G, int radius, real* res, real* best, const unsigned long long* gate = nullptr);
template <typename real> int gpk_projection_tiled(gpk_grid* G, int radius);
int gpk_recount_labels(gpk_grid* G);
int gpk_topology_simple_move_impl(gpk_grid* G, int cell, int32_t new_label, int* result);
int gpk_alloc(gpk_grid* G, void** p, size_t bytes);
int gpk_ensure_label_capacity(gpk_grid* G, int cap);
int gpk_sync_scalars(gpk_grid* G);
template <typename real> int gpk_remap_pass_graph(gpk_grid* G, const unsigned long long* gate);
template <typename real> int gpk_step_graph_body(gpk_grid* G, double dt_req, double dt_cap);
int gpk_step_graph_supported(gpk_grid* G, std::string* why);
// captures (or keeps) the grid's two-step graph for (dt, dt_cap); GPK_OK
// when G->step_graph holds a graph that replays two of its steps
int gpk_grid_graph_prepare(gpk_grid* G, double dt, double dt_cap);
void gpk_grid_graph_release(gpk_grid* G);
int gpk_remap_gates(gpk_grid* G, int stage);
