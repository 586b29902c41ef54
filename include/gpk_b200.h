/*
 * gpk_b200.h — C ABI of the B200 (sm_100a) implementation of the GPK
 * (Gaussian-Projected Kinetics) per-step hot path.
 *
 * The reference keeps its solver state in the C++ class gpk::GPKGrid
 * (include/gpk_core.hpp:205-326 of albert-hzbn/GPK) and evaluates the
 * constitutive law through virtual gpk::ThermoModel callbacks
 * (include/gpk_core.hpp:72-200).  This header is the flat boundary under that
 * class: every entry point takes plain pointers and sizes, returns an int
 * status (GPK_OK == 0) and never throws.  The C++ drop-in header
 * include/gpk_core.hpp of this repository implements GPKGrid on top of it,
 * and Python binds it with ctypes (gpk_b200/_lib.py).
 *
 * Grid layout is the reference's: flat index i = (z*Ny + y)*Nx + x, x fastest
 * (include/gpk_core.hpp:266-274).  Labels are int32.  Real-valued fields are
 * float in GPK_PREC_F32 grids and double in GPK_PREC_F64 grids.
 *
 * Threading: calls on one handle are serialised by the caller (the reference
 * has no concurrent calls on one grid either); distinct handles are
 * independent.  Each handle owns one CUDA stream.
 */
#ifndef GPK_B200_H
#define GPK_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define GPK_OK                     0
#define GPK_ERR_INVALID_ARGUMENT   1  /* bad size, null pointer, bad field id  */
#define GPK_ERR_UNSUPPORTED_MODEL  2  /* thermo model tag without device law   */
#define GPK_ERR_CUDA               3  /* a CUDA runtime call failed            */
#define GPK_ERR_OUT_OF_MEMORY      4  /* device allocation failed              */
#define GPK_ERR_LABEL_RANGE        5  /* a label lies outside [0, 2^26)        */
#define GPK_ERR_TIMEOUT            6  /* a bounded device wait gave up         */
#define GPK_ERR_NO_DEVICE          7  /* no CUDA device / wrong architecture   */
#define GPK_ERR_INTERNAL           8  /* device-side consistency check failed  */
#define GPK_ERR_INFEASIBLE         9  /* no admissible result (the reference raises) */

/* ---- arithmetic modes ---------------------------------------------------- */
/* GPK_PREC_F32: the reference's own FP32 arithmetic, operation for operation
 * (no FMA contraction, IEEE division and square root, reference tap order).
 * GPK_PREC_F64: the same algorithm with every real quantity in FP64.        */
#define GPK_PREC_F32 0
#define GPK_PREC_F64 1

/* ---- field identifiers (the public std::vector members of GPKGrid) ----- */
#define GPK_FIELD_PHI       0   /* int32  labels                 */
#define GPK_FIELD_ALPHA     1   /* real   sub-cell volume fraction */
#define GPK_FIELD_C         2   /* real   composition            */
#define GPK_FIELD_T         3   /* real   temperature            */
#define GPK_FIELD_G         4   /* real   orientation            */
#define GPK_FIELD_RHO       5   /* real   dislocation density    */
#define GPK_FIELD_NX        6   /* real   normal x               */
#define GPK_FIELD_NY        7   /* real   normal y               */
#define GPK_FIELD_NZ        8   /* real   normal z               */
#define GPK_FIELD_KAPPA     9   /* real   mean curvature         */
#define GPK_FIELD_VN       10   /* real   projected velocity     */
#define GPK_FIELD_E_EL     11   /* real   elastic energy density */
#define GPK_FIELD_PHI_COMP 12   /* int32  competitor label       */
#define GPK_FIELD_G_COMP   13   /* real   competitor orientation */
#define GPK_FIELD_MASK     14   /* uint8  interface mask         */
#define GPK_NUM_FIELDS     15

/* ---- thermodynamic model descriptor ------------------------------------- */
/* One tag per ThermoModel subclass of the reference
 * (include/gpk_thermo.hpp:18-591); GPK_MODEL_BASE is the plain ThermoModel
 * with its default virtuals (src/gpk_thermo.cpp:9-47).                     */
#define GPK_MODEL_BASE               0
#define GPK_MODEL_ISOTROPIC          1  /* IsotropicGrowthThermo       */
#define GPK_MODEL_ANISOTROPIC        2  /* AnisotropicGrowthThermo     */
#define GPK_MODEL_SOLIDIFICATION     3  /* SolidificationThermo        */
#define GPK_MODEL_RECRYSTALLISATION  4  /* RecrystallisationThermo     */
#define GPK_MODEL_DISLOCATION        5  /* DislocationThermo           */
#define GPK_MODEL_OSTWALD            6  /* OstwaldThermo               */
#define GPK_MODEL_TENSOR_ANISO       7  /* TensorAnisotropyThermo      */
#define GPK_MODEL_ANISO_OSTWALD      8  /* AnisoOstwaldThermo          */
#define GPK_MODEL_PRECIPITATION      9  /* PrecipitationThermo         */
#define GPK_MODEL_GROOVING          10  /* GroovingThermo              */
#define GPK_MODEL_REDUCTION         11  /* ReductionThermo             */
#define GPK_MODEL_MAGNETIC_ANNEAL   12  /* MagneticAnnealingThermo     */
#define GPK_MODEL_MAGNETOELASTIC    13  /* MagnetoelasticThermo        */
#define GPK_MODEL_NDFEB             14  /* NdFeBGrainBoundaryThermo    */
#define GPK_NUM_MODELS              15

#define GPK_THERMO_NPARAM 40
#define GPK_MAX_PHASES     8

/* Field-for-field image of ThermoModel (include/gpk_core.hpp:73-123) plus
 * the subclass parameters in p[]:
 *   SOLIDIFICATION   p = {m_liq, k_part, T_melt, L}
 *   RECRYSTALLISATION p = {E_stored}
 *   DISLOCATION      p = {mu, b, alphaT}
 *   OSTWALD          p = {c_sat, Omega}
 *   TENSOR_ANISO     p = {bxx, byy, bzz, dG_bias}
 *   ANISO_OSTWALD    p = {bxx, byy, bzz, c_sat, Omega}
 *   PRECIPITATION    p = {n_phases, T_ref, a[8], b[8], c2[8], dT[8]}
 *   GROOVING         p = {sigma_gb, sigma_sv}
 *   REDUCTION        p = {pH2_over_pH2O, dG0_J_per_mol, V_molar_metal}
 *   NDFEB            p = {sigma_gb, sigma_gbphase_0, k_Cu, c_sat, Omega}   */
typedef struct gpk_thermo_desc {
    int32_t model;
    int32_t phase_selection, grain_network, stochastic;
    int32_t solute_rejection, elastic_enabled, elastic_smooth_iters;
    int32_t dislocation_enabled, magnetic_enabled;
    float sigma0, eps4, M0, Q, Rgas;
    float noise_scale, kB;
    float k_partition;
    float elastic_modulus, eigenstrain_coeff, c_ref;
    float disloc_coeff, rho_rex, recovery_rate;
    float Ku, Ms, H_ext, H_theta, g_easy_ref, lambda_s;
    float p[GPK_THERMO_NPARAM];
} gpk_thermo_desc;

/* The defaults of ThermoModel's member initialisers
 * (include/gpk_core.hpp:73-123) for the given model tag.                   */
void gpk_thermo_desc_init(gpk_thermo_desc* desc, int32_t model);

typedef struct gpk_grid gpk_grid;

/* ---- library / device -------------------------------------------------- */
/* Library version string and the last error text of this thread.          */
const char* gpk_version(void);
const char* gpk_last_error(void);
/* Selects and checks the CUDA device (must be sm_100).  Idempotent.        */
int gpk_device_init(int device);

/* ---- grid lifetime ------------------------------------------------------ */
/* Replaces GPKGrid::GPKGrid (src/gpk_grid.cpp:9-49): allocates every field
 * on the device with the reference's defaults (phi 0, alpha 1, c 0, T 800,
 * g 0, rho 0) and builds the Gaussian and derivative-of-Gaussian tap tables
 * (include/gpk_core.hpp:37-55, src/gpk_geometry.cpp:12-36) on the host.     */
int gpk_grid_create(int Nz, int Ny, int Nx, double dx,
                    const gpk_thermo_desc* thermo, double D,
                    double gaussian_sigma, int precision, gpk_grid** out);
int gpk_grid_destroy(gpk_grid* grid);
/* Swaps in a new thermodynamic model (the reference's shared ThermoModel
 * may be mutated by a driver between steps, e.g. dG_bias).                */
int gpk_grid_set_thermo(gpk_grid* grid, const gpk_thermo_desc* thermo);

/* ---- state transfer ------------------------------------------------------ */
/* Host <-> device copies of one public field (GPK_FIELD_*).  count is the
 * number of elements and must equal Nz*Ny*Nx.  Real fields are float or
 * double according to the grid's precision.                                */
int gpk_grid_upload(gpk_grid* grid, int field, const void* host, size_t count);
int gpk_grid_download(gpk_grid* grid, int field, void* host, size_t count);
/* Device pointer of a field, for callers that keep data on the GPU.        */
int gpk_grid_device_ptr(gpk_grid* grid, int field, void** dev_ptr);
int gpk_grid_get_time(gpk_grid* grid, double* time);
int gpk_grid_set_time(gpk_grid* grid, double time);
int gpk_grid_get_step_id(gpk_grid* grid, uint64_t* step_id);
int gpk_grid_set_step_id(gpk_grid* grid, uint64_t step_id);

/* ---- stepping --------------------------------------------------------------- */
/* GPKGrid::step(dt, dt_cap) (src/gpk_simulation.cpp:31-54): one complete
 * step.  dt < 0 selects the stable step.  *dt_used (may be null) receives
 * the step taken; reading it synchronises the stream.                      */
int gpk_grid_step(gpk_grid* grid, double dt, double dt_cap, double* dt_used);
/* n steps back to back with the same (dt, dt_cap), no host synchronisation
 * between them.  *time_out (may be null) receives the grid time after.     */
int gpk_grid_step_n(gpk_grid* grid, int n, double dt, double dt_cap,
                    double* time_out);
/* GPKGrid::run(t_end, dt) without a callback (src/gpk_simulation.cpp:60-73):
 * steps until time >= t_end, each capped by the remaining time.  At most
 * max_steps steps (<= 0: unbounded); *steps_out receives the count.        */
int gpk_grid_run(gpk_grid* grid, double t_end, double dt, int max_steps,
                 int* steps_out);
/* Waits for all work queued on the grid's stream.                          */
int gpk_grid_sync(gpk_grid* grid);
/* The interface mask and geometry of the current labels (the first two
 * stages of GPKGrid::step, src/gpk_geometry.cpp:42-183) without stepping:
 * fills mask, nx/ny/nz, kappa and phi_comp.  Returns when done.           */
int gpk_grid_geometry(gpk_grid* grid);

/* ---- diagnostics (src/gpk_simulation.cpp:11-144) ------------------------- */
int gpk_grid_max_dt(gpk_grid* grid, double* out);
int gpk_grid_phase_volume(gpk_grid* grid, int32_t label, double* out);
int gpk_grid_n_grains(gpk_grid* grid, int* out);
int gpk_grid_interface_fraction(gpk_grid* grid, double* out);
/* counters[0..2] = topology_accepted_last, topology_deferred_last,
 * gaussian_remap_exchanges_last (include/gpk_core.hpp:233-235).            */
int gpk_grid_counters(gpk_grid* grid, uint64_t counters[3]);
/* GPKGrid::topology_simple_move (src/gpk_connectivity.cpp:198-208).        */
int gpk_grid_topology_simple_move(gpk_grid* grid, int cell, int32_t new_label,
                                  int* result);
/* Device bytes held by the grid (the analogue of allocated_array_bytes).
 * Not counted: the 16 MiB static array of gpk_gaussian_filter_3d_noalloc,
 * resident on every GPU that loads the library.                           */
int gpk_grid_device_bytes(gpk_grid* grid, size_t* out);
/* Cumulative kernel-launch count issued by this grid (instrumentation).   */
int gpk_grid_launch_count(gpk_grid* grid, uint64_t* out);

/* gaussian_filter_3d (src/gpk_gaussian.cpp:9-72 of the reference): periodic
 * separable filter of an Nz x Ny x Nx float field with 2*radius+1 taps,
 * x then y then z (no z pass when Nz == 1), host buffers in and out.      */
int gpk_gaussian_filter_3d(const float* in, float* out, int Nz, int Ny, int Nx,
                           const float* taps, int radius);

/* Allocation-free variant of gpk_gaussian_filter_3d (no counterpart in the
 * reference).  For callers that cannot call cudaMalloc — processes whose
 * device memory belongs to another allocator or a fixed budget, loops that
 * must not allocate, hosts that only link this library — it takes the same
 * host buffers and returns the same result, but uses a file-scope static
 * device array (taps + two fields of at most GPK_NOALLOC_MAX_CELLS floats,
 * 16 MiB held by every GPU that loads the library until exit) instead of
 * cudaMalloc, and no stream of its own.  Larger grids return
 * GPK_ERR_INVALID_ARGUMENT.  The first call on a device looks up the array's
 * address (cudaGetSymbolAddress) with that device current: make it before
 * any stream capture.  Every call copies with synchronous cudaMemcpy on the
 * legacy default stream, which CUDA refuses while any stream of the process
 * is capturing in global mode: no call, first or later, may overlap such a
 * capture.  Calls share the array and keep the last call's contents; calls
 * in one process are serialised, calls overlapping on the GPU by any other
 * route race.                                                              */
#define GPK_NOALLOC_MAX_CELLS (1 << 21)
int gpk_gaussian_filter_3d_noalloc(const float* in, float* out, int Nz, int Ny, int Nx,
                                   const float* taps, int radius);

/* ---- instrumentation ------------------------------------------------------ */
/* The CUDA stream (cudaStream_t) all of this grid's work is queued on.     */
int gpk_grid_stream(gpk_grid* grid, void** stream);
/* Stage timing with CUDA events on the grid's stream.  enable != 0 records
 * an event pair around each stage of every following step; the per-stage
 * device milliseconds accumulate until read.  Stages (GPK_STAGE_*):       */
#define GPK_STAGE_MASK        0  /* interface mask + compaction          */
#define GPK_STAGE_GEOMETRY    1  /* Gaussian-Hessian geometry + competitor */
#define GPK_STAGE_VELOCITY    2  /* elastic proxy + constitutive velocity */
#define GPK_STAGE_PROJECTION  3  /* pair projection + stable dt          */
#define GPK_STAGE_ALPHA       4  /* alpha integration + candidates       */
#define GPK_STAGE_CROSSINGS   5  /* certified label crossings            */
#define GPK_STAGE_REMAP       6  /* balanced Gaussian remap              */
#define GPK_STAGE_EXTINCTION  7  /* unresolved-grain extinction          */
#define GPK_STAGE_TRANSPORT   8  /* diffusion / partitioning / recovery  */
#define GPK_NUM_STAGES        9
int gpk_grid_profile(gpk_grid* grid, int enable);
/* ms[k] = device milliseconds of stage k summed over profiled steps;
 * calls[k] = profiled steps; both reset after reading.                     */
int gpk_grid_stage_times(gpk_grid* grid, double ms[GPK_NUM_STAGES], uint64_t calls[GPK_NUM_STAGES]);
/* out = {waves of the crossing sweeps, waves of the remap exchange loops,
 * crossing candidates, remap proposals, global flood fills, cells they
 * visited, exact label counts, candidates those counts scanned, interface
 * cells given remap scores, those of them summed tap by tap}, summed since
 * the last read.                                                           */
int gpk_grid_wave_stats(gpk_grid* grid, uint64_t out[10]);
/* Kernel selection (all give identical results): 0 = tiled shared-memory
 * kernels where an instantiation exists (default), 1 = the per-interface-
 * cell kernels, 2 = tiled kernels with one label per geometry bitmap batch
 * (exercises the many-label path of the tiled geometry kernel; the remap
 * scores then skip their bitmap screening), 3 = tiled kernels with every
 * remap score summed tap by tap (no screening) and the pair-compare
 * projection tiles.  4 = separable tiles, FP64 grids only (the throughput
 * geometry): the reference's separable geometry (src/gpk_geometry.cpp:
 * 185-347: Gaussian smoothing of each label's indicator, fourth-order
 * differences) evaluated per tile; the fields agree with the direct stencil
 * to rounding (far below 1e-10), not bit for bit, so a label may differ
 * where a decision lies within rounding of its threshold (see the
 * near-threshold listing).  Kind 4 on an FP32 grid, or at a kernel radius
 * outside 4..10, returns GPK_ERR_INVALID_ARGUMENT.                        */
int gpk_grid_set_geometry_kernel(gpk_grid* grid, int kind);
/* External elastic energy (no counterpart in the reference): when on, the
 * E_el field is what the caller last wrote (an upload, a device write, or
 * gpk_spectral_couple_grid) and enters every interface velocity as
 * E_el(product neighbour) - E_el(cell) (src/gpk_physics.cpp:118-125), even
 * when the thermodynamic model's elastic flag is off; the model's own elastic
 * proxy (src/gpk_physics.cpp:10-63) is not run.                            */
int gpk_grid_set_external_elastic(gpk_grid* grid, int on);

/* Near-threshold listing (no counterpart in the reference).  The crossing
 * decision of src/gpk_transitions.cpp:291-292 is
 *     alpha_new <= 1e-6  &&  phi_comp != phi
 * with alpha_new = min(alpha + v dt / dx, 1) (:251-271).  Every step lists
 * the interface cells with phi_comp != phi whose margin alpha_new - 1e-6
 * lies within tol of zero: the decisions that an arithmetic of another
 * precision or operation order could flip.  tol defaults to 1e-12 and is
 * compared in the grid's real type.
 * gpk_grid_near_threshold returns in *n the number of cells listed by the
 * last step and writes the first min(*n, cap) of them, in increasing cell
 * order, to cells.                                                         */
int gpk_grid_set_near_threshold(gpk_grid* grid, double tol);
int gpk_grid_near_threshold(gpk_grid* grid, int32_t* cells, int cap, int* n);

/* Solid/liquid diffusivity ratio of the partitioned solute transport (no
 * counterpart in the reference, whose face flux is D x the smaller liquid
 * fraction of the two cells times the jump of cL, src/gpk_transport.cpp:
 * 102-135).  With ratio r > 0 the solid composition k cL also diffuses, with
 * r D, through the face's shared solid fraction: the face weight becomes
 * min(l_i, l_j) + r k min(s_i, s_j).  r = 0 (the default) is the reference's
 * transport bit for bit; r must lie in [0, 1] (r <= 1 keeps the reference's
 * stable time step valid).                                                  */
int gpk_grid_set_solid_diffusivity_ratio(gpk_grid* grid, double ratio);

/* The step as a captured CUDA graph (no counterpart in the reference, whose
 * step is host code).  gpk_grid_step_graph takes n steps of
 * GPKGrid::step(dt, dt_cap) like gpk_grid_step_n, replaying a graph of two
 * captured steps that takes no decision on the host: counts are read on
 * the device, the remap runs under a device-side gate on the step's
 * accepted crossings, and its proposals are ordered by one block.  The
 * results are bit-identical to gpk_grid_step_n.  The graph is captured on
 * first use (a fresh grid first takes one ordinary step) and again when the
 * model, a setting or the step arguments change; an odd last step is
 * ordinary.  gpk_grid_graph_supported tells whether the grid's model
 * qualifies (no region-identity topology certificates, no stochastic noise,
 * no recovery, no global-separable geometry; gpk_last_error says why not);
 * gpk_grid_step_graph returns GPK_ERR_UNSUPPORTED_MODEL otherwise.       */
int gpk_grid_step_graph(gpk_grid* grid, int n, double dt, double dt_cap, double* time_out);
/* Height of the 2-D geometry tiles at kernel radius 8 (sigma 1.5): the
 * 1024-cell tile's rows divided by 1, 2 or 4 (1024, 512 or 256 cells per
 * CTA).  Results do not depend on it; small grids get more CTAs from
 * smaller tiles.  gpk_batch_autotune_tiles picks it per instance size.     */
int gpk_grid_set_tile_rows(gpk_grid* grid, int divisor);
int gpk_grid_graph_supported(gpk_grid* grid, int* supported);

/* Failure injection for tests (no counterpart in the reference).  The next
 * cooperative launch of the grid (the ordered crossing sweep, or a remap
 * exchange loop) waits at its first grid barrier for one block more than it
 * launched, gives up after spin_limit polls (1 .. 2^24; about 100 ns each),
 * and returns; the step then fails with GPK_ERR_TIMEOUT.  The grid's state
 * is unspecified afterwards and it keeps reporting the error; the CUDA
 * context stays usable for other grids.                                    */
int gpk_grid_inject_wait_timeout(gpk_grid* grid, long long spin_limit);

#ifdef __cplusplus
}
#endif

#endif /* GPK_B200_H */
