/*
 * gpk_spectral.h — C ABI of the FP64 spectral micro-elasticity solve.
 *
 * Replaces `spectral_elasticity(variant_fractions, p)` of the reference's
 * Al-Cu material module (scripts/run_alcu_gpk_microstructure.py:99-190 of
 * albert-hzbn/GPK): the periodic Fourier solution of div(C:(eps - eps*)) = 0
 * for a homogeneous cubic solid (C11, C12, C44) carrying three eigenstrain
 * variants with volume fractions f_v.  Inputs and outputs keep the reference's
 * array layout: C order over the field shape (n0, n1[, n2]), the wave vector
 * component k_a running along array axis a (k_z = 0 in 2-D), and
 * variant-major stacks of 3 fields.
 *
 *   eps*_j     = sum_v eig[3*v + j] * f_v          (j = xx, yy, zz)
 *   driving_v  = -sigma : eps*_v                  (3 fields)
 *   energy     = (sigma : (eps - eps*)) / 2
 *   hydro      = trace(sigma) / 3
 *   residual   = rms |k . sigma^(k)| / rms |b(k)|  (the reference's audit)
 *
 * Transforms are real-to-complex / complex-to-real FP64 cuFFT on half
 * spectra; the strain is the inverse transform of the Hermitian part of the
 * reference's strain transform, which is exactly what the reference's
 * `ifftn(...).real` keeps (the two differ only on the Nyquist planes of even
 * extents, handled explicitly).  Everything else (the eigenstrain assembly,
 * the per-wave-vector 3x3 acoustic-tensor solve, the stress/energy epilogue,
 * the residual reduction) is hand-written CUDA.
 * Results agree with the reference to about 1e-15 relative (FFT rounding).
 *
 * All functions return GPK_OK (0) or a GPK_ERR_* status of gpk_b200.h; the
 * message is in gpk_last_error().
 */
#ifndef GPK_SPECTRAL_H
#define GPK_SPECTRAL_H

#include <stddef.h>
#include <stdint.h>

#include "gpk_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gpk_spectral gpk_spectral;

/* shape: ndim (2 or 3) extents, each >= 1; dx: grid spacing (the `d` of the
 * reference's fftfreq); c11, c12, c44: cubic constants; eig: 3x3 row-major,
 * row v = (xx, yy, zz) eigenstrain of variant v (the reference's
 * variant_eigenstrains, lines 93-96).  Plans the transforms and allocates
 * 144 bytes per cell of device memory on the current device.              */
int gpk_spectral_create(int ndim, const int* shape, double dx, double c11, double c12, double c44,
                        const double eig[9], gpk_spectral** out);
int gpk_spectral_destroy(gpk_spectral* s);
/* Change the constants without re-planning.                               */
int gpk_spectral_set_constants(gpk_spectral* s, double dx, double c11, double c12, double c44, const double eig[9]);
/* Run on this CUDA stream (cudaStream_t) from now on; 0 is the legacy
 * default stream.  A new handle runs on a stream of its own.              */
int gpk_spectral_set_stream(gpk_spectral* s, void* stream);
/* Device pointers: fractions (3*N doubles, variant-major), driving (3*N),
 * energy (N), hydro (N); any output may be NULL.  Enqueued on the handle's
 * stream.  residual (host pointer) may be NULL; when given, the call waits
 * for the stream and stores the residual.                                 */
int gpk_spectral_solve(gpk_spectral* s, const double* fractions, double* driving, double* energy, double* hydro,
                       double* residual);
/* The same with host pointers (copies in and out; returns when done).     */
int gpk_spectral_solve_host(gpk_spectral* s, const double* fractions, double* driving, double* energy, double* hydro,
                            double* residual);
/* Coupling to a grid (no counterpart in the reference): variant 0 = every
 * cell whose label is not matrix_label (variants 1, 2 empty), solved on the
 * grid's stream, the elastic energy density written into the grid's E_el
 * field (converted to float for a GPK_PREC_F32 grid).  With
 * gpk_grid_set_external_elastic on, the next step drives the interfaces by
 * it.  The solve's shape must be the grid's ((Nz, Ny, Nx), or (Ny, Nx) for
 * Nz = 1).  residual (host) may be NULL.                                   */
int gpk_spectral_couple_grid(gpk_spectral* s, gpk_grid* grid, int32_t matrix_label, double* residual);
/* Cells N = product of the extents; device bytes held by the handle.      */
int gpk_spectral_info(const gpk_spectral* s, int64_t* cells, int64_t* device_bytes);

#ifdef __cplusplus
}
#endif
#endif /* GPK_SPECTRAL_H */
