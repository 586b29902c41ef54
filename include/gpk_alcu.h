/*
 * gpk_alcu.h — C ABI of the Al-Cu material module's per-step Cu transport
 * and volume-conserving label remap (FP64, int8 labels).
 *
 * Replaces, function for function, the numpy/scipy code that the reference's
 * Al-Cu driver runs once per step (scripts/run_alcu_gpk_microstructure.py of
 * albert-hzbn/GPK):
 *
 *   gpk_alcu_competitor             neighbor_competitor             (260-276)
 *   gpk_alcu_precip_fraction        precip_fraction                 (675-676)
 *   gpk_alcu_variant_fractions      variant_fraction_fields         (278-283)
 *   gpk_alcu_matrix_composition     c_m of the lever rule           (917-919)
 *   gpk_alcu_diffuse                diffuse_conservative_subcycled  (679-699)
 *   gpk_alcu_partition_transfer     conservative_partition_transfer (702-737)
 *   gpk_alcu_interface_composition  interface_matrix_composition    (740-755)
 *   gpk_alcu_gaussian_remap         conservative_gaussian_remap     (562-594)
 *   gpk_alcu_balanced_remap         balanced_gaussian_remap         (597-672)
 *   gpk_alcu_commit_transactions    commit_topology_transactions    (526-559)
 *   gpk_alcu_sum                    np.sum of a float64 field
 *
 * Arrays keep the reference's layout: C order over the shape (n0, n1[, n2]),
 * periodic where the reference uses np.roll or mode="wrap".  Every result is
 * bit-identical to the reference's: the arithmetic follows numpy's operand
 * order, sums follow numpy's pairwise summation of the flattened array, and
 * Gaussian smoothing follows scipy.ndimage.gaussian_filter(mode="wrap")
 * (taps applied from the outermost inwards, axis 0 first).
 *
 * Gaussian taps.  scipy samples exp(-x^2 / (2 sigma^2)) with numpy's exp and
 * normalises by numpy's sum; numpy's vectorised exp and the C library's exp
 * differ in the last bit for a few percent of arguments, so the functions
 * that smooth take the taps (2 radius + 1 doubles, symmetric, radius <= 32)
 * from the caller.  gpk_alcu_gauss_taps computes them with the C library's
 * exp; a caller that wants the reference's exact bits passes the taps numpy
 * computes (the Python layer does).
 *
 * Pointers are device pointers unless said otherwise; work is enqueued on the
 * handle's stream, and calls that return a host value wait for it.  All
 * functions return GPK_OK or a GPK_ERR_* status (gpk_b200.h); the message is
 * in gpk_last_error().
 */
#ifndef GPK_ALCU_H
#define GPK_ALCU_H

#include <stddef.h>
#include <stdint.h>

#include "gpk_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#define GPK_ALCU_MAX_RADIUS 32

typedef struct gpk_alcu gpk_alcu;

/* The reference's Parameters fields these functions read (lines 43-76).   */
typedef struct gpk_alcu_params {
    double dx;           /* m                                              */
    double diffusivity;  /* m^2/s                                          */
    double c_matrix_eq;  /* equilibrium matrix Cu fraction                 */
    double c_theta;      /* theta-prime Cu fraction                        */
} gpk_alcu_params;

/* ndim 2 or 3, extents >= 1, fewer than 2^31 - 1 cells.  Allocates about
 * 127 bytes per cell of device memory on the current device; the balanced
 * remap adds 8 bytes per cell per distinct label at its first call.       */
int gpk_alcu_create(int ndim, const int* shape, const gpk_alcu_params* p, gpk_alcu** out);
int gpk_alcu_destroy(gpk_alcu* h);
int gpk_alcu_set_params(gpk_alcu* h, const gpk_alcu_params* p);
/* cudaStream_t; 0 is the legacy default stream.  A new handle has its own. */
int gpk_alcu_set_stream(gpk_alcu* h, void* stream);

/* Host only: scipy's taps for sigma (radius int(4 sigma + 0.5)), with the C
 * library's exp.  taps receives 2 radius + 1 values (max_taps >= that).    */
int gpk_alcu_gauss_taps(double sigma, double* taps, int max_taps, int* radius);

/* mask (uint8 0/1) and competitor (int8) of int8 labels.                  */
int gpk_alcu_competitor(gpk_alcu* h, const int8_t* labels, uint8_t* mask, int8_t* competitor);
/* fprec = labels > 0 ? alpha : (competitor > 0 ? 1 - alpha : 0)           */
int gpk_alcu_precip_fraction(gpk_alcu* h, const int8_t* labels, const double* alpha, const int8_t* competitor,
                             double* fprec);
/* fractions (3 N doubles, variant-major, the input of gpk_spectral_solve):
 * fractions[v - 1] = fprec * (variant == v), variant = labels > 0 ? labels
 * : competitor, v = 1, 2, 3.                                              */
int gpk_alcu_variant_fractions(gpk_alcu* h, const int8_t* labels, const double* alpha, const int8_t* competitor,
                               double* fractions);
/* cm = clip((ctot - fprec c_theta) / max(1 - fprec, 1e-8), 0, c_theta),
 * c_matrix_eq where the matrix fraction is below 1e-7.                    */
int gpk_alcu_matrix_composition(gpk_alcu* h, const double* ctot, const double* fprec, double* cm);
/* ctot advanced by dt in ceil(dt / (0.4 dx^2 / (2 ndim D))) explicit
 * substeps, in place; cm (may be NULL) gets the matrix composition the last
 * substep used; substeps (host, may be NULL) the count.                   */
int gpk_alcu_diffuse(gpk_alcu* h, double* ctot, const double* fprec, double dt, double* cm, int* substeps);
/* ctot += the partition transfer of old -> clip(new, 0, 1) at the matrix
 * composition, drawn from the Gaussian matrix neighbourhood so that the
 * summed Cu is unchanged (the rounding residue goes to the cell of largest
 * weight).  GPK_ERR_INFEASIBLE when the matrix holds too little Cu above
 * equilibrium or the neighbourhood is empty; ctot then holds the transfer
 * but no correction, as the reference leaves it when it raises.           */
int gpk_alcu_partition_transfer(gpk_alcu* h, double* ctot, const double* old_fraction, const double* new_fraction,
                                const double* matrix_composition, const double* taps, int radius);
/* trace = clip(G(cm m) / max(G(m), 1e-12), 0, c_theta), m = clip(1 - fprec,
 * 0, 1), G the wrapped Gaussian of the taps.                              */
int gpk_alcu_interface_composition(gpk_alcu* h, const double* cm, const double* fprec, double* trace,
                                   const double* taps, int radius);
/* Every face-connected component (no wrap) of every nonzero label, in the
 * reference's order (label ascending, then first cell in C order), is
 * replaced by the equal-volume upper level set of the wrapped Gaussian of its
 * own indicator inside its 3^d dilation, restricted to cells that are zero
 * or its own at that point; components of one cell are left alone.  labels
 * is updated in place, alpha is set to 1 where a label changed, changed
 * (host, may be NULL) gets the count.  Components whose dilations are
 * disjoint are processed together: the result is that of the serial order. */
int gpk_alcu_gaussian_remap(gpk_alcu* h, int8_t* labels, double* alpha, const double* taps, int radius,
                            int64_t* changed);
/* The crossing cells (crossing != 0) relabelled to their competitor in C
 * order, each only if the local certificate of topology_simple_relabel
 * (lines 464-523, local_only=True: one face-connected component of the old
 * label and of the new one around the cell within its periodic 3^d patch, or
 * the old label's last cell) holds against the labels left by the earlier
 * ones; accepted cells get alpha = 1, deferred ones alpha = max(alpha, 1e-6).
 * The certificates run in that order on one device thread; deferred (host,
 * may be NULL) gets the deferred count.                                    */
int gpk_alcu_commit_transactions(gpk_alcu* h, int8_t* labels, double* alpha, const int8_t* competitor,
                                 const uint8_t* crossing, int64_t* deferred);
/* Every interface cell proposes the face-neighbour label of largest wrapped-
 * Gaussian score gain over its own; for each pair of labels of one phase
 * class (both nonzero, or both zero) the k-th strongest proposals of the two
 * directions (gain descending, then cell descending) are exchanged when both
 * pass the local certificate, so every label keeps its volume.  labels in
 * place, alpha = 1 where a label changed, changed (host, may be NULL) the
 * count.  At most 8 distinct label values; the proposals and their ordering
 * run in parallel, the exchanges in the reference's order on one device
 * thread.                                                                  */
int gpk_alcu_balanced_remap(gpk_alcu* h, int8_t* labels, double* alpha, const double* taps, int radius,
                            int64_t* changed);
/* out (host) = np.sum(x) of an N-cell field, same bits.                   */
int gpk_alcu_sum(gpk_alcu* h, const double* x, double* out);
/* out = scipy.ndimage.gaussian_filter(in, sigma, mode="wrap") for the taps;
 * in and out may not alias.                                                */
int gpk_alcu_gaussian_filter(gpk_alcu* h, const double* in, double* out, const double* taps, int radius);
/* Cells; device bytes held; components, waves and scored (cell, component)
 * pairs of the last Gaussian remap (pairs above the cell count are handled
 * wave by wave instead).  Any output may be NULL.                         */
int gpk_alcu_info(const gpk_alcu* h, int64_t* cells, int64_t* device_bytes, int64_t* last_components,
                  int64_t* last_waves, int64_t* last_pairs);

#ifdef __cplusplus
}
#endif
#endif /* GPK_ALCU_H */
