/*
 * gpk_adjoint.h — gradients of an interface-velocity loss at a fixed label map.
 *
 * No counterpart exists in the reference (albert-hzbn/GPK has no adjoint or
 * gradient code).  The forward model is assembled from the reference's own
 * step, at fixed labels, in FP64:
 *
 *   geometry   n, kappa, phi_comp of the labels (src/gpk_geometry.cpp:42-183,
 *              via gpk_grid_geometry; constant at a fixed label map)
 *   elastic    plane-strain spectral solve for the eigenstrain field
 *              eta(x) * (E_xx, E_yy, E_xy), eta = 1 on precipitate labels,
 *              cubic C11/C12/C44, free mean normal expansion as in the
 *              reference's spectral_elasticity
 *              (scripts/run_alcu_gpk_microstructure.py:99-190); e(x) the
 *              elastic energy density
 *   velocity   v_raw = M_l * (e(q) - e(i) - sigma_a(n, g) * kappa) at every
 *              interface cell i of label l, q its first face neighbour of the
 *              competitor label (the elastic term of src/gpk_physics.cpp:
 *              118-125), M_l a per-grain mobility, and
 *              sigma_a = sigma0 * (1 + sum_m a_m cos(4 m theta_c)), theta_c
 *              the normal's angle in the grain frame (g); a = (eps4, 0, 0, 0)
 *              is the reference's 2-D sigma (src/gpk_thermo.cpp:9-30)
 *   projection v = pair-restricted Gaussian average of v_raw
 *              (src/gpk_physics.cpp:152-193, FP64 accumulation)
 *   loss       L = 1/2 sum_i (v_i - v*_i)^2 + w_E * sum_x e(x) dx^2
 *
 * Parameters theta = (E_xx, E_yy, E_xy, a_1..a_4, M_0..M_{n_mob-1}).
 * The gradient is the exact discrete adjoint: the transposed projection
 * stencil, a gather for the elastic term, and one adjoint spectral solve
 * (the elastic operator is self-adjoint), so a gradient costs two spectral
 * solves and a few stencil passes.  No FFT buffer is kept between calls.
 */
#ifndef GPK_ADJOINT_H
#define GPK_ADJOINT_H

#include <stddef.h>
#include <stdint.h>

#include "gpk_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gpk_adjoint gpk_adjoint;

/* grid: a 2-D GPK_PREC_F64 grid holding the label map and the per-cell
 * orientation g; its geometry is computed here (gpk_grid_geometry).
 * mob_index[l] (n_labels entries, labels in [0, n_labels)): index into the
 * n_mob mobility parameters, or -1 for a precipitate label, which carries
 * the eigenstrain and moves with the fixed mobility m_fixed.
 * The grid must outlive the handle and keep its labels.                   */
int gpk_adjoint_create(gpk_grid* grid, int n_labels, const int32_t* mob_index, int n_mob, double m_fixed,
                       double sigma0, double c11, double c12, double c44, double energy_weight,
                       gpk_adjoint** out);
int gpk_adjoint_destroy(gpk_adjoint* a);
/* 7 + n_mob                                                                */
int gpk_adjoint_num_params(const gpk_adjoint* a, int* n);
/* Target velocity (host, N doubles, row-major like the grid); read at
 * interface cells only.  Zero until set.                                   */
int gpk_adjoint_set_target(gpk_adjoint* a, const double* v_target);
/* theta (host, 7 + n_mob); loss (host); v_out (host, N doubles or NULL):
 * the projected velocity, zero away from the interface.                   */
int gpk_adjoint_forward(gpk_adjoint* a, const double* theta, double* loss, double* v_out);
/* loss and dL/dtheta (host, 7 + n_mob doubles).                           */
int gpk_adjoint_gradient(gpk_adjoint* a, const double* theta, double* loss, double* grad);

#ifdef __cplusplus
}
#endif
#endif /* GPK_ADJOINT_H */
