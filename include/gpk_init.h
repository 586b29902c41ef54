/*
 * gpk_init.h — host-side initial conditions for gpk_b200 label grids.
 *
 * The reference builds its polycrystals in the driver, voronoi_init
 * (demos/gpk.cpp:51-189 of albert-hzbn/GPK).  This is the same construction
 * with this library's own seeded random stream, exported so that drivers,
 * tests and benchmarks can produce identical input buffers for the GPU path
 * and for CPU checkers.
 */
#ifndef GPK_INIT_H
#define GPK_INIT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Fills phi (labels 1..n_seeds) and, when g is not null, g (one orientation
 * per grain in [0, pi/2)) for an Nz x Ny x Nx periodic grid.  Returns 0 on
 * success, 1 on bad arguments, 2 if the normalisation stalls.  *reassigned
 * (may be null) receives the number of raster-tie cells that were moved to
 * make every label one face-connected component.                          */
int gpk_voronoi_init(int Nz, int Ny, int Nx, int n_seeds, uint64_t seed, int32_t* phi, float* g, int* reassigned);

/* The same polycrystal built on the device, straight into a grid's phi and
 * g fields (and its label counts): cell for cell the result of
 * gpk_voronoi_init for the grid's dimensions, n_seeds and seed.  Returns a
 * GPK_* status (gpk_b200.h).                                               */
typedef struct gpk_grid gpk_grid;
int gpk_grid_voronoi(gpk_grid* grid, int n_seeds, uint64_t seed, int* reassigned);

/* The same construction on the device for an explicit seed list: seed k sits
 * at cell (seed_z[k], seed_y[k], seed_x[k]) with orientation seed_g[k] and
 * labels its Voronoi cell k + 1.  This is the reference driver's
 * voronoi_init (demos/gpk.cpp:73-189 of albert-hzbn/GPK) after its seed
 * draws, so that handing it the seeds the reference draws for a seed value
 * gives the reference's polycrystal.  Seeds must be distinct cells of the
 * grid (GPK_ERR_INVALID_ARGUMENT otherwise).                               */
int gpk_grid_voronoi_seeds(gpk_grid* grid, int n_seeds, const int* seed_z, const int* seed_y, const int* seed_x,
                           const float* seed_g, int* reassigned);

#ifdef __cplusplus
}
#endif

#endif /* GPK_INIT_H */
