/*
 * ref_voronoi.cpp — the reference driver's own voronoi_init behind a C call
 * (TEST INFRASTRUCTURE ONLY).
 *
 * voronoi_init is a file-local function of the reference's driver
 * (demos/gpk.cpp:51-189 of albert-hzbn/GPK), so this translation unit
 * compiles that driver source unchanged, with its main renamed by the
 * command line (-Dmain=gpk_driver_main, oracle/Makefile), and calls the
 * function on a grid of the requested shape.  ref_voronoi_seeds returns the
 * seed list the function draws for a given seed: the same std::mt19937 and
 * libstdc++ distributions in the same order as demos/gpk.cpp:56-71, so that
 * another construction can be handed the reference's own seeds.
 */
#include "gpk.cpp"

#include <cstdint>
#include <cstring>
#include <memory>
#include <random>
#include <unordered_set>

extern "C" {

/* Labels and orientations of voronoi_init(grid, n_seeds, seed).  Returns 0,
 * or 1 when the reference rejects the arguments. */
int ref_voronoi_init(int Nz, int Ny, int Nx, int n_seeds, uint32_t seed, int32_t* phi, float* g) {
    try {
        gpk::GPKGrid grid(Nz, Ny, Nx, 1.0f, std::make_shared<gpk::IsotropicGrowthThermo>(1.0f, 1.0f), 0.0f, 1.5f);
        voronoi_init(grid, n_seeds, seed);
        std::memcpy(phi, grid.phi.data(), sizeof(int32_t) * grid.phi.size());
        if (g) std::memcpy(g, grid.g.data(), sizeof(float) * grid.g.size());
        return 0;
    } catch (const std::exception&) {
        return 1;
    }
}

/* The seed cells and orientations voronoi_init draws for (shape, n, seed). */
int ref_voronoi_seeds(int Nz, int Ny, int Nx, int n_seeds, uint32_t seed, int* sz, int* sy, int* sx, float* sg) {
    if (n_seeds <= 0 || (long long)n_seeds > (long long)Nz * Ny * Nx) return 1;
    std::mt19937 rng(seed);
    std::uniform_int_distribution<int> rz(0, Nz - 1), ry(0, Ny - 1), rx(0, Nx - 1);
    std::uniform_real_distribution<float> rg(0.f, (float)M_PI * 0.5f);
    std::unordered_set<int> taken;
    for (int k = 0; k < n_seeds; ++k) {
        int lin;
        do {
            sz[k] = rz(rng); sy[k] = ry(rng); sx[k] = rx(rng);
            lin = (sz[k] * Ny + sy[k]) * Nx + sx[k];
        } while (!taken.insert(lin).second);
        sg[k] = rg(rng);
    }
    return 0;
}

}  // extern "C"
