/*
 * ref_harness.cpp — extern "C" harness around the reference's own GPKGrid.
 *
 * TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile against the
 * reference's unmodified sources (src/*.cpp, include/gpk_core.hpp,
 * include/gpk_thermo.hpp of albert-hzbn/GPK) into oracle/_ref/libgpk_ref.so.
 * It lets the tests and bench.py drive the reference through plain C calls:
 * create a grid from a gpk_thermo_desc, write/read its public fields, step
 * it, and time step() loops.  Nothing in the product links it.
 */
#include "gpk_core.hpp"
#include "gpk_thermo.hpp"

#include <omp.h>

#include <chrono>
#include <cstring>
#include <memory>
#include <vector>

#include "../include/gpk_b200.h"

using namespace gpk;

namespace {

std::shared_ptr<ThermoModel> make_model(const gpk_thermo_desc& d) {
    std::shared_ptr<ThermoModel> m;
    const float* p = d.p;
    switch (d.model) {
    case GPK_MODEL_BASE: m = std::make_shared<ThermoModel>(); break;
    case GPK_MODEL_ISOTROPIC: m = std::make_shared<IsotropicGrowthThermo>(d.M0, d.sigma0); break;
    case GPK_MODEL_ANISOTROPIC: m = std::make_shared<AnisotropicGrowthThermo>(d.M0, d.sigma0, d.eps4); break;
    case GPK_MODEL_SOLIDIFICATION:
        m = std::make_shared<SolidificationThermo>(d.M0, d.sigma0, d.eps4, p[0], p[1], p[2], p[3]);
        break;
    case GPK_MODEL_RECRYSTALLISATION:
        m = std::make_shared<RecrystallisationThermo>(d.M0, d.sigma0, p[0]);
        break;
    case GPK_MODEL_DISLOCATION:
        m = std::make_shared<DislocationThermo>(d.M0, d.sigma0, p[0], p[1], p[2], d.recovery_rate, d.rho_rex);
        break;
    case GPK_MODEL_OSTWALD: m = std::make_shared<OstwaldThermo>(d.M0, d.sigma0, p[0], p[1]); break;
    case GPK_MODEL_TENSOR_ANISO: {
        auto t = std::make_shared<TensorAnisotropyThermo>(d.M0, d.sigma0, p[0], p[1], p[2]);
        t->dG_bias = p[3];
        m = t;
        break;
    }
    case GPK_MODEL_ANISO_OSTWALD:
        m = std::make_shared<AnisoOstwaldThermo>(d.M0, d.sigma0, p[0], p[1], p[2], p[3], p[4]);
        break;
    case GPK_MODEL_PRECIPITATION: {
        const int n = (int)p[0];
        std::vector<float> a(p + 2, p + 2 + n), b(p + 10, p + 10 + n), c2(p + 18, p + 18 + n),
            dT(p + 26, p + 26 + n);
        m = std::make_shared<PrecipitationThermo>(d.M0, d.sigma0, n, a, b, c2, dT, p[1]);
        break;
    }
    case GPK_MODEL_GROOVING: m = std::make_shared<GroovingThermo>(d.M0, p[0], p[1]); break;
    case GPK_MODEL_REDUCTION:
        m = std::make_shared<ReductionThermo>(d.M0, d.sigma0, p[0], p[1], p[2]);
        break;
    case GPK_MODEL_MAGNETIC_ANNEAL:
        m = std::make_shared<MagneticAnnealingThermo>(d.M0, d.sigma0, d.Ku, d.Ms, d.H_ext, d.H_theta,
                                                      d.g_easy_ref);
        break;
    case GPK_MODEL_MAGNETOELASTIC:
        m = std::make_shared<MagnetoelasticThermo>(d.M0, d.sigma0, d.elastic_modulus, d.lambda_s, d.H_theta,
                                                   d.H_ext, d.Ku, d.Ms);
        break;
    case GPK_MODEL_NDFEB:
        m = std::make_shared<NdFeBGrainBoundaryThermo>(d.M0, p[0], p[1], p[2], p[3], p[4]);
        break;
    default: return nullptr;
    }
    /* base-class fields the drivers set after construction */
    m->sigma0 = d.sigma0; m->eps4 = d.eps4; m->M0 = d.M0; m->Q = d.Q; m->Rgas = d.Rgas;
    m->phase_selection = d.phase_selection != 0; m->grain_network = d.grain_network != 0;
    m->stochastic = d.stochastic != 0; m->noise_scale = d.noise_scale; m->kB = d.kB;
    m->solute_rejection = d.solute_rejection != 0; m->k_partition = d.k_partition;
    m->elastic_enabled = d.elastic_enabled != 0; m->elastic_modulus = d.elastic_modulus;
    m->eigenstrain_coeff = d.eigenstrain_coeff; m->c_ref = d.c_ref;
    m->elastic_smooth_iters = d.elastic_smooth_iters;
    m->dislocation_enabled = d.dislocation_enabled != 0; m->disloc_coeff = d.disloc_coeff;
    m->rho_rex = d.rho_rex; m->recovery_rate = d.recovery_rate;
    m->magnetic_enabled = d.magnetic_enabled != 0; m->Ku = d.Ku; m->Ms = d.Ms; m->H_ext = d.H_ext;
    m->H_theta = d.H_theta; m->g_easy_ref = d.g_easy_ref; m->lambda_s = d.lambda_s;
    return m;
}

}  // namespace

extern "C" {

void* ref_create(int Nz, int Ny, int Nx, double dx, const gpk_thermo_desc* d, double D, double sigma) {
    auto m = make_model(*d);
    if (!m) return nullptr;
    return new GPKGrid(Nz, Ny, Nx, (float)dx, m, (float)D, (float)sigma);
}
void ref_destroy(void* h) { delete static_cast<GPKGrid*>(h); }

void* ref_field(void* h, int field) {
    GPKGrid* g = static_cast<GPKGrid*>(h);
    switch (field) {
    case GPK_FIELD_PHI: return g->phi.data();
    case GPK_FIELD_ALPHA: return g->alpha.data();
    case GPK_FIELD_C: return g->c.data();
    case GPK_FIELD_T: return g->T.data();
    case GPK_FIELD_G: return g->g.data();
    case GPK_FIELD_RHO: return g->rho.data();
    case GPK_FIELD_NX: return g->nx_f.data();
    case GPK_FIELD_NY: return g->ny_f.data();
    case GPK_FIELD_NZ: return g->nz_f.data();
    case GPK_FIELD_KAPPA: return g->kappa_f.data();
    case GPK_FIELD_VN: return g->vn_f.data();
    case GPK_FIELD_E_EL: return g->E_el.data();
    case GPK_FIELD_PHI_COMP: return g->phi_comp.data();
    case GPK_FIELD_G_COMP: return g->g_comp.data();
    case GPK_FIELD_MASK: return g->mask.data();
    default: return nullptr;
    }
}

double ref_step(void* h, double dt, double dt_cap) {
    return (double)static_cast<GPKGrid*>(h)->step((float)dt, (float)dt_cap);
}
int ref_run(void* h, double t_end, double dt) { return static_cast<GPKGrid*>(h)->run(t_end, (float)dt); }
double ref_get_time(void* h) { return static_cast<GPKGrid*>(h)->time; }
void ref_set_time(void* h, double t) { static_cast<GPKGrid*>(h)->time = t; }
void ref_counters(void* h, uint64_t out[3]) {
    GPKGrid* g = static_cast<GPKGrid*>(h);
    out[0] = g->topology_accepted_last; out[1] = g->topology_deferred_last;
    out[2] = g->gaussian_remap_exchanges_last;
}
double ref_max_dt(void* h) { return (double)static_cast<GPKGrid*>(h)->max_dt(); }
double ref_phase_volume(void* h, int32_t label) { return static_cast<GPKGrid*>(h)->phase_volume(label); }
int ref_n_grains(void* h) { return static_cast<GPKGrid*>(h)->n_grains(); }
double ref_interface_fraction(void* h) { return (double)static_cast<GPKGrid*>(h)->interface_fraction(); }
int ref_topology_simple_move(void* h, int cell, int32_t label) {
    return static_cast<GPKGrid*>(h)->topology_simple_move(cell, label) ? 1 : 0;
}

/* Times n steps of step(dt) with the given OpenMP thread count (<= 0: keep
 * the default); returns wall seconds of the step() loop only. */
double ref_time_steps(void* h, int n, double dt, int threads) {
    if (threads > 0) omp_set_num_threads(threads);
    GPKGrid* g = static_cast<GPKGrid*>(h);
    auto t0 = std::chrono::steady_clock::now();
    for (int k = 0; k < n; ++k) g->step((float)dt);
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}
int ref_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
