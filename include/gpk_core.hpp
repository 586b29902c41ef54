#pragma once
/*
 * gpk_core.hpp — drop-in replacement for the reference's include/gpk_core.hpp
 * (albert-hzbn/GPK), backed by the B200 library libgpk_b200.so.
 *
 * The public interface is the reference's, name for name and signature for
 * signature (include/gpk_core.hpp:37-326 there): GaussKernel,
 * gaussian_filter_3d, ThermoModel with its fields and virtual callbacks, and
 * GPKGrid with its public field vectors, step/run and diagnostics.  Callers
 * such as the reference's `gpk` driver and validate_* programs compile
 * unchanged against this header together with the reference's unchanged
 * gpk_thermo.hpp.
 *
 * What differs is underneath:
 *   - the state lives on the GPU.  The public std::vector members are host
 *     mirrors: step() and run() upload them on entry and download them on
 *     exit (run() also before each callback), so code that reads or writes
 *     the vectors between steps sees exactly what it sees with the reference.
 *   - the ThermoModel subclass is translated once per step call into the flat
 *     descriptor of include/gpk_b200.h (gpk_thermo_desc); the device evaluates
 *     the same constitutive formulas.  The subclasses of the reference's
 *     gpk_thermo.hpp are recognised by type; other subclasses describe
 *     themselves by overriding ThermoModel::gpk_describe, and a subclass that
 *     does neither makes step() throw (there is no CPU fallback).
 */

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <functional>
#include <memory>
#include <numeric>
#include <vector>

#include "gpk_b200.h"

namespace gpk {

class GPKGrid;

// Gaussian kernel (precomputed, separable) — include/gpk_core.hpp:37-55.
struct GaussKernel {
    std::vector<float> w;
    int radius;
    float sigma_cells;

    explicit GaussKernel(float sigma = 2.0f) : sigma_cells(std::max(sigma, 0.5f)) {
        sigma = sigma_cells;
        radius = static_cast<int>(std::ceil(3.5f * sigma));
        const int sz = 2 * radius + 1;
        w.resize(sz);
        float sum = 0.f;
        for (int i = 0; i < sz; ++i) {
            const float x = float(i - radius);
            w[i] = std::exp(-x * x / (2.f * sigma * sigma));
            sum += w[i];
        }
        for (auto& v : w) v /= sum;
    }
};

// Separable periodic 3-D Gaussian filter, evaluated on the GPU.  tmp1/tmp2
// are accepted for interface compatibility and left untouched.
void gaussian_filter_3d(const float* __restrict__ in, float* __restrict__ out, float* __restrict__ tmp1,
                        float* __restrict__ tmp2, int Nz, int Ny, int Nx, const GaussKernel& K);

// Thermodynamic model — include/gpk_core.hpp:72-200.
struct ThermoModel {
    float sigma0 = 0.5f;
    float eps4 = 0.0f;
    float M0 = 1e-8f;
    float Q = 0.0f;
    float Rgas = 8.314f;
    bool phase_selection = false;
    bool grain_network = false;

    bool stochastic = false;
    float noise_scale = 1.0f;
    float kB = 1.380649e-23f;

    bool solute_rejection = false;
    float k_partition = 1.0f;

    bool elastic_enabled = false;
    float elastic_modulus = 0.0f;
    float eigenstrain_coeff = 0.0f;
    float c_ref = 0.0f;
    int elastic_smooth_iters = 8;

    bool dislocation_enabled = false;
    float disloc_coeff = 0.0f;
    float rho_rex = 0.0f;
    float recovery_rate = 0.0f;

    bool magnetic_enabled = false;
    float Ku = 0.f;
    float Ms = 0.f;
    float H_ext = 0.f;
    float H_theta = 0.f;
    float g_easy_ref = 0.f;
    static constexpr float MU0 = 4.0e-7f * 3.14159265358979323846f;

    float lambda_s = 0.f;

    virtual float bulk_driving_force(int, int, float, float) const { return 0.f; }
    virtual float interface_composition(int, int, float c_parent, float) const { return c_parent; }
    virtual int select_product_phase(int phi_parent, float c_val, float T_val, const int32_t* candidates,
                                     int n_cands) const {
        (void)phi_parent; (void)c_val; (void)T_val; (void)candidates; (void)n_cands;
        return -1;
    }
    virtual float interfacial_energy(float nx, float ny, float nz, float g_val) const;
    virtual float interfacial_energy_pair(float nx, float ny, float nz, float g_val, int32_t, int32_t) const {
        return interfacial_energy(nx, ny, nz, g_val);
    }
    virtual float interfacial_energy_pair_comp(float nx, float ny, float nz, float g_val, int32_t phi_parent,
                                               int32_t phi_product, float) const {
        return interfacial_energy_pair(nx, ny, nz, g_val, phi_parent, phi_product);
    }
    virtual float E_mag(float g_val) const {
        if (!magnetic_enabled) return 0.f;
        const float c1 = std::cos(g_val - g_easy_ref);
        const float c2 = std::cos(g_val - H_theta);
        return -Ku * c1 * c1 - MU0 * Ms * H_ext * c2;
    }
    virtual float mobility(float nx, float ny, float nz, float g_parent, float g_product, float T_val) const;

    // Device description of this model (no counterpart in the reference).
    // Subclasses outside the reference's gpk_thermo.hpp override this to run
    // on the GPU; return false when the model has no device form.
    virtual bool gpk_describe(gpk_thermo_desc* desc) const {
        (void)desc;
        return false;
    }

    virtual ~ThermoModel() = default;
};

// GPKGrid — include/gpk_core.hpp:205-326.
class GPKGrid {
public:
    const int Nz, Ny, Nx;
    const float dx;
    double time = 0.0;

    std::vector<int32_t> phi;
    std::vector<float> alpha;
    std::vector<float> c;
    std::vector<float> T;
    std::vector<float> g;
    std::vector<float> rho;

    std::vector<float> nx_f, ny_f, nz_f;
    std::vector<float> kappa_f;
    std::vector<float> vn_f;
    std::vector<float> E_el;
    std::vector<int32_t> phi_comp;
    std::vector<float> g_comp;
    std::vector<uint8_t> mask;

    uint64_t topology_accepted_last = 0;
    uint64_t topology_deferred_last = 0;
    uint64_t gaussian_remap_exchanges_last = 0;

    GPKGrid(int Nz, int Ny, int Nx, float dx, std::shared_ptr<ThermoModel> thermo, float D = 0.f,
            float gaussian_sigma = 2.0f);
    // Copyable like the reference's GPKGrid: a copy takes every public
    // member and builds its own device grid from them at its first use.
    ~GPKGrid() = default;
    GPKGrid(const GPKGrid&) = default;
    GPKGrid& operator=(const GPKGrid&) = default;

    float step(float dt = -1.f, float dt_cap = 1.0e30f);
    int run(double t_end, float dt = -1.f, std::function<void(const GPKGrid&, int)> cb = nullptr,
            int cb_interval = 100);

    float max_dt() const;
    double phase_volume(int32_t label) const;
    double mean_grain_radius() const;
    int n_grains() const;
    float solid_fraction() const;
    float interface_fraction() const;
    std::size_t allocated_array_bytes() const;
    bool topology_simple_move(int cell, int32_t new_label) const;

    int N() const { return Nz * Ny * Nx; }
    inline int idx(int z, int y, int x) const { return z * Ny * Nx + y * Nx + x; }
    inline void decode(int i, int& z, int& y, int& x) const {
        x = i % Nx;
        y = (i / Nx) % Ny;
        z = i / (Ny * Nx);
    }

    // The device grid behind this object (no counterpart in the reference).
    gpk_grid* device_grid() const { return dev(); }
    // run() with a callback: when the environment variable
    // GPK_ASYNC_CALLBACKS is 1, each callback receives a snapshot copy of the
    // grid on a writer thread (in order) while the steps go on, so a driver's
    // snapshot output overlaps the computation; run() returns after the last
    // callback and rethrows a callback's exception.  (No counterpart in the
    // reference, whose callbacks run between steps.)
    // Host members -> device, and device -> host members, for code that
    // advances device_grid() directly (e.g. a gpk_batch); step() and run()
    // do both themselves.  No counterpart in the reference.
    void to_device() { push_state(); }
    void from_device() { pull_state(); }

private:
    std::shared_ptr<ThermoModel> thermo_;
    float D_;
    float gaussian_sigma_;
    // owns one device grid; a copy or assignment starts without one
    struct DeviceGrid {
        gpk_grid* p = nullptr;
        DeviceGrid() = default;
        DeviceGrid(const DeviceGrid&) {}
        DeviceGrid& operator=(const DeviceGrid&) {
            release();
            return *this;
        }
        ~DeviceGrid() { release(); }
        void release();
    };
    mutable DeviceGrid grid_;
    uint64_t step_id_ = 0;

    gpk_grid* dev() const;  // the device grid, created on first use
    void push_state();      // host mirrors -> device (state + time)
    void pull_state();      // device -> host mirrors (every public field)
    void push_thermo();     // ThermoModel -> gpk_thermo_desc
};

// Translates a ThermoModel into the device descriptor; throws
// std::runtime_error for a model with no device form.
gpk_thermo_desc describe_thermo(const ThermoModel& model);

}  // namespace gpk
