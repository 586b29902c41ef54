// gpk_core_shim.cpp — the reference's C++ interface (include/gpk_core.hpp of
// albert-hzbn/GPK) implemented over the C ABI of libgpk_b200.
//
// GPKGrid keeps the reference's public std::vector members as host mirrors
// of the device state: step() uploads the state fields, advances on the GPU
// and downloads every public field; run() uploads once, steps on the device
// and downloads before each callback and at the end.  Host-side diagnostics
// (phase_volume, n_grains, ...) read the mirrors exactly as the reference's
// own diagnostics read its vectors (src/gpk_simulation.cpp:78-144).
#include <condition_variable>
#include <cstdlib>
#include <deque>
#include <exception>
#include <memory>
#include <mutex>
#include <thread>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>
#include <typeinfo>
#include <vector>

#include "../../include/gpk_core.hpp"

namespace gpk {

// ---- default constitutive laws (src/gpk_thermo.cpp:9-47) -------------------
float ThermoModel::interfacial_energy(float nx, float ny, float nz, float g_val) const {
    if (eps4 == 0.f) return sigma0;
    const float cg = std::cos(g_val), sg = std::sin(g_val);
    const float nc_x = nx * cg + ny * sg;
    const float nc_y = -nx * sg + ny * cg;
    const float nc_z = nz;
    float aniso;
    if (nc_z == 0.f) aniso = std::cos(4.f * std::atan2(nc_y, nc_x));
    else aniso = nc_x * nc_x * nc_x * nc_x + nc_y * nc_y * nc_y * nc_y + nc_z * nc_z * nc_z * nc_z - 0.6f;
    return sigma0 * (1.f + eps4 * aniso);
}

float ThermoModel::mobility(float, float, float, float g_parent, float g_product, float T_val) const {
    const float pi = (float)M_PI;
    float dg = std::fabs(g_parent - g_product);
    dg = std::fmod(dg + pi * 0.5f, pi * 0.5f);
    if (dg > pi * 0.25f) dg = pi * 0.5f - dg;
    const float theta_m = 15.f * pi / 180.f;
    float mis;
    if (dg < 1e-6f) mis = 0.f;
    else if (dg >= theta_m) mis = 1.f;
    else { const float frac = dg / theta_m; mis = frac * (1.f - std::log(frac)); }
    const float arr = (Q > 0.f) ? std::exp(-Q / (Rgas * std::max(T_val, 1.f))) : 1.f;
    return M0 * mis * arr;
}

// ---- ThermoModel -> gpk_thermo_desc ---------------------------------------------
// The subclasses of the reference's gpk_thermo.hpp are recognised by their
// type name; their own members (declared after the ThermoModel base) are read
// through structs with the same member sequence.
namespace {

struct LSolidification : ThermoModel { float m_liq, k_part, T_melt, L; };
struct LRecrystallisation : ThermoModel { float E_stored; };
struct LDislocation : ThermoModel { float mu, b, alphaT; };
struct LOstwald : ThermoModel { float c_sat, Omega; };
struct LTensorAniso : ThermoModel { float bxx, byy, bzz; mutable float dG_bias; };
struct LAnisoOstwald : ThermoModel { float bxx, byy, bzz, c_sat, Omega; };
struct LPrecipitation : ThermoModel {
    int n_phases;
    float T_ref;
    std::vector<float> a, b, c2, dT;
};
struct LGrooving : ThermoModel { float sigma_gb, sigma_sv; };
struct LReduction : ThermoModel { float pH2_over_pH2O, dG0_J_per_mol, V_molar_metal; };
struct LNdFeB : ThermoModel { float sigma_gb, sigma_gbphase_0, k_Cu, c_sat, Omega; };

std::string mangled(const char* cls) { return "N3gpk" + std::to_string(std::strlen(cls)) + cls + "E"; }

void base_fields(const ThermoModel& m, gpk_thermo_desc& d) {
    d.sigma0 = m.sigma0; d.eps4 = m.eps4; d.M0 = m.M0; d.Q = m.Q; d.Rgas = m.Rgas;
    d.phase_selection = m.phase_selection; d.grain_network = m.grain_network;
    d.stochastic = m.stochastic; d.noise_scale = m.noise_scale; d.kB = m.kB;
    d.solute_rejection = m.solute_rejection; d.k_partition = m.k_partition;
    d.elastic_enabled = m.elastic_enabled; d.elastic_modulus = m.elastic_modulus;
    d.eigenstrain_coeff = m.eigenstrain_coeff; d.c_ref = m.c_ref; d.elastic_smooth_iters = m.elastic_smooth_iters;
    d.dislocation_enabled = m.dislocation_enabled; d.disloc_coeff = m.disloc_coeff;
    d.rho_rex = m.rho_rex; d.recovery_rate = m.recovery_rate;
    d.magnetic_enabled = m.magnetic_enabled; d.Ku = m.Ku; d.Ms = m.Ms; d.H_ext = m.H_ext;
    d.H_theta = m.H_theta; d.g_easy_ref = m.g_easy_ref; d.lambda_s = m.lambda_s;
}

// A subclass not known by name is described by behaviour: each virtual the
// step calls is evaluated on the host at a fixed sample set and compared, bit
// for bit, with a law the device implements.  Described: no bulk driving
// force, the parent's interface composition, no product-phase selection, the
// base interfacial energy (sigma0, eps4; src/gpk_thermo.cpp:9-30), the base
// magnetic energy, and a mobility that is either a constant (the
// AnisotropicGrowthThermo law) or the base Read-Shockley law
// (src/gpk_thermo.cpp:32-47).  Anything else is left undescribed.
bool describe_by_behaviour(const ThermoModel& m, gpk_thermo_desc& d) {
    if (m.phase_selection) return false;
    const int pairs[4][2] = {{0, 1}, {1, 0}, {2, 3}, {5, 2}};
    const float cs[3] = {0.f, 0.15f, 0.9f}, Ts[3] = {300.f, 800.f, 1250.f};
    for (const auto& pq : pairs)
        for (float c : cs)
            for (float T : Ts) {
                if (m.bulk_driving_force(pq[0], pq[1], c, T) != 0.f) return false;
                if (m.interface_composition(pq[0], pq[1], c, 0.5f * c + 0.1f) != c) return false;
            }
    const float nrm[8][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {0.6f, 0.8f, 0}, {-0.28f, 0.96f, 0},
                             {0.48f, 0.6f, 0.64f}, {-0.36f, -0.48f, 0.8f}, {0.8f, 0, -0.6f}};
    const float gs[5] = {0.f, 0.3f, 1.1f, -0.7f, 2.5f};
    for (const auto& n : nrm)
        for (float g : gs) {
            if (m.interfacial_energy_pair_comp(n[0], n[1], n[2], g, 1, 2, 0.1f) !=
                m.ThermoModel::interfacial_energy(n[0], n[1], n[2], g))
                return false;
            if (m.E_mag(g) != m.ThermoModel::E_mag(g)) return false;
        }
    bool constant = true, base = true;
    float first = 0.f;
    int k = 0;
    for (const auto& n : nrm)
        for (float gp : gs)
            for (float gq : gs)
                for (float T : Ts) {
                    const float v = m.mobility(n[0], n[1], n[2], gp, gq, T);
                    if (k++ == 0) first = v;
                    constant = constant && v == first;
                    base = base && v == m.ThermoModel::mobility(n[0], n[1], n[2], gp, gq, T);
                }
    if (!constant && !base) return false;
    base_fields(m, d);
    if (constant) {
        d.model = GPK_MODEL_ANISOTROPIC;
        d.M0 = first;
    } else {
        d.model = GPK_MODEL_BASE;
    }
    return true;
}

}  // namespace

gpk_thermo_desc describe_thermo(const ThermoModel& m) {
    gpk_thermo_desc d;
    gpk_thermo_desc_init(&d, GPK_MODEL_BASE);
    if (m.gpk_describe(&d)) return d;
    const std::string t = typeid(m).name();
    int model = -1;
    if (t == typeid(ThermoModel).name()) model = GPK_MODEL_BASE;
    else if (t == mangled("IsotropicGrowthThermo")) model = GPK_MODEL_ISOTROPIC;
    else if (t == mangled("AnisotropicGrowthThermo")) model = GPK_MODEL_ANISOTROPIC;
    else if (t == mangled("SolidificationThermo")) model = GPK_MODEL_SOLIDIFICATION;
    else if (t == mangled("RecrystallisationThermo")) model = GPK_MODEL_RECRYSTALLISATION;
    else if (t == mangled("DislocationThermo")) model = GPK_MODEL_DISLOCATION;
    else if (t == mangled("OstwaldThermo")) model = GPK_MODEL_OSTWALD;
    else if (t == mangled("TensorAnisotropyThermo")) model = GPK_MODEL_TENSOR_ANISO;
    else if (t == mangled("AnisoOstwaldThermo")) model = GPK_MODEL_ANISO_OSTWALD;
    else if (t == mangled("PrecipitationThermo")) model = GPK_MODEL_PRECIPITATION;
    else if (t == mangled("GroovingThermo")) model = GPK_MODEL_GROOVING;
    else if (t == mangled("ReductionThermo")) model = GPK_MODEL_REDUCTION;
    else if (t == mangled("MagneticAnnealingThermo")) model = GPK_MODEL_MAGNETIC_ANNEAL;
    else if (t == mangled("MagnetoelasticThermo")) model = GPK_MODEL_MAGNETOELASTIC;
    else if (t == mangled("NdFeBGrainBoundaryThermo")) model = GPK_MODEL_NDFEB;
    if (model < 0) {
        if (describe_by_behaviour(m, d)) return d;
        throw std::runtime_error(std::string("gpk_b200: ThermoModel subclass '") + t +
                                 "' has no device form (its virtual functions match no device law); "
                                 "override ThermoModel::gpk_describe");
    }
    d.model = model;
    base_fields(m, d);
    float* p = d.p;
    switch (model) {
    case GPK_MODEL_SOLIDIFICATION: {
        const auto& s = static_cast<const LSolidification&>(m);
        p[0] = s.m_liq; p[1] = s.k_part; p[2] = s.T_melt; p[3] = s.L;
        break;
    }
    case GPK_MODEL_RECRYSTALLISATION: p[0] = static_cast<const LRecrystallisation&>(m).E_stored; break;
    case GPK_MODEL_DISLOCATION: {
        const auto& s = static_cast<const LDislocation&>(m);
        p[0] = s.mu; p[1] = s.b; p[2] = s.alphaT;
        break;
    }
    case GPK_MODEL_OSTWALD: {
        const auto& s = static_cast<const LOstwald&>(m);
        p[0] = s.c_sat; p[1] = s.Omega;
        break;
    }
    case GPK_MODEL_TENSOR_ANISO: {
        const auto& s = static_cast<const LTensorAniso&>(m);
        p[0] = s.bxx; p[1] = s.byy; p[2] = s.bzz; p[3] = s.dG_bias;
        break;
    }
    case GPK_MODEL_ANISO_OSTWALD: {
        const auto& s = static_cast<const LAnisoOstwald&>(m);
        p[0] = s.bxx; p[1] = s.byy; p[2] = s.bzz; p[3] = s.c_sat; p[4] = s.Omega;
        break;
    }
    case GPK_MODEL_PRECIPITATION: {
        const auto& s = static_cast<const LPrecipitation&>(m);
        if (s.n_phases > GPK_MAX_PHASES)
            throw std::runtime_error("gpk_b200: PrecipitationThermo with more than 8 phases");
        p[0] = (float)s.n_phases; p[1] = s.T_ref;
        for (int q = 0; q < s.n_phases; ++q) {
            p[2 + q] = s.a[q]; p[10 + q] = s.b[q]; p[18 + q] = s.c2[q]; p[26 + q] = s.dT[q];
        }
        break;
    }
    case GPK_MODEL_GROOVING: {
        const auto& s = static_cast<const LGrooving&>(m);
        p[0] = s.sigma_gb; p[1] = s.sigma_sv;
        break;
    }
    case GPK_MODEL_REDUCTION: {
        const auto& s = static_cast<const LReduction&>(m);
        p[0] = s.pH2_over_pH2O; p[1] = s.dG0_J_per_mol; p[2] = s.V_molar_metal;
        break;
    }
    case GPK_MODEL_NDFEB: {
        const auto& s = static_cast<const LNdFeB&>(m);
        p[0] = s.sigma_gb; p[1] = s.sigma_gbphase_0; p[2] = s.k_Cu; p[3] = s.c_sat; p[4] = s.Omega;
        break;
    }
    default: break;
    }
    return d;
}

// ---- GPKGrid ---------------------------------------------------------------------
static void throw_if(int rc, const char* what) {
    if (rc != GPK_OK) throw std::runtime_error(std::string("gpk_b200: ") + what + ": " + gpk_last_error());
}

GPKGrid::GPKGrid(int Nz_, int Ny_, int Nx_, float dx_, std::shared_ptr<ThermoModel> thermo, float D,
                 float gaussian_sigma)
    : Nz(Nz_), Ny(Ny_), Nx(Nx_), dx(dx_),
      phi(Nz_ * Ny_ * Nx_, 0), alpha(Nz_ * Ny_ * Nx_, 1.f), c(Nz_ * Ny_ * Nx_, 0.f), T(Nz_ * Ny_ * Nx_, 800.f),
      g(Nz_ * Ny_ * Nx_, 0.f), rho(Nz_ * Ny_ * Nx_, 0.f), nx_f(Nz_ * Ny_ * Nx_, 0.f), ny_f(Nz_ * Ny_ * Nx_, 0.f),
      nz_f(Nz_ * Ny_ * Nx_, 0.f), kappa_f(Nz_ * Ny_ * Nx_, 0.f), vn_f(Nz_ * Ny_ * Nx_, 0.f),
      E_el(Nz_ * Ny_ * Nx_, 0.f), phi_comp(Nz_ * Ny_ * Nx_, 0), g_comp(Nz_ * Ny_ * Nx_, 0.f),
      mask(Nz_ * Ny_ * Nx_, 0), thermo_(std::move(thermo)), D_(D), gaussian_sigma_(gaussian_sigma) {
    dev();
}

void GPKGrid::DeviceGrid::release() {
    if (p) gpk_grid_destroy(p);
    p = nullptr;
}

gpk_grid* GPKGrid::dev() const {
    if (!grid_.p) {
        const gpk_thermo_desc d = describe_thermo(*thermo_);
        throw_if(gpk_grid_create(Nz, Ny, Nx, (double)dx, &d, (double)D_, (double)gaussian_sigma_, GPK_PREC_F32,
                                 &grid_.p),
                 "grid creation");
    }
    return grid_.p;
}


void GPKGrid::push_thermo() {
    const gpk_thermo_desc d = describe_thermo(*thermo_);
    throw_if(gpk_grid_set_thermo(dev(), &d), "thermo update");
}

void GPKGrid::push_state() {
    const size_t n = (size_t)N();
    throw_if(gpk_grid_upload(dev(), GPK_FIELD_PHI, phi.data(), n), "upload phi");
    throw_if(gpk_grid_upload(dev(), GPK_FIELD_ALPHA, alpha.data(), n), "upload alpha");
    throw_if(gpk_grid_upload(dev(), GPK_FIELD_C, c.data(), n), "upload c");
    throw_if(gpk_grid_upload(dev(), GPK_FIELD_T, T.data(), n), "upload T");
    throw_if(gpk_grid_upload(dev(), GPK_FIELD_G, g.data(), n), "upload g");
    throw_if(gpk_grid_upload(dev(), GPK_FIELD_RHO, rho.data(), n), "upload rho");
    // phi_comp keeps stale values outside the interface in the reference;
    // upload it so those cells read back unchanged
    throw_if(gpk_grid_upload(dev(), GPK_FIELD_PHI_COMP, phi_comp.data(), n), "upload phi_comp");
    throw_if(gpk_grid_set_time(dev(), time), "set time");
    throw_if(gpk_grid_set_step_id(dev(), step_id_), "set step id");
}

void GPKGrid::pull_state() {
    const size_t n = (size_t)N();
    struct F { int id; void* p; };
    const F fs[] = {{GPK_FIELD_PHI, phi.data()},       {GPK_FIELD_ALPHA, alpha.data()},
                    {GPK_FIELD_C, c.data()},           {GPK_FIELD_T, T.data()},
                    {GPK_FIELD_G, g.data()},           {GPK_FIELD_RHO, rho.data()},
                    {GPK_FIELD_NX, nx_f.data()},       {GPK_FIELD_NY, ny_f.data()},
                    {GPK_FIELD_NZ, nz_f.data()},       {GPK_FIELD_KAPPA, kappa_f.data()},
                    {GPK_FIELD_VN, vn_f.data()},       {GPK_FIELD_E_EL, E_el.data()},
                    {GPK_FIELD_PHI_COMP, phi_comp.data()}, {GPK_FIELD_G_COMP, g_comp.data()},
                    {GPK_FIELD_MASK, mask.data()}};
    for (const F& f : fs) throw_if(gpk_grid_download(dev(), f.id, f.p, n), "download");
    uint64_t cnt[3];
    throw_if(gpk_grid_counters(dev(), cnt), "counters");
    topology_accepted_last = cnt[0];
    topology_deferred_last = cnt[1];
    gaussian_remap_exchanges_last = cnt[2];
    throw_if(gpk_grid_get_time(dev(), &time), "time");
}

float GPKGrid::step(float dt, float dt_cap) {
    push_thermo();
    push_state();
    double used = 0.0;
    throw_if(gpk_grid_step(dev(), (double)dt, (double)dt_cap, &used), "step");
    ++step_id_;
    pull_state();
    return (float)used;
}

namespace {

// Callbacks on a writer thread, in order, each on a snapshot copy of the
// grid taken at its step: the snapshot I/O of a driver (CSV/VTK writers in
// its callback) then overlaps the following steps.  At most two snapshots
// wait at a time.  An exception from a callback stops later callbacks and is
// rethrown by run().
class CallbackWriter {
public:
    explicit CallbackWriter(const std::function<void(const GPKGrid&, int)>& cb) : cb_(cb) {
        thread_ = std::thread([this] { loop(); });
    }
    ~CallbackWriter() { finish(); }
    void push(std::unique_ptr<GPKGrid> g, int step) {
        std::unique_lock<std::mutex> lk(m_);
        space_.wait(lk, [this] { return q_.size() < 2; });
        q_.emplace_back(std::move(g), step);
        ready_.notify_one();
    }
    // waits for every queued callback; rethrows the first callback error
    void finish() {
        {
            std::lock_guard<std::mutex> lk(m_);
            if (done_) return;
            done_ = true;
        }
        ready_.notify_all();
        thread_.join();
    }
    std::exception_ptr error() const { return err_; }

private:
    void loop() {
        while (true) {
            std::pair<std::unique_ptr<GPKGrid>, int> item;
            {
                std::unique_lock<std::mutex> lk(m_);
                ready_.wait(lk, [this] { return done_ || !q_.empty(); });
                if (q_.empty()) return;
                item = std::move(q_.front());
                q_.pop_front();
                space_.notify_one();
            }
            if (!err_) {
                try {
                    cb_(*item.first, item.second);
                } catch (...) {
                    err_ = std::current_exception();
                }
            }
        }
    }
    const std::function<void(const GPKGrid&, int)>& cb_;
    std::deque<std::pair<std::unique_ptr<GPKGrid>, int>> q_;
    std::mutex m_;
    std::condition_variable ready_, space_;
    bool done_ = false;
    std::exception_ptr err_;
    std::thread thread_;
};

bool async_callbacks() {
    const char* e = std::getenv("GPK_ASYNC_CALLBACKS");
    return e && e[0] == '1';
}

}  // namespace

int GPKGrid::run(double t_end, float dt, std::function<void(const GPKGrid&, int)> cb, int cb_interval) {
    push_thermo();
    push_state();
    int step_count = 0;
    double t = time;
    std::unique_ptr<CallbackWriter> writer;
    if (cb && async_callbacks()) writer.reset(new CallbackWriter(cb));
    while (t < t_end) {
        const float remaining = static_cast<float>(t_end - t);
        double used = 0.0;
        throw_if(gpk_grid_step(dev(), (double)dt, (double)remaining, &used), "step");
        ++step_id_;
        t += (double)(float)used;
        ++step_count;
        if (cb && step_count % cb_interval == 0) {
            pull_state();
            if (writer) writer->push(std::unique_ptr<GPKGrid>(new GPKGrid(*this)), step_count);
            else cb(*this, step_count);
        }
    }
    pull_state();
    if (writer) {
        writer->finish();
        if (writer->error()) std::rethrow_exception(writer->error());
    }
    return step_count;
}

float GPKGrid::max_dt() const {
    float vmax = 1e-30f;
    for (int i = 0; i < N(); ++i)
        if (mask[i]) vmax = std::max(vmax, std::fabs(vn_f[i]));
    const float neighbors = (Nz > 1) ? 6.f : 4.f;
    const float dt_iface = 0.125f * dx / vmax;
    const float dt_diff = (D_ > 0.f) ? 0.4f * dx * dx / (neighbors * D_) : 1e30f;
    return std::min(dt_iface, dt_diff);
}

double GPKGrid::phase_volume(int32_t label) const {
    double volume = 0.0;
    for (int i = 0; i < N(); ++i) {
        if (phi[i] == label) volume += alpha[i];
        if (mask[i] && phi_comp[i] == label && phi_comp[i] != phi[i]) volume += 1.0 - alpha[i];
    }
    return volume;
}

int GPKGrid::n_grains() const {
    std::vector<int32_t> tmp(phi);
    std::sort(tmp.begin(), tmp.end());
    return static_cast<int>(std::unique(tmp.begin(), tmp.end()) - tmp.begin());
}

double GPKGrid::mean_grain_radius() const {
    const int ng = n_grains();
    if (ng == 0) return 0.0;
    const double mean_volume = static_cast<double>(N()) / ng;
    const double R = (Nz > 1) ? std::cbrt(3.0 * mean_volume / (4.0 * M_PI)) : std::sqrt(mean_volume / M_PI);
    return R * dx;
}

float GPKGrid::solid_fraction() const { return static_cast<float>(phase_volume(1) / static_cast<double>(N())); }

float GPKGrid::interface_fraction() const {
    int cnt = 0;
    for (auto v : mask) if (v) ++cnt;
    return static_cast<float>(cnt) / static_cast<float>(N());
}

std::size_t GPKGrid::allocated_array_bytes() const {
    auto bytes = [](const auto& v) -> std::size_t {
        using value_type = typename std::decay_t<decltype(v)>::value_type;
        return v.capacity() * sizeof(value_type);
    };
    std::size_t total = 0;
    total += bytes(phi) + bytes(alpha) + bytes(c) + bytes(T) + bytes(g) + bytes(rho);
    total += bytes(nx_f) + bytes(ny_f) + bytes(nz_f) + bytes(kappa_f) + bytes(vn_f);
    total += bytes(E_el) + bytes(phi_comp) + bytes(g_comp) + bytes(mask);
    return total;
}

bool GPKGrid::topology_simple_move(int cell, int32_t new_label) const {
    if (cell < 0 || cell >= N()) return false;
    // evaluate on the labels currently held in the host mirror
    throw_if(gpk_grid_upload(dev(), GPK_FIELD_PHI, phi.data(), (size_t)N()), "upload phi");
    int r = 0;
    throw_if(gpk_grid_topology_simple_move(dev(), cell, new_label, &r), "topology_simple_move");
    return r != 0;
}

void gaussian_filter_3d(const float* __restrict__ in, float* __restrict__ out, float* __restrict__ tmp1,
                        float* __restrict__ tmp2, int Nz, int Ny, int Nx, const GaussKernel& K) {
    (void)tmp1; (void)tmp2;
    throw_if(gpk_gaussian_filter_3d(in, out, Nz, Ny, Nx, K.w.data(), K.radius), "gaussian_filter_3d");
}

}  // namespace gpk
