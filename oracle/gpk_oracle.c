/*
 * gpk_oracle.c — CPU restatement of the GPK per-step algorithm.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path of
 * gpk_b200: only tests/, __graft_entry__.smoke() and the CPU-baseline leg of
 * bench.py may load it.  The product never links or calls it.
 *
 * It restates, in plain C and in the reference's order of floating-point
 * operations, GPKGrid::step() of albert-hzbn/GPK:
 *   mask/compaction        src/gpk_geometry.cpp:42-82
 *   geometry (direct)      src/gpk_geometry.cpp:88-183
 *   geometry (separable)   src/gpk_geometry.cpp:185-390, src/gpk_gaussian.cpp:9-72
 *   elastic proxy          src/gpk_physics.cpp:10-63
 *   velocities             src/gpk_physics.cpp:67-148
 *   pair projection        src/gpk_physics.cpp:152-193
 *   dt control / step      src/gpk_simulation.cpp:11-54
 *   crossings              src/gpk_transitions.cpp:251-326
 *   certificates           src/gpk_connectivity.cpp:10-208
 *   balanced remap         src/gpk_transitions.cpp:38-178
 *   extinction             src/gpk_transitions.cpp:180-249
 *   transport / recovery   src/gpk_transport.cpp:11-152
 *   constitutive laws      src/gpk_thermo.cpp:9-47, include/gpk_thermo.hpp
 *
 * Compiled twice: with -DOR_F64 every real quantity is double (symbols end
 * in _f64); without it the arithmetic is the reference's float arithmetic
 * (symbols end in _f32).  The float build must be compiled without FMA
 * contraction (-ffp-contract=off) so that it reproduces the reference's
 * x86-64 SSE results bit for bit.
 *
 * Parity pin: the float build is checked against the reference library
 * built from its own sources (oracle/_ref) and against the reference's
 * committed golden label grids (tests/golden/).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/gpk_b200.h"

#ifdef OR_F64
typedef double real;
#define RL(x) x
#define SFX(n) n##_f64
#define R_EXP exp
#define R_SQRT sqrt
#define R_CEIL ceil
#define R_FABS fabs
#define R_COS cos
#define R_SIN sin
#define R_ATAN2 atan2
#define R_LOG log
#define R_FMOD fmod
#define R_PI 3.14159265358979323846
#else
typedef float real;
#define RL(x) x##f
#define SFX(n) n##_f32
#define R_EXP expf
#define R_SQRT sqrtf
#define R_CEIL ceilf
#define R_FABS fabsf
#define R_COS cosf
#define R_SIN sinf
#define R_ATAN2 atan2f
#define R_LOG logf
#define R_FMOD fmodf
#define R_PI ((float)3.14159265358979323846)
#endif

static inline real rmax(real a, real b) { return (a < b) ? b : a; }  /* std::max */
static inline real rmin(real a, real b) { return (b < a) ? b : a; }  /* std::min */
static inline real rclamp(real v, real lo, real hi) {                /* std::clamp */
    return (v < lo) ? lo : (hi < v) ? hi : v;
}
static inline int imax(int a, int b) { return a < b ? b : a; }

/* ----------------------------------------------------------------------- */
/* label -> int map (open addressing) standing in for unordered_map         */
/* ----------------------------------------------------------------------- */
typedef struct { int32_t* keys; int* vals; uint8_t* used; size_t cap; size_t n; } lmap;

static void lmap_init(lmap* m, size_t hint) {
    size_t cap = 64;
    while (cap < 2 * hint + 16) cap <<= 1;
    m->cap = cap; m->n = 0;
    m->keys = (int32_t*)calloc(cap, sizeof(int32_t));
    m->vals = (int*)calloc(cap, sizeof(int));
    m->used = (uint8_t*)calloc(cap, 1);
}
static void lmap_free(lmap* m) { free(m->keys); free(m->vals); free(m->used); }
static size_t lmap_slot(const lmap* m, int32_t k) {
    uint64_t h = (uint64_t)(uint32_t)k * 0x9e3779b97f4a7c15ULL;
    size_t s = (size_t)(h >> 17) & (m->cap - 1);
    while (m->used[s] && m->keys[s] != k) s = (s + 1) & (m->cap - 1);
    return s;
}
static void lmap_grow(lmap* m);
static int* lmap_ref(lmap* m, int32_t k) {   /* operator[]: inserts 0 */
    size_t s = lmap_slot(m, k);
    if (!m->used[s]) {
        if (2 * (m->n + 1) > m->cap) { lmap_grow(m); s = lmap_slot(m, k); }
        m->used[s] = 1; m->keys[s] = k; m->vals[s] = 0; m->n++;
    }
    return &m->vals[s];
}
static int lmap_find(const lmap* m, int32_t k, int* out) {
    size_t s = lmap_slot(m, k);
    if (!m->used[s]) return 0;
    *out = m->vals[s];
    return 1;
}
static void lmap_grow(lmap* m) {
    lmap n2; lmap_init(&n2, m->cap);
    for (size_t s = 0; s < m->cap; ++s)
        if (m->used[s]) *lmap_ref(&n2, m->keys[s]) = m->vals[s];
    lmap_free(m); *m = n2;
}

/* ----------------------------------------------------------------------- */
/* Gaussian kernel: include/gpk_core.hpp:37-55                              */
/* ----------------------------------------------------------------------- */
typedef struct { real* w; int radius; real sigma_cells; } gk_t;

static void gk_init(gk_t* k, real sigma) {
    k->sigma_cells = rmax(sigma, RL(0.5));
    sigma = k->sigma_cells;
    k->radius = (int)R_CEIL(RL(3.5) * sigma);
    const int sz = 2 * k->radius + 1;
    k->w = (real*)malloc(sizeof(real) * sz);
    real sum = RL(0.);
    for (int i = 0; i < sz; ++i) {
        real x = (real)(i - k->radius);
        k->w[i] = R_EXP(-x * x / (RL(2.) * sigma * sigma));
        sum += k->w[i];
    }
    for (int i = 0; i < sz; ++i) k->w[i] /= sum;
}

/* ----------------------------------------------------------------------- */
/* grid                                                                     */
/* ----------------------------------------------------------------------- */
typedef struct OrGrid {
    int Nz, Ny, Nx, N;
    real dx;
    double time;
    int32_t* phi; real* alpha; real* c; real* T; real* g; real* rho;
    real *nx_f, *ny_f, *nz_f, *kappa_f, *vn_f, *E_el;
    int32_t* phi_comp; real* g_comp; uint8_t* mask;
    uint64_t topology_accepted_last, topology_deferred_last, gaussian_remap_exchanges_last;

    gpk_thermo_desc th;
    real D;
    gk_t gauss, velocity_gauss, remap_gauss;
    int* active; int nactive;
    real *geom_w0, *geom_w1, *geom_w2; int geom_radius; int geom_global_separable;
    real *geom_I, *geom_smooth, *geom_tmp1, *geom_tmp2;
    real *alpha_new, *c_new, *eps_star, *eps_smooth, *eps_tmp;
    real* solid_old; int have_solid_old;
    uint64_t step_id;
    uint32_t* ff_stamp; uint32_t ff_epoch; int* ff_stack;   /* flood-fill scratch */
    /* near-threshold listing (builder-defined, no reference counterpart):
     * interface cells with phi_comp != phi whose alpha_new lies within
     * near_tol of the switching threshold 1e-6, in increasing cell order   */
    double near_tol; int* near; int n_near;
    /* solid/liquid diffusivity ratio of the partitioned transport
     * (builder-defined; 0 is the reference's transport)                    */
    double solid_ratio;
} OrGrid;

static inline int IDX(const OrGrid* G, int z, int y, int x) { return z * G->Ny * G->Nx + y * G->Nx + x; }
static inline void DECODE(const OrGrid* G, int i, int* z, int* y, int* x) {
    *x = i % G->Nx; *y = (i / G->Nx) % G->Ny; *z = i / (G->Ny * G->Nx);
}
/* face neighbours in the reference's order: x-, x+, y-, y+, z-, z+        */
static inline void FACES(const OrGrid* G, int i, int nb[6]) {
    int z, y, x; DECODE(G, i, &z, &y, &x);
    const int Nx = G->Nx, Ny = G->Ny, Nz = G->Nz;
    const int xm = (x == 0 ? Nx - 1 : x - 1), xp = (x == Nx - 1 ? 0 : x + 1);
    const int ym = (y == 0 ? Ny - 1 : y - 1), yp = (y == Ny - 1 ? 0 : y + 1);
    const int zm = (z == 0 ? Nz - 1 : z - 1), zp = (z == Nz - 1 ? 0 : z + 1);
    nb[0] = IDX(G, z, y, xm); nb[1] = IDX(G, z, y, xp);
    nb[2] = IDX(G, z, ym, x); nb[3] = IDX(G, z, yp, x);
    nb[4] = IDX(G, zm, y, x); nb[5] = IDX(G, zp, y, x);
}

/* ----------------------------------------------------------------------- */
/* constitutive laws: src/gpk_thermo.cpp:9-47, include/gpk_thermo.hpp      */
/* ----------------------------------------------------------------------- */
static real th_interfacial_energy_base(const gpk_thermo_desc* th, real nx, real ny, real nz, real g) {
    if ((real)th->eps4 == RL(0.)) return (real)th->sigma0;
    const real cg = R_COS(g), sg = R_SIN(g);
    const real ncx = nx * cg + ny * sg;
    const real ncy = -nx * sg + ny * cg;
    const real ncz = nz;
    real aniso;
    if (ncz == RL(0.)) aniso = R_COS(RL(4.) * R_ATAN2(ncy, ncx));
    else aniso = ncx * ncx * ncx * ncx + ncy * ncy * ncy * ncy + ncz * ncz * ncz * ncz - RL(0.6);
    return (real)th->sigma0 * (RL(1.) + (real)th->eps4 * aniso);
}
static real th_tensor_sigma(const gpk_thermo_desc* th, real bxx, real byy, real bzz,
                            real nx, real ny, real nz, real g) {
    const real cg = R_COS(g), sg = R_SIN(g);
    const real ncx = nx * cg + ny * sg;
    const real ncy = -nx * sg + ny * cg;
    const real ncz = nz;
    const real K = bxx * ncx * ncx + byy * ncy * ncy + bzz * ncz * ncz;
    return (real)th->sigma0 * R_SQRT(rmax(K, RL(1e-12)));
}
static real th_sigma(const gpk_thermo_desc* th, real nx, real ny, real nz, real g,
                     int32_t p, int32_t q, real c) {
    switch (th->model) {
    case GPK_MODEL_TENSOR_ANISO:
    case GPK_MODEL_ANISO_OSTWALD:
        return th_tensor_sigma(th, (real)th->p[0], (real)th->p[1], (real)th->p[2], nx, ny, nz, g);
    case GPK_MODEL_GROOVING:
        return (p == 0 || q == 0) ? (real)th->p[1] : (real)th->p[0];
    case GPK_MODEL_NDFEB: {
        if (p == 0 || q == 0) {
            const real s0 = (real)th->p[1];
            real s = s0 * (RL(1.) - (real)th->p[2] * c);
            return rclamp(s, RL(0.), s0);
        }
        return (real)th->p[0];
    }
    default:
        return th_interfacial_energy_base(th, nx, ny, nz, g);
    }
}
static real th_mobility(const gpk_thermo_desc* th, real gp, real gq, real T) {
    if (th->model != GPK_MODEL_BASE) return (real)th->M0;
    real dg = R_FABS(gp - gq);
    dg = R_FMOD(dg + (real)R_PI * RL(0.5), (real)R_PI * RL(0.5));
    if (dg > (real)R_PI * RL(0.25)) dg = (real)R_PI * RL(0.5) - dg;
    const real theta_m = RL(15.) * (real)R_PI / RL(180.);
    real mis;
    if (dg < RL(1e-6)) mis = RL(0.);
    else if (dg >= theta_m) mis = RL(1.);
    else { real frac = dg / theta_m; mis = frac * (RL(1.) - R_LOG(frac)); }
    real arr = ((real)th->Q > RL(0.)) ? R_EXP(-(real)th->Q / ((real)th->Rgas * rmax(T, RL(1.)))) : RL(1.);
    return (real)th->M0 * mis * arr;
}
static real th_precip_G(const gpk_thermo_desc* th, int q, real c, real T) {
    const real a = (real)th->p[2 + q], b = (real)th->p[10 + q], c2 = (real)th->p[18 + q], dT = (real)th->p[26 + q];
    return a + b * c + c2 * c * c + dT * (T - (real)th->p[1]);
}
static real th_bulk(const gpk_thermo_desc* th, int32_t p, int32_t q, real c, real T) {
    switch (th->model) {
    case GPK_MODEL_SOLIDIFICATION: {
        const real m_liq = (real)th->p[0], T_melt = (real)th->p[2], L = (real)th->p[3];
        real T_liq = T_melt + m_liq * c;
        real dT = T_liq - T;
        real dG = (L / T_melt) * dT;
        if (p == 0 && q == 1) return -dG;
        if (p == 1 && q == 0) return +dG;
        return RL(0.);
    }
    case GPK_MODEL_RECRYSTALLISATION: {
        const real E = (real)th->p[0];
        if (p == 0 && q >= 1) return -E;
        if (p >= 1 && q == 0) return +E;
        return RL(0.);
    }
    case GPK_MODEL_OSTWALD: {
        const real c_sat = (real)th->p[0], Omega = (real)th->p[1];
        if (p == 0) return Omega * (c_sat - c);
        if (p >= 1) return Omega * (c - c_sat);
        return RL(0.);
    }
    case GPK_MODEL_TENSOR_ANISO: {
        const real bias = (real)th->p[3];
        if (bias == RL(0.)) return RL(0.);
        return (p != 0) ? bias : -bias;
    }
    case GPK_MODEL_ANISO_OSTWALD: {
        const real c_sat = (real)th->p[3], Omega = (real)th->p[4];
        if (p == 0) return Omega * (c_sat - c);
        return Omega * (c - c_sat);
    }
    case GPK_MODEL_PRECIPITATION: {
        const int np = (int)th->p[0];
        if (p < 0 || p >= np || q < 0 || q >= np) return RL(0.);
        return th_precip_G(th, q, c, T) - th_precip_G(th, p, c, T);
    }
    case GPK_MODEL_REDUCTION: {
        const real Rg = RL(8.314);
        real dG_mol = (real)th->p[1] - Rg * T * R_LOG((real)th->p[0]);
        real dG_vol = dG_mol / (real)th->p[2];
        if (p == 0 && q >= 1) return dG_vol;
        if (p >= 1 && q == 0) return -dG_vol;
        return RL(0.);
    }
    case GPK_MODEL_NDFEB: {
        const real c_sat = (real)th->p[3], Omega = (real)th->p[4];
        if (p != 0) return Omega * (c_sat - c);
        return Omega * (c - c_sat);
    }
    default:
        return RL(0.);
    }
}
static real th_iface_comp(const gpk_thermo_desc* th, int32_t p, int32_t q, real cp, real cq) {
    if (th->model == GPK_MODEL_OSTWALD || th->model == GPK_MODEL_ANISO_OSTWALD) {
        if (p == 0) return cp;
        if (q == 0) return cq;
        return cp;
    }
    return cp;
}
static int th_select(const gpk_thermo_desc* th, int32_t p, real c, real T, const int32_t* cand, int n) {
    if (th->model != GPK_MODEL_PRECIPITATION) return -1;
    const int np = (int)th->p[0];
    real best = RL(1e30);
    int best_q = -1;
    for (int k = 0; k < n; ++k) {
        int32_t q = cand[k];
        if (q < 0 || q >= np || q == p) continue;
        real dG = th_precip_G(th, q, c, T) - th_precip_G(th, p, c, T);
        if (dG < best) { best = dG; best_q = q; }
    }
    return best_q;
}
static real th_Emag(const gpk_thermo_desc* th, real g) {
    if (!th->magnetic_enabled) return RL(0.);
    const real MU0 = RL(4.0e-7) * (real)R_PI;
    real c1 = R_COS(g - (real)th->g_easy_ref);
    real c2 = R_COS(g - (real)th->H_theta);
    return -(real)th->Ku * c1 * c1 - MU0 * (real)th->Ms * (real)th->H_ext * c2;
}

/* ----------------------------------------------------------------------- */
/* construction: src/gpk_grid.cpp:9-49, src/gpk_geometry.cpp:12-36         */
/* ----------------------------------------------------------------------- */
static real* ralloc(int n, real v) {
    real* p = (real*)malloc(sizeof(real) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; ++i) p[i] = v;
    return p;
}

static void build_geometry_kernels(OrGrid* G) {
    G->geom_radius = G->gauss.radius + 2;
    const int width = 2 * G->geom_radius + 1;
    G->geom_w0 = ralloc(width, RL(0.)); G->geom_w1 = ralloc(width, RL(0.)); G->geom_w2 = ralloc(width, RL(0.));
    const int first_offset[4] = {-2, -1, 1, 2};
    const real first_coeff[4] = {RL(1.) / RL(12.), -RL(8.) / RL(12.), RL(8.) / RL(12.), -RL(1.) / RL(12.)};
    const int second_offset[5] = {-2, -1, 0, 1, 2};
    const real second_coeff[5] = {-RL(1.) / RL(12.), RL(16.) / RL(12.), -RL(30.) / RL(12.),
                                  RL(16.) / RL(12.), -RL(1.) / RL(12.)};
    for (int o = -G->geom_radius; o <= G->geom_radius; ++o) {
        const int j = o + G->geom_radius;
#define GAT(off) (((off) < -G->gauss.radius || (off) > G->gauss.radius) ? RL(0.) : G->gauss.w[(off) + G->gauss.radius])
        G->geom_w0[j] = GAT(o);
        for (int k = 0; k < 4; ++k) G->geom_w1[j] += first_coeff[k] * GAT(o - first_offset[k]);
        for (int k = 0; k < 5; ++k) G->geom_w2[j] += second_coeff[k] * GAT(o - second_offset[k]);
#undef GAT
    }
}

OrGrid* SFX(or_create)(int Nz, int Ny, int Nx, double dx, const gpk_thermo_desc* th,
                       double D, double gaussian_sigma) {
    OrGrid* G = (OrGrid*)calloc(1, sizeof(OrGrid));
    G->Nz = Nz; G->Ny = Ny; G->Nx = Nx; G->N = Nz * Ny * Nx;
    G->dx = (real)dx; G->D = (real)D; G->th = *th;
    const int N = G->N;
    G->phi = (int32_t*)calloc((size_t)N, sizeof(int32_t));
    G->alpha = ralloc(N, RL(1.)); G->c = ralloc(N, RL(0.)); G->T = ralloc(N, RL(800.));
    G->g = ralloc(N, RL(0.)); G->rho = ralloc(N, RL(0.));
    G->nx_f = ralloc(N, RL(0.)); G->ny_f = ralloc(N, RL(0.)); G->nz_f = ralloc(N, RL(0.));
    G->kappa_f = ralloc(N, RL(0.)); G->vn_f = ralloc(N, RL(0.)); G->E_el = ralloc(N, RL(0.));
    G->phi_comp = (int32_t*)calloc((size_t)N, sizeof(int32_t));
    G->g_comp = ralloc(N, RL(0.));
    G->mask = (uint8_t*)calloc((size_t)N, 1);
    const real gs = (real)gaussian_sigma;
    gk_init(&G->gauss, gs);
    gk_init(&G->velocity_gauss, Nz > 1 ? rclamp(RL(0.375) * gs, RL(0.85), RL(3.00)) : RL(0.85));
    gk_init(&G->remap_gauss, Nz > 1 ? rclamp(RL(0.125) * gs, RL(0.70), RL(1.00)) : RL(0.70));
    G->alpha_new = ralloc(N, RL(0.)); G->c_new = ralloc(N, RL(0.));
    G->eps_star = ralloc(N, RL(0.)); G->eps_smooth = ralloc(N, RL(0.)); G->eps_tmp = ralloc(N, RL(0.));
    G->active = (int*)malloc(sizeof(int) * (size_t)N);
    G->solid_old = ralloc(N, RL(0.));
    G->ff_stamp = (uint32_t*)calloc((size_t)N, sizeof(uint32_t));
    G->ff_stack = (int*)malloc(sizeof(int) * (size_t)N);
    G->near = (int*)malloc(sizeof(int) * (size_t)N);
    G->near_tol = 1e-12;
    build_geometry_kernels(G);
    G->geom_global_separable = Nz > 1 && G->geom_radius > 18;
    if (G->geom_global_separable) {
        G->geom_I = ralloc(N, RL(0.)); G->geom_smooth = ralloc(N, RL(0.));
        G->geom_tmp1 = ralloc(N, RL(0.)); G->geom_tmp2 = ralloc(N, RL(0.));
    }
    return G;
}

void SFX(or_destroy)(OrGrid* G) {
    if (!G) return;
    free(G->phi); free(G->alpha); free(G->c); free(G->T); free(G->g); free(G->rho);
    free(G->nx_f); free(G->ny_f); free(G->nz_f); free(G->kappa_f); free(G->vn_f); free(G->E_el);
    free(G->phi_comp); free(G->g_comp); free(G->mask);
    free(G->gauss.w); free(G->velocity_gauss.w); free(G->remap_gauss.w);
    free(G->alpha_new); free(G->c_new); free(G->eps_star); free(G->eps_smooth); free(G->eps_tmp);
    free(G->active); free(G->solid_old); free(G->ff_stamp); free(G->ff_stack); free(G->near);
    free(G->geom_w0); free(G->geom_w1); free(G->geom_w2);
    free(G->geom_I); free(G->geom_smooth); free(G->geom_tmp1); free(G->geom_tmp2);
    free(G);
}

void* SFX(or_field)(OrGrid* G, int field) {
    switch (field) {
    case GPK_FIELD_PHI: return G->phi;
    case GPK_FIELD_ALPHA: return G->alpha;
    case GPK_FIELD_C: return G->c;
    case GPK_FIELD_T: return G->T;
    case GPK_FIELD_G: return G->g;
    case GPK_FIELD_RHO: return G->rho;
    case GPK_FIELD_NX: return G->nx_f;
    case GPK_FIELD_NY: return G->ny_f;
    case GPK_FIELD_NZ: return G->nz_f;
    case GPK_FIELD_KAPPA: return G->kappa_f;
    case GPK_FIELD_VN: return G->vn_f;
    case GPK_FIELD_E_EL: return G->E_el;
    case GPK_FIELD_PHI_COMP: return G->phi_comp;
    case GPK_FIELD_G_COMP: return G->g_comp;
    case GPK_FIELD_MASK: return G->mask;
    default: return NULL;
    }
}
double SFX(or_get_time)(OrGrid* G) { return G->time; }
void SFX(or_set_time)(OrGrid* G, double t) { G->time = t; }
uint64_t SFX(or_get_step_id)(OrGrid* G) { return G->step_id; }
void SFX(or_set_step_id)(OrGrid* G, uint64_t s) { G->step_id = s; }
void SFX(or_counters)(OrGrid* G, uint64_t out[3]) {
    out[0] = G->topology_accepted_last; out[1] = G->topology_deferred_last;
    out[2] = G->gaussian_remap_exchanges_last;
}
void SFX(or_set_thermo)(OrGrid* G, const gpk_thermo_desc* th) { G->th = *th; }
int SFX(or_nactive)(OrGrid* G) { return G->nactive; }
void SFX(or_set_near_tol)(OrGrid* G, double tol) { G->near_tol = tol; }
/* cells of the last step's near-threshold list (at most cap written); returns its length */
int SFX(or_near_threshold)(OrGrid* G, int* out, int cap) {
    for (int k = 0; k < G->n_near && k < cap; ++k) out[k] = G->near[k];
    return G->n_near;
}
void SFX(or_set_solid_ratio)(OrGrid* G, double r) { G->solid_ratio = r; }
const int* SFX(or_active)(OrGrid* G) { return G->active; }

/* ----------------------------------------------------------------------- */
/* interface mask + sorted compaction: src/gpk_geometry.cpp:42-82          */
/* ----------------------------------------------------------------------- */
static void step_interface_mask(OrGrid* G) {
    const int32_t* p = G->phi;
    int n = 0;
    for (int i = 0; i < G->N; ++i) {
        int nb[6]; FACES(G, i, nb);
        const int32_t v = p[i];
        const uint8_t act = (uint8_t)((v != p[nb[0]]) | (v != p[nb[1]]) | (v != p[nb[2]]) |
                                      (v != p[nb[3]]) | (v != p[nb[4]]) | (v != p[nb[5]]));
        G->mask[i] = act;
        if (act) G->active[n++] = i;
    }
    G->nactive = n;
}

/* ----------------------------------------------------------------------- */
/* competitor choice: src/gpk_geometry.cpp:154-182                          */
/* ----------------------------------------------------------------------- */
static void competitor_at(OrGrid* G, int i) {
    const int Nz = G->Nz, Ny = G->Ny, Nx = G->Nx;
    int z, y, x; DECODE(G, i, &z, &y, &x);
    int nei[6]; FACES(G, i, nei);
    const real score[6] = {-G->nx_f[i], G->nx_f[i], -G->ny_f[i], G->ny_f[i], -G->nz_f[i], G->nz_f[i]};
    const int nface = Nz > 1 ? 6 : 4;
    int best = -1, best_support = -1; real best_score = RL(-2.);
    for (int k = 0; k < nface; ++k) {
        const int32_t q = G->phi[nei[k]];
        if (q == G->phi[i]) continue;
        int support = 0;
        for (int dz = (Nz > 1 ? -1 : 0); dz <= (Nz > 1 ? 1 : 0); ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dxs = -1; dxs <= 1; ++dxs) {
                    if (dxs == 0 && dy == 0 && dz == 0) continue;
                    int xx = x + dxs; if (xx < 0) xx += Nx; else if (xx >= Nx) xx -= Nx;
                    int yy = y + dy; if (yy < 0) yy += Ny; else if (yy >= Ny) yy -= Ny;
                    int zz = z + dz; if (zz < 0) zz += Nz; else if (zz >= Nz) zz -= Nz;
                    support += G->phi[IDX(G, zz, yy, xx)] == q;
                }
        if (support > best_support || (support == best_support && score[k] > best_score)) {
            best = k; best_support = support; best_score = score[k];
        }
    }
    G->phi_comp[i] = (best >= 0) ? G->phi[nei[best]] : G->phi[i];
}

/* ----------------------------------------------------------------------- */
/* direct Gaussian-Hessian geometry: src/gpk_geometry.cpp:88-152            */
/* ----------------------------------------------------------------------- */
static void finish_geometry(OrGrid* G, int i, real Ix, real Iy, real Iz, real Ixx, real Iyy,
                            real Izz, real Ixy, real Ixz, real Iyz) {
    const real dx = G->dx;
    const real kappa_limit = RL(1.) / (G->gauss.sigma_cells * dx);
    const real grad_sq = Ix * Ix + Iy * Iy + Iz * Iz;
    if (grad_sq * dx * dx > RL(1e-8)) {
        const real grad = R_SQRT(grad_sq);
        G->nx_f[i] = -Ix / grad;
        G->ny_f[i] = -Iy / grad;
        G->nz_f[i] = -Iz / grad;
        const real trace_H = Ixx + Iyy + Izz;
        const real gHg = Ix * Ix * Ixx + Iy * Iy * Iyy + Iz * Iz * Izz
                       + RL(2.) * (Ix * Iy * Ixy + Ix * Iz * Ixz + Iy * Iz * Iyz);
        real curvature = (gHg - grad_sq * trace_H) / (grad_sq * grad);
        if (R_FABS(curvature * dx) < RL(1e-6)) curvature = RL(0.);
        G->kappa_f[i] = rclamp(curvature, -kappa_limit, kappa_limit);
    }
}

static void step_geometry_direct(OrGrid* G) {
    const int N = G->N, Nz = G->Nz, Ny = G->Ny, Nx = G->Nx;
    memset(G->nx_f, 0, sizeof(real) * N); memset(G->ny_f, 0, sizeof(real) * N);
    memset(G->nz_f, 0, sizeof(real) * N); memset(G->kappa_f, 0, sizeof(real) * N);
    const int radius = G->geom_radius;
    const real inv_dx = RL(1.) / G->dx;
    const real inv_dx2 = inv_dx * inv_dx;
    const real *w0 = G->geom_w0, *w1 = G->geom_w1, *w2 = G->geom_w2;
    for (int a = 0; a < G->nactive; ++a) {
        const int i = G->active[a];
        const int32_t resident = G->phi[i];
        int z0, y0, x0; DECODE(G, i, &z0, &y0, &x0);
        real Ix = 0, Iy = 0, Iz = 0, Ixx = 0, Iyy = 0, Izz = 0, Ixy = 0, Ixz = 0, Iyz = 0;
        const int dz_begin = Nz > 1 ? -radius : 0;
        const int dz_end = Nz > 1 ? radius : 0;
        for (int dz = dz_begin; dz <= dz_end; ++dz) {
            int z = z0 + dz; while (z < 0) z += Nz; while (z >= Nz) z -= Nz;
            const int jz = dz + radius;
            const real gz0 = Nz > 1 ? w0[jz] : RL(1.);
            const real gz1 = Nz > 1 ? w1[jz] : RL(0.);
            const real gz2 = Nz > 1 ? w2[jz] : RL(0.);
            for (int dy = -radius; dy <= radius; ++dy) {
                int y = y0 + dy; while (y < 0) y += Ny; while (y >= Ny) y -= Ny;
                const int jy = dy + radius;
                const real gy0 = w0[jy], gy1 = w1[jy], gy2 = w2[jy];
                for (int dxs = -radius; dxs <= radius; ++dxs) {
                    int x = x0 + dxs; while (x < 0) x += Nx; while (x >= Nx) x -= Nx;
                    if (G->phi[IDX(G, z, y, x)] != resident) continue;
                    const int jx = dxs + radius;
                    const real gx0 = w0[jx], gx1 = w1[jx], gx2 = w2[jx];
                    Ix += gx1 * gy0 * gz0; Iy += gx0 * gy1 * gz0;
                    Ixx += gx2 * gy0 * gz0; Iyy += gx0 * gy2 * gz0; Ixy += gx1 * gy1 * gz0;
                    if (Nz > 1) {
                        Iz += gx0 * gy0 * gz1; Izz += gx0 * gy0 * gz2;
                        Ixz += gx1 * gy0 * gz1; Iyz += gx0 * gy1 * gz1;
                    }
                }
            }
        }
        Ix *= inv_dx; Iy *= inv_dx; Iz *= inv_dx;
        Ixx *= inv_dx2; Iyy *= inv_dx2; Izz *= inv_dx2;
        Ixy *= inv_dx2; Ixz *= inv_dx2; Iyz *= inv_dx2;
        finish_geometry(G, i, Ix, Iy, Iz, Ixx, Iyy, Izz, Ixy, Ixz, Iyz);
    }
    for (int a = 0; a < G->nactive; ++a) competitor_at(G, G->active[a]);
}

static int int32_cmp(const void* a, const void* b) {
    const int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
    return (x > y) - (x < y);
}

/* separable variant for broad 3-D kernels: src/gpk_geometry.cpp:185-390     */
static void step_geometry_separable(OrGrid* G) {
    const int N = G->N, Nz = G->Nz, Ny = G->Ny, Nx = G->Nx;
    const real dx = G->dx;
    const real idx12 = RL(1.) / (RL(12.) * dx);
    const real idx_sq = RL(1.) / (dx * dx);
    const real idx12_sq = idx_sq / RL(12.);
    const real idx144_sq = idx_sq / RL(144.);
    /* distinct interface labels, ascending */
    int32_t* labs = (int32_t*)malloc(sizeof(int32_t) * (size_t)(G->nactive + 1));
    int nl = 0;
    for (int i = 0; i < N; ++i) if (G->mask[i]) labs[nl++] = G->phi[i];
    qsort(labs, (size_t)nl, sizeof(int32_t), int32_cmp);
    int ng = 0;
    for (int a = 0; a < nl; ++a) if (ng == 0 || labs[ng - 1] != labs[a]) labs[ng++] = labs[a];
    memset(G->nx_f, 0, sizeof(real) * N); memset(G->ny_f, 0, sizeof(real) * N);
    memset(G->nz_f, 0, sizeof(real) * N); memset(G->kappa_f, 0, sizeof(real) * N);
    const int krad = G->gauss.radius; const real* kw = G->gauss.w;
    real *I = G->geom_I, *S = G->geom_smooth, *t1 = G->geom_tmp1, *t2 = G->geom_tmp2;
    for (int gi = 0; gi < ng; ++gi) {
        const int32_t p = labs[gi];
        for (int i = 0; i < N; ++i) I[i] = (G->phi[i] == p) ? RL(1.) : RL(0.);
        for (int z = 0; z < Nz; ++z) for (int y = 0; y < Ny; ++y) for (int x = 0; x < Nx; ++x) {
            real acc = RL(0.);
            for (int k = 0, ki = -krad; ki <= krad; ++k, ++ki) {
                int xx = x + ki; if (xx < 0) xx += Nx; else if (xx >= Nx) xx -= Nx;
                acc += kw[k] * I[(z * Ny + y) * Nx + xx];
            }
            t1[(z * Ny + y) * Nx + x] = acc;
        }
        for (int z = 0; z < Nz; ++z) for (int y = 0; y < Ny; ++y) for (int x = 0; x < Nx; ++x) {
            real acc = RL(0.);
            for (int k = 0, ki = -krad; ki <= krad; ++k, ++ki) {
                int yy = y + ki; if (yy < 0) yy += Ny; else if (yy >= Ny) yy -= Ny;
                acc += kw[k] * t1[(z * Ny + yy) * Nx + x];
            }
            t2[(z * Ny + y) * Nx + x] = acc;
        }
        if (Nz == 1) memcpy(S, t2, sizeof(real) * N);
        else
            for (int z = 0; z < Nz; ++z) for (int y = 0; y < Ny; ++y) for (int x = 0; x < Nx; ++x) {
                real acc = RL(0.);
                for (int k = 0, ki = -krad; ki <= krad; ++k, ++ki) {
                    int zz = z + ki; if (zz < 0) zz += Nz; else if (zz >= Nz) zz -= Nz;
                    acc += kw[k] * t2[(zz * Ny + y) * Nx + x];
                }
                S[(z * Ny + y) * Nx + x] = acc;
            }
        for (int z = 0; z < Nz; ++z) for (int y = 0; y < Ny; ++y) for (int x = 0; x < Nx; ++x) {
            const int i = IDX(G, z, y, x);
            if (!G->mask[i] || G->phi[i] != p) continue;
            const int xm = (x == 0 ? Nx - 1 : x - 1), xp = (x == Nx - 1 ? 0 : x + 1);
            const int ym = (y == 0 ? Ny - 1 : y - 1), yp = (y == Ny - 1 ? 0 : y + 1);
            const int zm = (z == 0 ? Nz - 1 : z - 1), zp = (z == Nz - 1 ? 0 : z + 1);
            const int xmm = (x < 2 ? x + Nx - 2 : x - 2), xpp = (x >= Nx - 2 ? x - Nx + 2 : x + 2);
            const int ymm = (y < 2 ? y + Ny - 2 : y - 2), ypp = (y >= Ny - 2 ? y - Ny + 2 : y + 2);
            const int zmm = (z < 2 ? z + Nz - 2 : z - 2), zpp = (z >= Nz - 2 ? z - Nz + 2 : z + 2);
            const real I0 = S[i];
            const real Ix = (S[IDX(G, z, y, xmm)] - RL(8.) * S[IDX(G, z, y, xm)]
                             + RL(8.) * S[IDX(G, z, y, xp)] - S[IDX(G, z, y, xpp)]) * idx12;
            const real Iy = (S[IDX(G, z, ymm, x)] - RL(8.) * S[IDX(G, z, ym, x)]
                             + RL(8.) * S[IDX(G, z, yp, x)] - S[IDX(G, z, ypp, x)]) * idx12;
            const real Iz = (Nz > 1) ? (S[IDX(G, zmm, y, x)] - RL(8.) * S[IDX(G, zm, y, x)]
                                        + RL(8.) * S[IDX(G, zp, y, x)] - S[IDX(G, zpp, y, x)]) * idx12
                                     : RL(0.);
            const real Ixx = (-S[IDX(G, z, y, xpp)] + RL(16.) * S[IDX(G, z, y, xp)]
                              - RL(30.) * I0 + RL(16.) * S[IDX(G, z, y, xm)] - S[IDX(G, z, y, xmm)]) * idx12_sq;
            const real Iyy = (-S[IDX(G, z, ypp, x)] + RL(16.) * S[IDX(G, z, yp, x)]
                              - RL(30.) * I0 + RL(16.) * S[IDX(G, z, ym, x)] - S[IDX(G, z, ymm, x)]) * idx12_sq;
            const real Izz = (Nz > 1) ? (-S[IDX(G, zpp, y, x)] + RL(16.) * S[IDX(G, zp, y, x)]
                                         - RL(30.) * I0 + RL(16.) * S[IDX(G, zm, y, x)] - S[IDX(G, zmm, y, x)]) * idx12_sq
                                      : RL(0.);
            const int xo[4] = {xmm, xm, xp, xpp};
            const int yo[4] = {ymm, ym, yp, ypp};
            const int zo[4] = {zmm, zm, zp, zpp};
            const real dc[4] = {RL(1.), RL(-8.), RL(8.), RL(-1.)};
            real Ixy_sum = RL(0.), Ixz_sum = RL(0.), Iyz_sum = RL(0.);
            for (int a = 0; a < 4; ++a)
                for (int b = 0; b < 4; ++b) {
                    const real w = dc[a] * dc[b];
                    Ixy_sum += w * S[IDX(G, z, yo[b], xo[a])];
                    if (Nz > 1) {
                        Ixz_sum += w * S[IDX(G, zo[b], y, xo[a])];
                        Iyz_sum += w * S[IDX(G, zo[b], yo[a], x)];
                    }
                }
            const real Ixy = Ixy_sum * idx144_sq;
            const real Ixz = (Nz > 1) ? Ixz_sum * idx144_sq : RL(0.);
            const real Iyz = (Nz > 1) ? Iyz_sum * idx144_sq : RL(0.);
            const real grad_sq = Ix * Ix + Iy * Iy + Iz * Iz;
            if (grad_sq * dx * dx > RL(1e-8)) {
                const real inv_grad = RL(1.) / R_SQRT(grad_sq);
                G->nx_f[i] = -Ix * inv_grad;
                G->ny_f[i] = -Iy * inv_grad;
                G->nz_f[i] = -Iz * inv_grad;
                const real trace_H = Ixx + Iyy + Izz;
                const real gHg = Ix * Ix * Ixx + Iy * Iy * Iyy + Iz * Iz * Izz
                               + RL(2.) * (Ix * Iy * Ixy + Ix * Iz * Ixz + Iy * Iz * Iyz);
                G->kappa_f[i] = (gHg - grad_sq * trace_H) / (grad_sq * R_SQRT(grad_sq));
                if (R_FABS(G->kappa_f[i] * dx) < RL(1e-6)) G->kappa_f[i] = RL(0.);
                const real kappa_limit = RL(1.) / (G->gauss.sigma_cells * dx);
                G->kappa_f[i] = rclamp(G->kappa_f[i], -kappa_limit, kappa_limit);
            }
        }
    }
    free(labs);
    for (int i = 0; i < N; ++i) if (G->mask[i]) competitor_at(G, i);
}

static void step_geometry(OrGrid* G) {
    if (G->geom_global_separable) step_geometry_separable(G);
    else step_geometry_direct(G);
}

/* ----------------------------------------------------------------------- */
/* elastic proxy: src/gpk_physics.cpp:10-63                                  */
/* ----------------------------------------------------------------------- */
static void step_elastic(OrGrid* G) {
    const gpk_thermo_desc* th = &G->th;
    const int N = G->N, Nz = G->Nz;
    if (!th->elastic_enabled || (real)th->elastic_modulus <= RL(0.) ||
        ((real)th->eigenstrain_coeff == RL(0.) && (real)th->lambda_s == RL(0.))) {
        memset(G->E_el, 0, sizeof(real) * N);
        return;
    }
    for (int i = 0; i < N; ++i) {
        real eps = (real)th->eigenstrain_coeff * (G->c[i] - (real)th->c_ref);
        if ((real)th->lambda_s != RL(0.)) {
            real cg = R_COS(G->g[i] - (real)th->H_theta);
            eps += RL(1.5) * (real)th->lambda_s * (cg * cg - (RL(1.) / RL(3.)));
        }
        G->eps_star[i] = eps; G->eps_smooth[i] = eps;
    }
    const int iters = imax(1, th->elastic_smooth_iters);
    for (int it = 0; it < iters; ++it) {
        const real* src = G->eps_smooth; real* dst = G->eps_tmp;
        for (int i = 0; i < N; ++i) {
            int nb[6]; FACES(G, i, nb);
            real avg = src[nb[0]] + src[nb[1]] + src[nb[2]] + src[nb[3]];
            if (Nz > 1) { avg += src[nb[4]] + src[nb[5]]; avg /= RL(6.); }
            else avg /= RL(4.);
            dst[i] = RL(0.5) * src[i] + RL(0.5) * avg;
        }
        real* t = G->eps_smooth; G->eps_smooth = G->eps_tmp; G->eps_tmp = t;
    }
    for (int i = 0; i < N; ++i) {
        real d = G->eps_star[i] - G->eps_smooth[i];
        G->E_el[i] = RL(0.5) * (real)th->elastic_modulus * d * d;
    }
}

/* ----------------------------------------------------------------------- */
/* velocities: src/gpk_physics.cpp:67-148                                    */
/* ----------------------------------------------------------------------- */
static void step_velocities(OrGrid* G) {
    const gpk_thermo_desc* th = &G->th;
    memset(G->vn_f, 0, sizeof(real) * G->N);
    for (int a = 0; a < G->nactive; ++a) {
        const int i = G->active[a];
        int nei[6]; FACES(G, i, nei);
        if (th->phase_selection) {
            int32_t cand[6]; int ncand = 0;
            for (int k = 0; k < 6; ++k) {
                int32_t q = G->phi[nei[k]];
                if (q == G->phi[i]) continue;
                int seen = 0;
                for (int cc = 0; cc < ncand; ++cc) if (cand[cc] == q) { seen = 1; break; }
                if (!seen) cand[ncand++] = q;
            }
            int sel = th_select(th, G->phi[i], G->c[i], G->T[i], cand, ncand);
            if (sel >= 0) G->phi_comp[i] = sel;
        }
        const int32_t qid = G->phi_comp[i];
        real g_p = G->g[i], g_q = g_p;
        real c_q = G->c[i];
        for (int k = 0; k < 6; ++k)
            if (G->phi[nei[k]] == qid) { g_q = G->g[nei[k]]; c_q = G->c[nei[k]]; break; }
        G->g_comp[i] = g_q;
        const real c_iface = th_iface_comp(th, G->phi[i], qid, G->c[i], c_q);
        real dG = th_bulk(th, G->phi[i], qid, c_iface, G->T[i]);
        real sig = th_sigma(th, G->nx_f[i], G->ny_f[i], G->nz_f[i], g_p, G->phi[i], qid, G->c[i]);
        real mob = th_mobility(th, g_p, g_q, G->T[i]);
        if (th->elastic_enabled) {
            real E_prod = G->E_el[i];
            for (int k = 0; k < 6; ++k) if (G->phi[nei[k]] == qid) { E_prod = G->E_el[nei[k]]; break; }
            dG += (E_prod - G->E_el[i]);
        }
        if (th->dislocation_enabled) {
            real rho_prod = G->rho[i];
            for (int k = 0; k < 6; ++k) if (G->phi[nei[k]] == qid) { rho_prod = G->rho[nei[k]]; break; }
            dG += (real)th->disloc_coeff * (rho_prod - G->rho[i]);
        }
        if (th->magnetic_enabled) dG += th_Emag(th, g_q) - th_Emag(th, g_p);
        G->vn_f[i] = mob * (dG - sig * G->kappa_f[i]);
    }
}

/* ----------------------------------------------------------------------- */
/* pair velocity projection: src/gpk_physics.cpp:152-193                     */
/* ----------------------------------------------------------------------- */
static void step_velocity_projection(OrGrid* G) {
    const int Nz = G->Nz, Ny = G->Ny, Nx = G->Nx;
    memcpy(G->alpha_new, G->vn_f, sizeof(real) * G->N);
    const real vs = G->velocity_gauss.sigma_cells;
    const int radius = imax(1, (int)R_CEIL(RL(3.) * vs));
    const real inv_two_sigma2 = RL(0.5) / (vs * vs);
    for (int a = 0; a < G->nactive; ++a) {
        const int i = G->active[a];
        if (G->phi[i] == G->phi_comp[i]) continue;
        const int32_t low = G->phi[i] < G->phi_comp[i] ? G->phi[i] : G->phi_comp[i];
        const int32_t high = G->phi[i] < G->phi_comp[i] ? G->phi_comp[i] : G->phi[i];
        const real orientation_i = G->phi[i] == low ? RL(1.) : RL(-1.);
        int z0, y0, x0; DECODE(G, i, &z0, &y0, &x0);
        double numerator = 0.0, denominator = 0.0;
        const int dz0 = Nz > 1 ? -radius : 0, dz1 = Nz > 1 ? radius : 0;
        for (int dz = dz0; dz <= dz1; ++dz)
            for (int dy = -radius; dy <= radius; ++dy)
                for (int dxs = -radius; dxs <= radius; ++dxs) {
                    int z = (z0 + dz) % Nz; if (z < 0) z += Nz;
                    int y = (y0 + dy) % Ny; if (y < 0) y += Ny;
                    int x = (x0 + dxs) % Nx; if (x < 0) x += Nx;
                    const int j = IDX(G, z, y, x);
                    const int32_t pj = G->phi[j], qj = G->phi_comp[j];
                    if (!G->mask[j] || pj == qj || (pj < qj ? pj : qj) != low || (pj < qj ? qj : pj) != high)
                        continue;
                    const real r2 = (real)(dxs * dxs + dy * dy + dz * dz);
                    const double weight = (double)R_EXP(-r2 * inv_two_sigma2);
                    const real orientation_j = pj == low ? RL(1.) : RL(-1.);
                    numerator += weight * orientation_j * G->vn_f[j];
                    denominator += weight;
                }
        if (denominator > 0.0) G->alpha_new[i] = orientation_i * (real)(numerator / denominator);
    }
    real* t = G->vn_f; G->vn_f = G->alpha_new; G->alpha_new = t;
}

/* ----------------------------------------------------------------------- */
/* timestep: src/gpk_simulation.cpp:11-23                                   */
/* ----------------------------------------------------------------------- */
static real max_dt_impl(OrGrid* G) {
    real vmax = RL(1e-30);
    for (int a = 0; a < G->nactive; ++a) vmax = rmax(vmax, R_FABS(G->vn_f[G->active[a]]));
    const real neighbors = (G->Nz > 1) ? RL(6.) : RL(4.);
    const real dt_iface = RL(0.125) * G->dx / vmax;
    const real dt_diff = (G->D > RL(0.)) ? RL(0.4) * G->dx * G->dx / (neighbors * G->D) : RL(1e30);
    return rmin(dt_iface, dt_diff);
}
double SFX(or_max_dt)(OrGrid* G) { return (double)max_dt_impl(G); }

/* ----------------------------------------------------------------------- */
/* digital-topology certificate: src/gpk_connectivity.cpp:10-195             */
/* ----------------------------------------------------------------------- */
static int topological_number(const OrGrid* G, int cell, int32_t label) {
    const int Nz = G->Nz, Ny = G->Ny, Nx = G->Nx;
    int z0, y0, x0; DECODE(G, cell, &z0, &y0, &x0);
    const int lz_count = (Nz > 1) ? 3 : 1;
    const int lz_centre = (Nz > 1) ? 1 : 0;
    const int centre = lz_centre * 9 + 4;
    uint8_t occupied[27] = {0}, seen[27] = {0};
    for (int lz = 0; lz < lz_count; ++lz) {
        const int dz = (Nz > 1) ? lz - 1 : 0;
        int z = z0 + dz; if (z < 0) z += Nz; else if (z >= Nz) z -= Nz;
        for (int ly = 0; ly < 3; ++ly) {
            int y = y0 + ly - 1; if (y < 0) y += Ny; else if (y >= Ny) y -= Ny;
            for (int lx = 0; lx < 3; ++lx) {
                int x = x0 + lx - 1; if (x < 0) x += Nx; else if (x >= Nx) x -= Nx;
                occupied[lz * 9 + ly * 3 + lx] = G->phi[IDX(G, z, y, x)] == label;
            }
        }
    }
    occupied[centre] = 0;
    int component_count = 0;
    for (int seed = 0; seed < 27; ++seed) {
        const int sz = seed / 9;
        if (sz >= lz_count || !occupied[seed] || seen[seed]) continue;
        int queue[27]; int head = 0, tail = 0;
        queue[tail++] = seed; seen[seed] = 1;
        int touches = 0;
        while (head < tail) {
            const int cur = queue[head++];
            const int cz = cur / 9, rem = cur % 9, cy = rem / 3, cx = rem % 3;
            const int man = abs(cz - lz_centre) + abs(cy - 1) + abs(cx - 1);
            if (man == 1) touches = 1;
            for (int dz = -1; dz <= 1; ++dz)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dxc = -1; dxc <= 1; ++dxc) {
                        if (abs(dz) + abs(dy) + abs(dxc) != 1) continue;
                        const int nz = cz + dz, ny = cy + dy, nx = cx + dxc;
                        if (nz < 0 || nz >= lz_count || ny < 0 || ny >= 3 || nx < 0 || nx >= 3) continue;
                        const int next = nz * 9 + ny * 3 + nx;
                        if (occupied[next] && !seen[next]) { seen[next] = 1; queue[tail++] = next; }
                    }
        }
        if (touches) ++component_count;
    }
    return component_count;
}

static int global_branches_connected(const OrGrid* G, int cell, int32_t label, int exclude_centre) {
    int nb[6]; FACES(G, cell, nb);
    const int nface = G->Nz > 1 ? 6 : 4;
    int branches[6], nbr = 0;
    for (int k = 0; k < nface; ++k) if (G->phi[nb[k]] == label) branches[nbr++] = nb[k];
    if (nbr <= 1) return 1;
    /* targets = distinct branches[1..] */
    int targets[6], nt = 0;
    for (int k = 1; k < nbr; ++k) {
        int dup = 0; for (int t = 0; t < nt; ++t) dup |= targets[t] == branches[k];
        if (!dup) targets[nt++] = branches[k];
    }
    OrGrid* GM = (OrGrid*)G;
    if (++GM->ff_epoch == 0) { memset(GM->ff_stamp, 0, sizeof(uint32_t) * (size_t)G->N); GM->ff_epoch = 1; }
    const uint32_t ep = GM->ff_epoch;
    uint32_t* visited = GM->ff_stamp;
    int* stack = GM->ff_stack;
    int sp = 0;
    stack[sp++] = branches[0]; visited[branches[0]] = ep;
    int result = -1;
    while (sp > 0 && result < 0) {
        const int cur = stack[--sp];
        int nx[6]; FACES(G, cur, nx);
        for (int k = 0; k < nface; ++k) {
            const int next = nx[k];
            if (visited[next] == ep || G->phi[next] != label || (exclude_centre && next == cell)) continue;
            visited[next] = ep;
            for (int t = 0; t < nt; ++t)
                if (targets[t] == next) { targets[t] = targets[--nt]; break; }
            if (nt == 0) { result = 1; break; }
            stack[sp++] = next;
        }
    }
    if (result < 0) result = nt == 0;
    return result;
}

static int bounded_branches_connected(const OrGrid* G, int cell, int32_t label, int exclude_centre) {
    const int Nz = G->Nz, Ny = G->Ny, Nx = G->Nx;
    enum { radius = 2, side = 5, plane = 25, capacity = 125 };
    int z0, y0, x0; DECODE(G, cell, &z0, &y0, &x0);
    const int zcount = Nz > 1 ? side : 1, zcentre = Nz > 1 ? radius : 0;
    const int local_centre = zcentre * plane + radius * side + radius;
    uint8_t occupied[capacity] = {0}, seen[capacity] = {0};
    for (int lz = 0; lz < zcount; ++lz) {
        const int dz = Nz > 1 ? lz - radius : 0;
        int z = z0 + dz; while (z < 0) z += Nz; while (z >= Nz) z -= Nz;
        for (int ly = 0; ly < side; ++ly) {
            int y = y0 + ly - radius; while (y < 0) y += Ny; while (y >= Ny) y -= Ny;
            for (int lx = 0; lx < side; ++lx) {
                int x = x0 + lx - radius; while (x < 0) x += Nx; while (x >= Nx) x -= Nx;
                occupied[lz * plane + ly * side + lx] = G->phi[IDX(G, z, y, x)] == label;
            }
        }
    }
    if (exclude_centre) occupied[local_centre] = 0;
    const int branch_local[6] = {
        zcentre * plane + radius * side + (radius - 1), zcentre * plane + radius * side + (radius + 1),
        zcentre * plane + (radius - 1) * side + radius, zcentre * plane + (radius + 1) * side + radius,
        (zcentre - 1) * plane + radius * side + radius, (zcentre + 1) * plane + radius * side + radius};
    const int nface = Nz > 1 ? 6 : 4;
    int branches[6], nbranch = 0;
    for (int k = 0; k < nface; ++k) if (occupied[branch_local[k]]) branches[nbranch++] = branch_local[k];
    if (nbranch <= 1) return 1;
    int queue[capacity], head = 0, tail = 0;
    queue[tail++] = branches[0]; seen[branches[0]] = 1;
    const int dzv[6] = {0, 0, 0, 0, -1, 1}, dyv[6] = {0, 0, -1, 1, 0, 0}, dxv[6] = {-1, 1, 0, 0, 0, 0};
    while (head < tail) {
        const int cur = queue[head++];
        const int cz = cur / plane, rem = cur % plane, cy = rem / side, cx = rem % side;
        for (int k = 0; k < nface; ++k) {
            const int zz = cz + dzv[k], yy = cy + dyv[k], xx = cx + dxv[k];
            if (zz < 0 || zz >= zcount || yy < 0 || yy >= side || xx < 0 || xx >= side) continue;
            const int next = zz * plane + yy * side + xx;
            if (occupied[next] && !seen[next]) { seen[next] = 1; queue[tail++] = next; }
        }
    }
    for (int k = 1; k < nbranch; ++k) if (!seen[branches[k]]) return 0;
    return 1;
}

static int topology_simple_move_counted(const OrGrid* G, int cell, int32_t new_label,
                                        int old_count, int new_count, int local_only) {
    (void)new_count;
    if (cell < 0 || cell >= G->N) return 0;
    const int32_t old_label = G->phi[cell];
    if (old_label == new_label) return 0;
    const int old_object = topological_number(G, cell, old_label);
    const int old_extinction = old_count <= 1;
    if (old_object == 0 && !old_extinction) return 0;
    if (old_object > 1 && !(local_only ? bounded_branches_connected(G, cell, old_label, 1)
                                       : global_branches_connected(G, cell, old_label, 1)))
        return 0;
    const int new_object = topological_number(G, cell, new_label);
    if (new_object == 0) return 0;
    if (new_object > 1 && !(local_only ? bounded_branches_connected(G, cell, new_label, 0)
                                       : global_branches_connected(G, cell, new_label, 0)))
        return 0;
    return 1;
}

int SFX(or_topology_simple_move)(OrGrid* G, int cell, int32_t new_label) {
    if (cell < 0 || cell >= G->N) return 0;
    const int32_t old_label = G->phi[cell];
    int oc = 0, nc = 0;
    for (int i = 0; i < G->N; ++i) { oc += G->phi[i] == old_label; nc += G->phi[i] == new_label; }
    return topology_simple_move_counted(G, cell, new_label, oc, nc, 0);
}

/* ----------------------------------------------------------------------- */
/* balanced Gaussian remap: src/gpk_transitions.cpp:38-178                   */
/* ----------------------------------------------------------------------- */
typedef struct { int32_t low, high; int dir; real gain; int cell; } proposal_t;

static int proposal_cmp(const void* pa, const void* pb) {
    const proposal_t* a = (const proposal_t*)pa; const proposal_t* b = (const proposal_t*)pb;
    if (a->low != b->low) return a->low < b->low ? -1 : 1;
    if (a->high != b->high) return a->high < b->high ? -1 : 1;
    if (a->dir != b->dir) return a->dir < b->dir ? -1 : 1;
    if (a->gain != b->gain) return a->gain > b->gain ? -1 : 1;
    return a->cell < b->cell ? -1 : (a->cell > b->cell ? 1 : 0);
}

static real target_orientation(const OrGrid* G, int cell, int32_t target) {
    int nei[6]; FACES(G, cell, nei);
    const int nface = G->Nz > 1 ? 6 : 4;
    for (int k = 0; k < nface; ++k) if (G->phi[nei[k]] == target) return G->g[nei[k]];
    return G->g[cell];
}
static int mismatch_count(const OrGrid* G, int cell, int32_t proposed, int paired, int32_t paired_proposed) {
    int nei[6]; FACES(G, cell, nei);
    const int nface = G->Nz > 1 ? 6 : 4;
    int m = 0;
    for (int k = 0; k < nface; ++k) {
        const int32_t q = (nei[k] == paired) ? paired_proposed : G->phi[nei[k]];
        m += q != proposed;
    }
    return m;
}

static void step_balanced_gaussian_remap(OrGrid* G) {
    const int Nz = G->Nz, Ny = G->Ny, Nx = G->Nx, N = G->N;
    G->gaussian_remap_exchanges_last = 0;
    if (G->topology_accepted_last == 0) return;
    step_interface_mask(G);
    for (int i = 0; i < N; ++i) { G->eps_star[i] = (real)-INFINITY; G->eps_smooth[i] = (real)-INFINITY; }
    memcpy(G->phi_comp, G->phi, sizeof(int32_t) * N);
    const real rs = G->remap_gauss.sigma_cells;
    const int radius = imax(1, (int)R_CEIL(RL(3.) * rs));
    const real inv_two_sigma2 = RL(0.5) / (rs * rs);
    for (int a = 0; a < G->nactive; ++a) {
        const int i = G->active[a];
        int z0, y0, x0; DECODE(G, i, &z0, &y0, &x0);
        int face[6]; FACES(G, i, face);
        const int nface = Nz > 1 ? 6 : 4;
        int32_t candidate[6]; int ncand = 0;
        for (int k = 0; k < nface; ++k) {
            const int32_t v = G->phi[face[k]];
            if (v == G->phi[i]) continue;
            int known = 0; for (int q = 0; q < ncand; ++q) known |= candidate[q] == v;
            if (!known) candidate[ncand++] = v;
        }
        double resident = 0.0, best = -1.0; int32_t best_label = G->phi[i];
        double support[6] = {0, 0, 0, 0, 0, 0};
        const int dz0 = Nz > 1 ? -radius : 0, dz1 = Nz > 1 ? radius : 0;
        for (int dz = dz0; dz <= dz1; ++dz)
            for (int dy = -radius; dy <= radius; ++dy)
                for (int dxs = -radius; dxs <= radius; ++dxs) {
                    int z = (z0 + dz) % Nz; if (z < 0) z += Nz;
                    int y = (y0 + dy) % Ny; if (y < 0) y += Ny;
                    int x = (x0 + dxs) % Nx; if (x < 0) x += Nx;
                    const int32_t v = G->phi[IDX(G, z, y, x)];
                    const real r2 = (real)(dxs * dxs + dy * dy + dz * dz);
                    const double weight = (double)R_EXP(-r2 * inv_two_sigma2);
                    if (v == G->phi[i]) resident += weight;
                    for (int q = 0; q < ncand; ++q) if (v == candidate[q]) support[q] += weight;
                }
        G->eps_star[i] = (real)resident;
        for (int q = 0; q < ncand; ++q) if (support[q] > best) { best = support[q]; best_label = candidate[q]; }
        G->eps_smooth[i] = (real)best;
        G->phi_comp[i] = best_label;
    }
    /* proposals grouped by unordered label pair, ranked within each direction */
    proposal_t* props = (proposal_t*)malloc(sizeof(proposal_t) * (size_t)(G->nactive + 1));
    int np = 0;
    for (int a = 0; a < G->nactive; ++a) {
        const int i = G->active[a];
        const int32_t p = G->phi[i], q = G->phi_comp[i];
        const real gain = G->eps_smooth[i] - G->eps_star[i];
        if (p == q || !(gain > RL(1e-7))) continue;
        proposal_t pr; pr.low = p < q ? p : q; pr.high = p < q ? q : p;
        pr.dir = (p == pr.low) ? 0 : 1; pr.gain = gain; pr.cell = i;
        props[np++] = pr;
    }
    qsort(props, (size_t)np, sizeof(proposal_t), proposal_cmp);
    lmap cnt; lmap_init(&cnt, 256);
    for (int i = 0; i < N; ++i) ++*lmap_ref(&cnt, G->phi[i]);
    const int sweep_rho = G->th.dislocation_enabled;
    int s = 0;
    while (s < np) {
        int e = s;
        while (e < np && props[e].low == props[s].low && props[e].high == props[s].high) ++e;
        int f0 = s, f1 = s;
        while (f1 < e && props[f1].dir == 0) ++f1;
        const int r0 = f1, r1 = e;
        const int count = (f1 - f0) < (r1 - r0) ? (f1 - f0) : (r1 - r0);
        const int32_t low = props[s].low, high = props[s].high;
        for (int k = 0; k < count; ++k) {
            const int a = props[f0 + k].cell, b = props[r0 + k].cell;
            if (G->phi[a] != low || G->phi[b] != high) continue;
            const real ga = target_orientation(G, a, high);
            const real gb = target_orientation(G, b, low);
            const int before = mismatch_count(G, a, low, b, high) + mismatch_count(G, b, high, a, low);
            const int after = mismatch_count(G, a, high, b, low) + mismatch_count(G, b, low, a, high);
            if (after >= before) continue;
            const int cl = *lmap_ref(&cnt, low), ch = *lmap_ref(&cnt, high);
            if (!topology_simple_move_counted(G, a, high, cl, ch, 1)) continue;
            G->phi[a] = high;
            if (!topology_simple_move_counted(G, b, low, ch + 1, cl - 1, 1)) { G->phi[a] = low; continue; }
            G->phi[b] = low; G->g[a] = ga; G->g[b] = gb; G->alpha[a] = G->alpha[b] = RL(1.);
            if (sweep_rho) G->rho[a] = G->rho[b] = (real)G->th.rho_rex;
            G->gaussian_remap_exchanges_last += 2;
        }
        s = e;
    }
    lmap_free(&cnt);
    free(props);
    step_interface_mask(G);
}

/* ----------------------------------------------------------------------- */
/* unresolved-grain extinction: src/gpk_transitions.cpp:180-249              */
/* ----------------------------------------------------------------------- */
static void step_complete_unresolved_grains(OrGrid* G) {
    if (!G->th.grain_network) return;
    if ((G->step_id & 7ULL) != 0ULL) return;
    const int N = G->N, Nz = G->Nz, Ny = G->Ny, Nx = G->Nx;
    lmap cnt; lmap_init(&cnt, 256);
    for (int i = 0; i < N; ++i) ++*lmap_ref(&cnt, G->phi[i]);
    const double sigma = (double)rmax(G->gauss.sigma_cells, RL(1.));
    const double support_volume = (Nz > 1) ? (4.0 * 3.14159265358979323846 * sigma * sigma * sigma / 3.0)
                                           : (3.14159265358979323846 * sigma * sigma);
    const int min_resolved = imax(2, (int)ceil(support_volume));
    /* unresolved set = labels with count < min_resolved (value 1 marks it) */
    lmap unres; lmap_init(&unres, 64);
    size_t n_unres = 0;
    for (size_t s = 0; s < cnt.cap; ++s)
        if (cnt.used[s] && cnt.vals[s] < min_resolved) { *lmap_ref(&unres, cnt.keys[s]) = 1; ++n_unres; }
    if (n_unres == 0 || n_unres == cnt.n) { lmap_free(&cnt); lmap_free(&unres); return; }
    const int sweep_rho = G->th.dislocation_enabled;
    int* cells = (int*)malloc(sizeof(int) * (size_t)N);
    int32_t* targets = (int32_t*)malloc(sizeof(int32_t) * (size_t)N);
    real* tg = (real*)malloc(sizeof(real) * (size_t)N);
    for (;;) {
        int nc = 0;
        for (int i = 0; i < N; ++i) {
            int dummy;
            if (!lmap_find(&unres, G->phi[i], &dummy)) continue;
            int z, y, x; DECODE(G, i, &z, &y, &x);
            int face[6]; FACES(G, i, face);
            const int nface = Nz > 1 ? 6 : 4;
            int best = -1, best_support = -1;
            for (int k = 0; k < nface; ++k) {
                const int32_t q = G->phi[face[k]];
                if (lmap_find(&unres, q, &dummy)) continue;
                int support = 0;
                for (int dz = (Nz > 1 ? -1 : 0); dz <= (Nz > 1 ? 1 : 0); ++dz)
                    for (int dy = -1; dy <= 1; ++dy)
                        for (int dxs = -1; dxs <= 1; ++dxs) {
                            int zz = (z + dz + Nz) % Nz, yy = (y + dy + Ny) % Ny, xx = (x + dxs + Nx) % Nx;
                            support += G->phi[IDX(G, zz, yy, xx)] == q;
                        }
                if (support > best_support) { best = k; best_support = support; }
            }
            if (best >= 0) { cells[nc] = i; targets[nc] = G->phi[face[best]]; tg[nc] = G->g[face[best]]; ++nc; }
        }
        if (nc == 0) break;
        for (int k = 0; k < nc; ++k) {
            const int i = cells[k]; G->phi[i] = targets[k]; G->g[i] = tg[k]; G->alpha[i] = RL(1.);
            if (sweep_rho) G->rho[i] = (real)G->th.rho_rex;
        }
    }
    free(cells); free(targets); free(tg);
    lmap_free(&cnt); lmap_free(&unres);
    step_interface_mask(G);
}

/* ----------------------------------------------------------------------- */
/* noise: src/gpk_transitions.cpp:17-35                                      */
/* ----------------------------------------------------------------------- */
static inline uint64_t mix64(uint64_t x) {
    x ^= x >> 30; x *= 0xbf58476d1ce4e5b9ULL;
    x ^= x >> 27; x *= 0x94d049bb133111ebULL;
    x ^= x >> 31;
    return x;
}
static inline real u01_from_u64(uint64_t x) {
    const uint64_t m = (x >> 11) | 1ULL;
    return (real)((double)(m & ((1ULL << 53) - 1)) * (1.0 / (double)(1ULL << 53)));
}
static inline real normal_from_cell_step(int i, uint64_t step_id, uint64_t salt) {
    uint64_t a = mix64(((uint64_t)i + 0x9e3779b97f4a7c15ULL) ^ (step_id << 1) ^ salt);
    uint64_t b = mix64(((uint64_t)i + 0xd2b74407b1ce6e93ULL) ^ (step_id << 3) ^ (salt + 17ULL));
    real u1 = rmax(RL(1e-12), u01_from_u64(a));
    real u2 = u01_from_u64(b);
    return R_SQRT(RL(-2.) * R_LOG(u1)) * R_COS(RL(2.) * (real)R_PI * u2);
}

/* ----------------------------------------------------------------------- */
/* alpha integration + serial crossings: src/gpk_transitions.cpp:251-326     */
/* ----------------------------------------------------------------------- */
static void step_alpha(OrGrid* G, real dt) {
    const gpk_thermo_desc* th = &G->th;
    const int N = G->N;
    const real dx = G->dx;
    const real idt = dt / dx;
    const real cell_vol = dx * dx * dx;
    const real inv_dt = (dt > RL(0.)) ? (RL(1.) / dt) : RL(0.);
    const int do_noise = th->stochastic && dt > RL(0.);
    const real noise_amp = do_noise
        ? (real)th->noise_scale * R_SQRT(RL(2.) * (real)th->M0 * (real)th->kB * inv_dt / rmax(cell_vol, RL(1e-30)))
        : RL(0.);
    memcpy(G->alpha_new, G->alpha, sizeof(real) * N);
    for (int a = 0; a < G->nactive; ++a) {
        const int i = G->active[a];
        real vn_eff = G->vn_f[i];
        if (do_noise)
            vn_eff += noise_amp * R_SQRT(rmax(G->T[i], RL(1.))) * normal_from_cell_step(i, G->step_id, 0xabcddcbaULL);
        G->alpha_new[i] = rmin(G->alpha[i] + vn_eff * idt, RL(1.));
    }
    /* the decision alpha_new <= 1e-6 && phi_comp != phi, listed where the
     * margin alpha_new - 1e-6 lies within near_tol of zero */
    G->n_near = 0;
    const real near_tol = (real)G->near_tol;
    for (int a = 0; a < G->nactive; ++a) {
        const int i = G->active[a];
        if (G->phi_comp[i] != G->phi[i] && R_FABS(G->alpha_new[i] - RL(1e-6)) <= near_tol) G->near[G->n_near++] = i;
    }
    lmap cnt; lmap_init(&cnt, 256);
    for (int i = 0; i < N; ++i) ++*lmap_ref(&cnt, G->phi[i]);
    G->topology_accepted_last = 0;
    G->topology_deferred_last = 0;
    const int sweep_rho = th->dislocation_enabled;
    const real rho_rex = (real)th->rho_rex;
    const int tracks = th->grain_network;
    for (int a = 0; a < G->nactive; ++a) {
        const int i = G->active[a];
        if (!(G->alpha_new[i] <= RL(1e-6) && G->phi_comp[i] != G->phi[i])) {
            G->alpha[i] = G->alpha_new[i];
            continue;
        }
        const int32_t old_label = G->phi[i];
        const int32_t new_label = G->phi_comp[i];
        int* oc = lmap_ref(&cnt, old_label);
        const int old_count = *oc;
        const int new_count = *lmap_ref(&cnt, new_label);
        if (!tracks || topology_simple_move_counted(G, i, new_label, old_count, new_count, 0)) {
            G->phi[i] = new_label;
            G->g[i] = G->g_comp[i];
            G->alpha[i] = RL(1.);
            --*lmap_ref(&cnt, old_label);
            ++*lmap_ref(&cnt, new_label);
            ++G->topology_accepted_last;
            if (sweep_rho) G->rho[i] = rho_rex;
        } else {
            G->alpha[i] = rmax(G->alpha_new[i], RL(1e-6));
            ++G->topology_deferred_last;
        }
    }
    lmap_free(&cnt);
    step_balanced_gaussian_remap(G);
    if (G->Nz > 1 && G->gaussian_remap_exchanges_last > 0) {
        const uint64_t first = G->gaussian_remap_exchanges_last;
        step_balanced_gaussian_remap(G);
        G->gaussian_remap_exchanges_last += first;
    }
    step_complete_unresolved_grains(G);
}

/* ----------------------------------------------------------------------- */
/* transport + recovery: src/gpk_transport.cpp:11-152                        */
/* ----------------------------------------------------------------------- */
static void step_diffusion(OrGrid* G, real dt) {
    if (G->D <= RL(0.)) return;
    const real* cm = G->c;
    const real dx2 = G->dx * G->dx;
    for (int i = 0; i < G->N; ++i) {
        int nb[6]; FACES(G, i, nb);
        real lap = cm[nb[1]] + cm[nb[0]] + cm[nb[3]] + cm[nb[2]];
        if (G->Nz > 1) lap += cm[nb[5]] + cm[nb[4]] - RL(6.) * cm[i];
        else lap -= RL(4.) * cm[i];
        real D_eff = G->mask[i] ? G->D * G->alpha[i] : G->D;
        G->c_new[i] = cm[i] + dt * D_eff * lap / dx2;
    }
    real* t = G->c; G->c = G->c_new; G->c_new = t;
}

static void cell_solid_fraction(const OrGrid* G, real* s) {
    for (int i = 0; i < G->N; ++i) s[i] = (G->phi[i] != 0) ? G->alpha[i] : RL(1.) - G->alpha[i];
}

/* rejection-side neighbour order: x+, x-, y+, y-, z+, z- (src/gpk_transport.cpp:71-79) */
static int faces_transport(const OrGrid* G, int i, int nb[6]) {
    int z, y, x; DECODE(G, i, &z, &y, &x);
    const int Nx = G->Nx, Ny = G->Ny, Nz = G->Nz;
    int nn = 0;
    nb[nn++] = IDX(G, z, y, x == Nx - 1 ? 0 : x + 1);
    nb[nn++] = IDX(G, z, y, x == 0 ? Nx - 1 : x - 1);
    nb[nn++] = IDX(G, z, y == Ny - 1 ? 0 : y + 1, x);
    nb[nn++] = IDX(G, z, y == 0 ? Ny - 1 : y - 1, x);
    if (Nz > 1) {
        nb[nn++] = IDX(G, z == Nz - 1 ? 0 : z + 1, y, x);
        nb[nn++] = IDX(G, z == 0 ? Nz - 1 : z - 1, y, x);
    }
    return nn;
}

static void step_solute_rejection(OrGrid* G) {
    const real k = (real)G->th.k_partition;
    if (k >= RL(1.) || !G->have_solid_old) return;
    const int N = G->N;
    real* s_new = ralloc(N, RL(0.));
    cell_solid_fraction(G, s_new);
    real* delta = ralloc(N, RL(0.));
    for (int i = 0; i < N; ++i) {
        const real ds = s_new[i] - G->solid_old[i];
        if (ds <= RL(0.)) continue;
        const real s0 = rclamp(G->solid_old[i], RL(0.), RL(1.));
        const real cL = G->c[i] / rmax(RL(1.) - s0 * (RL(1.) - k), RL(1e-6));
        real q = (RL(1.) - k) * cL * rmin(ds, RL(1.));
        q = rmin(q, G->c[i]);
        if (q <= RL(0.)) continue;
        int nb[6]; const int nn = faces_transport(G, i, nb);
        real wsum = RL(0.), w[6];
        for (int a = 0; a < nn; ++a) {
            const int j = nb[a];
            w[a] = (G->phi[j] == 0) ? rmax(RL(1.) - s_new[j], RL(0.)) : RL(0.);
            wsum += w[a];
        }
        if (wsum <= RL(0.)) continue;
        delta[i] -= q;
        for (int a = 0; a < nn; ++a) if (w[a] > RL(0.)) delta[nb[a]] += q * w[a] / wsum;
    }
    for (int i = 0; i < N; ++i) G->c[i] += delta[i];
    free(s_new); free(delta);
}

static void step_diffusion_partitioned(OrGrid* G, real dt) {
    if (G->D <= RL(0.)) return;
    const real k = (real)G->th.k_partition;
    const int N = G->N;
    real* s = ralloc(N, RL(0.));
    real* cL = ralloc(N, RL(0.));
    cell_solid_fraction(G, s);
    for (int i = 0; i < N; ++i) cL[i] = G->c[i] / rmax(RL(1.) - s[i] * (RL(1.) - k), RL(1e-6));
    const real coef = dt * G->D / (G->dx * G->dx);
    /* solid diffusion (builder-defined): the solid composition k cL diffuses
     * with ratio x D through the face's shared solid fraction, so the face
     * weight is lf + ratio k min(s_i, s_j); ratio 0 is the reference */
    const real rsk = (real)G->solid_ratio * k;
    for (int i = 0; i < N; ++i) {
        int nb[6]; const int nn = faces_transport(G, i, nb);
        const real li = RL(1.) - s[i];
        real flux = RL(0.);
        for (int a = 0; a < nn; ++a) {
            const int j = nb[a];
            const real lf = rmin(li, RL(1.) - s[j]);
            if (rsk > RL(0.)) {
                const real w = lf + rsk * rmin(s[i], s[j]);
                if (w > RL(0.)) flux += w * (cL[j] - cL[i]);
            } else if (lf > RL(0.)) {
                flux += lf * (cL[j] - cL[i]);
            }
        }
        G->c_new[i] = G->c[i] + coef * flux;
    }
    real* t = G->c; G->c = G->c_new; G->c_new = t;
    free(s); free(cL);
}

static void step_recovery(OrGrid* G, real dt) {
    const gpk_thermo_desc* th = &G->th;
    if (!th->dislocation_enabled || (real)th->recovery_rate <= RL(0.) || dt <= RL(0.)) return;
    const real decay = R_EXP(-(real)th->recovery_rate * dt);
    for (int i = 0; i < G->N; ++i) G->rho[i] *= decay;
}

/* ----------------------------------------------------------------------- */
/* one step: src/gpk_simulation.cpp:31-54                                   */
/* ----------------------------------------------------------------------- */
double SFX(or_step)(OrGrid* G, double dt_d, double dt_cap_d) {
    real dt = (real)dt_d;
    const real dt_cap = (real)dt_cap_d;
    step_interface_mask(G);
    step_geometry(G);
    step_elastic(G);
    step_velocities(G);
    step_velocity_projection(G);
    const real dt_stable = max_dt_impl(G);
    if (dt < RL(0.)) dt = dt_stable;
    else dt = rmin(dt, dt_stable);
    dt = rmin(dt, dt_cap);
    const int partition = G->th.solute_rejection;
    if (partition) { cell_solid_fraction(G, G->solid_old); G->have_solid_old = 1; }
    step_alpha(G, dt);
    if (partition) {
        step_solute_rejection(G);
        step_diffusion_partitioned(G, dt);
    } else {
        step_diffusion(G, dt);
    }
    step_recovery(G, dt);
    G->time += dt;
    ++G->step_id;
    return (double)dt;
}

/* run(): src/gpk_simulation.cpp:60-73, without callback */
int SFX(or_run)(OrGrid* G, double t_end, double dt, int max_steps) {
    int n = 0;
    while (G->time < t_end && (max_steps <= 0 || n < max_steps)) {
        const real remaining = (real)(t_end - G->time);
        SFX(or_step)(G, dt, (double)remaining);
        ++n;
    }
    return n;
}

/* ----------------------------------------------------------------------- */
/* diagnostics: src/gpk_simulation.cpp:78-124                                */
/* ----------------------------------------------------------------------- */
double SFX(or_phase_volume)(OrGrid* G, int32_t label) {
    double v = 0.0;
    for (int i = 0; i < G->N; ++i) {
        if (G->phi[i] == label) v += G->alpha[i];
        if (G->mask[i] && G->phi_comp[i] == label && G->phi_comp[i] != G->phi[i]) v += 1.0 - G->alpha[i];
    }
    return v;
}
int SFX(or_n_grains)(OrGrid* G) {
    lmap m; lmap_init(&m, 256);
    for (int i = 0; i < G->N; ++i) *lmap_ref(&m, G->phi[i]) = 1;
    const int n = (int)m.n;
    lmap_free(&m);
    return n;
}
double SFX(or_interface_fraction)(OrGrid* G) {
    int cnt = 0;
    for (int i = 0; i < G->N; ++i) if (G->mask[i]) ++cnt;
    return (double)((float)cnt / (float)G->N);
}
/* mask + active list without stepping (used by tests of the compaction) */
void SFX(or_interface_mask)(OrGrid* G) { step_interface_mask(G); }
