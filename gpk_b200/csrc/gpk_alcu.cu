// gpk_alcu.cu — Al-Cu per-step Cu transport and Gaussian label remap (FP64, sm_100a).
//
// Restates the numpy/scipy functions the reference's Al-Cu driver runs once
// per step (scripts/run_alcu_gpk_microstructure.py): neighbor_competitor
// (260-276), precip_fraction (675-676), diffuse_conservative[_subcycled]
// (679-699), conservative_partition_transfer (702-737),
// interface_matrix_composition (740-755) and conservative_gaussian_remap
// (562-594), bit for bit:
//
//  * elementwise arithmetic in numpy's operand order, built without FMA
//    contraction; numpy's maximum/clip keep their own argument on ties;
//  * np.sum of a float64 field = numpy's pairwise summation of the flattened
//    array: leaves of at most 128 values, each summed by 8 running partials
//    (here 8 lanes, combined ((r0+r1)+(r2+r3))+((r4+r5)+(r6+r7))), ranges
//    above 128 split at half the length rounded down to a multiple of 8.  The
//    tree depends on N only; the host cuts it at sizes 128 * 32^k, and each
//    level is one launch (a thread per node walks its subtree);
//  * scipy.ndimage.gaussian_filter(mode="wrap") = three periodic passes (axis
//    0, 1, 2), each output x[i] w0 + (x[i-j] + x[i+j]) w_j added for
//    j = r, ..., 1;
//  * the remap's components (scipy `label`: face connectivity, no wrap,
//    numbered by first cell) come from a union-find that links to the smaller
//    root, so a component's root is its first cell.  The reference relabels
//    components one after the other; a component reads and writes only cells
//    of its 3^d dilation, so two components interact only when their
//    dilations meet.  Components are scheduled in waves (the longest chain of
//    earlier interacting components, relaxed to a fixed point over the cells
//    where dilations meet); a wave's components run together and the result
//    is that of the serial order.  The cells of any component's dilation
//    (the band: the 3^d box maximum of the active cells, three separable
//    passes, then an exact test) are compacted once per call; per wave,
//    candidates are compacted from the band in cell order, scores evaluated
//    per candidate from the component's indicator
//    (the three passes restricted to the (2r+1)^d box, same operations), two
//    stable radix sorts (score descending, then component), and the first
//    `size` entries of each component's run take its label.
//
// Cell kernels take their coordinates from a 3-D launch (a 2-D field is held
// as 1 x n0 x n1); periodic neighbours wrap by a compare.  Every kernel is
// HBM- or latency-bound FP64 work; none is a contraction.
#include <cuda_runtime.h>
#include <cub/cub.cuh>

#include <cmath>
#include <string>
#include <vector>

#include "../../include/gpk_alcu.h"
#include "gpk_grid.h"

namespace {

#define ALCU_TRY(expr)                                                                 \
    do {                                                                               \
        cudaError_t _e = (expr);                                                       \
        if (_e != cudaSuccess) {                                                       \
            gpk_set_error(std::string(#expr " failed: ") + cudaGetErrorString(_e));    \
            return GPK_ERR_CUDA;                                                       \
        }                                                                              \
    } while (0)

struct Ext {
    int e[3];        // extents; a 2-D field (n0, n1) is held as (1, n0, n1)
    long long st[3]; // strides of the C-order layout
    int ndim;
    int a0;          // first axis that belongs to the field (3 - ndim)
    long long N;
};

struct Taps {
    double w[GPK_ALCU_MAX_RADIUS + 1];  // w[j]: the tap at offsets -j and +j
    int r;
};

struct Phys {
    double dx, D, ceq, ct;
};

__device__ __forceinline__ int wrapi(int x, int n) {
    const int r = x % n;
    return r < 0 ? r + n : r;
}
// x + off on a periodic axis of n points; `near` when |off| <= n
__device__ __forceinline__ int wrap_off(int y, int n, bool near) {
    if (near) return y < 0 ? y + n : (y >= n ? y - n : y);
    return wrapi(y, n);
}
// numpy's float maximum / clip (no NaN reaches these here): the first
// argument is kept only when strictly beyond the bound
__device__ __forceinline__ double np_max(double a, double b) { return a > b ? a : b; }
__device__ __forceinline__ double np_clip(double x, double lo, double hi) { return x < lo ? lo : (x > hi ? hi : x); }

#define GRID_STRIDE(i, n) \
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (n); i += (long long)gridDim.x * blockDim.x)

// one thread per cell of a (32 x 4) block tile of axes 2 and 1, looping over
// axis 0: the coordinates come from the launch, not from divisions
#define CELLS3(d)                                                                           \
    for (int x1 = blockIdx.y * 4 + threadIdx.y; x1 < (d).e[1]; x1 += gridDim.y * 4)         \
        for (int x0 = blockIdx.z; x0 < (d).e[0]; x0 += gridDim.z)                           \
            if (const int x2 = blockIdx.x * 32 + threadIdx.x; x2 < (d).e[2])
#define CELL_INDEX(d) (((long long)x0 * (d).e[1] + x1) * (d).e[2] + x2)

// ---------------------------------------------------------------- elementwise

__global__ void __launch_bounds__(128) k_competitor(Ext d, const int8_t* __restrict__ lab, uint8_t* __restrict__ mask,
                                                    int8_t* __restrict__ comp) {
    CELLS3(d) {
        const long long i = CELL_INDEX(d);
        const int x[3] = {x0, x1, x2};
        const int8_t l = lab[i];
        bool m = false, mat = false;
        int s1 = 0, s2 = 0, s3 = 0;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            if (a < d.a0) continue;
            const int n = d.e[a];
            const long long ip = i + (long long)((x[a] + 1 == n ? 0 : x[a] + 1) - x[a]) * d.st[a];
            const long long im = i + (long long)((x[a] == 0 ? n - 1 : x[a] - 1) - x[a]) * d.st[a];
            const int8_t nbs[2] = {lab[im], lab[ip]};
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int8_t nb = nbs[q];
                m |= nb != l;
                mat |= nb == 0;
                s1 += nb == 1;
                s2 += nb == 2;
                s3 += nb == 3;
            }
        }
        // argmax over (s1, s2, s3), first maximum
        int8_t c = 1;
        int best = s1;
        if (s2 > best) { c = 2; best = s2; }
        if (s3 > best) { c = 3; }
        if (l > 0 && mat) c = 0;
        if (!m) c = l;
        mask[i] = m ? 1 : 0;
        comp[i] = c;
    }
}

__global__ void k_precip_fraction(long long N, const int8_t* __restrict__ lab, const double* __restrict__ alpha,
                                  const int8_t* __restrict__ comp, double* __restrict__ fp) {
    GRID_STRIDE(i, N) fp[i] = lab[i] > 0 ? alpha[i] : (comp[i] > 0 ? 1.0 - alpha[i] : 0.0);
}

// variant_fraction_fields (lines 278-283): fraction * (variant == v), the
// product taken as numpy takes it (times 1.0 or 0.0, so a negative fraction
// gives -0.0 off its variant)
__global__ void k_variant_fractions(long long N, const int8_t* __restrict__ lab, const double* __restrict__ alpha,
                                    const int8_t* __restrict__ comp, double* __restrict__ out) {
    GRID_STRIDE(i, N) {
        const int l = lab[i], c = comp[i];
        const double f = l > 0 ? alpha[i] : (c > 0 ? 1.0 - alpha[i] : 0.0);
        const int v = l > 0 ? l : c;
#pragma unroll
        for (int k = 0; k < 3; ++k) out[k * N + i] = f * (v == k + 1 ? 1.0 : 0.0);
    }
}

// matrix fraction max(1 - f, 1e-8) and the clipped lever-rule composition
__device__ __forceinline__ void lever(double c, double f, const Phys& p, double& m, double& cm) {
    if (f == 0.0) {
        // matrix cell: m = 1 exactly, and x / 1 = x for every x
        m = 1.0;
        cm = np_clip(c - f * p.ct, 0.0, p.ct);
        return;
    }
    m = np_max(1.0 - f, 1e-8);
    const double raw = m > 1e-7 ? (c - f * p.ct) / m : p.ceq;
    cm = np_clip(raw, 0.0, p.ct);
}

__global__ void k_matrix_composition(long long N, Phys p, const double* __restrict__ c, const double* __restrict__ f,
                                     double* __restrict__ cm) {
    GRID_STRIDE(i, N) {
        double m, v;
        lever(c[i], f[i], p, m, v);
        cm[i] = v;
    }
}

// one explicit substep of diffuse_conservative (lines 679-688)
__global__ void __launch_bounds__(128) k_diffuse(Ext d, Phys p, double dt, const double* __restrict__ c,
                                                 const double* __restrict__ f, double* __restrict__ out,
                                                 double* __restrict__ cm_out) {
    CELLS3(d) {
        const long long i = CELL_INDEX(d);
        const int x[3] = {x0, x1, x2};
        double mc, cmc;
        lever(c[i], f[i], p, mc, cmc);
        const double nD = -p.D;
        double dc = 0.0;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            if (a < d.a0) continue;
            const int n = d.e[a];
            const long long ip = i + (long long)((x[a] + 1 == n ? 0 : x[a] + 1) - x[a]) * d.st[a];
            const long long im = i + (long long)((x[a] == 0 ? n - 1 : x[a] - 1) - x[a]) * d.st[a];
            double mp, cmp, mm, cmm;
            lever(c[ip], f[ip], p, mp, cmp);
            lever(c[im], f[im], p, mm, cmm);
            const double mfp = 0.5 * (mc + mp);
            double fpl = (nD * mfp) * (cmp - cmc);
            fpl = fpl / p.dx;
            const double mfm = 0.5 * (mm + mc);
            double fmi = (nD * mfm) * (cmc - cmm);
            fmi = fmi / p.dx;
            dc = dc - (fpl - fmi) / p.dx;
        }
        out[i] = c[i] + dt * dc;
        if (cm_out) cm_out[i] = cmc;
    }
}

// The same substep for a 3-D field, tiled: a (32 x 8) block marches along
// axis 0 through zc planes.  The lever rule (one division) is evaluated once
// per cell and plane (own cells carried in registers from the plane before,
// the halo ring recomputed), and the flux through each face is evaluated once
// and read by both of its cells, with the reference's operands: for the face
// between cell lo and its + neighbour hi, ((-D) (0.5 (m_lo + m_hi)))
// (cm_hi - cm_lo) / dx.  dc then takes the axes in the reference's order.
constexpr int DTX = 32, DTY = 8;

__device__ __forceinline__ double face_flux(double nD, const Phys& p, double m_lo, double cm_lo, double m_hi,
                                            double cm_hi) {
    const double mf = 0.5 * (m_lo + m_hi);
    const double fl = (nD * mf) * (cm_hi - cm_lo);
    return fl / p.dx;
}

__global__ void __launch_bounds__(DTX * DTY) k_diffuse_tiled(Ext d, Phys p, double dt, int zc,
                                                             const double* __restrict__ c,
                                                             const double* __restrict__ f, double* __restrict__ out,
                                                             double* __restrict__ cm_out) {
    __shared__ double sm[DTY + 2][DTX + 2];   // matrix fraction of the plane, halo included
    __shared__ double scm[DTY + 2][DTX + 2];  // lever composition of the plane
    __shared__ double fx[DTY][DTX + 1];       // fx[y][k]: the face between local x = k - 1 and k
    __shared__ double fy[DTY + 1][DTX];       // fy[k][x]: the face between local y = k - 1 and k
    const int n0 = d.e[0], n1 = d.e[1], n2 = d.e[2];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * DTX + tx;
    const int xs = blockIdx.x * DTX, ys = blockIdx.y * DTY;
    const bool valid = xs + tx < n2 && ys + ty < n1;
    const int ox = (xs + tx) % n2, oy = (ys + ty) % n1;  // own column (wrapped for idle threads)
    const long long plane = (long long)n1 * n2;
    const long long col = (long long)oy * n2 + ox;
    const double nD = -p.D;
    const int z0 = blockIdx.z * zc;
    const int z1 = z0 + zc < n0 ? z0 + zc : n0;
    // own column at planes z0 - 1 and z0
    const int zp = z0 == 0 ? n0 - 1 : z0 - 1;
    double m_prev, cm_prev, m_cur, cm_cur;
    lever(c[zp * plane + col], f[zp * plane + col], p, m_prev, cm_prev);
    double c_cur = c[z0 * plane + col];
    lever(c_cur, f[z0 * plane + col], p, m_cur, cm_cur);
    double fz_minus = face_flux(nD, p, m_prev, cm_prev, m_cur, cm_cur);
    for (int z = z0; z < z1; ++z) {
        const int zn = z + 1 == n0 ? 0 : z + 1;
        const double c_next = c[zn * plane + col];
        double m_next, cm_next;
        lever(c_next, f[zn * plane + col], p, m_next, cm_next);
        // the plane's tile: own cells from registers, the halo ring evaluated
        sm[ty + 1][tx + 1] = m_cur;
        scm[ty + 1][tx + 1] = cm_cur;
        constexpr int HALO = 2 * (DTX + 2) + 2 * DTY;
        for (int k = tid; k < HALO; k += DTX * DTY) {
            int ly, lx;
            if (k < DTX + 2) { ly = -1; lx = k - 1; }
            else if (k < 2 * (DTX + 2)) { ly = DTY; lx = k - (DTX + 2) - 1; }
            else if (k < 2 * (DTX + 2) + DTY) { ly = k - 2 * (DTX + 2); lx = -1; }
            else { ly = k - 2 * (DTX + 2) - DTY; lx = DTX; }
            int gy = ys + ly, gx = xs + lx;
            if (gy < 0) gy += n1;
            while (gy >= n1) gy -= n1;  // at most DTY + 1 times
            if (gx < 0) gx += n2;
            while (gx >= n2) gx -= n2;  // at most DTX + 1 times
            const long long q = z * plane + (long long)gy * n2 + gx;
            double mh, cmh;
            lever(c[q], f[q], p, mh, cmh);
            sm[ly + 1][lx + 1] = mh;
            scm[ly + 1][lx + 1] = cmh;
        }
        __syncthreads();
        fx[ty][tx + 1] = face_flux(nD, p, sm[ty + 1][tx + 1], scm[ty + 1][tx + 1], sm[ty + 1][tx + 2],
                                   scm[ty + 1][tx + 2]);
        if (tx == 0) fx[ty][0] = face_flux(nD, p, sm[ty + 1][0], scm[ty + 1][0], sm[ty + 1][1], scm[ty + 1][1]);
        fy[ty + 1][tx] = face_flux(nD, p, sm[ty + 1][tx + 1], scm[ty + 1][tx + 1], sm[ty + 2][tx + 1],
                                   scm[ty + 2][tx + 1]);
        if (ty == 0) fy[0][tx] = face_flux(nD, p, sm[0][tx + 1], scm[0][tx + 1], sm[1][tx + 1], scm[1][tx + 1]);
        const double fz_plus = face_flux(nD, p, m_cur, cm_cur, m_next, cm_next);
        __syncthreads();
        if (valid) {
            double dc = 0.0;
            dc = dc - (fz_plus - fz_minus) / p.dx;
            dc = dc - (fy[ty + 1][tx] - fy[ty][tx]) / p.dx;
            dc = dc - (fx[ty][tx + 1] - fx[ty][tx]) / p.dx;
            const long long i = z * plane + col;
            out[i] = c_cur + dt * dc;
            if (cm_out) cm_out[i] = cm_cur;
        }
        fz_minus = fz_plus;
        m_cur = m_next;
        cm_cur = cm_next;
        c_cur = c_next;
        // the next plane rewrites sm/scm only after every thread has read
        // them (second barrier above); fx/fy are rewritten after the next
        // plane's first barrier, which every thread reaches after its update
    }
}

// ---------------------------------------------------------------- Gaussian

// one periodic pass along axis AX of NF fields
template <int NF, int AX>
__global__ void __launch_bounds__(128) k_gauss_pass(Ext d, Taps t, const double* __restrict__ a0,
                                                    const double* __restrict__ a1, double* __restrict__ o0,
                                                    double* __restrict__ o1) {
    const int n = d.e[AX];
    const long long s = d.st[AX];
    const bool near = t.r <= n;
    CELLS3(d) {
        const long long i = CELL_INDEX(d);
        const int xa = AX == 0 ? x0 : (AX == 1 ? x1 : x2);
        const long long base = i - (long long)xa * s;
        double v0 = a0[i] * t.w[0];
        double v1 = 0.0;
        if (NF == 2) v1 = a1[i] * t.w[0];
        for (int j = t.r; j >= 1; --j) {
            const long long lo = base + (long long)wrap_off(xa - j, n, near) * s;
            const long long hi = base + (long long)wrap_off(xa + j, n, near) * s;
            v0 = v0 + (a0[lo] + a0[hi]) * t.w[j];
            if (NF == 2) v1 = v1 + (a1[lo] + a1[hi]) * t.w[j];
        }
        o0[i] = v0;
        if (NF == 2) o1[i] = v1;
    }
}

// The same pass along axis AX = 0 or 1 for radius R: a thread marches along
// AX through `chunk` outputs of one line, keeping the 2R + 1 inputs of the
// current output in registers, so that each input is read once per line
// chunk instead of 2R + 1 times.  Same operations and order as
// k_gauss_pass; requires 2R + 1 <= the axis extent.
// With PRE (NF = 2), the inputs are c_m and f of the interface composition
// and the window holds the reference's operands: c_m * m and m, with
// m = clip(1 - f, 0, 1).
template <int NF, int AX, int R, bool PRE = false>
__global__ void __launch_bounds__(128) k_gauss_march(Ext d, Taps t, int chunk, const double* __restrict__ a0,
                                                     const double* __restrict__ a1, double* __restrict__ o0,
                                                     double* __restrict__ o1) {
    constexpr int OX = AX == 0 ? 1 : 0;  // the axis across the lines (with axis 2)
    constexpr int W = 2 * R + 1;
    const int x2 = blockIdx.x * 32 + threadIdx.x;
    const int xo = blockIdx.y * 4 + threadIdx.y;
    if (x2 >= d.e[2] || xo >= d.e[OX]) return;
    const int n = d.e[AX];
    const long long s = d.st[AX];
    const long long base = (long long)xo * d.st[OX] + x2;
    const int z0 = blockIdx.z * chunk;
    const int z1 = z0 + chunk < n ? z0 + chunk : n;
    double u[W], v[W];
#pragma unroll
    for (int k = 0; k < W; ++k) {
        int z = z0 - R + k;
        z = z < 0 ? z + n : (z >= n ? z - n : z);
        if (PRE) {
            const double m = np_clip(1.0 - a1[base + z * s], 0.0, 1.0);
            u[k] = a0[base + z * s] * m;
            v[k] = m;
        } else {
            u[k] = a0[base + z * s];
            if (NF == 2) v[k] = a1[base + z * s];
        }
    }
    for (int z = z0; z < z1; ++z) {
        double r0 = u[R] * t.w[0];
        double r1 = 0.0;
        if (NF == 2) r1 = v[R] * t.w[0];
#pragma unroll
        for (int j = R; j >= 1; --j) {
            r0 = r0 + (u[R - j] + u[R + j]) * t.w[j];
            if (NF == 2) r1 = r1 + (v[R - j] + v[R + j]) * t.w[j];
        }
        o0[base + z * s] = r0;
        if (NF == 2) o1[base + z * s] = r1;
        if (z + 1 < z1) {
#pragma unroll
            for (int k = 0; k < W - 1; ++k) {
                u[k] = u[k + 1];
                if (NF == 2) v[k] = v[k + 1];
            }
            int zn = z + 1 + R;
            zn = zn >= n ? zn - n : zn;
            if (PRE) {
                const double m = np_clip(1.0 - a1[base + zn * s], 0.0, 1.0);
                u[W - 1] = a0[base + zn * s] * m;
                v[W - 1] = m;
            } else {
                u[W - 1] = a0[base + zn * s];
                if (NF == 2) v[W - 1] = a1[base + zn * s];
            }
        }
    }
}

// The last pass (axis 2) of the partition transfer's smoothing with the
// weight computed in its epilogue, as the reference computes it from the
// smoothed field (lines 721-729): w = G|transfer| * matrix, times the
// capacity max(ctot - c_eq matrix, 0) when Cu is drawn from the matrix
__global__ void __launch_bounds__(128) k_gauss_last_weight(Ext d, Taps t, const double* __restrict__ a0,
                                                           double* __restrict__ w, double* __restrict__ cap,
                                                           const double* __restrict__ newf,
                                                           const double* __restrict__ c, double ceq, int draw) {
    const int n = d.e[2];
    const bool near = t.r <= n;
    CELLS3(d) {
        const long long i = CELL_INDEX(d);
        const long long base = i - x2;
        double v0 = a0[i] * t.w[0];
        for (int j = t.r; j >= 1; --j)
            v0 = v0 + (a0[base + wrap_off(x2 - j, n, near)] + a0[base + wrap_off(x2 + j, n, near)]) * t.w[j];
        const double m = np_clip(1.0 - newf[i], 0.0, 1.0);
        double v = v0 * m;
        if (draw) {
            const double k = np_max(c[i] - ceq * m, 0.0);
            v = v * k;
            cap[i] = k;
        }
        w[i] = v;
    }
}

// The last pass (axis 2) of the interface composition's two smoothed fields
// with its epilogue: trace = clip(G(c_m m) / max(G(m), 1e-12), 0, c_theta)
__global__ void __launch_bounds__(128) k_gauss_last_trace(Ext d, Taps t, const double* __restrict__ a0,
                                                          const double* __restrict__ a1, double ct,
                                                          double* __restrict__ out) {
    const int n = d.e[2];
    const bool near = t.r <= n;
    CELLS3(d) {
        const long long i = CELL_INDEX(d);
        const long long base = i - x2;
        double v0 = a0[i] * t.w[0];
        double v1 = a1[i] * t.w[0];
        for (int j = t.r; j >= 1; --j) {
            const long long lo = base + wrap_off(x2 - j, n, near), hi = base + wrap_off(x2 + j, n, near);
            v0 = v0 + (a0[lo] + a0[hi]) * t.w[j];
            v1 = v1 + (a1[lo] + a1[hi]) * t.w[j];
        }
        out[i] = np_clip(v0 / np_max(v1, 1.0e-12), 0.0, ct);
    }
}

// ---------------------------------------------------------------- numpy's pairwise sum

// a field value, or (corr * w[i]) / wsum for the correction (added to c as it is summed)
struct LoadF {
    const double* a;
    __device__ __forceinline__ double operator()(long long i) const { return a[i]; }
};
// the same value, also added to c[i] (the leaf pass visits every i once)
struct CorrApplyF {
    const double* w;
    double* c;
    double corr, wsum;
    __device__ __forceinline__ double operator()(long long i) const {
        const double v = (corr * w[i]) / wsum;
        c[i] = c[i] + v;
        return v;
    }
};

// 8 lanes per leaf: lane j holds numpy's running partial r[j]
template <class F>
__global__ void k_pw_leaves(F f, const int* __restrict__ start, const int* __restrict__ len, int L,
                            double* __restrict__ out) {
    const long long gid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long leaf = gid >> 3;
    const int lane = (int)(gid & 7);
    const bool act = leaf < L;
    const long long s = act ? start[leaf] : 0;
    const int n = act ? len[leaf] : 0;
    double r = 0.0;
    if (act && n >= 8) {
        r = f(s + lane);
        const int end = n - n % 8;
        for (int i = 8; i < end; i += 8) r = r + f(s + i + lane);
    }
    const unsigned full = 0xffffffffu;
    const double t = r + __shfl_down_sync(full, r, 1);  // r0+r1, r2+r3, r4+r5, r6+r7 on even lanes
    const double u = t + __shfl_down_sync(full, t, 2);  // (r0+r1)+(r2+r3), (r4+r5)+(r6+r7)
    const double v = u + __shfl_down_sync(full, u, 4);  // lane 0 of the group: the 8-way total
    if (act && lane == 0) {
        double res;
        if (n < 8) {
            res = 0.0;
            for (int i = 0; i < n; ++i) res = res + f(s + i);
        } else {
            res = v;
            for (int i = n - n % 8; i < n; ++i) res = res + f(s + i);
        }
        out[leaf] = res;
    }
}

// the pairwise tree of a range of n values whose subtrees of size <= t have
// been summed into lower[k], lower[k + 1], ... (left to right)
__device__ double pw_walk(long long n, long long t, const double* __restrict__ lower, int k) {
    long long pend[40];
    double part[40];
    unsigned char state[40];
    int sp = 0;
    double v;
    for (;;) {
        while (n > t && sp < 40) {
            long long n2 = n / 2;
            n2 -= n2 % 8;
            pend[sp] = n - n2;
            state[sp] = 0;
            ++sp;
            n = n2;
        }
        v = lower[k++];
        for (;;) {
            if (sp == 0) return v;
            if (state[sp - 1] == 0) {
                part[sp - 1] = v;
                state[sp - 1] = 1;
                n = pend[sp - 1];
                break;
            }
            v = part[sp - 1] + v;
            --sp;
        }
    }
}

__global__ void k_pw_nodes(const int* __restrict__ node_n, const int* __restrict__ node_first, int M, long long t,
                           const double* __restrict__ lower, double* __restrict__ out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < M) out[k] = pw_walk(node_n[k], t, lower, node_first[k]);
}
// the small upper levels (at most 1024 nodes each) in one block, a barrier
// between levels; buffers alternate as in the per-level launches
struct PwTop {
    const int* n[12];
    const int* first[12];
    int count[12];
    long long below[12];
    int levels;
};
__global__ void __launch_bounds__(1024) k_pw_top(PwTop lv, double* b0, double* b1, int cur) {
    for (int l = 0; l < lv.levels; ++l) {
        const double* lower = cur ? b1 : b0;
        double* out = cur ? b0 : b1;
        for (int k = threadIdx.x; k < lv.count[l]; k += blockDim.x)
            out[k] = pw_walk(lv.n[l][k], lv.below[l], lower, lv.first[l][k]);
        __syncthreads();
        cur ^= 1;
    }
}

// ---------------------------------------------------------------- partition transfer

__global__ void k_pt_transfer(long long N, double ct, double* __restrict__ c, const double* __restrict__ oldf,
                              const double* __restrict__ newf, const double* __restrict__ mcomp,
                              double* __restrict__ tr, double* __restrict__ abs_tr) {
    GRID_STRIDE(i, N) {
        const double delta = np_clip(newf[i], 0.0, 1.0) - oldf[i];
        const double t = delta * (ct - mcomp[i]);
        tr[i] = t;
        c[i] = c[i] + t;
        abs_tr[i] = fabs(t);
    }
}

// order-preserving key of a double (larger value, larger key)
__device__ __forceinline__ unsigned long long okey(double v) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

__global__ void k_max_key(long long N, const double* __restrict__ w, unsigned long long* __restrict__ best) {
    typedef cub::BlockReduce<unsigned long long, 256> BR;
    __shared__ typename BR::TempStorage tmp;
    unsigned long long m = 0;
    GRID_STRIDE(i, N) {
        const unsigned long long k = okey(w[i]);
        m = k > m ? k : m;
    }
    const unsigned long long agg = BR(tmp).Reduce(m, cub::Max());
    if (threadIdx.x == 0) atomicMax(best, agg);
}
__global__ void k_first_at(long long N, const double* __restrict__ w, const unsigned long long* __restrict__ best,
                           unsigned long long* __restrict__ idx) {
    const unsigned long long b = *best;
    GRID_STRIDE(i, N) if (okey(w[i]) == b) atomicMin(idx, (unsigned long long)i);
}
__global__ void k_pt_residue(long long N, double* __restrict__ c, const unsigned long long* __restrict__ idx,
                             double residue) {
    const unsigned long long i = *idx;
    if (i < (unsigned long long)N) c[i] = c[i] - residue;
}

// ---------------------------------------------------------------- interface composition

__global__ void k_ic_pre(long long N, const double* __restrict__ cm, const double* __restrict__ f,
                         double* __restrict__ num, double* __restrict__ den) {
    GRID_STRIDE(i, N) {
        const double m = np_clip(1.0 - f[i], 0.0, 1.0);
        num[i] = cm[i] * m;
        den[i] = m;
    }
}

// ---------------------------------------------------------------- Gaussian remap

// Roots only decrease, so every walk ends; the loops are capped all the same
// (the cap sets *err).  Reads go to L2: other SMs change parents atomically.
constexpr int UF_CAP = 1 << 26;

__device__ __forceinline__ int uf_find(int* parent, int i, unsigned* err) {
    for (int it = 0; it < UF_CAP; ++it) {
        const int p = __ldcg(&parent[i]);
        if (p == i) return i;
        const int gp = __ldcg(&parent[p]);
        if (gp != p) atomicMin(&parent[i], gp);
        i = p;
    }
    atomicExch(err, 1u);
    return i;
}
__device__ void uf_unite(int* parent, int a, int b, unsigned* err) {
    for (int it = 0; it < UF_CAP; ++it) {
        a = uf_find(parent, a, err);
        b = uf_find(parent, b, err);
        if (a == b) return;
        const int lo = a < b ? a : b, hi = a < b ? b : a;
        const int old = atomicCAS(&parent[hi], hi, lo);
        if (old == hi) return;
        a = lo;
        b = old;
    }
    atomicExch(err, 1u);
}

// union-find state of the labelled cells (only they are ever read)
__global__ void k_cc_init(long long N, const int8_t* __restrict__ lab, int* __restrict__ parent,
                          int* __restrict__ size, int* __restrict__ wave) {
    GRID_STRIDE(i, N) if (lab[i] != 0) {
        parent[i] = (int)i;
        size[i] = 0;
        wave[i] = 0;
    }
}
// face neighbours without wrap, equal nonzero labels
__global__ void __launch_bounds__(128) k_cc_union(Ext d, const int8_t* __restrict__ lab, int* parent, unsigned* err) {
    CELLS3(d) {
        const long long i = CELL_INDEX(d);
        const int8_t l = lab[i];
        if (l == 0) continue;
        const int x[3] = {x0, x1, x2};
#pragma unroll
        for (int a = 0; a < 3; ++a)
            if (a >= d.a0 && x[a] + 1 < d.e[a] && lab[i + d.st[a]] == l)
                uf_unite(parent, (int)i, (int)(i + d.st[a]), err);
    }
}
__global__ void k_cc_finish(long long N, const int8_t* __restrict__ lab, int* parent, int* __restrict__ root,
                            int* __restrict__ size, unsigned* err) {
    GRID_STRIDE(i, N) {
        if (lab[i] == 0) {
            root[i] = -1;
            continue;
        }
        const int r = uf_find(parent, (int)i, err);
        root[i] = r;
        atomicAdd(&size[r], 1);
    }
}
// cells of components of more than one cell; their count of components
__global__ void k_cgr_active(long long N, const int* __restrict__ root, const int* __restrict__ size,
                             uint8_t* __restrict__ act, int* __restrict__ n_active) {
    GRID_STRIDE(i, N) {
        const int r = root[i];
        const bool a = r >= 0 && size[r] > 1;
        act[i] = a;
        if (a && r == (int)i) atomicAdd(n_active, 1);
    }
}
// one axis of the 3^d box maximum (no wrap)
template <int AX>
__global__ void __launch_bounds__(128) k_box_pass(Ext d, const uint8_t* __restrict__ in, uint8_t* __restrict__ out) {
    CELLS3(d) {
        const long long i = CELL_INDEX(d);
        const int xa = AX == 0 ? x0 : (AX == 1 ? x1 : x2);
        uint8_t v = in[i];
        if (xa > 0) v |= in[i - d.st[AX]];
        if (xa + 1 < d.e[AX]) v |= in[i + d.st[AX]];
        out[i] = v;
    }
}

// The whole 3^d box maximum (no wrap) in one pass: a (32 x 8) block marches
// along axis 0 through a chunk of BOX_ZC planes (and the plane on either
// side), ORs each plane's 3 x 3 box from a shared tile with a 1-cell halo, and
// keeps the last three plane results of its cell in registers.
constexpr int BOX_ZC = 8;
__global__ void __launch_bounds__(256) k_box_max3(Ext d, const uint8_t* __restrict__ in, uint8_t* __restrict__ out) {
    __shared__ uint8_t t[10][34];
    const int n0 = d.e[0], n1 = d.e[1], n2 = d.e[2];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
    const int xs = blockIdx.x * 32, ys = blockIdx.y * 8;
    const int x = xs + tx, y = ys + ty;
    const long long plane = (long long)n1 * n2;
    const int z0 = blockIdx.z * BOX_ZC;
    const int z1 = z0 + BOX_ZC < n0 ? z0 + BOX_ZC : n0;
    uint8_t prev = 0, cur = 0;
    for (int z = z0 - 1; z <= z1; ++z) {
        uint8_t next = 0;
        if (z >= 0 && z < n0) {
            for (int k = tid; k < 340; k += 256) {
                const int ly = k / 34 - 1, lx = k % 34 - 1;
                const int gy = ys + ly, gx = xs + lx;
                t[ly + 1][lx + 1] = (gy >= 0 && gy < n1 && gx >= 0 && gx < n2) ? in[z * plane + (long long)gy * n2 + gx]
                                                                            : (uint8_t)0;
            }
            __syncthreads();
            next = t[ty][tx] | t[ty][tx + 1] | t[ty][tx + 2] | t[ty + 1][tx] | t[ty + 1][tx + 1] | t[ty + 1][tx + 2] |
                   t[ty + 2][tx] | t[ty + 2][tx + 1] | t[ty + 2][tx + 2];
            __syncthreads();
        }
        // plane z - 1 is complete: its neighbours z - 2 (prev) and z (next)
        if (z - 1 >= z0 && x < n2 && y < n1) out[(z - 1) * plane + (long long)y * n2 + x] = prev | cur | next;
        prev = cur;
        cur = next;
    }
}

// the components (of more than one cell) with a cell in the 3^d box of x,
// without wrap; returns how many (at most 27)
// (act[c]: cell c belongs to such a component)
__device__ __forceinline__ int box_components(const Ext& d, int x0, int x1, int x2, long long i,
                                              const int* __restrict__ root, const uint8_t* __restrict__ act,
                                              int S[27]) {
    int n = 0;
    for (int o0 = -1; o0 <= 1; ++o0) {
        if (x0 + o0 < 0 || x0 + o0 >= d.e[0]) continue;
        for (int o1 = -1; o1 <= 1; ++o1) {
            if (x1 + o1 < 0 || x1 + o1 >= d.e[1]) continue;
            for (int o2 = -1; o2 <= 1; ++o2) {
                if (x2 + o2 < 0 || x2 + o2 >= d.e[2]) continue;
                const long long c = i + o0 * d.st[0] + o1 * d.st[1] + o2 * d.st[2];
                if (!act[c]) continue;
                const int r = root[c];
                bool seen = false;
                for (int q = 0; q < n; ++q) seen |= S[q] == r;
                if (!seen) S[n++] = r;
            }
        }
    }
    return n;
}
__device__ __forceinline__ void cell_coords(const Ext& d, long long i, int& x0, int& x1, int& x2) {
    unsigned u = (unsigned)i;
    x2 = (int)(u % (unsigned)d.e[2]);
    u /= (unsigned)d.e[2];
    x1 = (int)(u % (unsigned)d.e[1]);
    x0 = (int)(u / (unsigned)d.e[1]);
}

// the reference's processing order: label ascending, then first cell
__device__ __forceinline__ long long order_key(const int8_t* __restrict__ orig, int r) {
    return ((long long)((int)orig[r] + 128) << 32) | (long long)r;
}

// band = cells of some component's dilation; conflicts = cells of two or more
__global__ void __launch_bounds__(128) k_cgr_band(Ext d, const uint8_t* __restrict__ near, const int* __restrict__ root,
                                                  const uint8_t* __restrict__ act, int* __restrict__ flag,
                                                  int* __restrict__ list, int* __restrict__ count) {
    CELLS3(d) {
        const long long i = CELL_INDEX(d);
        int f = 0;
        if (near[i]) {
            int S[27];
            const int n = box_components(d, x0, x1, x2, i, root, act, S);
            f = n >= 1;
            if (n >= 2) list[atomicAdd(count, 1)] = (int)i;
        }
        flag[i] = f;
    }
}
// order-preserving compaction: out[pos[q]] = (idx ? idx[q] : q) where flag[q]
__global__ void k_compact(long long M, const int* __restrict__ flag, const int* __restrict__ pos,
                          const int* __restrict__ idx, int* __restrict__ out, int* __restrict__ count) {
    GRID_STRIDE(q, M) {
        if (flag[q]) out[pos[q]] = idx ? idx[q] : (int)q;
        if (q == M - 1) *count = pos[q] + flag[q];
    }
}

__global__ void k_cgr_relax(Ext d, const int* __restrict__ list, int M, const int8_t* __restrict__ orig,
                            const int* __restrict__ root, const uint8_t* __restrict__ act, int* wave,
                            int* __restrict__ changed) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < M; q += gridDim.x * blockDim.x) {
        const long long i = list[q];
        int x0, x1, x2;
        cell_coords(d, i, x0, x1, x2);
        int S[27];
        const int n = box_components(d, x0, x1, x2, i, root, act, S);
        for (int b = 0; b < n; ++b) {
            const long long kb = order_key(orig, S[b]);
            int m = __ldcg(&wave[S[b]]);
            const int m0 = m;
            for (int a = 0; a < n; ++a)
                if (order_key(orig, S[a]) < kb) {
                    const int wa = __ldcg(&wave[S[a]]) + 1;
                    m = wa > m ? wa : m;
                }
            if (m > m0) {
                atomicMax(&wave[S[b]], m);
                *changed = 1;
            }
        }
    }
}

// every active component's root lies in the band
__global__ void k_cgr_max_wave(const int* __restrict__ band, const int* __restrict__ n_band,
                               const int* __restrict__ root, const int* __restrict__ size,
                               const int* __restrict__ wave, int* __restrict__ max_wave) {
    const int M = *n_band;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < M; q += gridDim.x * blockDim.x) {
        const int i = band[q];
        if (root[i] == i && size[i] > 1) atomicMax(max_wave, wave[i]);
    }
}

// candidates of wave w among the band: cells of the dilation of a wave-w
// component that are zero or its own
__global__ void k_cgr_flags(Ext d, int w, const int* __restrict__ band, const int* __restrict__ n_band,
                            const int8_t* __restrict__ lab, const int* __restrict__ root,
                            const uint8_t* __restrict__ act, const int* __restrict__ wave, int* __restrict__ flag,
                            int* __restrict__ seg) {
    const int M = *n_band;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < M; q += gridDim.x * blockDim.x) {
        const long long i = band[q];
        int x0, x1, x2;
        cell_coords(d, i, x0, x1, x2);
        int S[27];
        const int n = box_components(d, x0, x1, x2, i, root, act, S);
        int B = -1;
        for (int k = 0; k < n; ++k)
            if (wave[S[k]] == w) B = S[k];
        flag[q] = B >= 0 && (root[i] == B || lab[i] == 0);
        seg[i] = B;
    }
}

// Pairs (cell, component B) of the band that can be admissible at B's wave:
// the cell is B's own, or zero, or a cell of a component processed in an
// earlier wave (which may vacate it).  Cells of later-wave components, and
// of components of one cell, are never zero when B runs.
__device__ __forceinline__ bool pair_possible(int cell, int B, const int8_t* __restrict__ orig,
                                              const int* __restrict__ root, const uint8_t* __restrict__ act,
                                              const int* __restrict__ wave) {
    if (orig[cell] == 0) return true;
    const int r = root[cell];
    if (r == B) return true;
    return act[cell] && wave[r] < wave[B];
}
__global__ void k_cgr_paircount(Ext d, const int* __restrict__ band, int Mb, const int8_t* __restrict__ orig,
                                const int* __restrict__ root, const uint8_t* __restrict__ act,
                                const int* __restrict__ wave, int* __restrict__ cnt) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < Mb; q += gridDim.x * blockDim.x) {
        const int i = band[q];
        int x0, x1, x2;
        cell_coords(d, i, x0, x1, x2);
        int S[27];
        const int n = box_components(d, x0, x1, x2, i, root, act, S);
        int c = 0;
        for (int k = 0; k < n; ++k) c += pair_possible(i, S[k], orig, root, act, wave);
        cnt[q] = c;
    }
}

// the wrapped Gaussian of component B's indicator at y: the pass along axis
// A0 (the first of the field) reads the indicator, each later axis AX reads
// the pass before it; each is y w0 + sum over j = r..1 of (y-j + y+j) w_j,
// evaluated on the (2r+1)^d box only
__device__ __forceinline__ double ind(const int* __restrict__ root, long long i, int B) {
    return root[i] == B ? 1.0 : 0.0;
}
template <int AX, int A0>
__device__ double gpass(const Ext& d, const Taps& t, const int* __restrict__ root, int B, int y0, int y1, int y2) {
    const int n = d.e[AX];
    const bool near = t.r <= n;
    const int ya = AX == 0 ? y0 : (AX == 1 ? y1 : y2);
    auto at = [&](int v) -> double {
        const int z0 = AX == 0 ? v : y0, z1 = AX == 1 ? v : y1, z2 = AX == 2 ? v : y2;
        if constexpr (AX == A0)
            return ind(root, ((long long)z0 * d.e[1] + z1) * d.e[2] + z2, B);
        else
            return gpass<(AX > A0 ? AX - 1 : A0), A0>(d, t, root, B, z0, z1, z2);
    };
    double v = at(ya) * t.w[0];
    for (int j = t.r; j >= 1; --j) v = v + (at(wrap_off(ya - j, n, near)) + at(wrap_off(ya + j, n, near))) * t.w[j];
    return v;
}

__global__ void k_cgr_score(Ext d, Taps t, const int* __restrict__ cand, const int* __restrict__ count,
                            const int* __restrict__ root, const int* __restrict__ seg,
                            unsigned long long* __restrict__ key) {
    const int M = *count;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < M; q += gridDim.x * blockDim.x) {
        const long long i = cand[q];
        int x0, x1, x2;
        cell_coords(d, i, x0, x1, x2);
        const int B = seg[i];
        const double s = d.a0 == 0 ? gpass<2, 0>(d, t, root, B, x0, x1, x2) : gpass<2, 1>(d, t, root, B, x0, x1, x2);
        key[q] = ~okey(s);  // ascending key = descending score
    }
}
// the pairs of band cell q at pos[q]..: cell, component, descending-score key
__global__ void k_cgr_pairs(Ext d, Taps t, const int* __restrict__ band, int Mb, const int* __restrict__ pos,
                            const int8_t* __restrict__ orig, const int* __restrict__ root,
                            const uint8_t* __restrict__ act, const int* __restrict__ wave, int* __restrict__ pcell,
                            int* __restrict__ pseg, unsigned long long* __restrict__ pkey, int* __restrict__ iota) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < Mb; q += gridDim.x * blockDim.x) {
        const int i = band[q];
        int x0, x1, x2;
        cell_coords(d, i, x0, x1, x2);
        int S[27];
        const int n = box_components(d, x0, x1, x2, i, root, act, S);
        int o = pos[q];
        for (int k = 0; k < n; ++k) {
            const int B = S[k];
            if (!pair_possible(i, B, orig, root, act, wave)) continue;
            const double sc = d.a0 == 0 ? gpass<2, 0>(d, t, root, B, x0, x1, x2) : gpass<2, 1>(d, t, root, B, x0, x1, x2);
            pcell[o] = i;
            pseg[o] = B;
            pkey[o] = ~okey(sc);  // ascending key = descending score
            iota[o] = o;
            ++o;
        }
    }
}
__global__ void k_total(int M, const int* __restrict__ cnt, const int* __restrict__ pos, int* __restrict__ out) {
    *out = M > 0 ? pos[M - 1] + cnt[M - 1] : 0;
}
// per sorted position: the pair's component (for the stable second sort)
__global__ void k_cgr_pairseg(int P, const int* __restrict__ perm, const int* __restrict__ pseg,
                              unsigned* __restrict__ out) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < P; q += gridDim.x * blockDim.x) out[q] = (unsigned)pseg[perm[q]];
}
// admissible now: wave-w pairs whose cell is B's own or zero
__global__ void k_cgr_adm(int P, int w, const int* __restrict__ perm, const unsigned* __restrict__ sk,
                          const int* __restrict__ pcell, const int* __restrict__ root, const int* __restrict__ wave,
                          const int8_t* __restrict__ lab, int* __restrict__ adm) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < P; q += gridDim.x * blockDim.x) {
        const int B = (int)sk[q];
        int a = 0;
        if (wave[B] == w) {
            const int c = pcell[perm[q]];
            a = root[c] == B || lab[c] == 0;
        }
        adm[q] = a;
    }
}
// the first size[B] admissible entries of B's run take its label
__global__ void k_cgr_take(int P, int w, const int* __restrict__ perm, const unsigned* __restrict__ sk,
                           const int* __restrict__ pcell, const int* __restrict__ adm, const int* __restrict__ rank,
                           const int* __restrict__ size, const int* __restrict__ wave, const int8_t* __restrict__ orig,
                           int8_t* __restrict__ lab) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < P; q += gridDim.x * blockDim.x) {
        const int B = (int)sk[q];
        if (adm[q] && wave[B] == w && rank[q] < size[B]) lab[pcell[perm[q]]] = orig[B];
    }
}

__global__ void k_cgr_segkeys(const int* __restrict__ cells, const int* __restrict__ count, const int* __restrict__ seg,
                              unsigned* __restrict__ out) {
    const int M = *count;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < M; q += gridDim.x * blockDim.x) out[q] = (unsigned)seg[cells[q]];
}
__global__ void k_cgr_starts(const unsigned* __restrict__ sk, const int* __restrict__ count, int* __restrict__ start) {
    const int M = *count;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < M; q += gridDim.x * blockDim.x)
        if (q == 0 || sk[q - 1] != sk[q]) start[sk[q]] = q;
}
// the wave's components give up their cells (all of them lie in the band)
__global__ void k_cgr_vacate(int w, const int* __restrict__ band, const int* __restrict__ n_band,
                             const int* __restrict__ root, const int* __restrict__ size, const int* __restrict__ wave,
                             int8_t* __restrict__ lab) {
    const int M = *n_band;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < M; q += gridDim.x * blockDim.x) {
        const int i = band[q];
        const int r = root[i];
        if (r >= 0 && size[r] > 1 && wave[r] == w) lab[i] = 0;
    }
}
__global__ void k_cgr_select(const unsigned* __restrict__ sk, const int* __restrict__ cells, const int* __restrict__ count,
                             const int* __restrict__ start, const int* __restrict__ size,
                             const int8_t* __restrict__ orig, int8_t* __restrict__ lab) {
    const int M = *count;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < M; q += gridDim.x * blockDim.x) {
        const int B = (int)sk[q];
        if (q - start[B] < size[B]) lab[cells[q]] = orig[B];
    }
}
// labels change only inside the band
__global__ void k_cgr_changed(const int* __restrict__ band, const int* __restrict__ n_band,
                              const int8_t* __restrict__ lab, const int8_t* __restrict__ orig,
                              double* __restrict__ alpha, unsigned long long* __restrict__ count) {
    typedef cub::BlockReduce<unsigned long long, 256> BR;
    __shared__ typename BR::TempStorage tmp;
    const int M = *n_band;
    unsigned long long n = 0;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < M; q += gridDim.x * blockDim.x) {
        const int i = band[q];
        if (lab[i] != orig[i]) {
            alpha[i] = 1.0;
            ++n;
        }
    }
    const unsigned long long agg = BR(tmp).Sum(n);
    if (threadIdx.x == 0 && agg) atomicAdd(count, agg);
}

// ---------------------------------------------------------------- topology transactions, balanced remap

// The local certificate of topology_simple_relabel(..., local_only=True)
// (lines 464-523) on bitmasks of the periodic 3^d patch (3^2 in 2-D):
// position p = 9 a + 3 b + c in 3-D, 3 b + c in 2-D, centre 13 or 4.
__device__ __forceinline__ unsigned face_nbr(int b, int nd) {
    unsigned m = 0;
    if (nd == 3) {
        const int a = b / 9, r = b % 9, y = r / 3, x = r % 3;
        if (a > 0) m |= 1u << (b - 9);
        if (a < 2) m |= 1u << (b + 9);
        if (y > 0) m |= 1u << (b - 3);
        if (y < 2) m |= 1u << (b + 3);
        if (x > 0) m |= 1u << (b - 1);
        if (x < 2) m |= 1u << (b + 1);
    } else {
        const int y = b / 3, x = b % 3;
        if (y > 0) m |= 1u << (b - 3);
        if (y < 2) m |= 1u << (b + 3);
        if (x > 0) m |= 1u << (b - 1);
        if (x < 2) m |= 1u << (b + 1);
    }
    return m;
}
// face-connected components of mask that touch a face neighbour of the centre
__device__ int topo_number(unsigned mask, int nd) {
    const unsigned incident = nd == 3 ? ((1u << 4) | (1u << 10) | (1u << 12) | (1u << 14) | (1u << 16) | (1u << 22))
                                      : ((1u << 1) | (1u << 3) | (1u << 5) | (1u << 7));
    int count = 0;
    unsigned unseen = mask;
    while (unseen) {
        unsigned comp = unseen & (~unseen + 1u);
        unsigned frontier = comp;
        while (frontier) {
            unsigned grow = 0;
            for (unsigned f = frontier; f; f &= f - 1u) grow |= face_nbr(__ffs(f) - 1, nd);
            grow &= unseen & ~comp;
            comp |= grow;
            frontier = grow;
        }
        unseen &= ~comp;
        if (comp & incident) ++count;
    }
    return count;
}
// positions of the periodic patch around cell i holding label a / b (centre excluded)
__device__ void patch_masks(const Ext& d, const int8_t* lab, long long i, int a, int b, unsigned& ma, unsigned& mb) {
    int x0, x1, x2;
    cell_coords(d, i, x0, x1, x2);
    const int y1[3] = {x1 == 0 ? d.e[1] - 1 : x1 - 1, x1, x1 + 1 == d.e[1] ? 0 : x1 + 1};
    const int y2[3] = {x2 == 0 ? d.e[2] - 1 : x2 - 1, x2, x2 + 1 == d.e[2] ? 0 : x2 + 1};
    const int y0[3] = {x0 == 0 ? d.e[0] - 1 : x0 - 1, x0, x0 + 1 == d.e[0] ? 0 : x0 + 1};
    ma = mb = 0;
    const int n0 = d.ndim == 3 ? 3 : 1;
    for (int p0 = 0; p0 < n0; ++p0)
        for (int p1 = 0; p1 < 3; ++p1)
            for (int p2 = 0; p2 < 3; ++p2) {
                const int bit = d.ndim == 3 ? 9 * p0 + 3 * p1 + p2 : 3 * p1 + p2;
                if (bit == (d.ndim == 3 ? 13 : 4)) continue;
                const int z0 = d.ndim == 3 ? y0[p0] : 0;
                const int v = lab[((long long)z0 * d.e[1] + y1[p1]) * d.e[2] + y2[p2]];
                if (v == a) ma |= 1u << bit;
                if (v == b) mb |= 1u << bit;
            }
}
// counts: label value + 128 -> cells holding it; null when no label can
// fall to one cell (extinction never applies)
__device__ bool cert_local(const Ext& d, const int8_t* lab, long long i, int old_label, int new_label,
                           const int* counts) {
    if (old_label == new_label) return false;
    unsigned mo, mn;
    patch_masks(d, lab, i, old_label, new_label, mo, mn);
    const int oc = topo_number(mo, d.ndim);
    const bool extinction = counts ? counts[old_label + 128] <= 1 : false;
    if (oc == 0 && !extinction) return false;
    if (oc > 1) return false;
    const int nc = topo_number(mn, d.ndim);
    if (nc == 0 || nc > 1) return false;
    return true;
}

__global__ void k_label_hist(long long N, const int8_t* __restrict__ lab, int* __restrict__ counts) {
    __shared__ int h[256];
    for (int k = threadIdx.x; k < 256; k += blockDim.x) h[k] = 0;
    __syncthreads();
    GRID_STRIDE(i, N) atomicAdd(&h[(int)lab[i] + 128], 1);
    __syncthreads();
    for (int k = threadIdx.x; k < 256; k += blockDim.x)
        if (h[k]) atomicAdd(&counts[k], h[k]);
}
__global__ void k_u8_flags(long long N, const uint8_t* __restrict__ m, int* __restrict__ flag) {
    GRID_STRIDE(i, N) flag[i] = m[i] != 0;
}

// commit_topology_transactions (lines 526-559): the crossing cells in C
// order, each certificate against the state the earlier ones left
__global__ void k_tx_commit(Ext d, const int* __restrict__ list, const int* __restrict__ n_list, int8_t* lab,
                            double* alpha, const int8_t* __restrict__ comp, int* counts,
                            unsigned long long* __restrict__ deferred) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const int M = *n_list;
    unsigned long long nd = 0;
    for (int q = 0; q < M; ++q) {
        const long long i = list[q];
        const int old_label = lab[i], new_label = comp[i];
        if (cert_local(d, lab, i, old_label, new_label, counts)) {
            lab[i] = (int8_t)new_label;
            alpha[i] = 1.0;
            counts[old_label + 128] -= 1;
            counts[new_label + 128] += 1;
        } else {
            ++nd;
            const double a = alpha[i];
            alpha[i] = 1.0e-6 > a ? 1.0e-6 : a;  // Python max(a, 1e-6)
        }
    }
    *deferred = nd;
}

// The same commits in rounds.  A transaction reads only its periodic 3^d
// patch, so it may run once every earlier (lower cell index) crossing cell in
// that patch has run in an earlier round; transactions ready in one round
// are never neighbours of one another, and their later neighbours have not
// run yet, so each sees exactly the state of the serial order.  Used when no
// label can fall to one cell during the sweep (then the extinction test is
// false throughout); done[i] = round of the commit, INT_MAX while pending.
constexpr int TX_PENDING = 0x7fffffff;

__global__ void k_tx_init(const int* __restrict__ list, const int* __restrict__ n_list, int* __restrict__ done,
                          int* __restrict__ crossing_hist, const int8_t* __restrict__ lab) {
    const int M = *n_list;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < M; q += gridDim.x * blockDim.x) {
        done[list[q]] = TX_PENDING;
        atomicAdd(&crossing_hist[(int)lab[list[q]] + 128], 1);
    }
}
__global__ void k_tx_round(Ext d, int round, const int* __restrict__ list, const int* __restrict__ n_list,
                           const uint8_t* __restrict__ crossing, int* done, int8_t* lab, double* alpha,
                           const int8_t* __restrict__ comp, unsigned long long* __restrict__ counters) {
    const int M = *n_list;
    // rounds launched after the last transaction ran return at once
    __shared__ int finished;
    if (threadIdx.x == 0) finished = __ldcg(&counters[0]) >= (unsigned long long)M;
    __syncthreads();
    if (finished) return;
    unsigned long long ran = 0, nd = 0;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < M; q += gridDim.x * blockDim.x) {
        const int j = list[q];
        if (__ldcg(&done[j]) != TX_PENDING) continue;
        int x0, x1, x2;
        cell_coords(d, j, x0, x1, x2);
        const int y1[3] = {x1 == 0 ? d.e[1] - 1 : x1 - 1, x1, x1 + 1 == d.e[1] ? 0 : x1 + 1};
        const int y2[3] = {x2 == 0 ? d.e[2] - 1 : x2 - 1, x2, x2 + 1 == d.e[2] ? 0 : x2 + 1};
        const int y0[3] = {x0 == 0 ? d.e[0] - 1 : x0 - 1, x0, x0 + 1 == d.e[0] ? 0 : x0 + 1};
        bool ready = true;
        const int n0 = d.ndim == 3 ? 3 : 1;
        for (int p0 = 0; p0 < n0 && ready; ++p0)
            for (int p1 = 0; p1 < 3 && ready; ++p1)
                for (int p2 = 0; p2 < 3; ++p2) {
                    const int z0 = d.ndim == 3 ? y0[p0] : 0;
                    const int nb = (int)(((long long)z0 * d.e[1] + y1[p1]) * d.e[2] + y2[p2]);
                    if (nb < j && crossing[nb] && __ldcg(&done[nb]) >= round) {
                        ready = false;
                        break;
                    }
                }
        if (!ready) continue;
        const int old_label = lab[j], new_label = comp[j];
        if (cert_local(d, lab, j, old_label, new_label, nullptr)) {
            lab[j] = (int8_t)new_label;
            alpha[j] = 1.0;
        } else {
            ++nd;
            const double a = alpha[j];
            alpha[j] = 1.0e-6 > a ? 1.0e-6 : a;  // Python max(a, 1e-6)
        }
        done[j] = round;
        ++ran;
    }
    if (ran) atomicAdd(&counters[0], ran);
    if (nd) atomicAdd(&counters[1], nd);
}

// the labels present, ascending (np.unique), at most 8
struct Vals {
    int n;
    int v[8];
};

__global__ void k_indicator(long long N, const int8_t* __restrict__ lab, int v, double* __restrict__ out) {
    GRID_STRIDE(i, N) out[i] = lab[i] == v ? 1.0 : 0.0;
}

// proposals of balanced_gaussian_remap (lines 611-636): an interface cell
// proposes the face-neighbour label of largest score gain over its own
// (labels in ascending order, strictly larger gains only)
__global__ void __launch_bounds__(128) k_bgr_propose(Ext d, Vals vals, const int8_t* __restrict__ lab,
                                                     const double* __restrict__ scores, int* __restrict__ flag,
                                                     int* __restrict__ pair, double* __restrict__ gain) {
    CELLS3(d) {
        const long long i = CELL_INDEX(d);
        const int x[3] = {x0, x1, x2};
        const int l = lab[i];
        unsigned near = 0;  // bit k: a face neighbour holds vals.v[k]
        bool iface = false;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            if (a < d.a0) continue;
            const int n = d.e[a];
            const long long ip = i + (long long)((x[a] + 1 == n ? 0 : x[a] + 1) - x[a]) * d.st[a];
            const long long im = i + (long long)((x[a] == 0 ? n - 1 : x[a] - 1) - x[a]) * d.st[a];
            const int nbs[2] = {lab[im], lab[ip]};
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                iface |= nbs[q] != l;
                for (int k = 0; k < vals.n; ++k)
                    if (nbs[q] == vals.v[k]) near |= 1u << k;
            }
        }
        int f = 0;
        if (iface) {
            int oi = 0;
            for (int k = 0; k < vals.n; ++k)
                if (vals.v[k] == l) oi = k;
            const double old_score = scores[(long long)oi * d.N + i];
            int best = oi;
            double best_gain = 0.0;
            for (int k = 0; k < vals.n; ++k) {
                if (k == oi || !((near >> k) & 1u)) continue;
                const double g = scores[(long long)k * d.N + i] - old_score;
                if (g > best_gain) {
                    best = k;
                    best_gain = g;
                }
            }
            if (best != oi) {
                f = 1;
                pair[i] = oi * 8 + best;
                gain[i] = best_gain;
            }
        }
        flag[i] = f;
    }
}
// records in descending cell order: key = descending gain
__global__ void k_bgr_records(long long N, const int* __restrict__ flag, const int* __restrict__ pos,
                              const int* __restrict__ count, const double* __restrict__ gain,
                              int* __restrict__ cells, unsigned long long* __restrict__ key) {
    const int M = *count;
    GRID_STRIDE(i, N) if (flag[i]) {
        const int q = M - 1 - pos[i];
        cells[q] = (int)i;
        key[q] = ~okey(gain[i]);
    }
}
__global__ void k_pair_hist(const unsigned* __restrict__ pk, const int* __restrict__ count, int* __restrict__ hist) {
    const int M = *count;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < M; q += gridDim.x * blockDim.x) atomicAdd(&hist[pk[q]], 1);
}

struct PairSegs {
    int start[64], len[64];
};

// the exchanges (lines 640-671), serially in the reference's order
__global__ void k_bgr_exchange(Ext d, Vals vals, PairSegs segs, const int* __restrict__ cells, int8_t* lab,
                               int* counts, uint8_t* __restrict__ changed) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    for (int ia = 0; ia < vals.n; ++ia)
        for (int ib = ia + 1; ib < vals.n; ++ib) {
            const int first = vals.v[ia], second = vals.v[ib];
            if ((first == 0) != (second == 0)) continue;
            const int sf = ia * 8 + ib, sr = ib * 8 + ia;
            const int cnt = segs.len[sf] < segs.len[sr] ? segs.len[sf] : segs.len[sr];
            for (int k = 0; k < cnt; ++k) {
                const long long f = cells[segs.start[sf] + k];
                const long long r = cells[segs.start[sr] + k];
                if (lab[f] != first || lab[r] != second) continue;
                if (!cert_local(d, lab, f, first, second, counts)) continue;
                lab[f] = (int8_t)second;
                counts[first + 128] -= 1;
                counts[second + 128] += 1;
                if (!cert_local(d, lab, r, second, first, counts)) {
                    lab[f] = (int8_t)first;
                    counts[first + 128] += 1;
                    counts[second + 128] -= 1;
                    continue;
                }
                lab[r] = (int8_t)first;
                counts[second + 128] -= 1;
                counts[first + 128] += 1;
                changed[f] = 1;
                changed[r] = 1;
            }
        }
}
// The same exchanges in rounds.  Exchange m (its place in the serial order)
// writes its cells f and r and reads their periodic 3^d patches, so it may
// run once every earlier exchange writing a cell of those patches has run in
// an earlier round.  Used when every label holds at least 3 cells: an
// exchange leaves the counts unchanged and moves them by one in between, so
// the extinction test is false throughout.  xid[c] = the exchange writing
// record cell c (TX_PENDING for proposals that take part in none).
struct PairList {
    int n;
    int sf[28], sr[28], cnt[28], base[28], first[28], second[28];
};

__global__ void k_bgr_xinit(const int* __restrict__ cells, const int* __restrict__ count, int* __restrict__ xid) {
    const int M = *count;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < M; q += gridDim.x * blockDim.x) xid[cells[q]] = TX_PENDING;
}
__global__ void k_bgr_xindex(PairList pl, PairSegs segs, const int* __restrict__ cells, int* __restrict__ xf,
                             int* __restrict__ xr, int* __restrict__ xp, int* __restrict__ xid, int* __restrict__ done,
                             int total) {
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < total; m += gridDim.x * blockDim.x) {
        int t = 0;
        while (t + 1 < pl.n && pl.base[t + 1] <= m) ++t;
        const int k = m - pl.base[t];
        const int f = cells[segs.start[pl.sf[t]] + k], r = cells[segs.start[pl.sr[t]] + k];
        xf[m] = f;
        xr[m] = r;
        xp[m] = t;
        xid[f] = m;
        xid[r] = m;
        done[m] = TX_PENDING;
    }
}
// no earlier exchange still pending writes a cell of the patch around i
__device__ bool patch_free(const Ext& d, long long i, int m, int round, const int* __restrict__ flag,
                           const int* xid, const int* done) {
    int x0, x1, x2;
    cell_coords(d, i, x0, x1, x2);
    const int y1[3] = {x1 == 0 ? d.e[1] - 1 : x1 - 1, x1, x1 + 1 == d.e[1] ? 0 : x1 + 1};
    const int y2[3] = {x2 == 0 ? d.e[2] - 1 : x2 - 1, x2, x2 + 1 == d.e[2] ? 0 : x2 + 1};
    const int y0[3] = {x0 == 0 ? d.e[0] - 1 : x0 - 1, x0, x0 + 1 == d.e[0] ? 0 : x0 + 1};
    const int n0 = d.ndim == 3 ? 3 : 1;
    for (int p0 = 0; p0 < n0; ++p0)
        for (int p1 = 0; p1 < 3; ++p1)
            for (int p2 = 0; p2 < 3; ++p2) {
                const int z0 = d.ndim == 3 ? y0[p0] : 0;
                const long long c = ((long long)z0 * d.e[1] + y1[p1]) * d.e[2] + y2[p2];
                if (!flag[c]) continue;
                const int w = __ldcg(&xid[c]);
                if (w < m && __ldcg(&done[w]) >= round) return false;
            }
    return true;
}
__global__ void k_bgr_round(Ext d, PairList pl, int round, int total, const int* __restrict__ xf,
                            const int* __restrict__ xr, const int* __restrict__ xp, const int* __restrict__ flag,
                            const int* xid, int* done, int8_t* lab, uint8_t* __restrict__ changed,
                            unsigned long long* __restrict__ ran_count) {
    __shared__ int finished;
    if (threadIdx.x == 0) finished = __ldcg(ran_count) >= (unsigned long long)total;
    __syncthreads();
    if (finished) return;
    unsigned long long ran = 0;
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < total; m += gridDim.x * blockDim.x) {
        if (__ldcg(&done[m]) != TX_PENDING) continue;
        const long long f = xf[m], r = xr[m];
        if (!patch_free(d, f, m, round, flag, xid, done) || !patch_free(d, r, m, round, flag, xid, done)) continue;
        const int first = pl.first[xp[m]], second = pl.second[xp[m]];
        if (lab[f] == first && lab[r] == second && cert_local(d, lab, f, first, second, nullptr)) {
            lab[f] = (int8_t)second;
            if (cert_local(d, lab, r, second, first, nullptr)) {
                lab[r] = (int8_t)first;
                changed[f] = 1;
                changed[r] = 1;
            } else {
                lab[f] = (int8_t)first;
            }
        }
        done[m] = round;
        ++ran;
    }
    if (ran) atomicAdd(ran_count, ran);
}

__global__ void k_bgr_finish(const int* __restrict__ cells, const int* __restrict__ count,
                             const uint8_t* __restrict__ changed, double* __restrict__ alpha,
                             unsigned long long* __restrict__ n_changed) {
    typedef cub::BlockReduce<unsigned long long, 256> BR;
    __shared__ typename BR::TempStorage tmp;
    const int M = *count;
    unsigned long long n = 0;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < M; q += gridDim.x * blockDim.x) {
        const int i = cells[q];
        if (changed[i]) {
            alpha[i] = 1.0;
            ++n;
        }
    }
    const unsigned long long agg = BR(tmp).Sum(n);
    if (threadIdx.x == 0 && agg) atomicAdd(n_changed, agg);
}

}  // namespace

// ============================================================== handle

struct gpk_alcu {
    Ext d{};
    Phys p{};
    int device = 0;
    int num_sms = 148;
    int grid = 0;
    cudaStream_t own = nullptr, stream = nullptr;
    long long bytes = 0;
    // transport scratch
    double* f[6] = {};  // six N-double fields
    // pairwise-sum tree: leaves, then upper levels up to the root
    int* leaf_start = nullptr;
    int* leaf_len = nullptr;
    int n_leaves = 0;
    std::vector<int*> lvl_n, lvl_first;
    std::vector<int> lvl_count;
    std::vector<long long> lvl_below;  // threshold of the level under each
    double* pw_buf[2] = {};
    // reductions
    unsigned long long* u64 = nullptr;  // [0] max key, [1] index, [2] changed count
    int* i32 = nullptr;                 // [0] candidates, [1] conflicts, [2] changed flag, [3] max wave, [4] active
    unsigned* err = nullptr;
    // remap scratch
    int8_t* orig = nullptr;
    int *parent = nullptr, *root = nullptr, *size = nullptr, *wave = nullptr, *seg = nullptr, *start = nullptr;
    int *flag = nullptr, *pos = nullptr, *cand = nullptr, *cells1 = nullptr, *cells2 = nullptr, *conflicts = nullptr;
    unsigned long long *key1 = nullptr, *key2 = nullptr;
    unsigned *sk1 = nullptr, *sk2 = nullptr;
    uint8_t *u8a = nullptr, *u8b = nullptr;  // active cells and their 3^d box maximum
    int* band = nullptr;                     // cells of some component's dilation, in order
    int* cnt256 = nullptr;                   // cells per label value (value + 128)
    int* aux = nullptr;                      // 512 ints: small histograms
    double* scores = nullptr;                // the balanced remap's per-label Gaussians
    int n_scores = 0;
    void* cub_tmp = nullptr;
    size_t cub_bytes = 0;
    int seg_bits = 1;
    long long last_components = 0, last_waves = 0, last_pairs = 0;
};

namespace {

int set_params(gpk_alcu* h, const gpk_alcu_params* p) {
    if (!p || !(p->dx > 0.0) || !(p->diffusivity > 0.0)) {
        gpk_set_error("alcu: params must be given with dx > 0 and diffusivity > 0");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    h->p.dx = p->dx;
    h->p.D = p->diffusivity;
    h->p.ceq = p->c_matrix_eq;
    h->p.ct = p->c_theta;
    return GPK_OK;
}

// launch shape of the CELLS3 kernels
const dim3 B3(32, 4);
dim3 grid3(const Ext& d) {
    const int gy = (d.e[1] + 3) / 4;
    return dim3((d.e[2] + 31) / 32, gy < 65535 ? gy : 65535, d.e[0] < 65535 ? d.e[0] : 65535);
}

// maximal subtrees of numpy's pairwise tree with at most t values, in order
void cut(long long lo, long long n, long long t, std::vector<long long>& s, std::vector<long long>& len) {
    if (n <= t) {
        s.push_back(lo);
        len.push_back(n);
        return;
    }
    long long n2 = n / 2;
    n2 -= n2 % 8;
    cut(lo, n2, t, s, len);
    cut(lo + n2, n - n2, t, s, len);
}

void free_all(gpk_alcu* h) {
    for (double*& q : h->f) cudaFree(q);
    cudaFree(h->leaf_start); cudaFree(h->leaf_len);
    for (int* q : h->lvl_n) cudaFree(q);
    for (int* q : h->lvl_first) cudaFree(q);
    cudaFree(h->pw_buf[0]); cudaFree(h->pw_buf[1]);
    cudaFree(h->u64); cudaFree(h->i32); cudaFree(h->err);
    cudaFree(h->orig); cudaFree(h->parent); cudaFree(h->root); cudaFree(h->size); cudaFree(h->wave);
    cudaFree(h->seg); cudaFree(h->start); cudaFree(h->flag); cudaFree(h->pos); cudaFree(h->cand);
    cudaFree(h->cells1); cudaFree(h->cells2); cudaFree(h->conflicts);
    cudaFree(h->key1); cudaFree(h->key2); cudaFree(h->sk1); cudaFree(h->sk2); cudaFree(h->cub_tmp);
    cudaFree(h->u8a); cudaFree(h->u8b); cudaFree(h->band); cudaFree(h->cnt256); cudaFree(h->aux); cudaFree(h->scores);
    if (h->own) cudaStreamDestroy(h->own);
}

int taps_of(const double* taps, int radius, Taps& t) {
    if (!taps || radius < 0 || radius > GPK_ALCU_MAX_RADIUS) {
        gpk_set_error("alcu: taps must be given with 0 <= radius <= " + std::to_string(GPK_ALCU_MAX_RADIUS));
        return GPK_ERR_INVALID_ARGUMENT;
    }
    t.r = radius;
    for (int j = 0; j <= radius; ++j) {
        if (taps[radius - j] != taps[radius + j]) {
            gpk_set_error("alcu: the taps must be symmetric");
            return GPK_ERR_INVALID_ARGUMENT;
        }
        t.w[j] = taps[radius + j];
    }
    return GPK_OK;
}

// np.sum of the values f(0..N-1); waits for the stream
template <class F>
int pw_sum(gpk_alcu* h, F f, double* out) {
    cudaStream_t st = h->stream;
    const long long threads = 8ll * h->n_leaves;
    k_pw_leaves<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(f, h->leaf_start, h->leaf_len, h->n_leaves,
                                                                     h->pw_buf[0]);
    ALCU_TRY(cudaGetLastError());
    int cur = 0;
    size_t k = 0;
    for (; k < h->lvl_n.size() && h->lvl_count[k] > 1024; ++k) {
        const int M = h->lvl_count[k];
        k_pw_nodes<<<(M + 127) / 128, 128, 0, st>>>(h->lvl_n[k], h->lvl_first[k], M, h->lvl_below[k],
                                                     h->pw_buf[cur], h->pw_buf[cur ^ 1]);
        ALCU_TRY(cudaGetLastError());
        cur ^= 1;
    }
    if (k < h->lvl_n.size()) {
        PwTop lv{};
        for (; k < h->lvl_n.size() && lv.levels < 12; ++k, ++lv.levels) {
            lv.n[lv.levels] = h->lvl_n[k];
            lv.first[lv.levels] = h->lvl_first[k];
            lv.count[lv.levels] = h->lvl_count[k];
            lv.below[lv.levels] = h->lvl_below[k];
        }
        if (k < h->lvl_n.size()) {
            gpk_set_error("alcu: summation tree deeper than expected");
            return GPK_ERR_INTERNAL;
        }
        k_pw_top<<<1, 1024, 0, st>>>(lv, h->pw_buf[0], h->pw_buf[1], cur);
        ALCU_TRY(cudaGetLastError());
        cur ^= lv.levels & 1;
    }
    ALCU_TRY(cudaMemcpyAsync(out, h->pw_buf[cur], sizeof(double), cudaMemcpyDeviceToHost, st));
    ALCU_TRY(cudaStreamSynchronize(st));
    return GPK_OK;
}

// CUB's scratch for the remap's scan and sorts at M items (sized for N at
// creation; grown here should a smaller problem ever ask for more)
int cub_reserve(gpk_alcu* h, int M) {
    size_t b1 = 0, b2 = 0, b3 = 0, b4 = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, b1, h->flag, h->pos, (int)h->d.N);
    cub::DeviceRadixSort::SortPairs(nullptr, b2, h->key1, h->key2, h->cand, h->cells1, M);
    cub::DeviceRadixSort::SortPairs(nullptr, b3, h->sk1, h->sk2, h->cells1, h->cells2, M, 0, h->seg_bits);
    cub::DeviceScan::ExclusiveSumByKey(nullptr, b4, h->sk2, h->flag, h->pos, M);
    size_t need = b1 > b2 ? b1 : b2;
    if (b3 > need) need = b3;
    if (b4 > need) need = b4;
    if (need <= h->cub_bytes) return GPK_OK;
    ALCU_TRY(cudaStreamSynchronize(h->stream));
    cudaFree(h->cub_tmp);
    h->cub_tmp = nullptr;
    if (cudaMalloc(&h->cub_tmp, need) != cudaSuccess) {
        cudaGetLastError();
        h->cub_bytes = 0;
        gpk_set_error("alcu: cudaMalloc of the sort scratch failed");
        return GPK_ERR_OUT_OF_MEMORY;
    }
    h->bytes += (long long)(need - h->cub_bytes);
    h->cub_bytes = need;
    return GPK_OK;
}

template <int NF>
void gauss_pass(gpk_alcu* h, int ax, const Taps& t, const double* a, const double* b, double* oa, double* ob) {
    const Ext& d = h->d;
    // lines along axes 0 and 1 marched with a register window when the radius
    // is 3 (the module's widths 0.70 and 0.75) and the axis holds the window
    if (ax < 2 && t.r == 3 && d.e[ax] >= 7) {
        const int ox = ax == 0 ? 1 : 0;
        const long long gy = (d.e[ox] + 3) / 4;
        const long long lines = (long long)((d.e[2] + 31) / 32) * gy;
        const long long want = (32ll * h->num_sms + lines - 1) / lines;  // line chunks for ~32 blocks per SM
        long long chunk = (d.e[ax] + want - 1) / want;
        chunk = chunk < 16 ? 16 : chunk;
        const long long gz = (d.e[ax] + chunk - 1) / chunk;
        if (gy <= 65535 && gz <= 65535) {
            const dim3 g((d.e[2] + 31) / 32, (unsigned)gy, (unsigned)gz);
            if (ax == 0)
                k_gauss_march<NF, 0, 3><<<g, B3, 0, h->stream>>>(d, t, (int)chunk, a, b, oa, ob);
            else
                k_gauss_march<NF, 1, 3><<<g, B3, 0, h->stream>>>(d, t, (int)chunk, a, b, oa, ob);
            return;
        }
    }
    const dim3 g = grid3(d);
    if (ax == 0)
        k_gauss_pass<NF, 0><<<g, B3, 0, h->stream>>>(d, t, a, b, oa, ob);
    else if (ax == 1)
        k_gauss_pass<NF, 1><<<g, B3, 0, h->stream>>>(d, t, a, b, oa, ob);
    else
        k_gauss_pass<NF, 2><<<g, B3, 0, h->stream>>>(d, t, a, b, oa, ob);
}

// out = the wrapped Gaussian of in (a pass per axis of the field, the first
// axis first); tmp: one N-double scratch
int gauss(gpk_alcu* h, const Taps& t, const double* in, double* out, double* tmp) {
    const Ext& d = h->d;
    // ping-pong so that the last pass lands in out
    const double* src = in;
    for (int a = d.a0; a < 3; ++a) {
        double* dst = ((2 - a) % 2 == 0) ? out : tmp;
        gauss_pass<1>(h, a, t, src, nullptr, dst, nullptr);
        ALCU_TRY(cudaGetLastError());
        src = dst;
    }
    return GPK_OK;
}

}  // namespace

// ============================================================== C ABI

extern "C" int gpk_alcu_gauss_taps(double sigma, double* taps, int max_taps, int* radius) {
    if (!(sigma > 0.0) || !taps || !radius) {
        gpk_set_error("alcu: sigma > 0 with taps and radius pointers");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    const int r = (int)(4.0 * sigma + 0.5);
    if (r > GPK_ALCU_MAX_RADIUS || max_taps < 2 * r + 1) {
        gpk_set_error("alcu: radius " + std::to_string(r) + " too large for the taps array or the limit");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    const double s2 = sigma * sigma;
    const double c = -0.5 / s2;
    std::vector<double> phi(2 * r + 1);
    for (int k = 0; k <= 2 * r; ++k) {
        const long long x = k - r;
        phi[k] = std::exp(c * (double)(x * x));
    }
    // numpy's sum of at most 65 values
    const int n = 2 * r + 1;
    double sum;
    if (n < 8) {
        sum = 0.0;
        for (int k = 0; k < n; ++k) sum = sum + phi[k];
    } else {
        double acc[8];
        for (int j = 0; j < 8; ++j) acc[j] = phi[j];
        int i = 8;
        for (; i < n - n % 8; i += 8)
            for (int j = 0; j < 8; ++j) acc[j] = acc[j] + phi[i + j];
        sum = ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
        for (; i < n; ++i) sum = sum + phi[i];
    }
    for (int k = 0; k < n; ++k) taps[k] = phi[k] / sum;
    *radius = r;
    return GPK_OK;
}

extern "C" int gpk_alcu_create(int ndim, const int* shape, const gpk_alcu_params* p, gpk_alcu** out) {
    if (!out || !shape || (ndim != 2 && ndim != 3)) {
        gpk_set_error("alcu: ndim must be 2 or 3 with a shape array and an output pointer");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    long long N = 1;
    for (int a = 0; a < ndim; ++a) {
        if (shape[a] < 1 || shape[a] > (1 << 20)) {
            gpk_set_error("alcu: extents must lie in [1, 2^20]");
            return GPK_ERR_INVALID_ARGUMENT;
        }
        N *= shape[a];
    }
    if (N >= (1ll << 31) - 1) {
        gpk_set_error("alcu: fewer than 2^31 - 1 cells");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        gpk_set_error("no CUDA device available");
        return GPK_ERR_NO_DEVICE;
    }
    gpk_alcu* h = new gpk_alcu();
    int rc = set_params(h, p);
    if (rc != GPK_OK) { delete h; return rc; }
    Ext& d = h->d;
    d.ndim = ndim;
    d.a0 = 3 - ndim;
    d.e[0] = ndim == 3 ? shape[0] : 1;
    d.e[1] = ndim == 3 ? shape[1] : shape[0];
    d.e[2] = ndim == 3 ? shape[2] : shape[1];
    d.st[2] = 1;
    d.st[1] = d.e[2];
    d.st[0] = (long long)d.e[1] * d.e[2];
    d.N = N;
    auto fail = [&](int code) { free_all(h); delete h; return code; };
    if (cudaGetDevice(&h->device) != cudaSuccess) return fail(GPK_ERR_CUDA);
    cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device);
    long long blocks = (N + 255) / 256;
    if (blocks > (long long)h->num_sms * 16) blocks = (long long)h->num_sms * 16;
    h->grid = (int)blocks;
    if (cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking) != cudaSuccess) {
        gpk_set_error("alcu: cudaStreamCreate failed");
        return fail(GPK_ERR_CUDA);
    }
    h->stream = h->own;
    auto alloc = [&](void** q, size_t b) -> bool {
        if (cudaMalloc(q, b < 16 ? 16 : b) != cudaSuccess) {
            cudaGetLastError();
            gpk_set_error("alcu: cudaMalloc of " + std::to_string(b) + " bytes failed");
            return false;
        }
        h->bytes += (long long)b;
        return true;
    };
    for (double*& q : h->f)
        if (!alloc((void**)&q, sizeof(double) * N)) return fail(GPK_ERR_OUT_OF_MEMORY);
    // pairwise-sum tree
    {
        std::vector<long long> s, len;
        cut(0, N, 128, s, len);
        h->n_leaves = (int)s.size();
        std::vector<int> s32(s.begin(), s.end()), l32(len.begin(), len.end());
        if (!alloc((void**)&h->leaf_start, sizeof(int) * s32.size()) ||
            !alloc((void**)&h->leaf_len, sizeof(int) * l32.size()))
            return fail(GPK_ERR_OUT_OF_MEMORY);
        if (cudaMemcpy(h->leaf_start, s32.data(), sizeof(int) * s32.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(h->leaf_len, l32.data(), sizeof(int) * l32.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
            gpk_set_error("alcu: upload of the summation tree failed");
            return fail(GPK_ERR_CUDA);
        }
        std::vector<long long> below_s = s;
        long long t_below = 128;
        while (below_s.size() > 1) {
            const long long t = t_below * 32;
            std::vector<long long> ns, nl;
            if (t >= N) {
                ns.push_back(0);
                nl.push_back(N);
            } else {
                cut(0, N, t, ns, nl);
            }
            // first lower-level node of each node: walk both ordered lists
            std::vector<int> first(ns.size()), n32(ns.size());
            size_t k = 0;
            for (size_t q = 0; q < ns.size(); ++q) {
                while (k < below_s.size() && below_s[k] < ns[q]) ++k;
                first[q] = (int)k;
                n32[q] = (int)nl[q];
            }
            int *dn = nullptr, *df = nullptr;
            if (!alloc((void**)&dn, sizeof(int) * ns.size()) || !alloc((void**)&df, sizeof(int) * ns.size()))
                return fail(GPK_ERR_OUT_OF_MEMORY);
            h->lvl_n.push_back(dn);
            h->lvl_first.push_back(df);
            if (cudaMemcpy(dn, n32.data(), sizeof(int) * ns.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
                cudaMemcpy(df, first.data(), sizeof(int) * ns.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
                gpk_set_error("alcu: upload of the summation tree failed");
                return fail(GPK_ERR_CUDA);
            }
            h->lvl_count.push_back((int)ns.size());
            h->lvl_below.push_back(t_below);
            below_s = ns;
            t_below = t;
        }
        if (!alloc((void**)&h->pw_buf[0], sizeof(double) * h->n_leaves) ||
            !alloc((void**)&h->pw_buf[1], sizeof(double) * h->n_leaves))
            return fail(GPK_ERR_OUT_OF_MEMORY);
    }
    if (!alloc((void**)&h->u64, sizeof(unsigned long long) * 4) || !alloc((void**)&h->i32, sizeof(int) * 8) ||
        !alloc((void**)&h->err, sizeof(unsigned) * 2))
        return fail(GPK_ERR_OUT_OF_MEMORY);
    // remap scratch
    int** ints[] = {&h->parent, &h->root, &h->size, &h->wave, &h->seg, &h->start,
                    &h->flag, &h->pos, &h->cand, &h->cells1, &h->cells2, &h->conflicts};
    for (int** q : ints)
        if (!alloc((void**)q, sizeof(int) * N)) return fail(GPK_ERR_OUT_OF_MEMORY);
    if (!alloc((void**)&h->orig, N) || !alloc((void**)&h->key1, 8 * N) || !alloc((void**)&h->key2, 8 * N) ||
        !alloc((void**)&h->sk1, 4 * N) || !alloc((void**)&h->sk2, 4 * N) || !alloc((void**)&h->u8a, N) ||
        !alloc((void**)&h->u8b, N) || !alloc((void**)&h->band, 4 * N) || !alloc((void**)&h->cnt256, 4 * 256) ||
        !alloc((void**)&h->aux, 4 * 512))
        return fail(GPK_ERR_OUT_OF_MEMORY);
    while ((1ll << h->seg_bits) < N) ++h->seg_bits;
    size_t b1 = 0, b2 = 0, b3 = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, b1, h->flag, h->pos, (int)N);
    cub::DeviceRadixSort::SortPairs(nullptr, b2, h->key1, h->key2, h->cand, h->cells1, (int)N);
    cub::DeviceRadixSort::SortPairs(nullptr, b3, h->sk1, h->sk2, h->cells1, h->cells2, (int)N, 0, h->seg_bits);
    h->cub_bytes = b1 > b2 ? b1 : b2;
    if (b3 > h->cub_bytes) h->cub_bytes = b3;
    if (!alloc(&h->cub_tmp, h->cub_bytes)) return fail(GPK_ERR_OUT_OF_MEMORY);
    *out = h;
    return GPK_OK;
}

extern "C" int gpk_alcu_destroy(gpk_alcu* h) {
    if (!h) return GPK_OK;
    cudaStreamSynchronize(h->stream);
    free_all(h);
    delete h;
    return GPK_OK;
}

extern "C" int gpk_alcu_set_params(gpk_alcu* h, const gpk_alcu_params* p) {
    if (!h) { gpk_set_error("alcu: null handle"); return GPK_ERR_INVALID_ARGUMENT; }
    return set_params(h, p);
}

extern "C" int gpk_alcu_set_stream(gpk_alcu* h, void* stream) {
    if (!h) { gpk_set_error("alcu: null handle"); return GPK_ERR_INVALID_ARGUMENT; }
    h->stream = (cudaStream_t)stream;
    return GPK_OK;
}

extern "C" int gpk_alcu_competitor(gpk_alcu* h, const int8_t* labels, uint8_t* mask, int8_t* competitor) {
    if (!h || !labels || !mask || !competitor) { gpk_set_error("alcu: null argument"); return GPK_ERR_INVALID_ARGUMENT; }
    k_competitor<<<grid3(h->d), B3, 0, h->stream>>>(h->d, labels, mask, competitor);
    ALCU_TRY(cudaGetLastError());
    return GPK_OK;
}

extern "C" int gpk_alcu_precip_fraction(gpk_alcu* h, const int8_t* labels, const double* alpha,
                                        const int8_t* competitor, double* fprec) {
    if (!h || !labels || !alpha || !competitor || !fprec) {
        gpk_set_error("alcu: null argument");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    k_precip_fraction<<<h->grid, 256, 0, h->stream>>>(h->d.N, labels, alpha, competitor, fprec);
    ALCU_TRY(cudaGetLastError());
    return GPK_OK;
}

extern "C" int gpk_alcu_variant_fractions(gpk_alcu* h, const int8_t* labels, const double* alpha,
                                          const int8_t* competitor, double* fractions) {
    if (!h || !labels || !alpha || !competitor || !fractions) {
        gpk_set_error("alcu: null argument");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    k_variant_fractions<<<h->grid, 256, 0, h->stream>>>(h->d.N, labels, alpha, competitor, fractions);
    ALCU_TRY(cudaGetLastError());
    return GPK_OK;
}

extern "C" int gpk_alcu_matrix_composition(gpk_alcu* h, const double* ctot, const double* fprec, double* cm) {
    if (!h || !ctot || !fprec || !cm) { gpk_set_error("alcu: null argument"); return GPK_ERR_INVALID_ARGUMENT; }
    k_matrix_composition<<<h->grid, 256, 0, h->stream>>>(h->d.N, h->p, ctot, fprec, cm);
    ALCU_TRY(cudaGetLastError());
    return GPK_OK;
}

extern "C" int gpk_alcu_diffuse(gpk_alcu* h, double* ctot, const double* fprec, double dt, double* cm, int* substeps) {
    if (!h || !ctot || !fprec) { gpk_set_error("alcu: null argument"); return GPK_ERR_INVALID_ARGUMENT; }
    const Phys& p = h->p;
    const double stable_dt = 0.4 * p.dx * p.dx / (2.0 * h->d.ndim * p.D);
    const double nsub = std::ceil(dt / stable_dt);
    if (!(nsub < 1e7) || dt != dt) {
        gpk_set_error("alcu: dt needs more than 10^7 diffusion substeps");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    const int n = nsub > 1.0 ? (int)nsub : 1;
    const double sub_dt = dt / n;
    double* bufs[2] = {ctot, h->f[0]};
    int cur = 0;
    const Ext& d = h->d;
    // planes per block: about 32 blocks per SM, from 4 to 16 planes
    const long long gx = (d.e[2] + DTX - 1) / DTX, gy = (d.e[1] + DTY - 1) / DTY;
    const long long chunks = (32ll * h->num_sms + gx * gy - 1) / (gx * gy);
    long long zc = (d.e[0] + chunks - 1) / chunks;
    zc = zc < 4 ? 4 : (zc > 16 ? 16 : zc);
    const long long gz = (d.e[0] + zc - 1) / zc;
    const bool tiled = d.ndim == 3 && gy <= 65535 && gz <= 65535;
    const dim3 tg((unsigned)gx, (unsigned)gy, (unsigned)gz);
    for (int s = 0; s < n; ++s) {
        double* cm_s = s == n - 1 ? cm : nullptr;
        if (tiled)
            k_diffuse_tiled<<<tg, dim3(DTX, DTY), 0, h->stream>>>(d, p, sub_dt, (int)zc, bufs[cur], fprec,
                                                                  bufs[cur ^ 1], cm_s);
        else
            k_diffuse<<<grid3(d), B3, 0, h->stream>>>(d, p, sub_dt, bufs[cur], fprec, bufs[cur ^ 1], cm_s);
        ALCU_TRY(cudaGetLastError());
        cur ^= 1;
    }
    if (cur != 0)
        ALCU_TRY(cudaMemcpyAsync(ctot, bufs[cur], sizeof(double) * h->d.N, cudaMemcpyDeviceToDevice, h->stream));
    if (substeps) *substeps = n;
    return GPK_OK;
}

extern "C" int gpk_alcu_sum(gpk_alcu* h, const double* x, double* out) {
    if (!h || !x || !out) { gpk_set_error("alcu: null argument"); return GPK_ERR_INVALID_ARGUMENT; }
    return pw_sum(h, LoadF{x}, out);
}

extern "C" int gpk_alcu_gaussian_filter(gpk_alcu* h, const double* in, double* out, const double* taps, int radius) {
    if (!h || !in || !out || in == out) {
        gpk_set_error("alcu: null or aliased arguments");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    Taps t;
    int rc = taps_of(taps, radius, t);
    if (rc != GPK_OK) return rc;
    return gauss(h, t, in, out, h->f[5]);
}

extern "C" int gpk_alcu_partition_transfer(gpk_alcu* h, double* ctot, const double* old_fraction,
                                           const double* new_fraction, const double* matrix_composition,
                                           const double* taps, int radius) {
    if (!h || !ctot || !old_fraction || !new_fraction || !matrix_composition) {
        gpk_set_error("alcu: null argument");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    Taps t;
    int rc = taps_of(taps, radius, t);
    if (rc != GPK_OK) return rc;
    const long long N = h->d.N;
    double *tr = h->f[0], *absd = h->f[1], *g = h->f[2], *w = h->f[3], *cap = h->f[4], *tmp = h->f[5];
    k_pt_transfer<<<h->grid, 256, 0, h->stream>>>(N, h->p.ct, ctot, old_fraction, new_fraction, matrix_composition, tr,
                                                  absd);
    ALCU_TRY(cudaGetLastError());
    double total = 0.0;
    if ((rc = pw_sum(h, LoadF{tr}, &total)) != GPK_OK) return rc;
    if (std::fabs(total) <= 1.0e-30) return GPK_OK;
    const double correction = -total;
    const int draw = correction < 0.0;
    {
        // passes along the field's axes; the last one (axis 2) computes the weight
        const double* src = absd;
        double* dst = g;
        for (int a = h->d.a0; a < 2; ++a) {
            gauss_pass<1>(h, a, t, src, nullptr, dst, nullptr);
            ALCU_TRY(cudaGetLastError());
            src = dst;
            dst = dst == g ? tmp : g;
        }
        k_gauss_last_weight<<<grid3(h->d), B3, 0, h->stream>>>(h->d, t, src, w, cap, new_fraction, ctot, h->p.ceq,
                                                              draw);
        ALCU_TRY(cudaGetLastError());
    }
    if (draw) {
        double cap_sum = 0.0;
        if ((rc = pw_sum(h, LoadF{cap}, &cap_sum)) != GPK_OK) return rc;
        if (cap_sum < -correction * (1.0 - 1.0e-12)) {
            gpk_set_error("insufficient matrix Cu for partition transfer");
            return GPK_ERR_INFEASIBLE;
        }
    }
    double wsum = 0.0;
    if ((rc = pw_sum(h, LoadF{w}, &wsum)) != GPK_OK) return rc;
    if (wsum <= 0.0) {
        gpk_set_error("empty matrix neighbourhood for partition transfer");
        return GPK_ERR_INFEASIBLE;
    }
    // ctot += (correction w) / wsum, summed as it is added
    double s = 0.0;
    if ((rc = pw_sum(h, CorrApplyF{w, ctot, correction, wsum}, &s)) != GPK_OK) return rc;
    const double residue = total + s;
    ALCU_TRY(cudaMemsetAsync(h->u64, 0, sizeof(unsigned long long), h->stream));
    ALCU_TRY(cudaMemsetAsync(h->u64 + 1, 0xff, sizeof(unsigned long long), h->stream));
    k_max_key<<<h->grid, 256, 0, h->stream>>>(N, w, h->u64);
    k_first_at<<<h->grid, 256, 0, h->stream>>>(N, w, h->u64, h->u64 + 1);
    k_pt_residue<<<1, 1, 0, h->stream>>>(N, ctot, h->u64 + 1, residue);
    ALCU_TRY(cudaGetLastError());
    return GPK_OK;
}

extern "C" int gpk_alcu_interface_composition(gpk_alcu* h, const double* cm, const double* fprec, double* trace,
                                              const double* taps, int radius) {
    if (!h || !cm || !fprec || !trace) { gpk_set_error("alcu: null argument"); return GPK_ERR_INVALID_ARGUMENT; }
    Taps t;
    int rc = taps_of(taps, radius, t);
    if (rc != GPK_OK) return rc;
    const Ext& d = h->d;
    const long long N = d.N;
    double *num = h->f[1], *den = h->f[2], *tn = h->f[3], *td = h->f[4];
    // passes along the field's axes, the first reading c_m and f (the
    // product and matrix fraction formed on load when it marches), the last
    // (axis 2) computing the trace
    double* sa = nullptr;
    double* sb = nullptr;
    const int ax0 = d.a0;
    const int ox = ax0 == 0 ? 1 : 0;
    const long long gy = (d.e[ox] + 3) / 4;
    const long long lines = (long long)((d.e[2] + 31) / 32) * gy;
    const long long want = (32ll * h->num_sms + lines - 1) / lines;
    long long chunk = (d.e[ax0] + want - 1) / want;
    chunk = chunk < 16 ? 16 : chunk;
    const long long gz = (d.e[ax0] + chunk - 1) / chunk;
    const bool march_first = t.r == 3 && d.e[ax0] >= 7 && gy <= 65535 && gz <= 65535;
    if (march_first) {
        const dim3 g((d.e[2] + 31) / 32, (unsigned)gy, (unsigned)gz);
        if (ax0 == 0)
            k_gauss_march<2, 0, 3, true><<<g, B3, 0, h->stream>>>(d, t, (int)chunk, cm, fprec, num, den);
        else
            k_gauss_march<2, 1, 3, true><<<g, B3, 0, h->stream>>>(d, t, (int)chunk, cm, fprec, num, den);
        ALCU_TRY(cudaGetLastError());
        sa = num;
        sb = den;
        if (ax0 == 0) {
            gauss_pass<2>(h, 1, t, num, den, tn, td);
            ALCU_TRY(cudaGetLastError());
            sa = tn;
            sb = td;
        }
    } else {
        k_ic_pre<<<h->grid, 256, 0, h->stream>>>(N, cm, fprec, num, den);
        ALCU_TRY(cudaGetLastError());
        sa = num;
        sb = den;
        double *da = tn, *db = td;
        for (int ax = ax0; ax < 2; ++ax) {
            gauss_pass<2>(h, ax, t, sa, sb, da, db);
            ALCU_TRY(cudaGetLastError());
            std::swap(sa, da);
            std::swap(sb, db);
        }
    }
    k_gauss_last_trace<<<grid3(d), B3, 0, h->stream>>>(d, t, sa, sb, h->p.ct, trace);
    ALCU_TRY(cudaGetLastError());
    return GPK_OK;
}

extern "C" int gpk_alcu_gaussian_remap(gpk_alcu* h, int8_t* labels, double* alpha, const double* taps, int radius,
                                       int64_t* changed) {
    if (!h || !labels || !alpha) { gpk_set_error("alcu: null argument"); return GPK_ERR_INVALID_ARGUMENT; }
    Taps t;
    int rc = taps_of(taps, radius, t);
    if (rc != GPK_OK) return rc;
    const Ext& d = h->d;
    const long long N = d.N;
    cudaStream_t st = h->stream;
    const int G = h->grid;
    const dim3 g3 = grid3(d);
    // i32: [0] candidates, [1] conflicts, [2] relax flag, [3] max wave,
    //      [4] active components, [5] band cells
    int* n_cand = h->i32;
    int* n_band = h->i32 + 5;
    ALCU_TRY(cudaMemcpyAsync(h->orig, labels, N, cudaMemcpyDeviceToDevice, st));
    ALCU_TRY(cudaMemsetAsync(h->i32, 0, sizeof(int) * 8, st));
    ALCU_TRY(cudaMemsetAsync(h->err, 0, sizeof(unsigned) * 2, st));
    ALCU_TRY(cudaMemsetAsync(h->u64 + 2, 0, sizeof(unsigned long long), st));
    k_cc_init<<<G, 256, 0, st>>>(N, h->orig, h->parent, h->size, h->wave);
    k_cc_union<<<g3, B3, 0, st>>>(d, h->orig, h->parent, h->err);
    k_cc_finish<<<G, 256, 0, st>>>(N, h->orig, h->parent, h->root, h->size, h->err);
    k_cgr_active<<<G, 256, 0, st>>>(N, h->root, h->size, h->u8a, h->i32 + 4);
    // 3^d box maximum of the active cells (u8a) into u8b: one marching pass,
    // or one pass per axis where the tile grid would be too tall
    {
        const long long gyb = (d.e[1] + 7) / 8, gzb = (d.e[0] + BOX_ZC - 1) / BOX_ZC;
        if (gyb <= 65535 && gzb <= 65535) {
            k_box_max3<<<dim3((d.e[2] + 31) / 32, (unsigned)gyb, (unsigned)gzb), dim3(32, 8), 0, st>>>(d, h->u8a,
                                                                                                     h->u8b);
        } else {
            // passes ping-pong through u8b and band (as bytes); the result in u8b
            uint8_t* tmp = reinterpret_cast<uint8_t*>(h->band);
            const uint8_t* src = h->u8a;
            for (int ax = d.a0; ax < 3; ++ax) {
                uint8_t* dst = ((2 - ax) % 2 == 0) ? h->u8b : tmp;
                if (ax == 0)
                    k_box_pass<0><<<g3, B3, 0, st>>>(d, src, dst);
                else if (ax == 1)
                    k_box_pass<1><<<g3, B3, 0, st>>>(d, src, dst);
                else
                    k_box_pass<2><<<g3, B3, 0, st>>>(d, src, dst);
                src = dst;
            }
        }
        k_cgr_band<<<g3, B3, 0, st>>>(d, h->u8b, h->root, h->u8a, h->flag, h->conflicts, h->i32 + 1);
    }
    ALCU_TRY(cudaGetLastError());
    size_t b = h->cub_bytes;
    ALCU_TRY(cub::DeviceScan::ExclusiveSum(h->cub_tmp, b, h->flag, h->pos, (int)N, st));
    k_compact<<<G, 256, 0, st>>>(N, h->flag, h->pos, nullptr, h->band, n_band);
    ALCU_TRY(cudaGetLastError());
    int hv[8];
    unsigned herr = 0;
    ALCU_TRY(cudaMemcpyAsync(hv, h->i32, sizeof(hv), cudaMemcpyDeviceToHost, st));
    ALCU_TRY(cudaMemcpyAsync(&herr, h->err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    ALCU_TRY(cudaStreamSynchronize(st));
    if (herr) {
        gpk_set_error("alcu: component search exceeded its iteration cap");
        return GPK_ERR_INTERNAL;
    }
    const int n_conf = hv[1], n_active = hv[4], Mb = hv[5];
    h->last_components = n_active;
    h->last_waves = 0;
    h->last_pairs = 0;
    if (n_active == 0) {
        if (changed) *changed = 0;
        return GPK_OK;
    }
    const int gb = (Mb + 255) / 256 < G ? (Mb + 255) / 256 : G;
    // waves: longest chain of earlier interacting components
    if (n_conf > 0) {
        for (int it = 0;; ++it) {
            if (it > n_active + 1) {
                gpk_set_error("alcu: wave relaxation did not settle");
                return GPK_ERR_INTERNAL;
            }
            int flag = 0;
            ALCU_TRY(cudaMemsetAsync(h->i32 + 2, 0, sizeof(int), st));
            const int blocks = (n_conf + 255) / 256 < G ? (n_conf + 255) / 256 : G;
            k_cgr_relax<<<blocks, 256, 0, st>>>(d, h->conflicts, n_conf, h->orig, h->root, h->u8a, h->wave,
                                                 h->i32 + 2);
            ALCU_TRY(cudaGetLastError());
            ALCU_TRY(cudaMemcpyAsync(&flag, h->i32 + 2, sizeof(int), cudaMemcpyDeviceToHost, st));
            ALCU_TRY(cudaStreamSynchronize(st));
            if (!flag) break;
        }
    }
    // the wave count, and the (cell, component) pairs that can be admissible
    k_cgr_max_wave<<<gb, 256, 0, st>>>(h->band, n_band, h->root, h->size, h->wave, h->i32 + 3);
    k_cgr_paircount<<<gb, 256, 0, st>>>(d, h->band, Mb, h->orig, h->root, h->u8a, h->wave, h->flag);
    ALCU_TRY(cudaGetLastError());
    b = h->cub_bytes;
    ALCU_TRY(cub::DeviceScan::ExclusiveSum(h->cub_tmp, b, h->flag, h->pos, Mb, st));
    k_total<<<1, 1, 0, st>>>(Mb, h->flag, h->pos, h->i32 + 7);
    ALCU_TRY(cudaGetLastError());
    int mw_p[5];
    ALCU_TRY(cudaMemcpyAsync(mw_p, h->i32 + 3, sizeof(mw_p), cudaMemcpyDeviceToHost, st));
    ALCU_TRY(cudaStreamSynchronize(st));
    const int max_wave = mw_p[0];
    const long long P = mw_p[4];
    h->last_waves = max_wave + 1;
    h->last_pairs = P;
    if (P > 0 && P <= N) {
        // every pair scored once and put in the reference's candidate order
        // (component, score descending, cell ascending) by two stable sorts;
        // a wave then takes, per component, the first `size` pairs that are
        // admissible on the labels the earlier waves left
        const int Pi = (int)P;
        const int sp = (Pi + 255) / 256 < G ? (Pi + 255) / 256 : G;
        k_cgr_pairs<<<gb, 256, 0, st>>>(d, t, h->band, Mb, h->pos, h->orig, h->root, h->u8a, h->wave, h->cand,
                                         h->seg, h->key1, h->start);
        ALCU_TRY(cudaGetLastError());
        if ((rc = cub_reserve(h, Pi)) != GPK_OK) return rc;
        b = h->cub_bytes;
        ALCU_TRY(cub::DeviceRadixSort::SortPairs(h->cub_tmp, b, h->key1, h->key2, h->start, h->cells1, Pi, 0, 64, st));
        k_cgr_pairseg<<<sp, 256, 0, st>>>(Pi, h->cells1, h->seg, h->sk1);
        ALCU_TRY(cudaGetLastError());
        b = h->cub_bytes;
        ALCU_TRY(cub::DeviceRadixSort::SortPairs(h->cub_tmp, b, h->sk1, h->sk2, h->cells1, h->cells2, Pi, 0,
                                                 h->seg_bits, st));
        for (int w = 0; w <= max_wave; ++w) {
            k_cgr_adm<<<sp, 256, 0, st>>>(Pi, w, h->cells2, h->sk2, h->cand, h->root, h->wave, labels, h->flag);
            ALCU_TRY(cudaGetLastError());
            b = h->cub_bytes;
            ALCU_TRY(cub::DeviceScan::ExclusiveSumByKey(h->cub_tmp, b, h->sk2, h->flag, h->pos, Pi,
                                                        ::cuda::std::equal_to<>(), st));
            k_cgr_vacate<<<gb, 256, 0, st>>>(w, h->band, n_band, h->root, h->size, h->wave, labels);
            k_cgr_take<<<sp, 256, 0, st>>>(Pi, w, h->cells2, h->sk2, h->cand, h->flag, h->pos, h->size, h->wave,
                                           h->orig, labels);
            ALCU_TRY(cudaGetLastError());
        }
    } else {
        // more pairs than cells (dilations stacked many deep): wave by wave
        for (int w = 0; w <= max_wave; ++w) {
            k_cgr_flags<<<gb, 256, 0, st>>>(d, w, h->band, n_band, labels, h->root, h->u8a, h->wave, h->flag,
                                            h->seg);
            ALCU_TRY(cudaGetLastError());
            b = h->cub_bytes;
            ALCU_TRY(cub::DeviceScan::ExclusiveSum(h->cub_tmp, b, h->flag, h->pos, Mb, st));
            k_compact<<<gb, 256, 0, st>>>(Mb, h->flag, h->pos, h->band, h->cand, n_cand);
            ALCU_TRY(cudaGetLastError());
            int M = 0;
            ALCU_TRY(cudaMemcpyAsync(&M, n_cand, sizeof(int), cudaMemcpyDeviceToHost, st));
            ALCU_TRY(cudaStreamSynchronize(st));
            if (M == 0) continue;
            if ((rc = cub_reserve(h, M)) != GPK_OK) return rc;
            const int sb = (M + 255) / 256 < G ? (M + 255) / 256 : G;
            k_cgr_score<<<sb, 256, 0, st>>>(d, t, h->cand, n_cand, h->root, h->seg, h->key1);
            ALCU_TRY(cudaGetLastError());
            b = h->cub_bytes;
            ALCU_TRY(cub::DeviceRadixSort::SortPairs(h->cub_tmp, b, h->key1, h->key2, h->cand, h->cells1, M, 0, 64,
                                                     st));
            k_cgr_segkeys<<<sb, 256, 0, st>>>(h->cells1, n_cand, h->seg, h->sk1);
            ALCU_TRY(cudaGetLastError());
            b = h->cub_bytes;
            ALCU_TRY(cub::DeviceRadixSort::SortPairs(h->cub_tmp, b, h->sk1, h->sk2, h->cells1, h->cells2, M, 0,
                                                     h->seg_bits, st));
            k_cgr_starts<<<sb, 256, 0, st>>>(h->sk2, n_cand, h->start);
            k_cgr_vacate<<<gb, 256, 0, st>>>(w, h->band, n_band, h->root, h->size, h->wave, labels);
            k_cgr_select<<<sb, 256, 0, st>>>(h->sk2, h->cells2, n_cand, h->start, h->size, h->orig, labels);
            ALCU_TRY(cudaGetLastError());
        }
    }
    k_cgr_changed<<<gb, 256, 0, st>>>(h->band, n_band, labels, h->orig, alpha, h->u64 + 2);
    ALCU_TRY(cudaGetLastError());
    unsigned long long n_changed = 0;
    ALCU_TRY(cudaMemcpyAsync(&n_changed, h->u64 + 2, sizeof(n_changed), cudaMemcpyDeviceToHost, st));
    ALCU_TRY(cudaStreamSynchronize(st));
    if (changed) *changed = (int64_t)n_changed;
    return GPK_OK;
}

extern "C" int gpk_alcu_commit_transactions(gpk_alcu* h, int8_t* labels, double* alpha, const int8_t* competitor,
                                            const uint8_t* crossing, int64_t* deferred) {
    if (!h || !labels || !alpha || !competitor || !crossing) {
        gpk_set_error("alcu: null argument");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    const Ext& d = h->d;
    const long long N = d.N;
    cudaStream_t st = h->stream;
    const int G = h->grid;
    int* n_list = h->i32 + 6;
    int* xhist = h->aux;  // 256 ints: crossing cells per label
    ALCU_TRY(cudaMemsetAsync(h->cnt256, 0, sizeof(int) * 256, st));
    ALCU_TRY(cudaMemsetAsync(xhist, 0, sizeof(int) * 256, st));
    ALCU_TRY(cudaMemsetAsync(h->u64, 0, sizeof(unsigned long long) * 4, st));
    k_label_hist<<<G, 256, 0, st>>>(N, labels, h->cnt256);
    k_u8_flags<<<G, 256, 0, st>>>(N, crossing, h->flag);
    ALCU_TRY(cudaGetLastError());
    size_t b = h->cub_bytes;
    ALCU_TRY(cub::DeviceScan::ExclusiveSum(h->cub_tmp, b, h->flag, h->pos, (int)N, st));
    k_compact<<<G, 256, 0, st>>>(N, h->flag, h->pos, nullptr, h->cand, n_list);
    k_tx_init<<<G, 256, 0, st>>>(h->cand, n_list, h->wave, xhist, labels);
    ALCU_TRY(cudaGetLastError());
    int M = 0;
    int hc[256], hx[256];
    ALCU_TRY(cudaMemcpyAsync(&M, n_list, sizeof(int), cudaMemcpyDeviceToHost, st));
    ALCU_TRY(cudaMemcpyAsync(hc, h->cnt256, sizeof(hc), cudaMemcpyDeviceToHost, st));
    ALCU_TRY(cudaMemcpyAsync(hx, xhist, sizeof(hx), cudaMemcpyDeviceToHost, st));
    ALCU_TRY(cudaStreamSynchronize(st));
    if (deferred) *deferred = 0;
    if (M == 0) return GPK_OK;
    // the extinction test can only fire for a label that the sweep may
    // reduce to one cell; then the serial order runs on one thread
    bool extinction_possible = false;
    for (int k = 0; k < 256; ++k)
        if (hx[k] && hc[k] - hx[k] < 2) extinction_possible = true;
    unsigned long long nd = 0;
    if (extinction_possible) {
        k_tx_commit<<<1, 32, 0, st>>>(d, h->cand, n_list, labels, alpha, competitor, h->cnt256, h->u64 + 1);
        ALCU_TRY(cudaGetLastError());
        ALCU_TRY(cudaMemcpyAsync(&nd, h->u64 + 1, sizeof(nd), cudaMemcpyDeviceToHost, st));
        ALCU_TRY(cudaStreamSynchronize(st));
    } else {
        const int gb = (M + 255) / 256 < G ? (M + 255) / 256 : G;
        unsigned long long hcnt[2] = {0, 0};
        // the earliest pending transaction is always ready: at most M rounds
        for (int round = 0; hcnt[0] < (unsigned long long)M;) {
            if (round > M) {
                gpk_set_error("alcu: transaction rounds did not finish");
                return GPK_ERR_INTERNAL;
            }
            for (int k = 0; k < 8; ++k, ++round)
                k_tx_round<<<gb, 256, 0, st>>>(d, round, h->cand, n_list, crossing, h->wave, labels, alpha,
                                                competitor, h->u64);
            ALCU_TRY(cudaGetLastError());
            ALCU_TRY(cudaMemcpyAsync(hcnt, h->u64, sizeof(hcnt), cudaMemcpyDeviceToHost, st));
            ALCU_TRY(cudaStreamSynchronize(st));
        }
        nd = hcnt[1];
    }
    if (deferred) *deferred = (int64_t)nd;
    return GPK_OK;
}

extern "C" int gpk_alcu_balanced_remap(gpk_alcu* h, int8_t* labels, double* alpha, const double* taps, int radius,
                                       int64_t* changed) {
    if (!h || !labels || !alpha) { gpk_set_error("alcu: null argument"); return GPK_ERR_INVALID_ARGUMENT; }
    Taps t;
    int rc = taps_of(taps, radius, t);
    if (rc != GPK_OK) return rc;
    const Ext& d = h->d;
    const long long N = d.N;
    cudaStream_t st = h->stream;
    const int G = h->grid;
    // the labels present (np.unique)
    ALCU_TRY(cudaMemsetAsync(h->cnt256, 0, sizeof(int) * 256, st));
    k_label_hist<<<G, 256, 0, st>>>(N, labels, h->cnt256);
    ALCU_TRY(cudaGetLastError());
    int hc[256];
    ALCU_TRY(cudaMemcpyAsync(hc, h->cnt256, sizeof(hc), cudaMemcpyDeviceToHost, st));
    ALCU_TRY(cudaStreamSynchronize(st));
    Vals vals{};
    for (int k = 0; k < 256; ++k)
        if (hc[k]) {
            if (vals.n == 8) {
                gpk_set_error("alcu: the balanced remap takes at most 8 distinct labels");
                return GPK_ERR_INVALID_ARGUMENT;
            }
            vals.v[vals.n++] = k - 128;
        }
    if (h->n_scores < vals.n) {
        ALCU_TRY(cudaStreamSynchronize(st));
        cudaFree(h->scores);
        h->scores = nullptr;
        h->n_scores = 0;
        if (cudaMalloc((void**)&h->scores, sizeof(double) * N * vals.n) != cudaSuccess) {
            cudaGetLastError();
            gpk_set_error("alcu: cudaMalloc of the balanced remap's score fields failed");
            return GPK_ERR_OUT_OF_MEMORY;
        }
        h->n_scores = vals.n;
        h->bytes += (long long)sizeof(double) * N * vals.n;
    }
    for (int k = 0; k < vals.n; ++k) {
        k_indicator<<<G, 256, 0, st>>>(N, labels, vals.v[k], h->f[1]);
        ALCU_TRY(cudaGetLastError());
        if ((rc = gauss(h, t, h->f[1], h->scores + (long long)k * N, h->f[5])) != GPK_OK) return rc;
    }
    k_bgr_propose<<<grid3(d), B3, 0, st>>>(d, vals, labels, h->scores, h->flag, h->seg, h->f[2]);
    ALCU_TRY(cudaGetLastError());
    size_t b = h->cub_bytes;
    ALCU_TRY(cub::DeviceScan::ExclusiveSum(h->cub_tmp, b, h->flag, h->pos, (int)N, st));
    int* n_rec = h->i32 + 7;
    k_compact<<<G, 256, 0, st>>>(N, h->flag, h->pos, nullptr, h->cells2, n_rec);  // count only
    k_bgr_records<<<G, 256, 0, st>>>(N, h->flag, h->pos, n_rec, h->f[2], h->cand, h->key1);
    ALCU_TRY(cudaGetLastError());
    int M = 0;
    ALCU_TRY(cudaMemcpyAsync(&M, n_rec, sizeof(int), cudaMemcpyDeviceToHost, st));
    ALCU_TRY(cudaStreamSynchronize(st));
    if (changed) *changed = 0;
    if (M == 0) return GPK_OK;
    if ((rc = cub_reserve(h, M)) != GPK_OK) return rc;
    const int sb = (M + 255) / 256 < G ? (M + 255) / 256 : G;
    // descending gain, ties in descending cell order (the records' order);
    // then grouped by (old, best) pair, stable
    b = h->cub_bytes;
    ALCU_TRY(cub::DeviceRadixSort::SortPairs(h->cub_tmp, b, h->key1, h->key2, h->cand, h->cells1, M, 0, 64, st));
    k_cgr_segkeys<<<sb, 256, 0, st>>>(h->cells1, n_rec, h->seg, h->sk1);
    ALCU_TRY(cudaGetLastError());
    b = h->cub_bytes;
    ALCU_TRY(cub::DeviceRadixSort::SortPairs(h->cub_tmp, b, h->sk1, h->sk2, h->cells1, h->cells2, M, 0, 6, st));
    ALCU_TRY(cudaMemsetAsync(h->aux, 0, sizeof(int) * 64, st));
    k_pair_hist<<<sb, 256, 0, st>>>(h->sk2, n_rec, h->aux);
    ALCU_TRY(cudaGetLastError());
    int hist[64];
    ALCU_TRY(cudaMemcpyAsync(hist, h->aux, sizeof(hist), cudaMemcpyDeviceToHost, st));
    ALCU_TRY(cudaStreamSynchronize(st));
    PairSegs segs{};
    for (int k = 0, acc = 0; k < 64; ++k) {
        segs.start[k] = acc;
        segs.len[k] = hist[k];
        acc += hist[k];
    }
    ALCU_TRY(cudaMemsetAsync(h->u8a, 0, N, st));
    ALCU_TRY(cudaMemsetAsync(h->u64 + 2, 0, sizeof(unsigned long long) * 2, st));
    // the exchanges of each pair, in the serial order
    PairList pl{};
    int total = 0;
    for (int ia = 0; ia < vals.n; ++ia)
        for (int ib = ia + 1; ib < vals.n; ++ib) {
            const int first = vals.v[ia], second = vals.v[ib];
            if ((first == 0) != (second == 0)) continue;
            const int sf = ia * 8 + ib, sr = ib * 8 + ia;
            const int cnt = segs.len[sf] < segs.len[sr] ? segs.len[sf] : segs.len[sr];
            if (cnt == 0) continue;
            pl.sf[pl.n] = sf;
            pl.sr[pl.n] = sr;
            pl.cnt[pl.n] = cnt;
            pl.base[pl.n] = total;
            pl.first[pl.n] = first;
            pl.second[pl.n] = second;
            ++pl.n;
            total += cnt;
        }
    bool few = false;  // a label of at most 2 cells: the extinction test may apply
    for (int k = 0; k < vals.n; ++k)
        if (hc[vals.v[k] + 128] <= 2) few = true;
    if (total > 0 && few) {
        k_bgr_exchange<<<1, 32, 0, st>>>(d, vals, segs, h->cells2, labels, h->cnt256, h->u8a);
        ALCU_TRY(cudaGetLastError());
    } else if (total > 0) {
        // exchange arrays: f, r, pair, done in key2 (as ints), xid in wave
        int* xf = reinterpret_cast<int*>(h->key2);
        int* xr = xf + total;
        int* xp = xr + total;
        int* done = h->pos;
        const int gx = (total + 255) / 256 < G ? (total + 255) / 256 : G;
        k_bgr_xinit<<<sb, 256, 0, st>>>(h->cells2, n_rec, h->wave);
        k_bgr_xindex<<<gx, 256, 0, st>>>(pl, segs, h->cells2, xf, xr, xp, h->wave, done, total);
        ALCU_TRY(cudaGetLastError());
        unsigned long long ran = 0;
        for (int round = 0; ran < (unsigned long long)total;) {
            if (round > total) {
                gpk_set_error("alcu: exchange rounds did not finish");
                return GPK_ERR_INTERNAL;
            }
            for (int k = 0; k < 8; ++k, ++round)
                k_bgr_round<<<gx, 256, 0, st>>>(d, pl, round, total, xf, xr, xp, h->flag, h->wave, done, labels,
                                                 h->u8a, h->u64 + 2);
            ALCU_TRY(cudaGetLastError());
            ALCU_TRY(cudaMemcpyAsync(&ran, h->u64 + 2, sizeof(ran), cudaMemcpyDeviceToHost, st));
            ALCU_TRY(cudaStreamSynchronize(st));
        }
    }
    k_bgr_finish<<<sb, 256, 0, st>>>(h->cells2, n_rec, h->u8a, alpha, h->u64 + 3);
    ALCU_TRY(cudaGetLastError());
    unsigned long long nc = 0;
    ALCU_TRY(cudaMemcpyAsync(&nc, h->u64 + 3, sizeof(nc), cudaMemcpyDeviceToHost, st));
    ALCU_TRY(cudaStreamSynchronize(st));
    if (changed) *changed = (int64_t)nc;
    return GPK_OK;
}

extern "C" int gpk_alcu_info(const gpk_alcu* h, int64_t* cells, int64_t* device_bytes, int64_t* last_components,
                             int64_t* last_waves, int64_t* last_pairs) {
    if (!h) { gpk_set_error("alcu: null handle"); return GPK_ERR_INVALID_ARGUMENT; }
    if (last_pairs) *last_pairs = h->last_pairs;
    if (cells) *cells = h->d.N;
    if (device_bytes) *device_bytes = h->bytes;
    if (last_components) *last_components = h->last_components;
    if (last_waves) *last_waves = h->last_waves;
    return GPK_OK;
}
