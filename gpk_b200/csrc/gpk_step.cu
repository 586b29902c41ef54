// gpk_step.cu — the per-step kernels of GPKGrid::step() and their sequencing.
//
// Reference (albert-hzbn/GPK):
//   step order           src/gpk_simulation.cpp:31-54
//   interface mask       src/gpk_geometry.cpp:42-82
//   geometry (direct)    src/gpk_geometry.cpp:88-183
//   geometry (separable) src/gpk_geometry.cpp:185-390, src/gpk_gaussian.cpp:9-72
//   elastic proxy        src/gpk_physics.cpp:10-63
//   velocities           src/gpk_physics.cpp:67-148
//   pair projection      src/gpk_physics.cpp:152-193
//   max_dt               src/gpk_simulation.cpp:11-23
//   alpha integration    src/gpk_transitions.cpp:251-271
//   transport, recovery  src/gpk_transport.cpp:11-152
//
// Every real-valued expression keeps the reference's operand order; with
// -fmad=false the float path rounds exactly like the reference build.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>

#include "gpk_grid.h"

namespace gpk_dev {

// ---------------------------------------------------------------------------
// interface mask + ordered compaction
// ---------------------------------------------------------------------------
static constexpr int MASK_TPB = 256;
static constexpr int MASK_IPT = 8;
static constexpr int MASK_TILE = MASK_TPB * MASK_IPT;

// `gate` (may be null): when it points to zero the launch does nothing
// (device-side skip of a stage inside a captured step)
__global__ void __launch_bounds__(MASK_TPB) k_mask_tiles(Dims D, const int32_t* __restrict__ phi,
                                                         uint8_t* __restrict__ mask, int32_t* __restrict__ tile_cnt,
                                                         const unsigned long long* gate = nullptr) {
    if (gate && *gate == 0ull) return;
    typedef cub::BlockReduce<int, MASK_TPB> BR;
    __shared__ typename BR::TempStorage tmp;
    const int base = blockIdx.x * MASK_TILE;
    int cnt = 0;
#pragma unroll
    for (int k = 0; k < MASK_IPT; ++k) {
        const int i = base + k * MASK_TPB + threadIdx.x;
        if (i < D.N) {
            int nb[6];
            D.faces(i, nb);
            const int32_t v = phi[i];
            const uint8_t act = (uint8_t)((v != phi[nb[0]]) | (v != phi[nb[1]]) | (v != phi[nb[2]]) |
                                          (v != phi[nb[3]]) | (v != phi[nb[4]]) | (v != phi[nb[5]]));
            mask[i] = act;
            cnt += act;
        }
    }
    const int total = BR(tmp).Sum(cnt);
    if (threadIdx.x == 0) tile_cnt[blockIdx.x] = total;
}

// The same mask when Nx is a multiple of 4: each thread takes groups of four
// cells of a row (one int4 load per face-neighbour row or plane, two scalar
// loads for the x neighbours of the group's ends) and stores four flags at once.
__global__ void __launch_bounds__(MASK_TPB) k_mask_tiles4(Dims D, const int32_t* __restrict__ phi,
                                                          uint8_t* __restrict__ mask, int32_t* __restrict__ tile_cnt,
                                                          const unsigned long long* gate = nullptr) {
    if (gate && *gate == 0ull) return;
    typedef cub::BlockReduce<int, MASK_TPB> BR;
    __shared__ typename BR::TempStorage tmp;
    const int nx4 = D.Nx >> 2, plane = D.Nx * D.Ny;
    int cnt = 0;
#pragma unroll
    for (int k = 0; k < MASK_IPT / 4; ++k) {
        const int g = blockIdx.x * (MASK_TILE / 4) + k * MASK_TPB + threadIdx.x;
        const int i = g * 4;
        if (i < D.N) {
            const int row = g / nx4, x = (g - row * nx4) * 4;
            const int y = row % D.Ny, z = row / D.Ny;
            const int oym = (y == 0 ? D.Ny - 1 : -1) * D.Nx, oyp = (y == D.Ny - 1 ? 1 - D.Ny : 1) * D.Nx;
            const int ozm = (z == 0 ? D.Nz - 1 : -1) * plane, ozp = (z == D.Nz - 1 ? 1 - D.Nz : 1) * plane;
            const int4 c = *reinterpret_cast<const int4*>(phi + i);
            const int4 a = *reinterpret_cast<const int4*>(phi + i + oym);
            const int4 b = *reinterpret_cast<const int4*>(phi + i + oyp);
            const int4 d = *reinterpret_cast<const int4*>(phi + i + ozm);
            const int4 e = *reinterpret_cast<const int4*>(phi + i + ozp);
            const int32_t l = phi[i - x + (x == 0 ? D.Nx - 1 : x - 1)];
            const int32_t r = phi[i - x + (x + 4 == D.Nx ? 0 : x + 4)];
            uchar4 m;
            m.x = (uint8_t)((c.x != l) | (c.x != c.y) | (c.x != a.x) | (c.x != b.x) | (c.x != d.x) | (c.x != e.x));
            m.y = (uint8_t)((c.y != c.x) | (c.y != c.z) | (c.y != a.y) | (c.y != b.y) | (c.y != d.y) | (c.y != e.y));
            m.z = (uint8_t)((c.z != c.y) | (c.z != c.w) | (c.z != a.z) | (c.z != b.z) | (c.z != d.z) | (c.z != e.z));
            m.w = (uint8_t)((c.w != c.z) | (c.w != r) | (c.w != a.w) | (c.w != b.w) | (c.w != d.w) | (c.w != e.w));
            *reinterpret_cast<uchar4*>(mask + i) = m;
            cnt += m.x + m.y + m.z + m.w;
        }
    }
    const int total = BR(tmp).Sum(cnt);
    if (threadIdx.x == 0) tile_cnt[blockIdx.x] = total;
}

// Exclusive scan of tile counts in one block; writes the total.
__global__ void __launch_bounds__(1024) k_scan_tiles(int32_t* __restrict__ tile, int ntiles, unsigned* __restrict__ total,
                                                     const unsigned long long* gate = nullptr) {
    if (gate && *gate == 0ull) return;
    typedef cub::BlockScan<int, 1024> BS;
    __shared__ typename BS::TempStorage tmp;
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < ntiles; base += 1024) {
        const int i = base + threadIdx.x;
        const int v = i < ntiles ? tile[i] : 0;
        int ex, agg;
        BS(tmp).ExclusiveSum(v, ex, agg);
        if (i < ntiles) tile[i] = ex + carry;
        __syncthreads();
        if (threadIdx.x == 0) carry += agg;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = (unsigned)carry;
}

// Writes the flat indices of flagged cells in increasing order.
__global__ void __launch_bounds__(MASK_TPB) k_compact_u8(int n, const uint8_t* __restrict__ flag,
                                                         const int32_t* __restrict__ tile_off, int32_t* __restrict__ out,
                                                         const unsigned long long* gate = nullptr) {
    if (gate && *gate == 0ull) return;
    typedef cub::BlockScan<int, MASK_TPB> BS;
    __shared__ typename BS::TempStorage tmp;
    const int base = blockIdx.x * MASK_TILE;
    int f[MASK_IPT];
    int cnt = 0;
#pragma unroll
    for (int k = 0; k < MASK_IPT; ++k) {
        const int i = base + threadIdx.x * MASK_IPT + k;
        f[k] = (i < n) ? flag[i] : 0;
        cnt += f[k];
    }
    int ex;
    BS(tmp).ExclusiveSum(cnt, ex);
    int pos = tile_off[blockIdx.x] + ex;
#pragma unroll
    for (int k = 0; k < MASK_IPT; ++k) {
        const int i = base + threadIdx.x * MASK_IPT + k;
        if (f[k]) out[pos++] = i;
    }
}

// Tile counts of a u8 flag array whose valid length is read on the device.
__global__ void __launch_bounds__(MASK_TPB) k_count_u8(const uint8_t* __restrict__ flag, const unsigned* __restrict__ n_ptr,
                                                       int32_t* __restrict__ tile_cnt) {
    typedef cub::BlockReduce<int, MASK_TPB> BR;
    __shared__ typename BR::TempStorage tmp;
    const int n = (int)*n_ptr;
    const int base = blockIdx.x * MASK_TILE;
    int cnt = 0;
    for (int k = 0; k < MASK_IPT; ++k) {
        const int i = base + k * MASK_TPB + threadIdx.x;
        if (i < n) cnt += flag[i];
    }
    const int total = BR(tmp).Sum(cnt);
    if (threadIdx.x == 0) tile_cnt[blockIdx.x] = total;
}

__global__ void __launch_bounds__(MASK_TPB) k_compact_u8_dyn(const unsigned* __restrict__ n_ptr,
                                                             const uint8_t* __restrict__ flag,
                                                             const int32_t* __restrict__ tile_off,
                                                             int32_t* __restrict__ out) {
    typedef cub::BlockScan<int, MASK_TPB> BS;
    __shared__ typename BS::TempStorage tmp;
    const int n = (int)*n_ptr;
    const int base = blockIdx.x * MASK_TILE;
    int f[MASK_IPT];
    int cnt = 0;
#pragma unroll
    for (int k = 0; k < MASK_IPT; ++k) {
        const int i = base + threadIdx.x * MASK_IPT + k;
        f[k] = (i < n) ? flag[i] : 0;
        cnt += f[k];
    }
    int ex;
    BS(tmp).ExclusiveSum(cnt, ex);
    int pos = tile_off[blockIdx.x] + ex;
#pragma unroll
    for (int k = 0; k < MASK_IPT; ++k) {
        const int i = base + threadIdx.x * MASK_IPT + k;
        if (f[k]) out[pos++] = i;
    }
}

// ---------------------------------------------------------------------------
// direct Gaussian-Hessian geometry + competitor choice
// ---------------------------------------------------------------------------
// table layout per tap t = ((dz+R)*W + (dy+R))*W + (dx+R), 12 reals:
//   [0] gx1*gy0*gz0 (Ix)   [1] gx0*gy1*gz0 (Iy)  [2] gx2*gy0*gz0 (Ixx) [3] gx0*gy2*gz0 (Iyy)
//   [4] gx1*gy1*gz0 (Ixy)  [5] gx0*gy0*gz1 (Iz)  [6] gx0*gy0*gz2 (Izz) [7] gx1*gy0*gz1 (Ixz)
//   [8] gx0*gy1*gz1 (Iyz)  [9..11] 0
// each product formed on the host exactly as the reference forms it, (a*b)*c.

template <typename real>
__device__ __forceinline__ void competitor_at(const Dims& D, const int32_t* __restrict__ phi, int i, real nx, real ny,
                                              real nz, int32_t* __restrict__ phi_comp) {
    int z, y, x;
    D.decode(i, z, y, x);
    int nei[6];
    D.faces(i, nei);
    const real score[6] = {-nx, nx, -ny, ny, -nz, nz};
    const int nf = D.nface();
    const bool is3d = D.is3d();
    const int32_t pi = phi[i];
    int best = -1, best_support = -1;
    real best_score = (real)-2;
    for (int k = 0; k < nf; ++k) {
        const int32_t q = phi[nei[k]];
        if (q == pi) continue;
        int support = 0;
        for (int dz = (is3d ? -1 : 0); dz <= (is3d ? 1 : 0); ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    if (!dx && !dy && !dz) continue;
                    const int xx = wrap1(x + dx, D.Nx), yy = wrap1(y + dy, D.Ny), zz = wrap1(z + dz, D.Nz);
                    support += phi[D.idx(zz, yy, xx)] == q;
                }
        if (support > best_support || (support == best_support && score[k] > best_score)) {
            best = k; best_support = support; best_score = score[k];
        }
    }
    phi_comp[i] = (best >= 0) ? phi[nei[best]] : pi;
}

template <typename real>
__device__ __forceinline__ void finish_geometry(int i, real Ix, real Iy, real Iz, real Ixx, real Iyy, real Izz, real Ixy,
                                                real Ixz, real Iyz, real dx, real kappa_limit, real* nxo, real* nyo,
                                                real* nzo, real* ko, real& nxv, real& nyv, real& nzv) {
    const real grad_sq = Ix * Ix + Iy * Iy + Iz * Iz;
    nxv = nyv = nzv = (real)0;
    if (grad_sq * dx * dx > (real)1e-8) {
        const real grad = sqrt(grad_sq);
        nxv = -Ix / grad;
        nyv = -Iy / grad;
        nzv = -Iz / grad;
        const real trace_H = Ixx + Iyy + Izz;
        const real gHg = Ix * Ix * Ixx + Iy * Iy * Iyy + Iz * Iz * Izz + (real)2 * (Ix * Iy * Ixy + Ix * Iz * Ixz + Iy * Iz * Iyz);
        real curvature = (gHg - grad_sq * trace_H) / (grad_sq * grad);
        if (fabs(curvature * dx) < (real)1e-6) curvature = (real)0;
        nxo[i] = nxv; nyo[i] = nyv; nzo[i] = nzv;
        ko[i] = dclamp(curvature, -kappa_limit, kappa_limit);
    }
}

template <typename real, bool IS3D>
__global__ void __launch_bounds__(128) k_geometry_direct(Dims D, const int32_t* __restrict__ active,
                                                         const unsigned* __restrict__ n_active,
                                                         const int32_t* __restrict__ phi, const real* __restrict__ table,
                                                         int R, real inv_dx, real inv_dx2, real dx, real kappa_limit,
                                                         real* __restrict__ nxo, real* __restrict__ nyo,
                                                         real* __restrict__ nzo, real* __restrict__ ko,
                                                         int32_t* __restrict__ phi_comp) {
    const int na = (int)*n_active;
    const int W = 2 * R + 1;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < na; a += gridDim.x * blockDim.x) {
        const int i = active[a];
        const int32_t resident = phi[i];
        int z0, y0, x0;
        D.decode(i, z0, y0, x0);
        real Ix = 0, Iy = 0, Iz = 0, Ixx = 0, Iyy = 0, Izz = 0, Ixy = 0, Ixz = 0, Iyz = 0;
        const int dzb = IS3D ? -R : 0, dze = IS3D ? R : 0;
        for (int dz = dzb; dz <= dze; ++dz) {
            const int z = IS3D ? wrap_any(z0 + dz, D.Nz) : z0;
            for (int dy = -R; dy <= R; ++dy) {
                const int y = wrap_any(y0 + dy, D.Ny);
                const int32_t* row = phi + (size_t)(z * D.Ny + y) * D.Nx;
                const int zoff = IS3D ? (dz + R) * W : 0;
                const real* trow = table + (size_t)((zoff + (dy + R)) * W) * 12;
                for (int dx = -R; dx <= R; ++dx) {
                    int x = x0 + dx;
                    if (x < 0 || x >= D.Nx) x = wrap_any(x, D.Nx);
                    if (row[x] != resident) continue;
                    const real* t = trow + (dx + R) * 12;
                    // table entry: (Ix, Ixx, Ixy, Ixz), (Iy, Iyy, Ixy, Iyz), (Iz, Izz, Ixz, Iyz)
                    Ix += t[0]; Iy += t[4]; Ixx += t[1]; Iyy += t[5]; Ixy += t[2];
                    if (IS3D) { Iz += t[8]; Izz += t[9]; Ixz += t[3]; Iyz += t[7]; }
                }
            }
        }
        Ix *= inv_dx; Iy *= inv_dx; Iz *= inv_dx;
        Ixx *= inv_dx2; Iyy *= inv_dx2; Izz *= inv_dx2;
        Ixy *= inv_dx2; Ixz *= inv_dx2; Iyz *= inv_dx2;
        real nxv, nyv, nzv;
        finish_geometry<real>(i, Ix, Iy, Iz, Ixx, Iyy, Izz, Ixy, Ixz, Iyz, dx, kappa_limit, nxo, nyo, nzo, ko, nxv, nyv, nzv);
        competitor_at<real>(D, phi, i, nxv, nyv, nzv, phi_comp);
    }
}

// ---- separable path (broad 3-D kernels) -----------------------------------
//
// One periodic 1-D Gaussian pass (src/gpk_gaussian.cpp:9-72): every output is
// acc = 0; acc += w[k] * in[wrap(q + k - R)] for k = 0 .. 2R, a multiply and
// an add per tap in tap order (no contraction).  The tiled kernel stages a
// tile of 32 lines x SEP_TL outputs plus the 2R halo in shared memory; each
// thread then produces SEP_M consecutive outputs of one line from a ring of
// SEP_M values in registers, so a tap costs one shared load per SEP_M
// outputs.  Lines are the cells sharing the other two coordinates; the 32
// lanes of a warp take 32 lines, so for the y and z passes every global load
// and store is a 128-byte row of consecutive x.  For the x pass the lines are
// rows of x: warps load and store whole rows (int4 label loads for the
// indicator when the rows are whole tiles) and the shared rows are padded to
// an odd length so that the 32 lanes, each walking its own row, hit 32 banks.
// With IND the input is the indicator phi == p, formed as the labels load.
static constexpr int SEP_TL = 128;      // outputs per line per tile
static constexpr int SEP_M = 8;         // outputs per thread
static constexpr int SEP_WARPS = SEP_TL / SEP_M;
static constexpr int SEP_TPB = 32 * SEP_WARPS;

__host__ __device__ __forceinline__ int sep_pitch(int axis, int R) {
    // positions staged per line: the tile, its halo, and SEP_M of slack for
    // the ring's last (unused) refill
    const int p = SEP_TL + 2 * R + SEP_M;
    return axis == 0 ? (p | 1) : p;
}

// One tap of the ring (KK = the tap's index within its chunk of SEP_M, so
// every register index is a compile-time constant): each output adds the
// product of the tap weight with its own ring value, in tap order.
template <int KK, typename real>
__device__ __forceinline__ void sep_tap(real (&acc)[SEP_M], const real (&v)[SEP_M], real wk) {
#pragma unroll
    for (int m = 0; m < SEP_M; ++m) acc[m] += wk * v[(m + KK) % SEP_M];
}

template <typename real, int AX, bool IND>
__global__ void __launch_bounds__(SEP_TPB) k_sep_pass(Dims D, const real* __restrict__ in,
                                                      const int32_t* __restrict__ phi, int32_t p,
                                                      real* __restrict__ out, const real* __restrict__ kw, int R) {
    extern __shared__ __align__(16) unsigned char sep_smem[];
    real* tw = (real*)sep_smem;
    const int K = 2 * R + 1;
    const int Kp = (K + 1) & ~1;
    real* s = tw + Kp;
    const int n = AX == 0 ? D.Nx : (AX == 1 ? D.Ny : D.Nz);
    const int nlines = AX == 0 ? D.Nz * D.Ny : (AX == 1 ? D.Nz * D.Nx : D.Ny * D.Nx);
    const int stride = AX == 0 ? 1 : (AX == 1 ? D.Nx : D.Ny * D.Nx);
    const int P = sep_pitch(AX, R);
    const int segs = (n + SEP_TL - 1) / SEP_TL;
    const int seg = blockIdx.x % segs;
    const int lb = blockIdx.x / segs;
    const int a0 = seg * SEP_TL;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    auto line_base = [&](int l) -> int {
        if (AX == 0) return l * D.Nx;
        if (AX == 1) return (l / D.Nx) * D.Ny * D.Nx + l % D.Nx;
        return l;
    };
    auto load = [&](int gi) -> real {
        if (IND) return phi[gi] == p ? (real)1 : (real)0;
        return in[gi];
    };
    for (int k = threadIdx.x; k < K; k += SEP_TPB) tw[k] = kw[k];
    const int span = SEP_TL + 2 * R;
    if (AX == 0) {
        // rows: warp w stages rows w, w + SEP_WARPS, ...; a lane's wrapped
        // x for pos = lane + 32 i advances by 32 (mod n)
        const bool vec = IND && (D.Nx % SEP_TL) == 0;
        const int gw0 = wrap_any(a0 - R + lane, n);
        for (int r = warp; r < 32; r += SEP_WARPS) {
            const int l = lb * 32 + r;
            if (l >= nlines) break;
            const int b = line_base(l);
            real* row = s + r * P;
            if (vec) {
                for (int c4 = lane; c4 < SEP_TL / 4; c4 += 32) {
                    const int4 q = *reinterpret_cast<const int4*>(phi + b + a0 + 4 * c4);
                    row[R + 4 * c4 + 0] = q.x == p ? (real)1 : (real)0;
                    row[R + 4 * c4 + 1] = q.y == p ? (real)1 : (real)0;
                    row[R + 4 * c4 + 2] = q.z == p ? (real)1 : (real)0;
                    row[R + 4 * c4 + 3] = q.w == p ? (real)1 : (real)0;
                }
                for (int h = lane; h < 2 * R; h += 32) {
                    const int pos = h < R ? h : SEP_TL + h;
                    row[pos] = load(b + wrap_any(a0 - R + pos, n));
                }
            } else {
                int gw = gw0;
                for (int pos = lane; pos < span; pos += 32) {
                    row[pos] = load(b + gw);
                    for (gw += 32; gw >= n;) gw -= n;
                }
            }
        }
    } else {
        const int l = lb * 32 + lane;
        if (l < nlines) {
            const int b = line_base(l);
            int gw = wrap_any(a0 - R + warp, n);
            for (int pos = warp; pos < span; pos += SEP_WARPS) {
                s[pos * 32 + lane] = load(b + gw * stride);
                for (gw += SEP_WARPS; gw >= n;) gw -= n;
            }
        }
    }
    __syncthreads();
    const int o0 = warp * SEP_M;
    auto S = [&](int j) -> real { return AX == 0 ? s[lane * P + j] : s[j * 32 + lane]; };
    real v[SEP_M], acc[SEP_M];
#pragma unroll
    for (int m = 0; m < SEP_M; ++m) {
        v[m] = S(o0 + m);
        acc[m] = 0;
    }
    // ring: slot i holds position o0 + j with j == i (mod SEP_M); after tap
    // kb + kk the value at o0 + kb + kk is dead and its slot takes the value
    // SEP_M further on.  Whole chunks of SEP_M taps run without guards, with
    // the tap and ring pointers advanced once per chunk; the last partial
    // chunk with guards.
    constexpr int SS = AX == 0 ? 1 : 32;  // shared-memory stride along the line
    const real* sp = AX == 0 ? &s[lane * P + o0 + SEP_M] : &s[(o0 + SEP_M) * 32 + lane];
    const real* tp = tw;
#define SEP_STEP(kk)                          \
    {                                         \
        sep_tap<kk>(acc, v, tp[kk]);          \
        v[kk] = sp[(kk) * SS];                \
    }
    int kb = 0;
    for (; kb + SEP_M <= K; kb += SEP_M, tp += SEP_M, sp += SEP_M * SS) {
        SEP_STEP(0) SEP_STEP(1) SEP_STEP(2) SEP_STEP(3) SEP_STEP(4) SEP_STEP(5) SEP_STEP(6) SEP_STEP(7)
    }
    static_assert(SEP_M == 8, "the chunk bodies list eight steps");
    const int rem = K - kb;
    if (rem > 0) SEP_STEP(0)
    if (rem > 1) SEP_STEP(1)
    if (rem > 2) SEP_STEP(2)
    if (rem > 3) SEP_STEP(3)
    if (rem > 4) SEP_STEP(4)
    if (rem > 5) SEP_STEP(5)
    if (rem > 6) SEP_STEP(6)
#undef SEP_STEP
    const int l = lb * 32 + lane;
    if (AX == 0) {
        // stage the outputs in the (now free) rows, then store whole rows
        __syncthreads();
#pragma unroll
        for (int m = 0; m < SEP_M; ++m) s[lane * P + o0 + m] = acc[m];
        __syncthreads();
        for (int r = warp; r < 32; r += SEP_WARPS) {
            const int lr = lb * 32 + r;
            if (lr >= nlines) break;
            const int b = line_base(lr);
            for (int pos = lane; pos < SEP_TL; pos += 32)
                if (a0 + pos < n) out[b + a0 + pos] = s[r * P + pos];
        }
    } else if (l < nlines) {
        const int b = line_base(l);
#pragma unroll
        for (int m = 0; m < SEP_M; ++m)
            if (a0 + o0 + m < n) out[b + (a0 + o0 + m) * stride] = acc[m];
    }
}

// Float x pass of an indicator with paired arithmetic.  The input is 0 or 1,
// so every product w * v is exact and round(acc + w * v) is also what one
// fused multiply-add gives: the pass may use fma.rn.f32x2 (two outputs per
// instruction, a quarter of the scalar multiply + add issue count) and still
// round exactly as the reference's multiply and add.  (For general inputs
// the products are inexact; those passes keep the scalar k_sep_pass, whose
// mul.rn / add.rn are not contracted.)  Each lane takes two rows, so a
// block covers 64 rows x SEP_TL outputs; shared memory and registers hold
// (row 2i, row 2i + 1) pairs as 64-bit words, row pitch odd in words so that
// the lanes' 64-bit reads fall in distinct banks.
typedef unsigned long long sep_u64;
__device__ __forceinline__ sep_u64 f2_pack(float a, float b) {
    return ((sep_u64)__float_as_uint(b) << 32) | (sep_u64)__float_as_uint(a);
}
__device__ __forceinline__ float f2_lo(sep_u64 v) { return __uint_as_float((unsigned)(v & 0xffffffffu)); }
__device__ __forceinline__ float f2_hi(sep_u64 v) { return __uint_as_float((unsigned)(v >> 32)); }
__device__ __forceinline__ sep_u64 f2_fma(sep_u64 w, sep_u64 v, sep_u64 acc) {
    sep_u64 r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(w), "l"(v), "l"(acc));
    return r;
}

template <int KK>
__device__ __forceinline__ void sep_tap_f2(sep_u64 (&acc)[SEP_M], const sep_u64 (&v)[SEP_M], sep_u64 wk) {
#pragma unroll
    for (int m = 0; m < SEP_M; ++m) acc[m] = f2_fma(wk, v[(m + KK) % SEP_M], acc[m]);
}

__global__ void __launch_bounds__(SEP_TPB) k_sep_x_indicator_f2(Dims D, const int32_t* __restrict__ phi, int32_t p,
                                                                float* __restrict__ out,
                                                                const float* __restrict__ kw, int R) {
    extern __shared__ __align__(16) unsigned char sep_smem[];
    sep_u64* tw = (sep_u64*)sep_smem;
    const int K = 2 * R + 1;
    sep_u64* s = tw + K;
    const int n = D.Nx;
    const int nlines = D.Nz * D.Ny;
    const int P = sep_pitch(0, R);
    const int segs = (n + SEP_TL - 1) / SEP_TL;
    const int seg = blockIdx.x % segs;
    const int lb = blockIdx.x / segs;
    const int a0 = seg * SEP_TL;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    auto ind = [&](int v) -> float { return v == p ? 1.f : 0.f; };
    for (int k = threadIdx.x; k < K; k += SEP_TPB) {
        const float w = kw[k];
        tw[k] = f2_pack(w, w);
    }
    const int span = SEP_TL + 2 * R;
    // pair q holds rows 2q and 2q + 1 of the block's 64
    if (n % SEP_TL == 0) {
        // body: one int4 of labels per row of a pair and thread
        constexpr int C4 = SEP_TL / 4;
        for (int it = threadIdx.x; it < 32 * C4; it += SEP_TPB) {
            const int q = it / C4, c4 = it % C4;
            const int l0 = lb * 64 + 2 * q;
            if (l0 >= nlines) continue;
            const int b0 = l0 * n;
            const int4 x = *reinterpret_cast<const int4*>(phi + b0 + a0 + 4 * c4);
            int4 y = make_int4(p + 1, p + 1, p + 1, p + 1);
            if (l0 + 1 < nlines) y = *reinterpret_cast<const int4*>(phi + b0 + n + a0 + 4 * c4);
            sep_u64* row = s + q * P + R + 4 * c4;
            row[0] = f2_pack(ind(x.x), ind(y.x));
            row[1] = f2_pack(ind(x.y), ind(y.y));
            row[2] = f2_pack(ind(x.z), ind(y.z));
            row[3] = f2_pack(ind(x.w), ind(y.w));
        }
        for (int q = warp; q < 32; q += SEP_WARPS) {
            const int l0 = lb * 64 + 2 * q;
            if (l0 >= nlines) break;
            const int b0 = l0 * n;
            const bool v1 = l0 + 1 < nlines;
            for (int h = lane; h < 2 * R; h += 32) {
                const int pos = h < R ? h : SEP_TL + h;
                const int g = wrap_any(a0 - R + pos, n);
                s[q * P + pos] = f2_pack(ind(phi[b0 + g]), v1 ? ind(phi[b0 + n + g]) : 0.f);
            }
        }
    } else {
        const int gw0 = wrap_any(a0 - R + lane, n);
        for (int q = warp; q < 32; q += SEP_WARPS) {
            const int l0 = lb * 64 + 2 * q;
            if (l0 >= nlines) break;
            const int b0 = l0 * n;
            const bool v1 = l0 + 1 < nlines;
            int gw = gw0;
            for (int pos = lane; pos < span; pos += 32) {
                s[q * P + pos] = f2_pack(ind(phi[b0 + gw]), v1 ? ind(phi[b0 + n + gw]) : 0.f);
                for (gw += 32; gw >= n;) gw -= n;
            }
        }
    }
    __syncthreads();
    const int o0 = warp * SEP_M;
    sep_u64 v[SEP_M], acc[SEP_M];
#pragma unroll
    for (int m = 0; m < SEP_M; ++m) {
        v[m] = s[lane * P + o0 + m];
        acc[m] = 0ull;  // (+0, +0)
    }
    const sep_u64* sp = &s[lane * P + o0 + SEP_M];
    const sep_u64* tp = tw;
#define SEP_STEP2(kk)                        \
    {                                        \
        sep_tap_f2<kk>(acc, v, tp[kk]);      \
        v[kk] = sp[kk];                      \
    }
    int kb = 0;
    for (; kb + SEP_M <= K; kb += SEP_M, tp += SEP_M, sp += SEP_M) {
        SEP_STEP2(0) SEP_STEP2(1) SEP_STEP2(2) SEP_STEP2(3) SEP_STEP2(4) SEP_STEP2(5) SEP_STEP2(6) SEP_STEP2(7)
    }
    const int rem = K - kb;
    if (rem > 0) SEP_STEP2(0)
    if (rem > 1) SEP_STEP2(1)
    if (rem > 2) SEP_STEP2(2)
    if (rem > 3) SEP_STEP2(3)
    if (rem > 4) SEP_STEP2(4)
    if (rem > 5) SEP_STEP2(5)
    if (rem > 6) SEP_STEP2(6)
#undef SEP_STEP2
    __syncthreads();
#pragma unroll
    for (int m = 0; m < SEP_M; ++m) s[lane * P + o0 + m] = acc[m];
    __syncthreads();
    for (int q = warp; q < 32; q += SEP_WARPS) {
        const int l0 = lb * 64 + 2 * q;
        if (l0 >= nlines) break;
        const int b0 = l0 * n;
        const bool v1 = l0 + 1 < nlines;
        for (int pos = lane; pos < SEP_TL; pos += 32) {
            if (a0 + pos >= n) break;
            const sep_u64 r = s[q * P + pos];
            out[b0 + a0 + pos] = f2_lo(r);
            if (v1) out[b0 + n + a0 + pos] = f2_hi(r);
        }
    }
}

// one periodic 1-D pass along axis (0 = x, 1 = y, 2 = z), one thread per
// output, taps from global memory: the form for radii whose tile does not fit
// in shared memory
template <typename real>
__global__ void k_gauss_pass(Dims D, const real* __restrict__ in, real* __restrict__ out, const real* __restrict__ kw,
                             int krad, int axis) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < D.N; i += gridDim.x * blockDim.x) {
        int z, y, x;
        D.decode(i, z, y, x);
        real acc = 0;
        for (int k = 0, ki = -krad; ki <= krad; ++k, ++ki) {
            int j;
            if (axis == 0) j = D.idx(z, y, wrap_any(x + ki, D.Nx));
            else if (axis == 1) j = D.idx(z, wrap_any(y + ki, D.Ny), x);
            else j = D.idx(wrap_any(z + ki, D.Nz), y, x);
            acc += kw[k] * in[j];
        }
        out[i] = acc;
    }
}

template <typename real>
__global__ void k_separable_eval(Dims D, const int32_t* __restrict__ active, const unsigned* __restrict__ n_active,
                                 const int32_t* __restrict__ phi, int32_t p, const real* __restrict__ S, real dx,
                                 real kappa_limit, real* __restrict__ nxo, real* __restrict__ nyo,
                                 real* __restrict__ nzo, real* __restrict__ ko) {
    const int Nx = D.Nx, Ny = D.Ny, Nz = D.Nz;
    const real idx12 = (real)1 / ((real)12 * dx);
    const real idx_sq = (real)1 / (dx * dx);
    const real idx12_sq = idx_sq / (real)12;
    const real idx144_sq = idx_sq / (real)144;
    // the interface cells of label p, from the ordered interface list
    const int na = (int)*n_active;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < na; a += gridDim.x * blockDim.x) {
        const int i = active[a];
        if (phi[i] != p) continue;
        int z, y, x;
        D.decode(i, z, y, x);
        const int xm = (x == 0 ? Nx - 1 : x - 1), xp = (x == Nx - 1 ? 0 : x + 1);
        const int ym = (y == 0 ? Ny - 1 : y - 1), yp = (y == Ny - 1 ? 0 : y + 1);
        const int zm = (z == 0 ? Nz - 1 : z - 1), zp = (z == Nz - 1 ? 0 : z + 1);
        const int xmm = (x < 2 ? x + Nx - 2 : x - 2), xpp = (x >= Nx - 2 ? x - Nx + 2 : x + 2);
        const int ymm = (y < 2 ? y + Ny - 2 : y - 2), ypp = (y >= Ny - 2 ? y - Ny + 2 : y + 2);
        const int zmm = (z < 2 ? z + Nz - 2 : z - 2), zpp = (z >= Nz - 2 ? z - Nz + 2 : z + 2);
        const real I0 = S[i];
        const real Ix = (S[D.idx(z, y, xmm)] - (real)8 * S[D.idx(z, y, xm)] + (real)8 * S[D.idx(z, y, xp)] -
                         S[D.idx(z, y, xpp)]) * idx12;
        const real Iy = (S[D.idx(z, ymm, x)] - (real)8 * S[D.idx(z, ym, x)] + (real)8 * S[D.idx(z, yp, x)] -
                         S[D.idx(z, ypp, x)]) * idx12;
        const real Iz = (Nz > 1) ? (S[D.idx(zmm, y, x)] - (real)8 * S[D.idx(zm, y, x)] + (real)8 * S[D.idx(zp, y, x)] -
                                    S[D.idx(zpp, y, x)]) * idx12
                                 : (real)0;
        const real Ixx = (-S[D.idx(z, y, xpp)] + (real)16 * S[D.idx(z, y, xp)] - (real)30 * I0 +
                          (real)16 * S[D.idx(z, y, xm)] - S[D.idx(z, y, xmm)]) * idx12_sq;
        const real Iyy = (-S[D.idx(z, ypp, x)] + (real)16 * S[D.idx(z, yp, x)] - (real)30 * I0 +
                          (real)16 * S[D.idx(z, ym, x)] - S[D.idx(z, ymm, x)]) * idx12_sq;
        const real Izz = (Nz > 1) ? (-S[D.idx(zpp, y, x)] + (real)16 * S[D.idx(zp, y, x)] - (real)30 * I0 +
                                     (real)16 * S[D.idx(zm, y, x)] - S[D.idx(zmm, y, x)]) * idx12_sq
                                  : (real)0;
        const int xo[4] = {xmm, xm, xp, xpp};
        const int yo[4] = {ymm, ym, yp, ypp};
        const int zo[4] = {zmm, zm, zp, zpp};
        const real dc[4] = {(real)1, (real)-8, (real)8, (real)-1};
        real Ixy_sum = 0, Ixz_sum = 0, Iyz_sum = 0;
        for (int aa = 0; aa < 4; ++aa)
            for (int b = 0; b < 4; ++b) {
                const real w = dc[aa] * dc[b];
                Ixy_sum += w * S[D.idx(z, yo[b], xo[aa])];
                if (Nz > 1) {
                    Ixz_sum += w * S[D.idx(zo[b], y, xo[aa])];
                    Iyz_sum += w * S[D.idx(zo[b], yo[aa], x)];
                }
            }
        const real Ixy = Ixy_sum * idx144_sq;
        const real Ixz = (Nz > 1) ? Ixz_sum * idx144_sq : (real)0;
        const real Iyz = (Nz > 1) ? Iyz_sum * idx144_sq : (real)0;
        const real grad_sq = Ix * Ix + Iy * Iy + Iz * Iz;
        if (grad_sq * dx * dx > (real)1e-8) {
            const real inv_grad = (real)1 / sqrt(grad_sq);
            nxo[i] = -Ix * inv_grad;
            nyo[i] = -Iy * inv_grad;
            nzo[i] = -Iz * inv_grad;
            const real trace_H = Ixx + Iyy + Izz;
            const real gHg = Ix * Ix * Ixx + Iy * Iy * Iyy + Iz * Iz * Izz + (real)2 * (Ix * Iy * Ixy + Ix * Iz * Ixz + Iy * Iz * Iyz);
            real k = (gHg - grad_sq * trace_H) / (grad_sq * sqrt(grad_sq));
            if (fabs(k * dx) < (real)1e-6) k = (real)0;
            ko[i] = dclamp(k, -kappa_limit, kappa_limit);
        }
    }
}

template <typename real>
__global__ void k_competitor_all(Dims D, const int32_t* __restrict__ active, const unsigned* __restrict__ n_active,
                                 const int32_t* __restrict__ phi, const real* __restrict__ nx, const real* __restrict__ ny,
                                 const real* __restrict__ nz, int32_t* __restrict__ phi_comp) {
    const int na = (int)*n_active;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < na; a += gridDim.x * blockDim.x) {
        const int i = active[a];
        competitor_at<real>(D, phi, i, nx[i], ny[i], nz[i], phi_comp);
    }
}

__global__ void k_label_flags(int N, const int32_t* __restrict__ phi, const uint8_t* __restrict__ mask,
                              uint8_t* __restrict__ present, int cap) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
        if (mask[i]) present[phi[i]] = 1;
}

// ---------------------------------------------------------------------------
// constitutive laws (src/gpk_thermo.cpp:9-47, include/gpk_thermo.hpp)
// ---------------------------------------------------------------------------
struct ThermoDev {
    gpk_thermo_desc t;
    float log_pH2;   // ReductionThermo: logf(pH2_over_pH2O), formed on the host
    float mu0;       // ThermoModel::MU0 = 4.0e-7f * pi (float)
};

template <typename real> __device__ __forceinline__ real dev_pi();
template <> __device__ __forceinline__ float dev_pi<float>() { return 3.14159265358979323846f; }
template <> __device__ __forceinline__ double dev_pi<double>() { return 3.14159265358979323846; }

template <typename real>
__device__ real th_sigma_base(const gpk_thermo_desc& th, real nx, real ny, real nz, real g) {
    if ((real)th.eps4 == (real)0) return (real)th.sigma0;
    const real cg = cos(g), sg = sin(g);
    const real ncx = nx * cg + ny * sg;
    const real ncy = -nx * sg + ny * cg;
    const real ncz = nz;
    real aniso;
    if (ncz == (real)0) aniso = cos((real)4 * atan2(ncy, ncx));
    else aniso = ncx * ncx * ncx * ncx + ncy * ncy * ncy * ncy + ncz * ncz * ncz * ncz - (real)0.6;
    return (real)th.sigma0 * ((real)1 + (real)th.eps4 * aniso);
}

template <typename real>
__device__ real th_sigma(const gpk_thermo_desc& th, real nx, real ny, real nz, real g, int32_t p, int32_t q, real c) {
    switch (th.model) {
    case GPK_MODEL_TENSOR_ANISO:
    case GPK_MODEL_ANISO_OSTWALD: {
        const real cg = cos(g), sg = sin(g);
        const real ncx = nx * cg + ny * sg;
        const real ncy = -nx * sg + ny * cg;
        const real ncz = nz;
        const real K = (real)th.p[0] * ncx * ncx + (real)th.p[1] * ncy * ncy + (real)th.p[2] * ncz * ncz;
        return (real)th.sigma0 * sqrt(dmax(K, (real)1e-12));
    }
    case GPK_MODEL_GROOVING: return (p == 0 || q == 0) ? (real)th.p[1] : (real)th.p[0];
    case GPK_MODEL_NDFEB:
        if (p == 0 || q == 0) {
            const real s0 = (real)th.p[1];
            const real s = s0 * ((real)1 - (real)th.p[2] * c);
            return dclamp(s, (real)0, s0);
        }
        return (real)th.p[0];
    default: return th_sigma_base<real>(th, nx, ny, nz, g);
    }
}

template <typename real>
__device__ real th_mobility(const gpk_thermo_desc& th, real gp, real gq, real T) {
    if (th.model != GPK_MODEL_BASE) return (real)th.M0;
    const real PI = dev_pi<real>();
    real dg = fabs(gp - gq);
    dg = fmod(dg + PI * (real)0.5, PI * (real)0.5);
    if (dg > PI * (real)0.25) dg = PI * (real)0.5 - dg;
    const real theta_m = (real)15 * PI / (real)180;
    real mis;
    if (dg < (real)1e-6) mis = 0;
    else if (dg >= theta_m) mis = 1;
    else { const real frac = dg / theta_m; mis = frac * ((real)1 - log(frac)); }
    const real arr = ((real)th.Q > (real)0) ? exp(-(real)th.Q / ((real)th.Rgas * dmax(T, (real)1))) : (real)1;
    return (real)th.M0 * mis * arr;
}

template <typename real>
__device__ __forceinline__ real th_precip_G(const gpk_thermo_desc& th, int q, real c, real T) {
    return (real)th.p[2 + q] + (real)th.p[10 + q] * c + (real)th.p[18 + q] * c * c + (real)th.p[26 + q] * (T - (real)th.p[1]);
}

template <typename real>
__device__ real th_bulk(const ThermoDev& TD, int32_t p, int32_t q, real c, real T) {
    const gpk_thermo_desc& th = TD.t;
    switch (th.model) {
    case GPK_MODEL_SOLIDIFICATION: {
        const real T_liq = (real)th.p[2] + (real)th.p[0] * c;
        const real dT = T_liq - T;
        const real dG = ((real)th.p[3] / (real)th.p[2]) * dT;
        if (p == 0 && q == 1) return -dG;
        if (p == 1 && q == 0) return +dG;
        return 0;
    }
    case GPK_MODEL_RECRYSTALLISATION: {
        const real E = (real)th.p[0];
        if (p == 0 && q >= 1) return -E;
        if (p >= 1 && q == 0) return +E;
        return 0;
    }
    case GPK_MODEL_OSTWALD:
        if (p == 0) return (real)th.p[1] * ((real)th.p[0] - c);
        if (p >= 1) return (real)th.p[1] * (c - (real)th.p[0]);
        return 0;
    case GPK_MODEL_TENSOR_ANISO: {
        const real bias = (real)th.p[3];
        if (bias == (real)0) return 0;
        return (p != 0) ? bias : -bias;
    }
    case GPK_MODEL_ANISO_OSTWALD:
        if (p == 0) return (real)th.p[4] * ((real)th.p[3] - c);
        return (real)th.p[4] * (c - (real)th.p[3]);
    case GPK_MODEL_PRECIPITATION: {
        const int np = (int)th.p[0];
        if (p < 0 || p >= np || q < 0 || q >= np) return 0;
        return th_precip_G<real>(th, q, c, T) - th_precip_G<real>(th, p, c, T);
    }
    case GPK_MODEL_REDUCTION: {
        const real dG_mol = (real)th.p[1] - (real)8.314 * T * (real)TD.log_pH2;
        const real dG_vol = dG_mol / (real)th.p[2];
        if (p == 0 && q >= 1) return dG_vol;
        if (p >= 1 && q == 0) return -dG_vol;
        return 0;
    }
    case GPK_MODEL_NDFEB:
        if (p != 0) return (real)th.p[4] * ((real)th.p[3] - c);
        return (real)th.p[4] * (c - (real)th.p[3]);
    default: return 0;
    }
}

template <typename real>
__device__ __forceinline__ real th_iface_comp(const gpk_thermo_desc& th, int32_t p, int32_t q, real cp, real cq) {
    if (th.model == GPK_MODEL_OSTWALD || th.model == GPK_MODEL_ANISO_OSTWALD) {
        if (p == 0) return cp;
        if (q == 0) return cq;
    }
    return cp;
}

template <typename real>
__device__ int th_select(const gpk_thermo_desc& th, int32_t p, real c, real T, const int32_t* cand, int n) {
    if (th.model != GPK_MODEL_PRECIPITATION) return -1;
    const int np = (int)th.p[0];
    real best = (real)1e30;
    int best_q = -1;
    for (int k = 0; k < n; ++k) {
        const int32_t q = cand[k];
        if (q < 0 || q >= np || q == p) continue;
        const real dG = th_precip_G<real>(th, q, c, T) - th_precip_G<real>(th, p, c, T);
        if (dG < best) { best = dG; best_q = q; }
    }
    return best_q;
}

template <typename real>
__device__ __forceinline__ real th_Emag(const ThermoDev& TD, real g) {
    const gpk_thermo_desc& th = TD.t;
    if (!th.magnetic_enabled) return 0;
    const real c1 = cos(g - (real)th.g_easy_ref);
    const real c2 = cos(g - (real)th.H_theta);
    return -(real)th.Ku * c1 * c1 - (real)TD.mu0 * (real)th.Ms * (real)th.H_ext * c2;
}

// ---------------------------------------------------------------------------
// velocities (src/gpk_physics.cpp:67-148)
// ---------------------------------------------------------------------------
template <typename real>
__global__ void k_velocities(Dims D, ThermoDev TD, const int32_t* __restrict__ active, const unsigned* __restrict__ n_active,
                             const int32_t* __restrict__ phi, int32_t* __restrict__ phi_comp, const real* __restrict__ c,
                             const real* __restrict__ T, const real* __restrict__ g, const real* __restrict__ rho,
                             const real* __restrict__ nx, const real* __restrict__ ny, const real* __restrict__ nz,
                             const real* __restrict__ kappa, const real* __restrict__ E_el, real* __restrict__ vn,
                             real* __restrict__ g_comp) {
    const gpk_thermo_desc& th = TD.t;
    const int na = (int)*n_active;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < na; a += gridDim.x * blockDim.x) {
        const int i = active[a];
        int nei[6];
        D.faces(i, nei);
        const int32_t pi = phi[i];
        if (th.phase_selection) {
            int32_t cand[6];
            int ncand = 0;
            for (int k = 0; k < 6; ++k) {
                const int32_t q = phi[nei[k]];
                if (q == pi) continue;
                bool seen = false;
                for (int cc = 0; cc < ncand; ++cc)
                    if (cand[cc] == q) { seen = true; break; }
                if (!seen) cand[ncand++] = q;
            }
            const int sel = th_select<real>(th, pi, c[i], T[i], cand, ncand);
            if (sel >= 0) phi_comp[i] = sel;
        }
        const int32_t qid = phi_comp[i];
        const real g_p = g[i];
        real g_q = g_p, c_q = c[i];
        int qk = -1;
        for (int k = 0; k < 6; ++k)
            if (phi[nei[k]] == qid) { qk = nei[k]; break; }
        if (qk >= 0) { g_q = g[qk]; c_q = c[qk]; }
        g_comp[i] = g_q;
        const real c_iface = th_iface_comp<real>(th, pi, qid, c[i], c_q);
        real dG = th_bulk<real>(TD, pi, qid, c_iface, T[i]);
        const real sig = th_sigma<real>(th, nx[i], ny[i], nz[i], g_p, pi, qid, c[i]);
        const real mob = th_mobility<real>(th, g_p, g_q, T[i]);
        if (th.elastic_enabled) {
            const real E_prod = qk >= 0 ? E_el[qk] : E_el[i];
            dG += (E_prod - E_el[i]);
        }
        if (th.dislocation_enabled) {
            const real rho_prod = qk >= 0 ? rho[qk] : rho[i];
            dG += (real)th.disloc_coeff * (rho_prod - rho[i]);
        }
        if (th.magnetic_enabled) dG += th_Emag<real>(TD, g_q) - th_Emag<real>(TD, g_p);
        vn[i] = mob * (dG - sig * kappa[i]);
    }
}

// ---------------------------------------------------------------------------
// pair projection (src/gpk_physics.cpp:152-193): double accumulation,
// weights (double)expf(-r2/(2 s^2)) tabulated on the host by r2.
// ---------------------------------------------------------------------------
template <typename real>
__global__ void k_projection(Dims D, const int32_t* __restrict__ active, const unsigned* __restrict__ n_active,
                             const int32_t* __restrict__ phi, const int32_t* __restrict__ phi_comp,
                             const uint8_t* __restrict__ mask, const real* __restrict__ vn, real* __restrict__ vn_out,
                             const double* __restrict__ wtab, int radius) {
    const int na = (int)*n_active;
    const bool is3d = D.is3d();
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < na; a += gridDim.x * blockDim.x) {
        const int i = active[a];
        const int32_t pi = phi[i], qi = phi_comp[i];
        real out = vn[i];
        if (pi != qi) {
            const int32_t low = min(pi, qi), high = max(pi, qi);
            const real orient_i = pi == low ? (real)1 : (real)-1;
            int z0, y0, x0;
            D.decode(i, z0, y0, x0);
            double num = 0.0, den = 0.0;
            const int dz0 = is3d ? -radius : 0, dz1 = is3d ? radius : 0;
            for (int dz = dz0; dz <= dz1; ++dz) {
                const int z = wrap_any(z0 + dz, D.Nz);
                for (int dy = -radius; dy <= radius; ++dy) {
                    const int y = wrap_any(y0 + dy, D.Ny);
                    for (int dx = -radius; dx <= radius; ++dx) {
                        const int x = wrap_any(x0 + dx, D.Nx);
                        const int j = D.idx(z, y, x);
                        if (!mask[j]) continue;
                        const int32_t pj = phi[j], qj = phi_comp[j];
                        if (pj == qj || min(pj, qj) != low || max(pj, qj) != high) continue;
                        const double w = wtab[dx * dx + dy * dy + dz * dz];
                        const real oj = pj == low ? (real)1 : (real)-1;
                        num += w * (double)oj * (double)vn[j];
                        den += w;
                    }
                }
            }
            if (den > 0.0) out = orient_i * (real)(num / den);
        }
        vn_out[i] = out;
    }
}

// ---------------------------------------------------------------------------
// max_dt (src/gpk_simulation.cpp:11-23)
// ---------------------------------------------------------------------------
template <typename real> struct RealBits;
template <> struct RealBits<float> {
    typedef unsigned int U;
    __device__ static U bits(float v) { return __float_as_uint(v); }
    __device__ static float val(U u) { return __uint_as_float(u); }
};
template <> struct RealBits<double> {
    typedef unsigned long long U;
    __device__ static U bits(double v) { return (U)__double_as_longlong(v); }
    __device__ static double val(U u) { return __longlong_as_double((long long)u); }
};

template <typename real>
__global__ void k_vmax(const int32_t* __restrict__ active, const unsigned* __restrict__ n_active,
                       const real* __restrict__ vn, typename RealBits<real>::U* out) {
    typedef typename RealBits<real>::U U;
    const int na = (int)*n_active;
    real m = (real)0;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < na; a += gridDim.x * blockDim.x)
        m = dmax(m, (real)fabs(vn[active[a]]));
    typedef cub::BlockReduce<U, 256> BR;
    __shared__ typename BR::TempStorage tmp;
    // non-negative reals order like their bit patterns
    const U agg = BR(tmp).Reduce(RealBits<real>::bits(m), cub::Max());
    if (threadIdx.x == 0) atomicMax(out, agg);
}

// dt selection of GPKGrid::step (src/gpk_simulation.cpp:31-37)
template <typename real>
__global__ void k_select_dt(StepScalars* s, const typename RealBits<real>::U* vbits, real dx, real D, int is3d,
                            double dt_req_d, double dt_cap_d) {
    real vmax = (real)1e-30;
    vmax = dmax(vmax, RealBits<real>::val(*vbits));
    const real neighbors = is3d ? (real)6 : (real)4;
    const real dt_iface = (real)0.125 * dx / vmax;
    const real dt_diff = (D > (real)0) ? (real)0.4 * dx * dx / (neighbors * D) : (real)1e30;
    const real dt_stable = dmin(dt_iface, dt_diff);
    real dt = (real)dt_req_d;
    if (dt < (real)0) dt = dt_stable;
    else dt = dmin(dt, dt_stable);
    dt = dmin(dt, (real)dt_cap_d);
    s->dt = (double)dt;
    s->vmax = (double)vmax;
}

// ---------------------------------------------------------------------------
// alpha integration + crossing candidates (src/gpk_transitions.cpp:251-292)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t mix64(uint64_t x) {
    x ^= x >> 30; x *= 0xbf58476d1ce4e5b9ULL;
    x ^= x >> 27; x *= 0x94d049bb133111ebULL;
    x ^= x >> 31;
    return x;
}
template <typename real>
__device__ __forceinline__ real u01_from_u64(uint64_t x) {
    const uint64_t m = (x >> 11) | 1ULL;
    return (real)((double)(m & ((1ULL << 53) - 1)) * (1.0 / (double)(1ULL << 53)));
}
template <typename real>
__device__ __forceinline__ real normal_from_cell_step(int i, uint64_t step_id, uint64_t salt) {
    const uint64_t a = mix64(((uint64_t)i + 0x9e3779b97f4a7c15ULL) ^ (step_id << 1) ^ salt);
    const uint64_t b = mix64(((uint64_t)i + 0xd2b74407b1ce6e93ULL) ^ (step_id << 3) ^ (salt + 17ULL));
    const real u1 = dmax((real)1e-12, u01_from_u64<real>(a));
    const real u2 = u01_from_u64<real>(b);
    return sqrt((real)-2 * log(u1)) * cos((real)2 * dev_pi<real>() * u2);
}

template <typename real>
__global__ void k_alpha(Dims D, const int32_t* __restrict__ active, const unsigned* __restrict__ n_active,
                        const int32_t* __restrict__ phi, const int32_t* __restrict__ phi_comp,
                        const real* __restrict__ vn, const real* __restrict__ T, real* __restrict__ alpha,
                        real* __restrict__ alpha_new_a, uint8_t* __restrict__ cand_flag, StepScalars* s, real dx,
                        int do_noise_flag, real M0, real kB, real noise_scale, uint64_t step_id,
                        real near_tol, int32_t* __restrict__ near_list, int near_cap) {
    const real dt = (real)s->dt;
    const real idt = dt / dx;
    const real cell_vol = dx * dx * dx;
    const real inv_dt = (dt > (real)0) ? ((real)1 / dt) : (real)0;
    const bool do_noise = do_noise_flag && dt > (real)0;
    const real noise_amp = do_noise ? noise_scale * sqrt((real)2 * M0 * kB * inv_dt / dmax(cell_vol, (real)1e-30)) : (real)0;
    const int na = (int)*n_active;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < na; a += gridDim.x * blockDim.x) {
        const int i = active[a];
        real vn_eff = vn[i];
        if (do_noise) vn_eff += noise_amp * sqrt(dmax(T[i], (real)1)) * normal_from_cell_step<real>(i, step_id, 0xabcddcbaULL);
        const real an = dmin(alpha[i] + vn_eff * idt, (real)1);
        alpha_new_a[a] = an;
        const bool other = phi_comp[i] != phi[i];
        const bool cand = an <= (real)1e-6 && other;
        cand_flag[a] = cand ? 1 : 0;
        if (!cand) alpha[i] = an;
        // near-threshold listing: the switching margin an - 1e-6 within
        // near_tol of zero (order restored when the list is read)
        if (other && fabs(an - (real)1e-6) <= near_tol) {
            const unsigned q = atomicAdd(&s->n_near, 1u);
            if (q < (unsigned)near_cap) near_list[q] = i;
        }
    }
}

// crossings without region identity: every candidate is accepted
template <typename real>
__global__ void k_accept_all(const int32_t* __restrict__ active, const int32_t* __restrict__ cpos, int m,
                             int32_t* __restrict__ phi, const int32_t* __restrict__ phi_comp, real* __restrict__ g,
                             const real* __restrict__ g_comp, real* __restrict__ alpha, real* __restrict__ rho,
                             int32_t* __restrict__ count, StepScalars* s, int sweep_rho, real rho_rex) {
    if (m < 0) m = (int)s->n_cand;  // count read on the device (captured step)
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        const int i = active[cpos[k]];
        const int32_t o = phi[i], n = phi_comp[i];
        phi[i] = n;
        g[i] = g_comp[i];
        alpha[i] = (real)1;
        atomicSub(&count[o], 1);
        atomicAdd(&count[n], 1);
        if (sweep_rho) rho[i] = rho_rex;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) s->accepted = (unsigned long long)m;
}

// ---------------------------------------------------------------------------
// elastic proxy (src/gpk_physics.cpp:10-63)
// ---------------------------------------------------------------------------
template <typename real>
__global__ void k_elastic_init(int N, ThermoDev TD, const real* __restrict__ c, const real* __restrict__ g,
                               real* __restrict__ es, real* __restrict__ sm) {
    const gpk_thermo_desc& th = TD.t;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        real eps = (real)th.eigenstrain_coeff * (c[i] - (real)th.c_ref);
        if ((real)th.lambda_s != (real)0) {
            const real cg = cos(g[i] - (real)th.H_theta);
            eps += (real)1.5 * (real)th.lambda_s * (cg * cg - ((real)1 / (real)3));
        }
        es[i] = eps;
        sm[i] = eps;
    }
}
template <typename real>
__global__ void k_elastic_jacobi(Dims D, const real* __restrict__ src, real* __restrict__ dst) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < D.N; i += gridDim.x * blockDim.x) {
        int nb[6];
        D.faces(i, nb);
        real avg = src[nb[0]] + src[nb[1]] + src[nb[2]] + src[nb[3]];
        if (D.Nz > 1) { avg += src[nb[4]] + src[nb[5]]; avg /= (real)6; }
        else avg /= (real)4;
        dst[i] = (real)0.5 * src[i] + (real)0.5 * avg;
    }
}
template <typename real>
__global__ void k_elastic_energy(int N, real E, const real* __restrict__ es, const real* __restrict__ sm, real* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const real d = es[i] - sm[i];
        out[i] = (real)0.5 * E * d * d;
    }
}

// ---------------------------------------------------------------------------
// transport (src/gpk_transport.cpp:11-135) and recovery (:143-152)
// ---------------------------------------------------------------------------
template <typename real>
__global__ void k_diffusion(Dims D, const real* __restrict__ c, real* __restrict__ c_new, const uint8_t* __restrict__ mask,
                            const real* __restrict__ alpha, real Dc, const StepScalars* s, real dx2) {
    const real dt = (real)s->dt;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < D.N; i += gridDim.x * blockDim.x) {
        int nb[6];
        D.faces(i, nb);
        real lap = c[nb[1]] + c[nb[0]] + c[nb[3]] + c[nb[2]];
        if (D.Nz > 1) lap += c[nb[5]] + c[nb[4]] - (real)6 * c[i];
        else lap -= (real)4 * c[i];
        const real D_eff = mask[i] ? Dc * alpha[i] : Dc;
        c_new[i] = c[i] + dt * D_eff * lap / dx2;
    }
}

template <typename real>
__global__ void k_solid_fraction(int N, const int32_t* __restrict__ phi, const real* __restrict__ alpha, real* __restrict__ s) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
        s[i] = (phi[i] != 0) ? alpha[i] : (real)1 - alpha[i];
}

// neighbour order of the transport routines: x+, x-, y+, y-, z+, z-
__device__ __forceinline__ int faces_transport(const Dims& D, int i, int nb[6]) {
    int z, y, x;
    D.decode(i, z, y, x);
    int nn = 0;
    nb[nn++] = D.idx(z, y, x == D.Nx - 1 ? 0 : x + 1);
    nb[nn++] = D.idx(z, y, x == 0 ? D.Nx - 1 : x - 1);
    nb[nn++] = D.idx(z, y == D.Ny - 1 ? 0 : y + 1, x);
    nb[nn++] = D.idx(z, y == 0 ? D.Ny - 1 : y - 1, x);
    if (D.Nz > 1) {
        nb[nn++] = D.idx(z == D.Nz - 1 ? 0 : z + 1, y, x);
        nb[nn++] = D.idx(z == 0 ? D.Nz - 1 : z - 1, y, x);
    }
    return nn;
}

// The rejection of source i (src/gpk_transport.cpp:64-88) with the
// reference's tests in its own form (a NaN passes them as it does there):
// false when i rejects nothing, else its solute q and liquid weight sum.
template <typename real>
__device__ __forceinline__ bool rejection_at(const Dims& D, const int32_t* __restrict__ phi,
                                             const real* __restrict__ c, const real* __restrict__ s_old,
                                             const real* __restrict__ s_new, real k, int i, real& q, real& wsum) {
    const real ds = s_new[i] - s_old[i];
    if (ds <= (real)0) return false;
    const real s0 = dclamp(s_old[i], (real)0, (real)1);
    const real cL = c[i] / dmax((real)1 - s0 * ((real)1 - k), (real)1e-6);
    q = ((real)1 - k) * cL * dmin(ds, (real)1);
    q = dmin(q, c[i]);
    if (q <= (real)0) return false;
    int nb[6];
    const int nn = faces_transport(D, i, nb);
    wsum = 0;
    for (int a = 0; a < nn; ++a) {
        const int j = nb[a];
        const real w = (phi[j] == 0) ? dmax((real)1 - s_new[j], (real)0) : (real)0;
        wsum += w;
    }
    return !(wsum <= (real)0);
}

// c_out = c + delta, delta gathered per cell in the reference's scatter
// order (increasing source index, then neighbour slot; src/gpk_transport.cpp:
// 89-96).  The sources of cell j are j and its face neighbours; a cell none
// of which grew (the common case) only copies c (c + 0).  Out of place: the
// sources' q reads the pre-rejection c of cells that other threads update.
// One block row of 128 x per (y, z): grid (ceil(Nx / 128) * Ny, Nz).
static constexpr int REJ_TPB = 128;

template <typename real>
__global__ void __launch_bounds__(REJ_TPB) k_rejection(Dims D, const int32_t* __restrict__ phi,
                                                       const real* __restrict__ s_old, const real* __restrict__ s_new,
                                                       const uint8_t* __restrict__ grew, real k,
                                                       const real* __restrict__ c, real* __restrict__ c_out) {
    const int Nx = D.Nx, Ny = D.Ny, Nz = D.Nz;
    const int nxb = (Nx + REJ_TPB - 1) / REJ_TPB;
    const int y = blockIdx.x / nxb;
    const int x = (blockIdx.x - y * nxb) * REJ_TPB + threadIdx.x;
    const int z = blockIdx.y;
    if (x >= Nx) return;
    const int j = (z * Ny + y) * Nx + x;
    {
        const int row = j - x, pl = z * Ny * Nx;
        int any = grew[j] | grew[row + (x == Nx - 1 ? 0 : x + 1)] | grew[row + (x == 0 ? Nx - 1 : x - 1)] |
                  grew[pl + (y == Ny - 1 ? 0 : y + 1) * Nx + x] | grew[pl + (y == 0 ? Ny - 1 : y - 1) * Nx + x];
        if (Nz > 1) {
            const int col = y * Nx + x, plane = Ny * Nx;
            any |= grew[(z == Nz - 1 ? 0 : z + 1) * plane + col] | grew[(z == 0 ? Nz - 1 : z - 1) * plane + col];
        }
        const real cj = c[j];
        if (!any) {
            c_out[j] = cj + (real)0;
            return;
        }
    }
    {
        int nbj[6];
        const int nn = faces_transport(D, j, nbj);
        const real cj = c[j];
        int src[7];
        int ns = 0;
        src[ns++] = j;
        for (int a = 0; a < nn; ++a) {
            bool dup = false;
            for (int b = 0; b < ns; ++b) dup |= src[b] == nbj[a];
            if (!dup) src[ns++] = nbj[a];
        }
        for (int a = 1; a < ns; ++a) {  // insertion sort, at most 7 entries
            const int v = src[a];
            int b = a - 1;
            while (b >= 0 && src[b] > v) { src[b + 1] = src[b]; --b; }
            src[b + 1] = v;
        }
        const real wj = (phi[j] == 0) ? dmax((real)1 - s_new[j], (real)0) : (real)0;
        real delta = 0;
        for (int t = 0; t < ns; ++t) {
            const int sidx = src[t];
            real q, wsum;
            if (!rejection_at<real>(D, phi, c, s_old, s_new, k, sidx, q, wsum)) continue;
            if (sidx == j) delta -= q;
            int nbs[6];
            const int ms = faces_transport(D, sidx, nbs);
            for (int a = 0; a < ms; ++a)
                if (nbs[a] == j && wj > (real)0) delta += q * wj / wsum;
        }
        c_out[j] = cj + delta;
    }
}

// s = the solid fraction of the labels; grew = s - s_old passes the
// reference's "ds <= 0 rejects nothing" test (a NaN passes it)
template <typename real>
__global__ void k_solid_fraction_grew(int N, const int32_t* __restrict__ phi, const real* __restrict__ alpha,
                                      const real* __restrict__ s_old, real* __restrict__ s,
                                      uint8_t* __restrict__ grew) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const real sv = (phi[i] != 0) ? alpha[i] : (real)1 - alpha[i];
        s[i] = sv;
        grew[i] = !(sv - s_old[i] <= (real)0);
    }
}

// Partitioned diffusion (src/gpk_transport.cpp:101-135) with the liquid
// composition cL = c / max(1 - s (1 - k), 1e-6) formed as the tile loads c
// and s (each cell once, plus a one-cell ring per plane) instead of being
// stored and re-read.  A 32 x 8 block marches zc planes along z with the
// column's s and cL at z - 1, z, z + 1 in registers and the plane's tile in
// shared memory; each cell's flux sums its faces in the reference's order
// x+, x-, y+, y-, z+, z-.
static constexpr int PDX = 32, PDY = 8;

template <typename real>
__global__ void __launch_bounds__(PDX * PDY) k_diffusion_partitioned_tiled(Dims D, const real* __restrict__ c,
                                                                           const real* __restrict__ s,
                                                                           real* __restrict__ c_new, real Dc, real k,
                                                                           const StepScalars* st, real dx, int zc,
                                                                           real rsk) {
    __shared__ real ts[PDY + 2][PDX + 2];
    __shared__ real tl[PDY + 2][PDX + 2];
    const int Nx = D.Nx, Ny = D.Ny, Nz = D.Nz;
    const real dt = (real)st->dt;
    const real coef = dt * Dc / (dx * dx);
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * PDX + tx;
    const int xs = blockIdx.x * PDX, ys = blockIdx.y * PDY;
    const bool valid = xs + tx < Nx && ys + ty < Ny;
    const int ox = (xs + tx) % Nx, oy = (ys + ty) % Ny;  // own column (wrapped for idle threads)
    const int plane = Ny * Nx;
    const int col = oy * Nx + ox;
    const bool is3 = Nz > 1;
    auto liquid = [&](real cv, real sv) -> real { return cv / dmax((real)1 - sv * ((real)1 - k), (real)1e-6); };
    const int z0 = blockIdx.z * zc;
    const int z1 = z0 + zc < Nz ? z0 + zc : Nz;
    real s_prev = 0, l_prev = 0, s_next = 0, l_next = 0, c_next = 0;
    if (is3) {
        const int zp = z0 == 0 ? Nz - 1 : z0 - 1;
        s_prev = s[zp * plane + col];
        l_prev = liquid(c[zp * plane + col], s_prev);
    }
    real c_cur = c[z0 * plane + col];
    real s_cur = s[z0 * plane + col];
    real l_cur = liquid(c_cur, s_cur);
    for (int z = z0; z < z1; ++z) {
        if (is3) {
            const int zn = z + 1 == Nz ? 0 : z + 1;
            c_next = c[zn * plane + col];
            s_next = s[zn * plane + col];
            l_next = liquid(c_next, s_next);
        }
        ts[ty + 1][tx + 1] = s_cur;
        tl[ty + 1][tx + 1] = l_cur;
        constexpr int HALO = 2 * (PDX + 2) + 2 * PDY;
        for (int h = tid; h < HALO; h += PDX * PDY) {
            int ly, lx;
            if (h < PDX + 2) { ly = -1; lx = h - 1; }
            else if (h < 2 * (PDX + 2)) { ly = PDY; lx = h - (PDX + 2) - 1; }
            else if (h < 2 * (PDX + 2) + PDY) { ly = h - 2 * (PDX + 2); lx = -1; }
            else { ly = h - 2 * (PDX + 2) - PDY; lx = PDX; }
            int gy = ys + ly, gx = xs + lx;
            if (gy < 0) gy += Ny;
            while (gy >= Ny) gy -= Ny;  // at most PDY + 1 times
            if (gx < 0) gx += Nx;
            while (gx >= Nx) gx -= Nx;  // at most PDX + 1 times
            const int q = z * plane + gy * Nx + gx;
            const real sh = s[q];
            ts[ly + 1][lx + 1] = sh;
            tl[ly + 1][lx + 1] = liquid(c[q], sh);
        }
        __syncthreads();
        const real li = (real)1 - s_cur;
        real flux = 0;
        // rsk = (solid/liquid diffusivity ratio) x k: the solid composition
        // k cL diffuses through the face's shared solid fraction; with
        // rsk = 0 this is the reference's liquid-fraction face weight
        auto face = [&](real sj, real lj) {
            const real lf = dmin(li, (real)1 - sj);
            if (rsk > (real)0) {
                const real w = lf + rsk * dmin(s_cur, sj);
                if (w > (real)0) flux += w * (lj - l_cur);
            } else if (lf > (real)0) {
                flux += lf * (lj - l_cur);
            }
        };
        face(ts[ty + 1][tx + 2], tl[ty + 1][tx + 2]);  // x+
        face(ts[ty + 1][tx], tl[ty + 1][tx]);          // x-
        face(ts[ty + 2][tx + 1], tl[ty + 2][tx + 1]);  // y+
        face(ts[ty][tx + 1], tl[ty][tx + 1]);          // y-
        if (is3) {
            face(s_next, l_next);  // z+
            face(s_prev, l_prev);  // z-
        }
        if (valid) c_new[z * plane + col] = c_cur + coef * flux;
        __syncthreads();  // the next plane rewrites the tile
        s_prev = s_cur;
        l_prev = l_cur;
        s_cur = s_next;
        l_cur = l_next;
        c_cur = c_next;
    }
}

template <typename real>
__global__ void k_scale(int N, real* __restrict__ v, real f) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) v[i] *= f;
}

__global__ void k_advance_time(StepScalars* s) { s->time += s->dt; }

__global__ void k_reset_step(StepScalars* s) {
    s->accepted = 0; s->deferred = 0; s->exchanges = 0; s->exch_pass = 0;
    s->n_cand = 0; s->n_prop = 0; s->waves = 0; s->n_near = 0;
}

}  // namespace gpk_dev

using namespace gpk_dev;

template <typename real> int gpk_crossings(gpk_grid* G, int m);
template <typename real> int gpk_remap_pass(gpk_grid* G, const unsigned long long* gate = nullptr);
template <typename real> int gpk_extinction(gpk_grid* G);

static inline int grid_for(gpk_grid* G, long long n, int block = 256) {
    long long b = (n + block - 1) / block;
    long long cap = (long long)G->num_sms * 8;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}

template <typename real>
__global__ void k_indicator(int N, const int32_t* __restrict__ phi, int32_t p, real* __restrict__ I) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
        I[i] = (phi[i] == p) ? (real)1 : (real)0;
}

// Shared memory of one tiled pass (word: bytes per staged value), or 0 when
// its tile does not fit.
static size_t sep_smem_bytes(size_t word, int axis, int R) {
    static int optin = -1;
    if (optin < 0) {
        int dev = 0, v = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
            v = 48 * 1024;
        optin = v;
    }
    const size_t b = word * ((size_t)(2 * R + 2) + 32 * (size_t)sep_pitch(axis, R));
    return b <= (size_t)optin ? b : 0;
}

template <typename real, int AX, bool IND>
static cudaError_t sep_launch(const Dims& D, const real* in, const int32_t* phi, int32_t p, real* out, const real* taps,
                              int R, size_t bytes, cudaStream_t st) {
    const int n = AX == 0 ? D.Nx : (AX == 1 ? D.Ny : D.Nz);
    const int segs = (n + SEP_TL - 1) / SEP_TL;
    if constexpr (sizeof(real) == 4 && AX == 0 && IND) {
        if (bytes > 48 * 1024) {
            const cudaError_t e = cudaFuncSetAttribute(k_sep_x_indicator_f2,
                                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
            if (e != cudaSuccess) return e;
        }
        const long long blocks = (long long)((D.N / n + 63) / 64) * segs;
        k_sep_x_indicator_f2<<<(unsigned)blocks, SEP_TPB, bytes, st>>>(D, phi, p, (float*)out, (const float*)taps, R);
    } else {
        if (bytes > 48 * 1024) {
            const cudaError_t e = cudaFuncSetAttribute(k_sep_pass<real, AX, IND>,
                                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
            if (e != cudaSuccess) return e;
        }
        const long long blocks = (long long)((D.N / n + 31) / 32) * segs;
        k_sep_pass<real, AX, IND><<<(unsigned)blocks, SEP_TPB, bytes, st>>>(D, in, phi, p, out, taps, R);
    }
    return cudaGetLastError();
}

// The periodic Gaussian of in (or, with phi, of the indicator phi == p)
// along x (into t1), y (into t2, or out when 2-D) and, in 3-D, z (into out);
// in may serve as t2, out may not be t1.  Tiled passes where their tiles fit in shared memory, else
// the one-thread-per-output form.  Returns the number of launches, or -1
// with the CUDA error in *err.
template <typename real>
static int sep_gauss3(const Dims& D, const real* in, const int32_t* phi, int32_t p, real* t1, real* t2, real* out,
                      real* ind_scratch, const real* taps, int R, int fallback_grid, cudaStream_t st,
                      cudaError_t* err) {
    // the float indicator pass stages 8-byte row pairs
    const size_t b0 = sep_smem_bytes(phi && sizeof(real) == 4 ? 8 : sizeof(real), 0, R);
    const size_t b1 = sep_smem_bytes(sizeof(real), 1, R), b2 = sep_smem_bytes(sizeof(real), 2, R);
    int launches = 0;
    cudaError_t e = cudaSuccess;
    if (b0 && b1 && b2) {
        e = phi ? sep_launch<real, 0, true>(D, nullptr, phi, p, t1, taps, R, b0, st)
                : sep_launch<real, 0, false>(D, in, nullptr, 0, t1, taps, R, b0, st);
        if (e == cudaSuccess) e = sep_launch<real, 1, false>(D, t1, nullptr, 0, D.Nz > 1 ? t2 : out, taps, R, b1, st);
        launches = 2;
        if (e == cudaSuccess && D.Nz > 1) {
            e = sep_launch<real, 2, false>(D, t2, nullptr, 0, out, taps, R, b2, st);
            ++launches;
        }
    } else {
        if (phi) {
            k_indicator<real><<<fallback_grid, 256, 0, st>>>(D.N, phi, p, ind_scratch);
            in = ind_scratch;
            ++launches;
        }
        k_gauss_pass<real><<<fallback_grid, 256, 0, st>>>(D, in, t1, taps, R, 0);
        k_gauss_pass<real><<<fallback_grid, 256, 0, st>>>(D, t1, D.Nz > 1 ? t2 : out, taps, R, 1);
        launches += 2;
        if (D.Nz > 1) {
            k_gauss_pass<real><<<fallback_grid, 256, 0, st>>>(D, t2, out, taps, R, 2);
            ++launches;
        }
        e = cudaGetLastError();
    }
    *err = e;
    return e == cudaSuccess ? launches : -1;
}

// mask + sorted interface list (src/gpk_geometry.cpp:42-82)
template <typename real>
int gpk_interface_mask(gpk_grid* G, const unsigned long long* gate) {
    const int nt = (G->d.N + MASK_TILE - 1) / MASK_TILE;
    if (G->d.Nx % 4 == 0)
        k_mask_tiles4<<<nt, MASK_TPB, 0, G->stream>>>(G->d, G->phi, G->mask, G->tile_off, gate);
    else
        k_mask_tiles<<<nt, MASK_TPB, 0, G->stream>>>(G->d, G->phi, G->mask, G->tile_off, gate);
    k_scan_tiles<<<1, 1024, 0, G->stream>>>(G->tile_off, nt, &G->scal->n_active, gate);
    k_compact_u8<<<nt, MASK_TPB, 0, G->stream>>>(G->d.N, G->mask, G->tile_off, G->active, gate);
    G->launches += 3;
    GPK_CUDA_TRY(cudaGetLastError());
    return GPK_OK;
}

template <typename real>
static int geometry(gpk_grid* G) {
    HostKernels<real>* hk = (HostKernels<real>*)G->host_kernels;
    const Dims D = G->d;
    const size_t nb = G->rsz * D.N;
    for (int f : {GPK_FIELD_NX, GPK_FIELD_NY, GPK_FIELD_NZ, GPK_FIELD_KAPPA})
        GPK_CUDA_TRY(cudaMemsetAsync(G->f[f], 0, nb, G->stream));
    const real dx = (real)G->dx;
    const real kappa_limit = (real)1 / (hk->gauss_sigma * dx);
    real* nx = (real*)G->f[GPK_FIELD_NX];
    real* ny = (real*)G->f[GPK_FIELD_NY];
    real* nz = (real*)G->f[GPK_FIELD_NZ];
    real* kp = (real*)G->f[GPK_FIELD_KAPPA];
    if (!hk->global_separable) {
        const real inv_dx = (real)1 / dx;
        const real inv_dx2 = inv_dx * inv_dx;
        if constexpr (sizeof(real) == 8) {
            if (G->geometry_kernel == 4) {
                const int rc = gpk_geometry_sep_tiles(G, hk->geom_radius, (const double*)hk->gauss_w.data(),
                                                      hk->gauss_radius, (double)dx, (double)kappa_limit);
                if (rc != -1) return rc;
            }
        }
        if (G->geometry_kernel != 1) {
            const int rc = gpk_geometry_tiled<real>(G, hk->geom_radius, inv_dx, inv_dx2, dx, kappa_limit);
            if (rc != -1) return rc;
        }
        const int grid = G->num_sms * 16;
        if (D.is3d())
            k_geometry_direct<real, true><<<grid, 128, 0, G->stream>>>(D, G->active, &G->scal->n_active, G->phi,
                                                                       (const real*)G->d_geom_table, hk->geom_radius,
                                                                       inv_dx, inv_dx2, dx, kappa_limit, nx, ny, nz, kp,
                                                                       G->phi_comp);
        else
            k_geometry_direct<real, false><<<grid, 128, 0, G->stream>>>(D, G->active, &G->scal->n_active, G->phi,
                                                                        (const real*)G->d_geom_table, hk->geom_radius,
                                                                        inv_dx, inv_dx2, dx, kappa_limit, nx, ny, nz,
                                                                        kp, G->phi_comp);
        G->launches++;
        GPK_CUDA_TRY(cudaGetLastError());
        return GPK_OK;
    }
    // separable path: one smoothed indicator per distinct interface label
    uint8_t* present = G->unres;  // label-indexed scratch
    GPK_CUDA_TRY(cudaMemsetAsync(present, 0, G->label_cap, G->stream));
    k_label_flags<<<grid_for(G, D.N), 256, 0, G->stream>>>(D.N, G->phi, G->mask, present, G->label_cap);
    std::vector<uint8_t> hp(G->label_cap);
    GPK_CUDA_TRY(cudaMemcpyAsync(hp.data(), present, G->label_cap, cudaMemcpyDeviceToHost, G->stream));
    GPK_CUDA_TRY(cudaStreamSynchronize(G->stream));
    const int gN = grid_for(G, D.N);
    for (int p = 0; p < G->label_cap; ++p) {
        if (!hp[p]) continue;
        cudaError_t ce = cudaSuccess;
        const int nl = sep_gauss3<real>(D, nullptr, G->phi, p, (real*)G->sep_t1, (real*)G->sep_t2, (real*)G->sep_S,
                                        (real*)G->sep_I, (const real*)G->d_gauss, hk->gauss_radius, gN, G->stream, &ce);
        GPK_CUDA_TRY(ce);
        k_separable_eval<real><<<gN, 256, 0, G->stream>>>(D, G->active, &G->scal->n_active, G->phi, p,
                                                          (const real*)G->sep_S, dx, kappa_limit, nx, ny, nz, kp);
        G->launches += nl + 1;
    }
    k_competitor_all<real><<<grid_for(G, D.N), 256, 0, G->stream>>>(D, G->active, &G->scal->n_active, G->phi, nx, ny,
                                                                     nz, G->phi_comp);
    G->launches += 2;
    GPK_CUDA_TRY(cudaGetLastError());
    return GPK_OK;
}

static ThermoDev make_thermo_dev(const gpk_thermo_desc& t) {
    ThermoDev TD;
    TD.t = t;
    TD.log_pH2 = (t.model == GPK_MODEL_REDUCTION) ? logf(t.p[0]) : 0.f;
    TD.mu0 = 4.0e-7f * 3.14159265358979323846f;
    return TD;
}

template <typename real>
static int elastic(gpk_grid* G) {
    const gpk_thermo_desc& th = G->th;
    const Dims D = G->d;
    real* E = (real*)G->f[GPK_FIELD_E_EL];
    if (G->external_elastic) return GPK_OK;  // E_el as the caller supplied it
    if (!th.elastic_enabled || (real)th.elastic_modulus <= (real)0 ||
        ((real)th.eigenstrain_coeff == (real)0 && (real)th.lambda_s == (real)0)) {
        GPK_CUDA_TRY(cudaMemsetAsync(E, 0, G->rsz * D.N, G->stream));
        return GPK_OK;
    }
    if (!G->eps_star) {
        GPK_TRY(gpk_alloc(G, &G->eps_star, G->rsz * D.N));
        GPK_TRY(gpk_alloc(G, &G->eps_smooth, G->rsz * D.N));
        GPK_TRY(gpk_alloc(G, &G->eps_tmp, G->rsz * D.N));
    }
    const int gN = grid_for(G, D.N);
    const ThermoDev TD = make_thermo_dev(th);
    k_elastic_init<real><<<gN, 256, 0, G->stream>>>(D.N, TD, (const real*)G->f[GPK_FIELD_C], (const real*)G->f[GPK_FIELD_G],
                                                    (real*)G->eps_star, (real*)G->eps_smooth);
    const int iters = std::max(1, th.elastic_smooth_iters);
    for (int it = 0; it < iters; ++it) {
        k_elastic_jacobi<real><<<gN, 256, 0, G->stream>>>(D, (const real*)G->eps_smooth, (real*)G->eps_tmp);
        std::swap(G->eps_smooth, G->eps_tmp);
    }
    k_elastic_energy<real><<<gN, 256, 0, G->stream>>>(D.N, (real)th.elastic_modulus, (const real*)G->eps_star,
                                                      (const real*)G->eps_smooth, E);
    G->launches += 2 + iters;
    GPK_CUDA_TRY(cudaGetLastError());
    return GPK_OK;
}

template <typename real>
static int transport(gpk_grid* G) {
    const Dims D = G->d;
    const gpk_thermo_desc& th = G->th;
    const real Dc = (real)G->D;
    const real dx = (real)G->dx;
    const int gN = grid_for(G, D.N);
    if (th.solute_rejection) {
        const real k = (real)th.k_partition;
        const bool rejected = k < (real)1 && G->have_solid_old;
        if (!rejected && !(Dc > (real)0)) return GPK_OK;
        if (rejected)
            k_solid_fraction_grew<real><<<gN, 256, 0, G->stream>>>(D.N, G->phi, (const real*)G->f[GPK_FIELD_ALPHA],
                                                                   (const real*)G->solid_old, (real*)G->s_new,
                                                                   G->grew);
        else
            k_solid_fraction<real><<<gN, 256, 0, G->stream>>>(D.N, G->phi, (const real*)G->f[GPK_FIELD_ALPHA],
                                                              (real*)G->s_new);
        G->launches++;
        if (rejected) {
            const dim3 rg((unsigned)(((D.Nx + REJ_TPB - 1) / REJ_TPB) * D.Ny), (unsigned)D.Nz);
            k_rejection<real><<<rg, REJ_TPB, 0, G->stream>>>(D, G->phi, (const real*)G->solid_old,
                                                             (const real*)G->s_new, G->grew, k,
                                                             (const real*)G->f[GPK_FIELD_C], (real*)G->c_new);
            std::swap(G->f[GPK_FIELD_C], G->c_new);
            G->launches++;
        }
        if (Dc > (real)0) {
            // about 16 blocks per SM over the z chunks, at most 16 planes each
            const int bx = (D.Nx + PDX - 1) / PDX, by = (D.Ny + PDY - 1) / PDY;
            long long zc = ((long long)D.Nz * bx * by + G->num_sms * 16 - 1) / ((long long)G->num_sms * 16);
            zc = std::max(1LL, std::min(zc, 16LL));
            const dim3 tg(bx, by, (unsigned)((D.Nz + zc - 1) / zc));
            k_diffusion_partitioned_tiled<real><<<tg, dim3(PDX, PDY), 0, G->stream>>>(
                D, (const real*)G->f[GPK_FIELD_C], (const real*)G->s_new, (real*)G->c_new, Dc, k, G->scal, dx,
                (int)zc, (real)G->solid_ratio * k);
            std::swap(G->f[GPK_FIELD_C], G->c_new);
            G->launches++;
        }
    } else if (Dc > (real)0) {
        k_diffusion<real><<<gN, 256, 0, G->stream>>>(D, (const real*)G->f[GPK_FIELD_C], (real*)G->c_new, G->mask,
                                                     (const real*)G->f[GPK_FIELD_ALPHA], Dc, G->scal, dx * dx);
        std::swap(G->f[GPK_FIELD_C], G->c_new);
        G->launches++;
    }
    GPK_CUDA_TRY(cudaGetLastError());
    return GPK_OK;
}

int gpk_stage_begin(gpk_grid* G, int stage) {
    if (!G->profile) return GPK_OK;
    if (!G->ev[stage][0]) {
        GPK_CUDA_TRY(cudaEventCreate(&G->ev[stage][0]));
        GPK_CUDA_TRY(cudaEventCreate(&G->ev[stage][1]));
    }
    GPK_CUDA_TRY(cudaEventRecord(G->ev[stage][0], G->stream));
    return GPK_OK;
}

int gpk_stage_end(gpk_grid* G, int stage) {
    if (!G->profile) return GPK_OK;
    GPK_CUDA_TRY(cudaEventRecord(G->ev[stage][1], G->stream));
    G->stage_open[stage] = true;
    return GPK_OK;
}

int gpk_stage_collect(gpk_grid* G) {
    if (!G->profile) return GPK_OK;
    for (int k = 0; k < GPK_NUM_STAGES; ++k) {
        if (!G->stage_open[k]) continue;
        GPK_CUDA_TRY(cudaEventSynchronize(G->ev[k][1]));
        float ms = 0.f;
        GPK_CUDA_TRY(cudaEventElapsedTime(&ms, G->ev[k][0], G->ev[k][1]));
        G->stage_ms[k] += ms;
        G->stage_calls[k] += 1;
        G->stage_open[k] = false;
    }
    return GPK_OK;
}

int gpk_sync_scalars(gpk_grid* G) {
    GPK_CUDA_TRY(cudaMemcpyAsync(G->h_scal, G->scal, sizeof(StepScalars), cudaMemcpyDeviceToHost, G->stream));
    GPK_CUDA_TRY(cudaStreamSynchronize(G->stream));
    if (G->h_scal->error) {
        const unsigned e = G->h_scal->error;
        gpk_set_error(e == GPK_ERR_TIMEOUT ? "a bounded device wait gave up" : "device consistency check failed");
        return (int)e;
    }
    return GPK_OK;
}

// GPKGrid::step (src/gpk_simulation.cpp:31-54)
template <typename real>
int gpk_step_impl(gpk_grid* G, double dt_req, double dt_cap) {
    HostKernels<real>* hk = (HostKernels<real>*)G->host_kernels;
    const Dims D = G->d;
    const gpk_thermo_desc& th = G->th;
    const int ga = G->num_sms * 8;
    k_reset_step<<<1, 1, 0, G->stream>>>(G->scal);
    G->launches++;
    // flood-fill stamps: restart before the 32-bit cursor can wrap
    if (G->h_scal->stamp > 0x70000000u) {
        GPK_CUDA_TRY(cudaMemsetAsync(G->stamp, 0, sizeof(uint32_t) * D.N, G->stream));
        GPK_CUDA_TRY(cudaMemsetAsync(G->stamp_rev, 0, sizeof(uint32_t) * D.N, G->stream));
        GPK_CUDA_TRY(cudaMemsetAsync(&G->scal->stamp, 0, sizeof(unsigned), G->stream));
        G->h_scal->stamp = 0;
    }
    GPK_TRY(gpk_stage_begin(G, GPK_STAGE_MASK));
    GPK_TRY(gpk_interface_mask<real>(G));
    GPK_TRY(gpk_stage_end(G, GPK_STAGE_MASK));
    GPK_TRY(gpk_stage_begin(G, GPK_STAGE_GEOMETRY));
    GPK_TRY(geometry<real>(G));
    GPK_TRY(gpk_stage_end(G, GPK_STAGE_GEOMETRY));
    GPK_TRY(gpk_stage_begin(G, GPK_STAGE_VELOCITY));
    GPK_TRY(elastic<real>(G));
    ThermoDev TD = make_thermo_dev(th);
    if (G->external_elastic) TD.t.elastic_enabled = 1;
    GPK_CUDA_TRY(cudaMemsetAsync(G->f[GPK_FIELD_VN], 0, G->rsz * D.N, G->stream));
    k_velocities<real><<<ga, 256, 0, G->stream>>>(
        D, TD, G->active, &G->scal->n_active, G->phi, G->phi_comp, (const real*)G->f[GPK_FIELD_C],
        (const real*)G->f[GPK_FIELD_T], (const real*)G->f[GPK_FIELD_G], (const real*)G->f[GPK_FIELD_RHO],
        (const real*)G->f[GPK_FIELD_NX], (const real*)G->f[GPK_FIELD_NY], (const real*)G->f[GPK_FIELD_NZ],
        (const real*)G->f[GPK_FIELD_KAPPA], (const real*)G->f[GPK_FIELD_E_EL], (real*)G->f[GPK_FIELD_VN],
        (real*)G->f[GPK_FIELD_G_COMP]);
    GPK_TRY(gpk_stage_end(G, GPK_STAGE_VELOCITY));
    // projection into vn2 (zero at bulk cells), then swap
    GPK_TRY(gpk_stage_begin(G, GPK_STAGE_PROJECTION));
    GPK_CUDA_TRY(cudaMemsetAsync(G->vn2, 0, G->rsz * D.N, G->stream));
    const int prc = G->geometry_kernel != 1 ? gpk_projection_tiled<real>(G, hk->proj_radius) : -1;
    if (prc == -1)
        k_projection<real><<<ga, 256, 0, G->stream>>>(D, G->active, &G->scal->n_active, G->phi, G->phi_comp, G->mask,
                                                      (const real*)G->f[GPK_FIELD_VN], (real*)G->vn2, G->d_proj_w,
                                                      hk->proj_radius);
    else if (prc != GPK_OK)
        return prc;
    std::swap(G->f[GPK_FIELD_VN], G->vn2);
    // stable dt
    typedef typename RealBits<real>::U U;
    U* vbits = (U*)&G->scal->vmax;
    GPK_CUDA_TRY(cudaMemsetAsync(vbits, 0, sizeof(double), G->stream));
    k_vmax<real><<<ga, 256, 0, G->stream>>>(G->active, &G->scal->n_active, (const real*)G->f[GPK_FIELD_VN], vbits);
    k_select_dt<real><<<1, 1, 0, G->stream>>>(G->scal, vbits, (real)G->dx, (real)G->D, D.is3d() ? 1 : 0, dt_req, dt_cap);
    G->launches += 4;
    GPK_TRY(gpk_stage_end(G, GPK_STAGE_PROJECTION));
    GPK_TRY(gpk_stage_begin(G, GPK_STAGE_ALPHA));
    if (th.solute_rejection) {
        if (!G->solid_old) {
            GPK_TRY(gpk_alloc(G, &G->solid_old, G->rsz * D.N));
            GPK_TRY(gpk_alloc(G, &G->s_new, G->rsz * D.N));
            GPK_TRY(gpk_alloc(G, (void**)&G->grew, D.N));
        }
        k_solid_fraction<real><<<grid_for(G, D.N), 256, 0, G->stream>>>(D.N, G->phi, (const real*)G->f[GPK_FIELD_ALPHA],
                                                                         (real*)G->solid_old);
        G->have_solid_old = 1;
        G->launches++;
    }
    // alpha integration and candidates
    uint8_t* cflag = (uint8_t*)G->ero_target;  // active-indexed scratch flags
    k_alpha<real><<<ga, 256, 0, G->stream>>>(D, G->active, &G->scal->n_active, G->phi, G->phi_comp,
                                             (const real*)G->f[GPK_FIELD_VN], (const real*)G->f[GPK_FIELD_T],
                                             (real*)G->f[GPK_FIELD_ALPHA], (real*)G->alpha_new_a, cflag, G->scal,
                                             (real)G->dx, th.stochastic, (real)th.M0, (real)th.kB, (real)th.noise_scale,
                                             G->step_id, (real)G->near_tol, G->near_list, D.N);
    const int nt = (D.N + MASK_TILE - 1) / MASK_TILE;
    int32_t* ctile = G->tile_off + nt + 1;
    k_count_u8<<<nt, MASK_TPB, 0, G->stream>>>(cflag, &G->scal->n_active, ctile);
    k_scan_tiles<<<1, 1024, 0, G->stream>>>(ctile, nt, &G->scal->n_cand);
    k_compact_u8_dyn<<<nt, MASK_TPB, 0, G->stream>>>(&G->scal->n_active, cflag, ctile, G->cand);
    G->launches += 4;
    GPK_CUDA_TRY(cudaGetLastError());
    GPK_TRY(gpk_stage_end(G, GPK_STAGE_ALPHA));
    GPK_TRY(gpk_sync_scalars(G));
    const int m = (int)G->h_scal->n_cand;
    GPK_TRY(gpk_stage_begin(G, GPK_STAGE_CROSSINGS));
    if (m > 0) {
        if (th.grain_network) {
            GPK_TRY(gpk_crossings<real>(G, m));
        } else {
            k_accept_all<real><<<grid_for(G, m), 256, 0, G->stream>>>(
                G->active, G->cand, m, G->phi, G->phi_comp, (real*)G->f[GPK_FIELD_G], (const real*)G->f[GPK_FIELD_G_COMP],
                (real*)G->f[GPK_FIELD_ALPHA], (real*)G->f[GPK_FIELD_RHO], G->count, G->scal, th.dislocation_enabled,
                (real)th.rho_rex);
            G->launches++;
        }
        GPK_CUDA_TRY(cudaGetLastError());
        GPK_TRY(gpk_stage_end(G, GPK_STAGE_CROSSINGS));
        GPK_TRY(gpk_sync_scalars(G));
        G->wave_stats[0] += G->h_scal->waves;
        G->wave_stats[2] += (uint64_t)m;
    }
    // balanced Gaussian remap, twice in 3-D when the first pass exchanged
    if (G->h_scal->accepted > 0) {
        GPK_TRY(gpk_stage_begin(G, GPK_STAGE_REMAP));
        GPK_TRY(gpk_interface_mask<real>(G));
        GPK_CUDA_TRY(cudaMemsetAsync(&G->scal->waves, 0, sizeof(unsigned), G->stream));
        GPK_TRY(gpk_remap_pass<real>(G));
        GPK_TRY(gpk_interface_mask<real>(G));
        const bool tiled_scores = G->geometry_kernel != 1 && hk->remap_radius == 3;
        if (D.is3d() && tiled_scores) {
            // the second pass under the device-side gate of the first pass's
            // exchanges (no host round trip between the passes); the pass
            // statistics and the exchange total are formed on the device
            GPK_TRY(gpk_remap_gates(G, 0));
            GPK_TRY(gpk_remap_pass<real>(G, &G->scal->gate2));
            GPK_TRY(gpk_interface_mask<real>(G, &G->scal->gate2));
            GPK_TRY(gpk_remap_gates(G, 1));
        } else if (!D.is3d()) {
            GPK_TRY(gpk_remap_gates(G, 1));
        } else {
            GPK_TRY(gpk_sync_scalars(G));
            G->wave_stats[1] += G->h_scal->waves;
            G->wave_stats[3] += G->h_scal->n_prop;
            const unsigned long long first = G->h_scal->exch_pass;
            unsigned long long total = first;
            if (first > 0) {
                GPK_CUDA_TRY(cudaMemsetAsync(&G->scal->exch_pass, 0, sizeof(unsigned long long), G->stream));
                GPK_CUDA_TRY(cudaMemsetAsync(&G->scal->waves, 0, sizeof(unsigned), G->stream));
                GPK_TRY(gpk_remap_pass<real>(G));
                GPK_TRY(gpk_interface_mask<real>(G));
                GPK_TRY(gpk_sync_scalars(G));
                total += G->h_scal->exch_pass;
                G->wave_stats[1] += G->h_scal->waves;
                G->wave_stats[3] += G->h_scal->n_prop;
            }
            G->h_scal->exchanges = total;
            GPK_CUDA_TRY(cudaMemcpyAsync(&G->scal->exchanges, &G->h_scal->exchanges, sizeof(unsigned long long),
                                         cudaMemcpyHostToDevice, G->stream));
        }
        GPK_TRY(gpk_stage_end(G, GPK_STAGE_REMAP));
    }
    if (th.grain_network && (G->step_id & 7ULL) == 0ULL) {
        GPK_TRY(gpk_stage_begin(G, GPK_STAGE_EXTINCTION));
        GPK_TRY(gpk_extinction<real>(G));
        GPK_TRY(gpk_stage_end(G, GPK_STAGE_EXTINCTION));
    }
    GPK_TRY(gpk_stage_begin(G, GPK_STAGE_TRANSPORT));
    GPK_TRY(transport<real>(G));
    if (th.dislocation_enabled && (real)th.recovery_rate > (real)0) {
        GPK_TRY(gpk_sync_scalars(G));
        const real dt = (real)G->h_scal->dt;
        if (dt > (real)0) {
            const real decay = (sizeof(real) == 4) ? (real)expf(-(float)th.recovery_rate * (float)dt)
                                                   : (real)exp(-(double)th.recovery_rate * (double)dt);
            k_scale<real><<<grid_for(G, D.N), 256, 0, G->stream>>>(D.N, (real*)G->f[GPK_FIELD_RHO], decay);
            G->launches++;
        }
    }
    GPK_TRY(gpk_stage_end(G, GPK_STAGE_TRANSPORT));
    k_advance_time<<<1, 1, 0, G->stream>>>(G->scal);
    G->launches++;
    GPK_CUDA_TRY(cudaGetLastError());
    GPK_TRY(gpk_stage_collect(G));
    ++G->step_id;
    return GPK_OK;
}

template <typename real>
int gpk_max_dt_impl(gpk_grid* G, double* out) {
    // the reference evaluates max_dt on its current interface list and vn_f
    typedef typename RealBits<real>::U U;
    U* vbits = (U*)G->alpha_new_a;  // scratch word
    GPK_CUDA_TRY(cudaMemsetAsync(vbits, 0, sizeof(U), G->stream));
    k_vmax<real><<<G->num_sms * 8, 256, 0, G->stream>>>(G->active, &G->scal->n_active, (const real*)G->f[GPK_FIELD_VN], vbits);
    U h = 0;
    GPK_CUDA_TRY(cudaMemcpyAsync(&h, vbits, sizeof(U), cudaMemcpyDeviceToHost, G->stream));
    GPK_CUDA_TRY(cudaStreamSynchronize(G->stream));
    real v;
    memcpy(&v, &h, sizeof(real));
    real vmax = dmax((real)1e-30, v);
    const real dx = (real)G->dx, Dc = (real)G->D;
    const real neighbors = G->d.is3d() ? (real)6 : (real)4;
    const real dt_iface = (real)0.125 * dx / vmax;
    const real dt_diff = (Dc > (real)0) ? (real)0.4 * dx * dx / (neighbors * Dc) : (real)1e30;
    *out = (double)dmin(dt_iface, dt_diff);
    return GPK_OK;
}

// gaussian_filter_3d (src/gpk_gaussian.cpp:9-72): host buffers in and out,
// the three periodic passes on the device.
extern "C" int gpk_gaussian_filter_3d(const float* in, float* out, int Nz, int Ny, int Nx, const float* taps,
                                      int radius) {
    if (!in || !out || !taps || Nz < 1 || Ny < 1 || Nx < 1 || radius < 0) {
        gpk_set_error("gpk_gaussian_filter_3d: bad arguments");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    const Dims D{Nz, Ny, Nx, Nz * Ny * Nx};
    const size_t nb = sizeof(float) * (size_t)D.N;
    float *a = nullptr, *b = nullptr, *w = nullptr;
    cudaStream_t st = nullptr;
    int rc = GPK_OK;
    auto done = [&](int code) {
        if (st) cudaStreamSynchronize(st);
        cudaFree(a); cudaFree(b); cudaFree(w);
        if (st) cudaStreamDestroy(st);
        return code;
    };
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess || cudaMalloc(&a, nb) != cudaSuccess ||
        cudaMalloc(&b, nb) != cudaSuccess || cudaMalloc(&w, sizeof(float) * (2 * radius + 1)) != cudaSuccess) {
        gpk_set_error("gpk_gaussian_filter_3d: device allocation failed");
        return done(GPK_ERR_OUT_OF_MEMORY);
    }
    const int grid = std::min((D.N + 255) / 256, 148 * 8);
    if (cudaMemcpyAsync(a, in, nb, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(w, taps, sizeof(float) * (2 * radius + 1), cudaMemcpyHostToDevice, st) != cudaSuccess)
        return done(GPK_ERR_CUDA);
    float* res = Nz > 1 ? b : a;
    cudaError_t ce = cudaSuccess;
    sep_gauss3<float>(D, a, nullptr, 0, b, a, res, nullptr, w, radius, grid, st, &ce);
    if (ce != cudaSuccess || cudaMemcpyAsync(out, res, nb, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        gpk_set_error("gpk_gaussian_filter_3d: CUDA failure");
        rc = GPK_ERR_CUDA;
    }
    return done(rc);
}

template int gpk_interface_mask<float>(gpk_grid*, const unsigned long long*);
template int gpk_interface_mask<double>(gpk_grid*, const unsigned long long*);
template int gpk_step_impl<float>(gpk_grid*, double, double);
template int gpk_step_impl<double>(gpk_grid*, double, double);

// ---------------------------------------------------------------------------
// The step as a captured CUDA graph.
//
// gpk_step_impl reads counts back on the host and branches on them (the
// crossing candidates, the remap passes, the extinction schedule).  For the
// configurations below the same kernels in the same order can run with no
// host decision: every launch is sized for the worst case and reads its
// count on the device, the remap stages run under a device-side gate on the
// step's accepted crossings (and, in 3-D, on the first pass's exchanges),
// and the proposals are ordered by one block instead of the radix sorts.
// Results are the step's, bit for bit.  Not covered (gpk_step_graph_supported
// says why): region-identity crossings with topology certificates (the
// ordered sweep's label-wide flood fills size their queues on the host),
// the extinction pass that goes with them, stochastic noise (its step index
// would be frozen into the graph), recovery (its decay is formed on the
// host from the step's dt) and the global-separable geometry (host loop
// over the interface labels).
// ---------------------------------------------------------------------------
int gpk_step_graph_supported(gpk_grid* G, std::string* why) {
    auto no = [&](const char* m) {
        if (why) *why = m;
        return 0;
    };
    const gpk_thermo_desc& th = G->th;
    if (th.grain_network) return no("region-identity crossings (grain_network) need the ordered sweep");
    if (th.stochastic) return no("stochastic noise depends on the step index");
    if (th.dislocation_enabled && th.recovery_rate > 0.f) return no("recovery forms its decay on the host");
    if (G->profile) return no("stage profiling is on");
    if (G->geometry_kernel == 1) return no("the per-cell kernels were selected");
    const bool sep = G->precision == GPK_PREC_F32 ? ((HostKernels<float>*)G->host_kernels)->global_separable
                                                  : ((HostKernels<double>*)G->host_kernels)->global_separable;
    if (sep) return no("the global-separable geometry loops over labels on the host");
    const int rr = G->precision == GPK_PREC_F32 ? ((HostKernels<float>*)G->host_kernels)->remap_radius
                                                : ((HostKernels<double>*)G->host_kernels)->remap_radius;
    if (rr != 3) return no("no tiled remap-score kernel for this remap radius");
    return 1;
}

template <typename real>
int gpk_step_graph_body(gpk_grid* G, double dt_req, double dt_cap) {
    HostKernels<real>* hk = (HostKernels<real>*)G->host_kernels;
    const Dims D = G->d;
    const gpk_thermo_desc& th = G->th;
    // grid-stride launches over at most N items, sized for the grid's cells
    const int ga = (int)std::max(1LL, std::min((long long)G->num_sms * 8, ((long long)D.N + 255) / 256));
    k_reset_step<<<1, 1, 0, G->stream>>>(G->scal);
    G->launches++;
    GPK_TRY(gpk_interface_mask<real>(G));
    GPK_TRY(geometry<real>(G));
    GPK_TRY(elastic<real>(G));
    ThermoDev TD = make_thermo_dev(th);
    if (G->external_elastic) TD.t.elastic_enabled = 1;
    GPK_CUDA_TRY(cudaMemsetAsync(G->f[GPK_FIELD_VN], 0, G->rsz * D.N, G->stream));
    k_velocities<real><<<ga, 256, 0, G->stream>>>(
        D, TD, G->active, &G->scal->n_active, G->phi, G->phi_comp, (const real*)G->f[GPK_FIELD_C],
        (const real*)G->f[GPK_FIELD_T], (const real*)G->f[GPK_FIELD_G], (const real*)G->f[GPK_FIELD_RHO],
        (const real*)G->f[GPK_FIELD_NX], (const real*)G->f[GPK_FIELD_NY], (const real*)G->f[GPK_FIELD_NZ],
        (const real*)G->f[GPK_FIELD_KAPPA], (const real*)G->f[GPK_FIELD_E_EL], (real*)G->f[GPK_FIELD_VN],
        (real*)G->f[GPK_FIELD_G_COMP]);
    GPK_CUDA_TRY(cudaMemsetAsync(G->vn2, 0, G->rsz * D.N, G->stream));
    const int prc = gpk_projection_tiled<real>(G, hk->proj_radius);
    if (prc == -1)
        k_projection<real><<<ga, 256, 0, G->stream>>>(D, G->active, &G->scal->n_active, G->phi, G->phi_comp, G->mask,
                                                      (const real*)G->f[GPK_FIELD_VN], (real*)G->vn2, G->d_proj_w,
                                                      hk->proj_radius);
    else if (prc != GPK_OK)
        return prc;
    std::swap(G->f[GPK_FIELD_VN], G->vn2);
    typedef typename RealBits<real>::U U;
    U* vbits = (U*)&G->scal->vmax;
    GPK_CUDA_TRY(cudaMemsetAsync(vbits, 0, sizeof(double), G->stream));
    k_vmax<real><<<ga, 256, 0, G->stream>>>(G->active, &G->scal->n_active, (const real*)G->f[GPK_FIELD_VN], vbits);
    k_select_dt<real><<<1, 1, 0, G->stream>>>(G->scal, vbits, (real)G->dx, (real)G->D, D.is3d() ? 1 : 0, dt_req, dt_cap);
    G->launches += 4;
    if (th.solute_rejection) {
        if (!G->solid_old) {
            gpk_set_error("captured step: solute buffers are made by a first ordinary step");
            return GPK_ERR_INVALID_ARGUMENT;
        }
        k_solid_fraction<real><<<grid_for(G, D.N), 256, 0, G->stream>>>(D.N, G->phi, (const real*)G->f[GPK_FIELD_ALPHA],
                                                                         (real*)G->solid_old);
        G->have_solid_old = 1;
        G->launches++;
    }
    uint8_t* cflag = (uint8_t*)G->ero_target;
    k_alpha<real><<<ga, 256, 0, G->stream>>>(D, G->active, &G->scal->n_active, G->phi, G->phi_comp,
                                             (const real*)G->f[GPK_FIELD_VN], (const real*)G->f[GPK_FIELD_T],
                                             (real*)G->f[GPK_FIELD_ALPHA], (real*)G->alpha_new_a, cflag, G->scal,
                                             (real)G->dx, th.stochastic, (real)th.M0, (real)th.kB, (real)th.noise_scale,
                                             G->step_id, (real)G->near_tol, G->near_list, D.N);
    const int nt = (D.N + MASK_TILE - 1) / MASK_TILE;
    int32_t* ctile = G->tile_off + nt + 1;
    k_count_u8<<<nt, MASK_TPB, 0, G->stream>>>(cflag, &G->scal->n_active, ctile);
    k_scan_tiles<<<1, 1024, 0, G->stream>>>(ctile, nt, &G->scal->n_cand);
    k_compact_u8_dyn<<<nt, MASK_TPB, 0, G->stream>>>(&G->scal->n_active, cflag, ctile, G->cand);
    // every candidate switches (no region identity); the count is read on the device
    k_accept_all<real><<<ga, 256, 0, G->stream>>>(
        G->active, G->cand, -1, G->phi, G->phi_comp, (real*)G->f[GPK_FIELD_G], (const real*)G->f[GPK_FIELD_G_COMP],
        (real*)G->f[GPK_FIELD_ALPHA], (real*)G->f[GPK_FIELD_RHO], G->count, G->scal, th.dislocation_enabled,
        (real)th.rho_rex);
    G->launches += 5;
    GPK_CUDA_TRY(cudaGetLastError());
    // balanced remap under the accepted-crossings gate; a second 3-D pass
    // under the first pass's exchanges
    const unsigned long long* gate = &G->scal->accepted;
    GPK_TRY(gpk_interface_mask<real>(G, gate));
    GPK_TRY(gpk_remap_pass_graph<real>(G, gate));
    GPK_TRY(gpk_interface_mask<real>(G, gate));
    if (D.is3d()) {
        GPK_TRY(gpk_remap_gates(G, 0));
        GPK_TRY(gpk_remap_pass_graph<real>(G, &G->scal->gate2));
        GPK_TRY(gpk_interface_mask<real>(G, &G->scal->gate2));
    }
    GPK_TRY(gpk_remap_gates(G, 1));
    GPK_TRY(transport<real>(G));
    k_advance_time<<<1, 1, 0, G->stream>>>(G->scal);
    G->launches++;
    GPK_CUDA_TRY(cudaGetLastError());
    ++G->step_id;
    return GPK_OK;
}
template int gpk_step_graph_body<float>(gpk_grid*, double, double);
template int gpk_step_graph_body<double>(gpk_grid*, double, double);

// The mask and geometry stages of GPKGrid::step on the current labels
// (src/gpk_geometry.cpp:42-183), without moving any interface.
template <typename real>
int gpk_geometry_only(gpk_grid* G) {
    GPK_TRY(gpk_interface_mask<real>(G));
    GPK_TRY(geometry<real>(G));
    GPK_CUDA_TRY(cudaStreamSynchronize(G->stream));
    return GPK_OK;
}
template int gpk_geometry_only<float>(gpk_grid*);
template int gpk_geometry_only<double>(gpk_grid*);
template int gpk_max_dt_impl<float>(gpk_grid*, double*);
template int gpk_max_dt_impl<double>(gpk_grid*, double*);

// ---------------------------------------------------------------------------
// Allocation-free separable Gaussian filter.
//
// Some callers cannot call cudaMalloc: processes whose device memory is
// owned up front by another allocator (a framework pool or a fixed budget),
// latency-critical loops that must not allocate, and hosts that only link
// this library without managing device memory themselves.  This entry point
// runs the same three periodic passes as gpk_gaussian_filter_3d on host
// input and output buffers, but its device scratch is the file-scope array
// below instead of cudaMalloc'd buffers, and it creates no stream.
//
//  - The array holds taps plus two fields of at most GPK_NOALLOC_MAX_CELLS
//    floats (16 MiB in all).  Every GPU that loads the library holds it until
//    the process exits.  Larger grids are rejected with
//    GPK_ERR_INVALID_ARGUMENT.
//  - The first call on a device looks up the array's device address with
//    cudaGetSymbolAddress while that device is current; make that first call
//    before any stream capture on the device.
//  - Every call overwrites the part of the array it reads before reading it,
//    so no region has to start at zero; the array keeps the last call's
//    contents.  All calls share the one array: calls in this process are
//    serialised by a mutex, and calls that overlap on the GPU from any other
//    route would race.
// ---------------------------------------------------------------------------
#include <mutex>

static constexpr int NOALLOC_TAP_PAD = 512;  // taps region, a multiple of 64 floats
static __device__ __align__(256) float g_noalloc_scratch[NOALLOC_TAP_PAD + 2 * (size_t)GPK_NOALLOC_MAX_CELLS];

static std::mutex g_noalloc_mutex;
static float* g_noalloc_ptr[64] = {};

extern "C" int gpk_gaussian_filter_3d_noalloc(const float* in, float* out, int Nz, int Ny, int Nx, const float* taps,
                                              int radius) {
    if (!in || !out || !taps || Nz < 1 || Ny < 1 || Nx < 1 || radius < 0) {
        gpk_set_error("gpk_gaussian_filter_3d_noalloc: bad arguments");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    const long long cells = (long long)Nz * Ny * Nx;
    if (cells > GPK_NOALLOC_MAX_CELLS || 2 * radius + 1 > NOALLOC_TAP_PAD) {
        gpk_set_error("gpk_gaussian_filter_3d_noalloc: " + std::to_string(cells) + " cells and " +
                      std::to_string(2 * radius + 1) + " taps exceed the static scratch limits of " +
                      std::to_string(GPK_NOALLOC_MAX_CELLS) + " cells and " + std::to_string(NOALLOC_TAP_PAD) +
                      " taps");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    int dev = 0;
    GPK_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) {
        gpk_set_error("gpk_gaussian_filter_3d_noalloc: device index beyond 63");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    if (!g_noalloc_ptr[dev]) {
        // set-up, once per device, with that device current
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            gpk_set_error(std::string("gpk_gaussian_filter_3d_noalloc: cudaGetSymbolAddress failed: ") +
                          cudaGetErrorString(e));
            return GPK_ERR_CUDA;
        }
        g_noalloc_ptr[dev] = (float*)p;
    }
    float* w = g_noalloc_ptr[dev];
    float* a = w + NOALLOC_TAP_PAD;
    float* b = a + GPK_NOALLOC_MAX_CELLS;
    const Dims D{Nz, Ny, Nx, (int)cells};
    const size_t nb = sizeof(float) * (size_t)cells;
    GPK_CUDA_TRY(cudaMemcpy(w, taps, sizeof(float) * (2 * radius + 1), cudaMemcpyHostToDevice));
    GPK_CUDA_TRY(cudaMemcpy(a, in, nb, cudaMemcpyHostToDevice));
    const int grid = std::min((D.N + 255) / 256, 148 * 8);
    float* res = Nz > 1 ? b : a;
    cudaError_t ce = cudaSuccess;
    sep_gauss3<float>(D, a, nullptr, 0, b, a, res, nullptr, w, radius, grid, 0, &ce);
    GPK_CUDA_TRY(ce);
    GPK_CUDA_TRY(cudaMemcpy(out, res, nb, cudaMemcpyDeviceToHost));
    return GPK_OK;
}
