// gpk_init.cpp — host-side initial conditions for the label grid.
//
// gpk_voronoi_init follows the reference driver's voronoi_init
// (demos/gpk.cpp:51-189 of albert-hzbn/GPK): distinct uniformly random seed
// cells, nearest seed under the periodic minimum-image squared distance with
// ties to the lowest seed index, one uniform orientation in [0, pi/2) per
// grain, then a connectivity normalisation that keeps the largest face-
// connected component of every label and attaches the remaining tie cells,
// layer by layer, to the best-supported attached face neighbour.
//
// The random stream is this library's own (splitmix64), not libstdc++'s
// mt19937 + distributions, whose mapping is implementation-defined; parity
// tests feed the same generated buffer to both sides.
#include <stdint.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <queue>
#include <unordered_set>
#include <vector>

#include "../../include/gpk_init.h"

namespace {

struct SplitMix {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9e3779b97f4a7c15ULL);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
        return z ^ (z >> 31);
    }
    // uniform integer in [0, n) without modulo bias
    uint32_t below(uint32_t n) {
        const uint64_t lim = (UINT64_MAX / n) * n;
        uint64_t v;
        do { v = next(); } while (v >= lim);
        return (uint32_t)(v % n);
    }
    float unit_float() { return (float)((next() >> 40) * (1.0 / 16777216.0)); }
};

inline long long pdist(int a, int b, int n) {
    long long d = std::llabs((long long)a - b);
    return std::min(d, (long long)n - d);
}

}  // namespace

extern "C" int gpk_voronoi_init(int Nz, int Ny, int Nx, int n_seeds, uint64_t seed, int32_t* phi, float* g,
                                int* reassigned) {
    const long long N = (long long)Nz * Ny * Nx;
    if (Nz < 1 || Ny < 1 || Nx < 1 || n_seeds <= 0 || n_seeds > N || !phi) return 1;
    SplitMix rng{seed};
    std::vector<int> sz(n_seeds), sy(n_seeds), sx(n_seeds);
    std::vector<float> sg(n_seeds);
    std::unordered_set<long long> used;
    used.reserve(2 * (size_t)n_seeds);
    for (int k = 0; k < n_seeds; ++k) {
        long long lin;
        do {
            sz[k] = (int)rng.below((uint32_t)Nz);
            sy[k] = (int)rng.below((uint32_t)Ny);
            sx[k] = (int)rng.below((uint32_t)Nx);
            lin = ((long long)sz[k] * Ny + sy[k]) * Nx + sx[k];
        } while (!used.insert(lin).second);
        sg[k] = rng.unit_float() * (float)(M_PI * 0.5);
    }
    // bucketed exact nearest-seed search
    const double cell_vol = (double)N / n_seeds;
    const int bs = std::max(1, (int)std::ceil(std::cbrt(cell_vol) * (Nz > 1 ? 1.0 : 0.0) +
                                              std::sqrt(cell_vol) * (Nz > 1 ? 0.0 : 1.0)));
    const int bz = std::max(1, (Nz + bs - 1) / bs), by = std::max(1, (Ny + bs - 1) / bs), bx = std::max(1, (Nx + bs - 1) / bs);
    std::vector<std::vector<int>> bucket((size_t)bz * by * bx);
    for (int k = 0; k < n_seeds; ++k)
        bucket[((size_t)(sz[k] / bs) * by + sy[k] / bs) * bx + sx[k] / bs].push_back(k);
    const int maxring = std::max(bz / 2, std::max(by / 2, bx / 2));
#pragma omp parallel for schedule(dynamic, 4)
    for (int z = 0; z < Nz; ++z) {
        for (int y = 0; y < Ny; ++y)
            for (int x = 0; x < Nx; ++x) {
                long long best_d = LLONG_MAX;
                int best = 0;
                const int cz = z / bs, cy = y / bs, cx = x / bs;
                for (int r = 0;; ++r) {
                    // visit the shell of buckets at Chebyshev ring r
                    const int rz = std::min(r, bz / 2), ry = std::min(r, by / 2), rx = std::min(r, bx / 2);
                    for (int dz = -rz; dz <= rz; ++dz)
                        for (int dy = -ry; dy <= ry; ++dy)
                            for (int dx = -rx; dx <= rx; ++dx) {
                                if (std::max(std::abs(dz), std::max(std::abs(dy), std::abs(dx))) != r) continue;
                                const int qz = ((cz + dz) % bz + bz) % bz, qy = ((cy + dy) % by + by) % by,
                                          qx = ((cx + dx) % bx + bx) % bx;
                                for (int k : bucket[((size_t)qz * by + qy) * bx + qx]) {
                                    const long long ddz = pdist(z, sz[k], Nz), ddy = pdist(y, sy[k], Ny),
                                                    ddx = pdist(x, sx[k], Nx);
                                    const long long d = ddz * ddz + ddy * ddy + ddx * ddx;
                                    if (d < best_d || (d == best_d && k < best)) { best_d = d; best = k; }
                                }
                            }
                    // every seed outside rings 0..r lies more than (r-1)*bs away along
                    // some axis (one bucket of slack covers a partial last bucket)
                    const long long reach = (long long)(r - 1) * bs;
                    if (r >= maxring || (r >= 1 && best_d < LLONG_MAX && best_d < reach * reach)) break;
                }
                const long long i = ((long long)z * Ny + y) * Nx + x;
                phi[i] = best + 1;
                if (g) g[i] = sg[best];
            }
    }
    // connectivity normalisation (demos/gpk.cpp:100-185)
    auto faces = [&](long long cell, long long out[6]) {
        const int x = (int)(cell % Nx), y = (int)((cell / Nx) % Ny), z = (int)(cell / ((long long)Ny * Nx));
        const int xm = x == 0 ? Nx - 1 : x - 1, xp = x == Nx - 1 ? 0 : x + 1;
        const int ym = y == 0 ? Ny - 1 : y - 1, yp = y == Ny - 1 ? 0 : y + 1;
        const int zm = z == 0 ? Nz - 1 : z - 1, zp = z == Nz - 1 ? 0 : z + 1;
        auto id = [&](int a, int b, int c) { return ((long long)a * Ny + b) * Nx + c; };
        out[0] = id(z, y, xm); out[1] = id(z, y, xp); out[2] = id(z, ym, x);
        out[3] = id(z, yp, x); out[4] = id(zm, y, x); out[5] = id(zp, y, x);
    };
    const int nface = Nz > 1 ? 6 : 4;
    std::vector<int> comp_of(N, -1);
    std::vector<long long> comp_size;
    std::vector<int32_t> comp_label;
    std::vector<int> largest(n_seeds + 1, -1);
    std::vector<long long> frontier;
    for (long long start = 0; start < N; ++start) {
        if (comp_of[start] >= 0) continue;
        const int c = (int)comp_size.size();
        const int32_t label = phi[start];
        long long size = 0;
        frontier.clear();
        frontier.push_back(start);
        comp_of[start] = c;
        for (size_t h = 0; h < frontier.size(); ++h) {
            const long long cell = frontier[h];
            ++size;
            long long nb[6];
            faces(cell, nb);
            for (int k = 0; k < nface; ++k)
                if (comp_of[nb[k]] < 0 && phi[nb[k]] == label) { comp_of[nb[k]] = c; frontier.push_back(nb[k]); }
        }
        comp_size.push_back(size);
        comp_label.push_back(label);
        const int prev = largest[label];
        if (prev < 0 || size > comp_size[prev]) largest[label] = c;
    }
    std::vector<uint8_t> attached(N, 0);
    long long n_att = 0;
    for (long long i = 0; i < N; ++i)
        if (largest[phi[i]] == comp_of[i]) { attached[i] = 1; ++n_att; }
    const long long reassigned_initial = N - n_att;
    std::vector<long long> cells;
    std::vector<int32_t> targets;
    std::vector<float> orient;
    while (n_att < N) {
        cells.clear(); targets.clear(); orient.clear();
        for (long long cell = 0; cell < N; ++cell) {
            if (attached[cell]) continue;
            long long nb[6];
            faces(cell, nb);
            int32_t cand[6]; int support[6] = {0, 0, 0, 0, 0, 0}; long long src[6]; int nc = 0;
            for (int k = 0; k < nface; ++k) {
                if (!attached[nb[k]]) continue;
                const int32_t v = phi[nb[k]];
                int q = 0;
                while (q < nc && cand[q] != v) ++q;
                if (q == nc) { cand[q] = v; src[q] = nb[k]; ++nc; }
                ++support[q];
            }
            if (nc == 0) continue;
            int best = 0;
            for (int q = 1; q < nc; ++q)
                if (support[q] > support[best] || (support[q] == support[best] && cand[q] < cand[best])) best = q;
            cells.push_back(cell); targets.push_back(cand[best]); orient.push_back(g ? g[src[best]] : 0.f);
        }
        if (cells.empty()) return 2;
        for (size_t k = 0; k < cells.size(); ++k) {
            phi[cells[k]] = targets[k];
            if (g) g[cells[k]] = orient[k];
            attached[cells[k]] = 1;
        }
        n_att += (long long)cells.size();
    }
    if (reassigned) *reassigned = (int)reassigned_initial;
    return 0;
}
