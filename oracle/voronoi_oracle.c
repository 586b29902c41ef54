/*
 * voronoi_oracle.c — CPU restatement of the reference driver's periodic
 * Voronoi initial condition (TEST INFRASTRUCTURE ONLY).
 *
 * Follows voronoi_init of albert-hzbn/GPK, demos/gpk.cpp:51-189:
 *   - seed k draws (z, y, x) until the cell is not yet a seed, then one
 *     orientation in [0, pi/2)                                  (:56-71)
 *   - every cell takes the nearest seed under the periodic minimum-image
 *     squared integer distance, the lowest seed index on ties   (:73-90)
 *   - connectivity normalisation: face-connected components found by a
 *     breadth-first search started at each unvisited cell in raster order;
 *     the first largest component of a label stays; every other cell is
 *     attached layer by layer (all decisions of a layer read the state
 *     before it) to the attached face neighbour label with the most
 *     support, the smaller label on ties, taking the orientation of the
 *     first face neighbour (order x-, x+, y-, y+, z-, z+) carrying it
 *                                                               (:92-185)
 * The random stream is not the reference's (libstdc++ mt19937 with its
 * implementation-defined distributions) but splitmix64, the stream
 * gpk_voronoi_init / gpk_grid_voronoi of the library draw from; with a seed
 * list given explicitly (or_voronoi_from_seeds) the construction is the
 * reference's own for those seeds.
 *
 * The nearest-seed search visits buckets of seeds in growing Chebyshev
 * rings and stops once no unvisited bucket can hold a seed at or below the
 * best distance, which gives the brute-force answer of the reference.
 */
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static uint64_t sm_next(uint64_t* s) {
    uint64_t z = (*s += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

/* uniform integer in [0, n) by rejection of the top partial block */
static uint32_t sm_below(uint64_t* s, uint32_t n) {
    const uint64_t lim = (UINT64_MAX / n) * n;
    uint64_t v;
    do { v = sm_next(s); } while (v >= lim);
    return (uint32_t)(v % n);
}

/* Seed cells and orientations in the library's draw order.  Returns 0, or 1
 * on bad arguments. */
int or_voronoi_seeds(int Nz, int Ny, int Nx, int n, uint64_t seed, int* sz, int* sy, int* sx, float* sg) {
    const long long N = (long long)Nz * Ny * Nx;
    if (Nz < 1 || Ny < 1 || Nx < 1 || n <= 0 || n > N) return 1;
    uint8_t* taken = (uint8_t*)calloc((size_t)N, 1);
    if (!taken) return 1;
    uint64_t s = seed;
    for (int k = 0; k < n; ++k) {
        long long lin;
        do {
            sz[k] = (int)sm_below(&s, (uint32_t)Nz);
            sy[k] = (int)sm_below(&s, (uint32_t)Ny);
            sx[k] = (int)sm_below(&s, (uint32_t)Nx);
            lin = ((long long)sz[k] * Ny + sy[k]) * Nx + sx[k];
        } while (taken[lin]);
        taken[lin] = 1;
        sg[k] = (float)((sm_next(&s) >> 40) * (1.0 / 16777216.0)) * (float)(M_PI * 0.5);
    }
    free(taken);
    return 0;
}

static long long per_d(int a, int b, int n) {
    long long d = a > b ? (long long)a - b : (long long)b - a;
    return d < n - d ? d : n - d;
}

/* bucket of coordinate v on an axis of n cells split into nb buckets */
static int bucket_of(int v, int n, int nb) { return (int)(((long long)v * nb) / n); }

/* Labels 1..n (and orientations when g is not null) for the given seeds.
 * Returns 0, 1 on bad arguments, 2 if the normalisation stalls. */
int or_voronoi_from_seeds(int Nz, int Ny, int Nx, int n, const int* sz, const int* sy, const int* sx,
                          const float* sg, int32_t* phi, float* g, int* reassigned) {
    const long long N = (long long)Nz * Ny * Nx;
    if (Nz < 1 || Ny < 1 || Nx < 1 || n <= 0 || n > N || N > INT_MAX) return 1;
    for (int k = 0; k < n; ++k)
        if (sz[k] < 0 || sz[k] >= Nz || sy[k] < 0 || sy[k] >= Ny || sx[k] < 0 || sx[k] >= Nx) return 1;
    /* about one seed per bucket; every bucket spans at least smin cells */
    const double per = (double)N / n;
    const int target = (int)(Nz > 1 ? cbrt(per) : sqrt(per));
    const int side = target < 1 ? 1 : target;
    const int bz = Nz / side > 0 ? Nz / side : 1, by = Ny / side > 0 ? Ny / side : 1,
              bx = Nx / side > 0 ? Nx / side : 1;
    /* an axis of one bucket never separates a seed from a cell */
    int smin = INT_MAX;
    if (bz > 1 && Nz / bz < smin) smin = Nz / bz;
    if (by > 1 && Ny / by < smin) smin = Ny / by;
    if (bx > 1 && Nx / bx < smin) smin = Nx / bx;
    if (smin == INT_MAX) smin = 1;
    const long long nbk = (long long)bz * by * bx;
    int* head = (int*)malloc(sizeof(int) * (size_t)(nbk + 1));
    int* list = (int*)malloc(sizeof(int) * (size_t)n);
    if (!head || !list) { free(head); free(list); return 1; }
    memset(head, 0, sizeof(int) * (size_t)(nbk + 1));
    for (int k = 0; k < n; ++k) {
        const long long b = ((long long)bucket_of(sz[k], Nz, bz) * by + bucket_of(sy[k], Ny, by)) * bx +
                            bucket_of(sx[k], Nx, bx);
        head[b + 1]++;
    }
    for (long long b = 0; b < nbk; ++b) head[b + 1] += head[b];
    {
        int* fill = (int*)malloc(sizeof(int) * (size_t)nbk);
        memcpy(fill, head, sizeof(int) * (size_t)nbk);
        for (int k = 0; k < n; ++k) {
            const long long b = ((long long)bucket_of(sz[k], Nz, bz) * by + bucket_of(sy[k], Ny, by)) * bx +
                                bucket_of(sx[k], Nx, bx);
            list[fill[b]++] = k;  /* increasing seed index within a bucket */
        }
        free(fill);
    }
    int rmax = bz / 2;
    if (by / 2 > rmax) rmax = by / 2;
    if (bx / 2 > rmax) rmax = bx / 2;
    for (int z = 0; z < Nz; ++z)
        for (int y = 0; y < Ny; ++y)
            for (int x = 0; x < Nx; ++x) {
                const int cz = bucket_of(z, Nz, bz), cy = bucket_of(y, Ny, by), cx = bucket_of(x, Nx, bx);
                long long best_d = LLONG_MAX;
                int best = -1;
                for (int r = 0; r <= rmax; ++r) {
                    /* offsets per axis, each bucket once: |o| <= nb/2, and
                     * +nb/2 dropped for an even count (it is -nb/2) */
                    const int rz = r < bz / 2 ? r : bz / 2, ry = r < by / 2 ? r : by / 2,
                              rx = r < bx / 2 ? r : bx / 2;
                    const int tz = (bz % 2 == 0 && rz == bz / 2) ? rz - 1 : rz;
                    const int ty = (by % 2 == 0 && ry == by / 2) ? ry - 1 : ry;
                    const int tx = (bx % 2 == 0 && rx == bx / 2) ? rx - 1 : rx;
                    for (int oz = -rz; oz <= tz; ++oz) {
                        const int qz = ((cz + oz) % bz + bz) % bz;
                        for (int oy = -ry; oy <= ty; ++oy) {
                            const int qy = ((cy + oy) % by + by) % by;
                            for (int ox = -rx; ox <= tx; ++ox) {
                                /* only the shell of this ring */
                                if (abs(oz) != r && abs(oy) != r && abs(ox) != r) continue;
                                const int qx = ((cx + ox) % bx + bx) % bx;
                                const long long b = ((long long)qz * by + qy) * bx + qx;
                                for (int t = head[b]; t < head[b + 1]; ++t) {
                                    const int k = list[t];
                                    const long long a = per_d(z, sz[k], Nz), c = per_d(y, sy[k], Ny),
                                                    e = per_d(x, sx[k], Nx);
                                    const long long d = a * a + c * c + e * e;
                                    if (d < best_d || (d == best_d && k < best)) { best_d = d; best = k; }
                                }
                            }
                        }
                    }
                    /* a seed beyond ring r is at least r*smin + 1 cells away
                     * along some axis */
                    const long long reach = (long long)r * smin + 1;
                    if (best >= 0 && best_d < reach * reach) break;
                }
                const long long i = ((long long)z * Ny + y) * Nx + x;
                phi[i] = best + 1;
                if (g) g[i] = sg[best];
            }
    free(head);
    free(list);

    /* connectivity normalisation */
    const int nface = Nz > 1 ? 6 : 4;
    int* comp = (int*)malloc(sizeof(int) * (size_t)N);
    int* queue = (int*)malloc(sizeof(int) * (size_t)N);
    long long* csize = (long long*)malloc(sizeof(long long) * (size_t)N);
    int* largest = (int*)malloc(sizeof(int) * (size_t)(n + 1));
    uint8_t* att = (uint8_t*)malloc((size_t)N);
    int* cells = (int*)malloc(sizeof(int) * (size_t)N);
    int32_t* tgt = (int32_t*)malloc(sizeof(int32_t) * (size_t)N);
    float* ori = (float*)malloc(sizeof(float) * (size_t)N);
    int rc = 0;
    if (!comp || !queue || !csize || !largest || !att || !cells || !tgt || !ori) { rc = 1; goto done; }
    for (long long i = 0; i < N; ++i) comp[i] = -1;
    for (int l = 0; l <= n; ++l) largest[l] = -1;
    int ncomp = 0;
    for (int start = 0; start < N; ++start) {
        if (comp[start] >= 0) continue;
        const int32_t lab = phi[start];
        int qh = 0, qt = 0;
        queue[qt++] = start;
        comp[start] = ncomp;
        while (qh < qt) {
            const int cell = queue[qh++];
            const int x = cell % Nx, y = (cell / Nx) % Ny, z = cell / (Nx * Ny);
            int nb[6];
            nb[0] = (z * Ny + y) * Nx + (x == 0 ? Nx - 1 : x - 1);
            nb[1] = (z * Ny + y) * Nx + (x == Nx - 1 ? 0 : x + 1);
            nb[2] = (z * Ny + (y == 0 ? Ny - 1 : y - 1)) * Nx + x;
            nb[3] = (z * Ny + (y == Ny - 1 ? 0 : y + 1)) * Nx + x;
            nb[4] = ((z == 0 ? Nz - 1 : z - 1) * Ny + y) * Nx + x;
            nb[5] = ((z == Nz - 1 ? 0 : z + 1) * Ny + y) * Nx + x;
            for (int f = 0; f < nface; ++f)
                if (comp[nb[f]] < 0 && phi[nb[f]] == lab) { comp[nb[f]] = ncomp; queue[qt++] = nb[f]; }
        }
        csize[ncomp] = qt;
        if (largest[lab] < 0 || qt > csize[largest[lab]]) largest[lab] = ncomp;
        ++ncomp;
    }
    long long n_att = 0;
    for (long long i = 0; i < N; ++i) {
        att[i] = largest[phi[i]] == comp[i];
        n_att += att[i];
    }
    if (reassigned) *reassigned = (int)(N - n_att);
    while (n_att < N) {
        int m = 0;
        for (int cell = 0; cell < N; ++cell) {
            if (att[cell]) continue;
            const int x = cell % Nx, y = (cell / Nx) % Ny, z = cell / (Nx * Ny);
            int nb[6];
            nb[0] = (z * Ny + y) * Nx + (x == 0 ? Nx - 1 : x - 1);
            nb[1] = (z * Ny + y) * Nx + (x == Nx - 1 ? 0 : x + 1);
            nb[2] = (z * Ny + (y == 0 ? Ny - 1 : y - 1)) * Nx + x;
            nb[3] = (z * Ny + (y == Ny - 1 ? 0 : y + 1)) * Nx + x;
            nb[4] = ((z == 0 ? Nz - 1 : z - 1) * Ny + y) * Nx + x;
            nb[5] = ((z == Nz - 1 ? 0 : z + 1) * Ny + y) * Nx + x;
            int32_t lab[6];
            int sup[6], src[6], nl = 0;
            for (int f = 0; f < nface; ++f) {
                if (!att[nb[f]]) continue;
                int q = 0;
                while (q < nl && lab[q] != phi[nb[f]]) ++q;
                if (q == nl) { lab[nl] = phi[nb[f]]; sup[nl] = 0; src[nl] = nb[f]; ++nl; }
                ++sup[q];
            }
            if (nl == 0) continue;
            int b = 0;
            for (int q = 1; q < nl; ++q)
                if (sup[q] > sup[b] || (sup[q] == sup[b] && lab[q] < lab[b])) b = q;
            cells[m] = cell;
            tgt[m] = lab[b];
            ori[m] = g ? g[src[b]] : 0.f;
            ++m;
        }
        if (m == 0) { rc = 2; goto done; }
        for (int k = 0; k < m; ++k) {
            phi[cells[k]] = tgt[k];
            if (g) g[cells[k]] = ori[k];
            att[cells[k]] = 1;
        }
        n_att += m;
    }
done:
    free(comp); free(queue); free(csize); free(largest); free(att); free(cells); free(tgt); free(ori);
    return rc;
}

/* The polycrystal of gpk_voronoi_init: seeds from the library's stream,
 * then the reference's construction. */
int or_voronoi_init(int Nz, int Ny, int Nx, int n, uint64_t seed, int32_t* phi, float* g, int* reassigned) {
    const long long N = (long long)Nz * Ny * Nx;
    if (Nz < 1 || Ny < 1 || Nx < 1 || n <= 0 || n > N) return 1;
    int* s = (int*)malloc(sizeof(int) * 3 * (size_t)n);
    float* sg = (float*)malloc(sizeof(float) * (size_t)n);
    if (!s || !sg) { free(s); free(sg); return 1; }
    int rc = or_voronoi_seeds(Nz, Ny, Nx, n, seed, s, s + n, s + 2 * n, sg);
    if (rc == 0) rc = or_voronoi_from_seeds(Nz, Ny, Nx, n, s, s + n, s + 2 * n, sg, phi, g, reassigned);
    free(s);
    free(sg);
    return rc;
}
