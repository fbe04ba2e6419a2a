/*
 * ndb_oracle.c -- CPU oracle for the DBSCAN hot path (TEST INFRASTRUCTURE ONLY).
 *
 * This file is the checker, never the product: only tests/, the smoke check in
 * __graft_entry__.py and the cpu_baseline leg of bench.py load it.  The product
 * path (libndb_b200.so) neither links nor calls anything here.
 *
 * It restates nextdbscan-exa's algorithm (data_process.cpp, data_process.h) in
 * plain C, in two forms that must agree bit for bit:
 *
 *   ndb_oracle_reference  literal O(n^2) restatement of the reference's phases:
 *                         neighbour counting (data_process.cpp:395-458), core
 *                         selection (:268-332), cluster seeding (:93-175),
 *                         label-propagation sweeps (:177-235) and flattening
 *                         (:236-260), and the result meta (:50-91).  Single
 *                         threaded, so each atomic_min of the reference becomes
 *                         a plain min and the sweep order is deterministic.
 *   ndb_oracle_grid       exact restatement of the same OUTPUT semantics with an
 *                         epsilon grid, so that inputs of 10^5..10^6 points can
 *                         be checked in seconds (OpenMP over points).
 *
 * Pinning: both are checked against the real reference, compiled from its own
 * sources by oracle/Makefile into oracle/_ref/, through the fixtures in
 * tests/golden/ (tests/test_oracle.py).
 *
 * Output semantics (identical for both functions, equal to the reference's
 * converged state):
 *   nn[i]            number of points j (i itself included) with
 *                    dist2(i, j) <= e2, where dist2 is the reference's FP32 loop
 *                    (data_process.cpp:443-447: length = 0; length += (a-b)*(a-b)
 *                    per dimension in order, each operation separately rounded)
 *                    and e2 = e*e in float (data_process.h:73).  A point whose
 *                    first coordinate is FLT_MAX is skipped as the "j" side
 *                    (padding test, data_process.cpp:440).
 *   core             nn[i] >= min_pts (data_process.cpp:282).
 *   cluster_index[i] NO_CLUSTER (INT32_MAX, data_process.h:26) for noise;
 *                    for a core, the rank among cores (index order) of the
 *                    smallest-index core in its core-connected component; for a
 *                    border point, the minimum of that value over the cores
 *                    within eps (data_process.cpp:204-209).
 *
 * Build with -ffp-contract=off: the reference's OMP build has no FMA contraction
 * (g++/icc -O3 without -march), so neither may the oracle.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define NDB_ORACLE_NO_CLUSTER INT32_MAX

/* data_process.cpp:443-447 -- the reference's distance predicate, same operation order. */
static inline int in_range(const float *p1, const float *p2, int d, float e2) {
    float length = 0.0f;
    for (int k = 0; k < d; ++k) {
        float t = p1[k] - p2[k];
        length += t * t;
    }
    return length <= e2;
}

/* ------------------------------------------------------------------------- */
/* Literal restatement                                                        */
/* ------------------------------------------------------------------------- */

/*
 * meta[0]=clusters meta[1]=noise meta[2]=cores meta[3]=n meta[4]=propagation sweeps.
 * cluster_label receives v_cluster_label (one entry per core, first meta[2] entries).
 * Returns 0 on success, -1 on allocation failure.
 */
int ndb_oracle_reference(const float *coord, int64_t n, int32_t d, float e, int32_t m,
                         int32_t is_approximate, int32_t *nn, int32_t *cluster_index,
                         int32_t *cluster_label, int32_t *meta) {
    const float e2 = e * e; /* data_process.h:73 */
    const float max_float = FLT_MAX;

    /* select_and_process / process_points (data_process.cpp:334-458): every sample j
     * that is not padding adds one to nn[i] of every i in range. */
    memset(nn, 0, sizeof(int32_t) * (size_t)n);
    for (int64_t j = 0; j < n; ++j) {
        const float *p2 = coord + j * d;
        if (p2[0] == max_float) continue; /* :440 */
        for (int64_t i = 0; i < n; ++i) {
            if (in_range(coord + i * d, p2, d, e2)) nn[i] += 1; /* :447-449 */
        }
    }

    /* select_cores_and_process (:268-283): ascending list of core ids. */
    int64_t n_cores = 0;
    for (int64_t i = 0; i < n; ++i)
        if (nn[i] >= m) ++n_cores;
    int32_t *core_id = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n_cores + 1));
    int32_t *core_cluster_index = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n_cores + 1));
    if (!core_id || !core_cluster_index) {
        free(core_id);
        free(core_cluster_index);
        return -1;
    }
    {
        int64_t c = 0;
        for (int64_t i = 0; i < n; ++i)
            if (nn[i] >= m) core_id[c++] = (int32_t)i;
    }

    /* v_coord_cluster_index.resize(n, NO_CLUSTER) (:291) */
    for (int64_t i = 0; i < n; ++i) cluster_index[i] = NDB_ORACLE_NO_CLUSTER;

    /* process_cores seeding (:105-171): every core starts unlabelled, so every core is a
     * new cluster; the exclusive scan of the marks gives core jj the id jj. */
    for (int64_t jj = 0; jj < n_cores; ++jj) {
        cluster_label[jj] = (int32_t)jj;          /* iota (:151) */
        core_cluster_index[jj] = (int32_t)jj;     /* :164 */
        cluster_index[core_id[jj]] = (int32_t)jj; /* :167 */
    }

    /* propagation sweeps (:183-261) */
    int running = 1;
    int sweeps = 0;
    while (running) {
        running = 0;
        ++sweeps;
        for (int64_t i = 0; i < n; ++i) {
            int keep_running = 0;
            const float *p1 = coord + i * d;
            for (int64_t jj = 0; jj < n_cores; ++jj) {
                const float *p2 = coord + (int64_t)core_id[jj] * d;
                if (p2[0] == max_float) continue; /* :196 */
                if (!in_range(p1, p2, d, e2)) continue;
                int32_t lab_j = cluster_label[core_cluster_index[jj]];
                if (cluster_index[i] == NDB_ORACLE_NO_CLUSTER) { /* :204-205 */
                    if (lab_j < cluster_index[i]) cluster_index[i] = lab_j;
                } else if (nn[i] < m) { /* :206-209 */
                    if (cluster_label[cluster_index[i]] > lab_j && lab_j < cluster_index[i])
                        cluster_index[i] = lab_j;
                } else { /* :210-221 */
                    int32_t lab_i = cluster_label[cluster_index[i]];
                    if (lab_i > lab_j) {
                        if (lab_j < cluster_label[cluster_index[i]])
                            cluster_label[cluster_index[i]] = lab_j;
                    } else if (lab_i < lab_j) {
                        if (!is_approximate) keep_running = 1;
                        if (lab_i < cluster_label[core_cluster_index[jj]])
                            cluster_label[core_cluster_index[jj]] = lab_i;
                    }
                }
            }
            if (keep_running) running = 1; /* :224-227 */
        }
        /* flatten cores (:237-247) */
        for (int64_t jj = 0; jj < n_cores; ++jj) {
            if (core_cluster_index[jj] == NDB_ORACLE_NO_CLUSTER) continue;
            while (cluster_label[core_cluster_index[jj]] != core_cluster_index[jj])
                core_cluster_index[jj] = cluster_label[core_cluster_index[jj]];
        }
        /* flatten coords (:250-260) */
        for (int64_t i = 0; i < n; ++i) {
            if (cluster_index[i] == NDB_ORACLE_NO_CLUSTER) continue;
            while (cluster_label[cluster_index[i]] != cluster_index[i])
                cluster_index[i] = cluster_label[cluster_index[i]];
        }
    }

    /* get_result_meta (:50-91) */
    int64_t noise = 0, clusters = 0;
    for (int64_t i = 0; i < n; ++i)
        if (cluster_index[i] == NDB_ORACLE_NO_CLUSTER) ++noise;
    for (int64_t k = 0; k < n_cores; ++k)
        if (cluster_label[k] == k) ++clusters;
    meta[0] = (int32_t)clusters;
    meta[1] = (int32_t)noise;
    meta[2] = (int32_t)n_cores;
    meta[3] = (int32_t)n;
    meta[4] = sweeps;
    free(core_id);
    free(core_cluster_index);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Grid restatement                                                           */
/* ------------------------------------------------------------------------- */

typedef struct {
    uint64_t key;
    int32_t idx;
} key_idx;

static int cmp_key_idx(const void *a, const void *b) {
    const key_idx *x = (const key_idx *)a, *y = (const key_idx *)b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    return x->idx < y->idx ? -1 : (x->idx > y->idx);
}

/* first position in ki[0..n) whose key >= k */
static int64_t lower_key(const key_idx *ki, int64_t n, uint64_t k) {
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        int64_t mid = (lo + hi) >> 1;
        if (ki[mid].key < k) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

static int32_t uf_find(int32_t *parent, int32_t x) {
    while (parent[x] != x) {
        parent[x] = parent[parent[x]];
        x = parent[x];
    }
    return x;
}

/* A point takes part in the grid iff every coordinate is finite and its first
 * coordinate is not FLT_MAX.  Any other point is never in range of anything when e2
 * is finite: a NaN or infinite coordinate makes one squared difference NaN or inf, and
 * a first coordinate of FLT_MAX is skipped as a sample (data_process.cpp:440) while
 * its difference to every other first coordinate squares to inf. */
static int point_valid(const float *p, int d) {
    if (p[0] == FLT_MAX) return 0;
    for (int k = 0; k < d; ++k)
        if (!isfinite(p[k])) return 0;
    return 1;
}

/*
 * meta[0]=clusters meta[1]=noise meta[2]=cores meta[3]=n.
 * Returns 0 on success, -1 on allocation failure, -2 when e*e is not finite.
 *
 * Exactness of the grid: if the FP32 loop accepts a pair then for every dimension the
 * rounded square of the rounded difference is <= e2, so the real difference is at most
 * r = max(sqrt(e2), 2^-63) * (1 + 2^-20).  Cells are at least r * (1 + 2^-12) wide and
 * are computed in double, so the cell coordinates of any accepted pair differ by at
 * most one in every gridded dimension.
 */
int ndb_oracle_grid(const float *coord, int64_t n, int32_t d, float e, int32_t m,
                    int32_t *nn, int32_t *cluster_index, int32_t *meta) {
    const float e2 = e * e;
    if (!isfinite(e2)) return -2;
    const int kd = d < 2 ? d : 2; /* gridded dimensions: 0 and (if d > 1) 1 */

    uint8_t *valid = (uint8_t *)malloc((size_t)n + 1);
    key_idx *ki = (key_idx *)malloc(sizeof(key_idx) * (size_t)(n + 1));
    int32_t *parent = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n + 1));
    int32_t *rank = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n + 1));
    int32_t *minrank = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n + 1));
    if (!valid || !ki || !parent || !rank || !minrank) {
        free(valid); free(ki); free(parent); free(rank); free(minrank);
        return -1;
    }

    double lo[2] = {0, 0}, hi[2] = {0, 0};
    int any = 0;
    for (int64_t i = 0; i < n; ++i) {
        valid[i] = (uint8_t)point_valid(coord + i * d, d);
        if (!valid[i]) continue;
        for (int k = 0; k < kd; ++k) {
            double v = coord[i * d + k];
            if (!any) {
                lo[k] = hi[k] = v;
            } else {
                if (v < lo[k]) lo[k] = v;
                if (v > hi[k]) hi[k] = v;
            }
        }
        any = 1;
    }
    double r = sqrt((double)e2);
    if (r < ldexp(1.0, -63)) r = ldexp(1.0, -63);
    r *= 1.0 + ldexp(1.0, -20);
    double w[2] = {1, 1};
    int64_t g[2] = {1, 1};
    for (int k = 0; k < kd; ++k) {
        w[k] = r * (1.0 + ldexp(1.0, -12));
        double span = hi[k] - lo[k];
        if (span / w[k] > ldexp(1.0, 24)) w[k] = span / ldexp(1.0, 24);
        g[k] = (int64_t)floor(span / w[k]) + 1;
    }

    int64_t nv = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (!valid[i]) continue;
        uint64_t key = 0, stride = 1;
        for (int k = 0; k < kd; ++k) {
            int64_t c = (int64_t)floor(((double)coord[i * d + k] - lo[k]) / w[k]);
            if (c < 0) c = 0;
            if (c > g[k] - 1) c = g[k] - 1;
            key += (uint64_t)c * stride;
            stride *= (uint64_t)g[k];
        }
        ki[nv].key = key;
        ki[nv].idx = (int32_t)i;
        ++nv;
    }
    qsort(ki, (size_t)nv, sizeof(key_idx), cmp_key_idx);

    /* neighbour counting (data_process.cpp:433-454) over the 3^kd neighbour cells */
    memset(nn, 0, sizeof(int32_t) * (size_t)n);
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t s = 0; s < nv; ++s) {
        const int32_t i = ki[s].idx;
        const float *p1 = coord + (int64_t)i * d;
        int64_t c[2] = {0, 0};
        uint64_t key = ki[s].key;
        c[0] = (int64_t)(key % (uint64_t)g[0]);
        if (kd > 1) c[1] = (int64_t)(key / (uint64_t)g[0]);
        int32_t cnt = 0;
        int64_t y0 = kd > 1 ? c[1] - 1 : 0, y1 = kd > 1 ? c[1] + 1 : 0;
        for (int64_t y = y0; y <= y1; ++y) {
            if (y < 0 || y >= g[1]) continue;
            int64_t x0 = c[0] > 0 ? c[0] - 1 : 0;
            int64_t x1 = c[0] + 1 < g[0] ? c[0] + 1 : g[0] - 1;
            uint64_t klo = (uint64_t)x0 + (uint64_t)y * (uint64_t)g[0];
            uint64_t khi = (uint64_t)x1 + (uint64_t)y * (uint64_t)g[0];
            int64_t a = lower_key(ki, nv, klo), b = lower_key(ki, nv, khi + 1);
            for (int64_t t = a; t < b; ++t)
                if (in_range(p1, coord + (int64_t)ki[t].idx * d, d, e2)) ++cnt;
        }
        nn[i] = cnt;
    }

    /* cores, ranks among cores in index order (data_process.cpp:276-283, :153) */
    int64_t n_cores = 0;
    for (int64_t i = 0; i < n; ++i) {
        rank[i] = (int32_t)n_cores;
        if (nn[i] >= m) ++n_cores;
    }

    /* union-find over core-core pairs (the reference's converged propagation) */
    for (int64_t i = 0; i < n; ++i) parent[i] = (int32_t)i;
    for (int64_t s = 0; s < nv; ++s) {
        const int32_t i = ki[s].idx;
        if (nn[i] < m) continue;
        const float *p1 = coord + (int64_t)i * d;
        uint64_t key = ki[s].key;
        int64_t c0 = (int64_t)(key % (uint64_t)g[0]);
        int64_t c1 = kd > 1 ? (int64_t)(key / (uint64_t)g[0]) : 0;
        int64_t y0 = kd > 1 ? c1 - 1 : 0, y1 = kd > 1 ? c1 + 1 : 0;
        for (int64_t y = y0; y <= y1; ++y) {
            if (y < 0 || y >= g[1]) continue;
            int64_t x0 = c0 > 0 ? c0 - 1 : 0;
            int64_t x1 = c0 + 1 < g[0] ? c0 + 1 : g[0] - 1;
            uint64_t klo = (uint64_t)x0 + (uint64_t)y * (uint64_t)g[0];
            uint64_t khi = (uint64_t)x1 + (uint64_t)y * (uint64_t)g[0];
            int64_t a = lower_key(ki, nv, klo), b = lower_key(ki, nv, khi + 1);
            for (int64_t t = a; t < b; ++t) {
                int32_t j = ki[t].idx;
                if (j <= i || nn[j] < m) continue;
                if (!in_range(p1, coord + (int64_t)j * d, d, e2)) continue;
                int32_t ri = uf_find(parent, i), rj = uf_find(parent, j);
                if (ri == rj) continue;
                if (ri < rj) parent[rj] = ri;
                else parent[ri] = rj;
            }
        }
    }

    /* cluster id of a component = rank of its smallest-index core */
    for (int64_t i = 0; i < n; ++i) minrank[i] = NDB_ORACLE_NO_CLUSTER;
    for (int64_t i = 0; i < n; ++i) {
        if (nn[i] < m) continue;
        int32_t root = uf_find(parent, (int32_t)i);
        if (rank[i] < minrank[root]) minrank[root] = rank[i];
    }
    int64_t clusters = 0;
    for (int64_t i = 0; i < n; ++i) {
        cluster_index[i] = NDB_ORACLE_NO_CLUSTER;
        if (nn[i] >= m) {
            int32_t root = uf_find(parent, (int32_t)i);
            cluster_index[i] = minrank[root];
            if (root == i) ++clusters;
        }
    }

    /* border points: minimum cluster id over the cores in range (data_process.cpp:204-209) */
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t s = 0; s < nv; ++s) {
        const int32_t i = ki[s].idx;
        if (nn[i] >= m) continue;
        const float *p1 = coord + (int64_t)i * d;
        uint64_t key = ki[s].key;
        int64_t c0 = (int64_t)(key % (uint64_t)g[0]);
        int64_t c1 = kd > 1 ? (int64_t)(key / (uint64_t)g[0]) : 0;
        int64_t y0 = kd > 1 ? c1 - 1 : 0, y1 = kd > 1 ? c1 + 1 : 0;
        int32_t best = NDB_ORACLE_NO_CLUSTER;
        for (int64_t y = y0; y <= y1; ++y) {
            if (y < 0 || y >= g[1]) continue;
            int64_t x0 = c0 > 0 ? c0 - 1 : 0;
            int64_t x1 = c0 + 1 < g[0] ? c0 + 1 : g[0] - 1;
            uint64_t klo = (uint64_t)x0 + (uint64_t)y * (uint64_t)g[0];
            uint64_t khi = (uint64_t)x1 + (uint64_t)y * (uint64_t)g[0];
            int64_t a = lower_key(ki, nv, klo), b = lower_key(ki, nv, khi + 1);
            for (int64_t t = a; t < b; ++t) {
                int32_t j = ki[t].idx;
                if (nn[j] < m) continue;
                if (cluster_index[j] >= best) continue;
                if (in_range(p1, coord + (int64_t)j * d, d, e2)) best = cluster_index[j];
            }
        }
        cluster_index[i] = best;
    }

    int64_t noise = 0;
    for (int64_t i = 0; i < n; ++i)
        if (cluster_index[i] == NDB_ORACLE_NO_CLUSTER) ++noise;
    meta[0] = (int32_t)clusters;
    meta[1] = (int32_t)noise;
    meta[2] = (int32_t)n_cores;
    meta[3] = (int32_t)n;
    free(valid); free(ki); free(parent); free(rank); free(minrank);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Cell restatement for large inputs                                          */
/* ------------------------------------------------------------------------- */
/*
 * ndb_oracle_cells computes the same outputs as ndb_oracle_grid for inputs of
 * 10^7..10^8 points, where the grid restatement's serial, pair-by-pair union
 * takes hours on dense clusters.  Differences in organisation only:
 *
 *   - OpenMP in every phase: a parallel LSD radix sort of (cell key, index), a
 *     lock-free union-find (larger root hooked under the smaller by
 *     compare-and-swap), parallel border search;
 *   - neighbour cells found by per-row merge cursors over the sorted cell keys
 *     (the targets of a row only grow as the cells are walked in key order);
 *   - early (optional): a point stops counting once it has min_pts neighbours,
 *     so nn[i] is exact below min_pts and some value >= min_pts otherwise;
 *   - clique cells for d <= 3: cells of width w = sqrt(e2 / d * (1 - 2^-8)).  Two
 *     points of one cell differ by less than w (1 + 2^-20) per dimension, so the
 *     reference's FP32 length is at most d w^2 (1 + 2^-18) < e2: every pair inside
 *     a cell is in range.  A cell's points then count each other without a test,
 *     all cores of a cell are one component (the cell is the union-find element),
 *     and two cells are joined by their first core pair in range.  Neighbour cells
 *     lie within R = ceil(r / w + 2^-18) cells per dimension.
 *   - otherwise an eps grid (cells >= r (1 + 2^-12) wide) on the three widest
 *     dimensions, with point-level unions that skip pairs already joined.
 *
 * The output semantics are the ones stated at the top of this file.
 */
typedef struct {
    uint64_t key;
    int32_t idx;
    int32_t pad;
} kv_t;

#define OC_MAX_ROWS 32 /* rows of a stencil: (2R+1)^(k-1) with R <= 2, k <= 3 */

typedef struct {
    int k;                    /* gridded dimensions */
    int dim[3];               /* which input dimension each one is */
    double lo[3], w[3];       /* origin and cell width */
    int64_t g[3];             /* cells per gridded dimension */
    int R;                    /* stencil reach in cells */
    int clique;               /* 1: every pair inside a cell is in range */
    int n_rows;
    int64_t row_delta[OC_MAX_ROWS]; /* key offset of each row's centre cell */
    int ro1[OC_MAX_ROWS], ro2[OC_MAX_ROWS];
} oc_grid;

static void oc_radix_sort(kv_t *a, kv_t *tmp, int64_t n, int bits, kv_t **out) {
    const int kDigit = 16, kBuckets = 1 << 16;
    int nt_max = 1;
#ifdef _OPENMP
    nt_max = omp_get_max_threads();
#endif
    int64_t *hist = (int64_t *)malloc(sizeof(int64_t) * (size_t)kBuckets * (size_t)nt_max);
    for (int shift = 0; shift < bits; shift += kDigit) {
#pragma omp parallel
        {
            int t = 0, nt = 1;
#ifdef _OPENMP
            t = omp_get_thread_num();
            nt = omp_get_num_threads();
#endif
            const int64_t lo = n * t / nt, hi = n * (t + 1) / nt;
            int64_t *h = hist + (size_t)t * kBuckets;
            memset(h, 0, sizeof(int64_t) * kBuckets);
            for (int64_t i = lo; i < hi; ++i) ++h[(a[i].key >> shift) & 0xffff];
#pragma omp barrier
#pragma omp single
            {
                int64_t run = 0;
                for (int b = 0; b < kBuckets; ++b)
                    for (int q = 0; q < nt; ++q) {
                        const int64_t c = hist[(size_t)q * kBuckets + b];
                        hist[(size_t)q * kBuckets + b] = run;
                        run += c;
                    }
            }
            for (int64_t i = lo; i < hi; ++i) tmp[h[(a[i].key >> shift) & 0xffff]++] = a[i];
        }
        kv_t *x = a;
        a = tmp;
        tmp = x;
    }
    free(hist);
    *out = a;
}

/* first cell index in [from, n_cells) whose key is >= k */
static int64_t oc_lower(const uint64_t *ck, int64_t n_cells, int64_t from, uint64_t k) {
    int64_t lo = from, hi = n_cells;
    while (lo < hi) {
        const int64_t mid = lo + ((hi - lo) >> 1);
        if (ck[mid] < k) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

/* Neighbour cells of cell c, as one [first, last) range of cell indices per row
 * (row[] = which stencil row).  cur[] are the rows' cursors (first cell whose key
 * reaches the row's lowest target); init != 0 places them by binary search.
 * Returns the number of ranges. */
static int oc_rows(const oc_grid *G, const uint64_t *ck, int64_t n_cells, int64_t c, int64_t *cur, int init,
                   int64_t *first, int64_t *last, int *row) {
    const uint64_t key = ck[c];
    int64_t cc[3] = {0, 0, 0};
    uint64_t rest = key;
    for (int a = 0; a < G->k; ++a) {
        if (a < G->k - 1) {
            cc[a] = (int64_t)(rest % (uint64_t)G->g[a]);
            rest /= (uint64_t)G->g[a];
        } else {
            cc[a] = (int64_t)rest;
        }
    }
    const int64_t x0 = cc[0] - G->R < 0 ? 0 : cc[0] - G->R;
    const int64_t x1 = cc[0] + G->R > G->g[0] - 1 ? G->g[0] - 1 : cc[0] + G->R;
    const uint64_t rowbase = key - (uint64_t)cc[0];
    int nr = 0;
    for (int q = 0; q < G->n_rows; ++q) {
        /* The row's lowest target, rowbase + max(x - R, 0) + delta, never decreases
         * as c walks the cells in key order (a later cell of the same x row has a
         * larger x; a later row starts g0 > x - R keys further).  So a cursor placed
         * once per chunk only moves forward.  Targets of rows outside the grid are
         * clamped at 0 and never used. */
        const int64_t tlo_s = (int64_t)rowbase + x0 + G->row_delta[q];
        const uint64_t tlo = tlo_s < 0 ? 0 : (uint64_t)tlo_s;
        const uint64_t thi = (uint64_t)((int64_t)rowbase + x1 + G->row_delta[q]);
        if (init) cur[q] = oc_lower(ck, n_cells, 0, tlo);
        const int64_t y = G->k >= 2 ? cc[1] + G->ro1[q] : 0, z = G->k >= 3 ? cc[2] + G->ro2[q] : 0;
        const int inside = (G->k < 2 || (y >= 0 && y < G->g[1])) && (G->k < 3 || (z >= 0 && z < G->g[2]));
        if (!inside) continue;
        int64_t p = cur[q];
        while (p < n_cells && ck[p] < tlo) ++p;
        cur[q] = p;
        int64_t e = p;
        while (e < n_cells && ck[e] <= thi) ++e;
        if (e > p) {
            first[nr] = p;
            last[nr] = e;
            row[nr] = q;
            ++nr;
        }
    }
    return nr;
}

static int32_t oc_find(int32_t *parent, int32_t x) {
    for (;;) {
        int32_t p = __atomic_load_n(parent + x, __ATOMIC_RELAXED);
        if (p == x) return x;
        const int32_t gp = __atomic_load_n(parent + p, __ATOMIC_RELAXED);
        if (gp != p) __atomic_compare_exchange_n(parent + x, &p, gp, 0, __ATOMIC_RELAXED, __ATOMIC_RELAXED);
        x = gp;
    }
}

static void oc_union(int32_t *parent, int32_t a, int32_t b) {
    for (;;) {
        a = oc_find(parent, a);
        b = oc_find(parent, b);
        if (a == b) return;
        if (a > b) {
            const int32_t t = a;
            a = b;
            b = t;
        }
        int32_t expect = b;
        if (__atomic_compare_exchange_n(parent + b, &expect, a, 0, __ATOMIC_ACQ_REL, __ATOMIC_RELAXED)) return;
    }
}

/*
 * early: 1 = counts stop at min_pts (exact below it).
 * meta[0]=clusters meta[1]=noise meta[2]=cores meta[3]=n meta[4]=1 when clique cells were used.
 * Returns 0 on success, -1 on allocation failure, -2 when e*e is not finite.
 */
int ndb_oracle_cells(const float *coord, int64_t n, int32_t d, float e, int32_t m, int32_t early,
                     int32_t *nn, int32_t *cluster_index, int32_t *meta) {
    const float e2 = e * e; /* data_process.h:73 */
    if (!isfinite(e2)) return -2;
    memset(meta, 0, 8 * sizeof(int32_t));
    uint8_t *valid = (uint8_t *)malloc((size_t)n + 1);
    if (!valid) return -1;
    int64_t nv = 0;
#pragma omp parallel for reduction(+ : nv)
    for (int64_t i = 0; i < n; ++i) {
        valid[i] = (uint8_t)point_valid(coord + i * d, d);
        nv += valid[i];
    }
    /* bounding box of the valid points */
    double lo[16], hi[16];
    for (int k = 0; k < d; ++k) {
        lo[k] = INFINITY;
        hi[k] = -INFINITY;
    }
    for (int64_t i = 0; i < n; ++i) {
        if (!valid[i]) continue;
        for (int k = 0; k < d; ++k) {
            const double v = coord[i * d + k];
            if (v < lo[k]) lo[k] = v;
            if (v > hi[k]) hi[k] = v;
        }
    }
    if (nv == 0)
        for (int k = 0; k < d; ++k) lo[k] = hi[k] = 0.0;

    /* the grid */
    oc_grid G;
    memset(&G, 0, sizeof(G));
    double r = sqrt((double)e2);
    if (r < ldexp(1.0, -63)) r = ldexp(1.0, -63);
    r *= 1.0 + ldexp(1.0, -20);
    const double cap = ldexp(1.0, 20); /* cells per dimension: keys < 2^60, exact in double */
    if (d <= 3 && (double)e2 >= ldexp(1.0, -100)) {
        const double wc = sqrt((double)e2 / d * (1.0 - ldexp(1.0, -8)));
        int fits = wc > 0;
        for (int k = 0; k < d && fits; ++k) fits = (hi[k] - lo[k]) / wc + 2.0 < cap;
        if (fits) {
            G.clique = 1;
            G.k = d;
            for (int k = 0; k < d; ++k) {
                G.dim[k] = k;
                G.w[k] = wc;
            }
            G.R = (int)ceil(r / wc + ldexp(1.0, -18));
        }
    }
    if (!G.clique) {
        G.k = d < 3 ? d : 3;
        /* the k widest dimensions, in input order */
        int used[16] = {0};
        for (int a = 0; a < G.k; ++a) {
            int best = -1;
            for (int k = 0; k < d; ++k)
                if (!used[k] && (best < 0 || hi[k] - lo[k] > hi[best] - lo[best])) best = k;
            used[best] = 1;
        }
        int a = 0;
        for (int k = 0; k < d; ++k)
            if (used[k]) G.dim[a++] = k;
        for (a = 0; a < G.k; ++a) {
            const double span = hi[G.dim[a]] - lo[G.dim[a]];
            G.w[a] = r * (1.0 + ldexp(1.0, -12));
            if (span / G.w[a] + 2.0 >= cap) G.w[a] = span / (cap - 4.0);
        }
        G.R = 1;
    }
    for (int a = 0; a < G.k; ++a) {
        G.lo[a] = lo[G.dim[a]];
        G.g[a] = (int64_t)floor((hi[G.dim[a]] - lo[G.dim[a]]) / G.w[a]) + 1;
    }
    for (int a = G.k; a < 3; ++a) G.g[a] = 1;
    {
        const int r1 = G.k >= 2 ? G.R : 0, r2 = G.k >= 3 ? G.R : 0;
        int q = 0;
        for (int o2 = -r2; o2 <= r2; ++o2)
            for (int o1 = -r1; o1 <= r1; ++o1) {
                G.ro1[q] = o1;
                G.ro2[q] = o2;
                G.row_delta[q] = (int64_t)o1 * G.g[0] + (int64_t)o2 * G.g[0] * G.g[1];
                ++q;
            }
        G.n_rows = q;
    }
    int key_bits = 1;
    {
        double total = (double)G.g[0] * (double)G.g[1] * (double)G.g[2];
        while (key_bits < 64 && ldexp(1.0, key_bits) < total) ++key_bits;
    }

    /* keys, stable sort by (key, index) */
    kv_t *kva = (kv_t *)malloc(sizeof(kv_t) * (size_t)(nv + 1));
    kv_t *kvb = (kv_t *)malloc(sizeof(kv_t) * (size_t)(nv + 1));
    if (!kva || !kvb) {
        free(valid); free(kva); free(kvb);
        return -1;
    }
    {
        int64_t s = 0;
        for (int64_t i = 0; i < n; ++i) {
            if (!valid[i]) continue;
            uint64_t key = 0, stride = 1;
            for (int a = 0; a < G.k; ++a) {
                int64_t c = (int64_t)floor(((double)coord[i * d + G.dim[a]] - G.lo[a]) / G.w[a]);
                if (c < 0) c = 0;
                if (c > G.g[a] - 1) c = G.g[a] - 1;
                key += (uint64_t)c * stride;
                stride *= (uint64_t)G.g[a];
            }
            kva[s].key = key;
            kva[s].idx = (int32_t)i;
            ++s;
        }
    }
    kv_t *sorted = kva;
    oc_radix_sort(kva, kvb, nv, key_bits, &sorted);
    kv_t *spare = sorted == kva ? kvb : kva;

    /* cells, the sorted order and the coordinates in it */
    int32_t *ord = (int32_t *)malloc(sizeof(int32_t) * (size_t)(nv + 1));
    float *xs = (float *)malloc(sizeof(float) * (size_t)(nv * d + 1));
    int64_t n_cells = 0;
    for (int64_t s = 0; s < nv; ++s)
        if (s == 0 || sorted[s].key != sorted[s - 1].key) ++n_cells;
    uint64_t *ck = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(n_cells + 1));
    int64_t *cs = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n_cells + 2));
    uint8_t *core_s = (uint8_t *)malloc((size_t)nv + 1);
    int32_t *rank = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n + 1));
    if (!ord || !xs || !ck || !cs || !core_s || !rank) {
        free(valid); free(kva); free(kvb); free(ord); free(xs); free(ck); free(cs); free(core_s); free(rank);
        return -1;
    }
    {
        int64_t c = 0;
        for (int64_t s = 0; s < nv; ++s) {
            if (s == 0 || sorted[s].key != sorted[s - 1].key) {
                ck[c] = sorted[s].key;
                cs[c] = s;
                ++c;
            }
            ord[s] = sorted[s].idx;
        }
        cs[n_cells] = nv;
    }
    free(spare);
    free(sorted);
#pragma omp parallel for schedule(static)
    for (int64_t s = 0; s < nv; ++s)
        for (int k = 0; k < d; ++k) xs[s * d + k] = coord[(int64_t)ord[s] * d + k];

    /* neighbour counts (data_process.cpp:433-454) */
    memset(nn, 0, sizeof(int32_t) * (size_t)n);
    const int64_t kChunk = 256;
#pragma omp parallel
    {
        int64_t cur[OC_MAX_ROWS], fr[OC_MAX_ROWS], lr[OC_MAX_ROWS];
        int rq[OC_MAX_ROWS];
#pragma omp for schedule(dynamic, 1)
        for (int64_t cb = 0; cb < n_cells; cb += kChunk) {
            const int64_t ce = cb + kChunk < n_cells ? cb + kChunk : n_cells;
            for (int64_t c = cb; c < ce; ++c) {
                const int nr = oc_rows(&G, ck, n_cells, c, cur, c == cb, fr, lr, rq);
                const int64_t a0 = cs[c], a1 = cs[c + 1];
                for (int64_t s = a0; s < a1; ++s) {
                    const float *p1 = xs + s * d;
                    int64_t cnt = 0;
                    if (G.clique) cnt = a1 - a0; /* the whole cell is in range, s included */
                    for (int q = 0; q < nr && !(early && cnt >= m); ++q) {
                        for (int64_t t = cs[fr[q]]; t < cs[lr[q]]; ++t) {
                            if (G.clique && t >= a0 && t < a1) continue;
                            if (in_range(p1, xs + t * d, d, e2)) {
                                ++cnt;
                                if (early && cnt >= m) break;
                            }
                        }
                    }
                    nn[ord[s]] = (int32_t)cnt;
                }
            }
        }
    }

    /* cores and their ranks in index order (data_process.cpp:276-283, :153) */
    int64_t n_cores = 0;
    for (int64_t i = 0; i < n; ++i) {
        rank[i] = (int32_t)n_cores;
        if (nn[i] >= m) ++n_cores;
    }
#pragma omp parallel for schedule(static)
    for (int64_t s = 0; s < nv; ++s) core_s[s] = nn[ord[s]] >= m;

    /* union-find: cells (clique cells) or sorted points */
    const int64_t n_units = G.clique ? n_cells : nv;
    int32_t *parent = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n_units + 1));
    int32_t *cmin = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n_units + 1));
    int32_t *ci_s = (int32_t *)malloc(sizeof(int32_t) * (size_t)(nv + 1));
    uint8_t *cell_core = (uint8_t *)calloc((size_t)n_cells + 1, 1);
    int32_t *cell_cid = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n_cells + 1));
    if (!parent || !cmin || !ci_s || !cell_core || !cell_cid) {
        free(valid); free(ord); free(xs); free(ck); free(cs); free(core_s); free(rank);
        free(parent); free(cmin); free(ci_s); free(cell_core); free(cell_cid);
        return -1;
    }
#pragma omp parallel for schedule(static)
    for (int64_t u = 0; u < n_units; ++u) {
        parent[u] = (int32_t)u;
        cmin[u] = NDB_ORACLE_NO_CLUSTER;
    }
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < n_cells; ++c)
        for (int64_t s = cs[c]; s < cs[c + 1]; ++s)
            if (core_s[s]) {
                cell_core[c] = 1;
                break;
            }
    /* Clique cells are joined in two passes: first the cells at most one cell away
     * in every dimension, then the rest.  Dense regions are connected by the first
     * pass, so the second finds their far pairs already joined; otherwise a far
     * pair of dense cells (at the stencil's corner, where almost no point pair is in
     * range) would be searched pair by pair. */
    for (int pass = 0; pass < (G.clique ? 2 : 1); ++pass)
#pragma omp parallel
    {
        int64_t cur[OC_MAX_ROWS], fr[OC_MAX_ROWS], lr[OC_MAX_ROWS];
        int rq[OC_MAX_ROWS];
#pragma omp for schedule(dynamic, 1)
        for (int64_t cb = 0; cb < n_cells; cb += kChunk) {
            const int64_t ce = cb + kChunk < n_cells ? cb + kChunk : n_cells;
            for (int64_t c = cb; c < ce; ++c) {
                const int nr = oc_rows(&G, ck, n_cells, c, cur, c == cb, fr, lr, rq);
                if (!cell_core[c]) continue;
                const int64_t a0 = cs[c], a1 = cs[c + 1];
                if (G.clique) {
                    const int64_t c0 = (int64_t)(ck[c] % (uint64_t)G.g[0]);
                    for (int q = 0; q < nr; ++q)
                        for (int64_t B = fr[q]; B < lr[q]; ++B) {
                            if (B <= c || !cell_core[B]) continue;
                            const int64_t dx = (int64_t)(ck[B] % (uint64_t)G.g[0]) - c0;
                            const int near = dx >= -1 && dx <= 1 && G.ro1[rq[q]] >= -1 && G.ro1[rq[q]] <= 1 &&
                                             G.ro2[rq[q]] >= -1 && G.ro2[rq[q]] <= 1;
                            if (near != (pass == 0)) continue;
                            if (oc_find(parent, (int32_t)c) == oc_find(parent, (int32_t)B)) continue;
                            int hit = 0;
                            for (int64_t s = a0; s < a1 && !hit; ++s) {
                                if (!core_s[s]) continue;
                                for (int64_t t = cs[B]; t < cs[B + 1]; ++t)
                                    if (core_s[t] && in_range(xs + s * d, xs + t * d, d, e2)) {
                                        hit = 1;
                                        break;
                                    }
                            }
                            if (hit) oc_union(parent, (int32_t)c, (int32_t)B);
                        }
                } else {
                    for (int64_t s = a0; s < a1; ++s) {
                        if (!core_s[s]) continue;
                        for (int q = 0; q < nr; ++q)
                            for (int64_t t = cs[fr[q]]; t < cs[lr[q]]; ++t) {
                                if (t <= s || !core_s[t]) continue;
                                if (oc_find(parent, (int32_t)s) == oc_find(parent, (int32_t)t)) continue;
                                if (in_range(xs + s * d, xs + t * d, d, e2)) oc_union(parent, (int32_t)s, (int32_t)t);
                            }
                    }
                }
            }
        }
    }
    /* component id = rank of the component's smallest-index core */
#pragma omp parallel for schedule(static)
    for (int64_t u = 0; u < n_units; ++u) parent[u] = oc_find(parent, (int32_t)u);
    {
        int64_t c = 0;
        for (int64_t s = 0; s < nv; ++s) {
            while (cs[c + 1] <= s) ++c;
            if (!core_s[s]) continue;
            const int64_t root = parent[G.clique ? c : s];
            const int32_t rk = rank[ord[s]];
            if (rk < cmin[root]) cmin[root] = rk;
        }
    }
    int64_t clusters = 0;
    for (int64_t u = 0; u < n_units; ++u)
        if (parent[u] == u && cmin[u] != NDB_ORACLE_NO_CLUSTER) ++clusters;
    {
        int64_t c = 0;
        for (int64_t s = 0; s < nv; ++s) {
            while (cs[c + 1] <= s) ++c;
            ci_s[s] = core_s[s] ? cmin[parent[G.clique ? c : s]] : NDB_ORACLE_NO_CLUSTER;
            if (core_s[s]) cell_cid[c] = ci_s[s];
        }
        for (c = 0; c < n_cells; ++c)
            if (!cell_core[c]) cell_cid[c] = NDB_ORACLE_NO_CLUSTER;
    }

    /* border points: minimum cluster id over the cores in range (data_process.cpp:204-209) */
#pragma omp parallel
    {
        int64_t cur[OC_MAX_ROWS], fr[OC_MAX_ROWS], lr[OC_MAX_ROWS];
        int rq[OC_MAX_ROWS];
#pragma omp for schedule(dynamic, 1)
        for (int64_t cb = 0; cb < n_cells; cb += kChunk) {
            const int64_t ce = cb + kChunk < n_cells ? cb + kChunk : n_cells;
            for (int64_t c = cb; c < ce; ++c) {
                const int nr = oc_rows(&G, ck, n_cells, c, cur, c == cb, fr, lr, rq);
                for (int64_t s = cs[c]; s < cs[c + 1]; ++s) {
                    if (core_s[s]) continue;
                    int32_t best = NDB_ORACLE_NO_CLUSTER;
                    for (int q = 0; q < nr; ++q)
                        for (int64_t B = fr[q]; B < lr[q]; ++B) {
                            if (!cell_core[B]) continue;
                            if (G.clique && cell_cid[B] >= best) continue;
                            for (int64_t t = cs[B]; t < cs[B + 1]; ++t) {
                                if (!core_s[t] || ci_s[t] >= best) continue;
                                if (in_range(xs + s * d, xs + t * d, d, e2)) {
                                    best = ci_s[t];
                                    if (G.clique) break;
                                }
                            }
                        }
                    ci_s[s] = best;
                }
            }
        }
    }

    int64_t noise = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (valid[i]) continue;
        /* outside the grid: in range of nothing; a core only when min_pts <= 0, then
         * a cluster of its own */
        cluster_index[i] = nn[i] >= m ? rank[i] : NDB_ORACLE_NO_CLUSTER;
        if (nn[i] >= m) ++clusters;
    }
#pragma omp parallel for schedule(static)
    for (int64_t s = 0; s < nv; ++s) cluster_index[ord[s]] = ci_s[s];
    for (int64_t i = 0; i < n; ++i)
        if (cluster_index[i] == NDB_ORACLE_NO_CLUSTER) ++noise;
    meta[0] = (int32_t)clusters;
    meta[1] = (int32_t)noise;
    meta[2] = (int32_t)n_cores;
    meta[3] = (int32_t)n;
    meta[4] = G.clique;
    free(valid); free(ord); free(xs); free(ck); free(cs); free(core_s); free(rank);
    free(parent); free(cmin); free(ci_s); free(cell_core); free(cell_cid);
    return 0;
}

/*
 * ndb_oracle_border_ids -- the border rule (data_process.cpp:204-209) with given
 * core ids: every non-core point takes the minimum of ids[j] over the core points j
 * in range (the reference's FP32 predicate), NO_CLUSTER when there is none; a core
 * keeps ids[i].  Cores are nn[i] >= m.  Brute force over all pairs (small inputs:
 * the checker of the sharded form's border pass).  Returns 0, or -2 when e*e is not
 * finite.
 */
int ndb_oracle_border_ids(const float *coord, int64_t n, int32_t d, float e, int32_t m, const int32_t *nn,
                          const int32_t *ids, int32_t *out) {
    const float e2 = e * e;
    if (!isfinite(e2)) return -2;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < n; ++i) {
        if (nn[i] >= m) {
            out[i] = ids[i];
            continue;
        }
        int32_t best = NDB_ORACLE_NO_CLUSTER;
        const float *p1 = coord + i * d;
        if (point_valid(p1, d)) {
            for (int64_t j = 0; j < n; ++j) {
                if (nn[j] < m || ids[j] >= best) continue;
                if (!point_valid(coord + j * d, d)) continue;
                if (in_range(p1, coord + j * d, d, e2)) best = ids[j];
            }
        }
        out[i] = best;
    }
    return 0;
}

/* Number of OpenMP threads the grid oracle uses (1 without OpenMP). */
int ndb_oracle_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
