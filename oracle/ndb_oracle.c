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

/* Number of OpenMP threads the grid oracle uses (1 without OpenMP). */
int ndb_oracle_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
