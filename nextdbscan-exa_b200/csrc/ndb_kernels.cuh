// ndb_kernels.cuh -- the DBSCAN hot-path kernels (sm_100a), templated on the
// dimensionality D and, for the grid, on the cell-key type K.
//
// Pipeline (one job):
//   bbox      per-dimension min/max of the grid-eligible points        (HBM bound)
//   keys      per-point cell key, invalid points get the all-ones key  (HBM bound)
//   sort      stable LSD radix sort of (key, point id)                  (ndb_prims.cu)
//   cells     cell boundaries, cell keys, point -> cell                 (HBM bound)
//   gather    coordinates in cell order, padded stride                  (HBM bound)
//   rows      per (cell, stencil row): range of neighbour cells         (L2 binary search)
//   count     per-point neighbour count / core flag                     (FP32 pipe)
//   union     core-core connectivity, lock-free union-find              (FP32 pipe + L2 atomics)
//   labels    canonical cluster ids (rank of the smallest core)          (HBM bound)
//   border    border points take the minimum adjacent cluster id        (FP32 pipe)
//
// Replaces data_process::process_points (data_process.cpp:395-458) and
// data_process::process_cores (data_process.cpp:93-266): the reference tests every
// pair of points; here only pairs whose cells are within the stencil are tested,
// with the identical FP32 predicate, so every accepted pair is the same.
#pragma once

#include <float.h>

#include <type_traits>

#include "ndb_common.cuh"

namespace ndb {

// Grid description passed by value to the kernels.
constexpr int kMaxGridDims = 4;

struct GridDev {
    int k;                                  // gridded dimensions (1..4)
    int dim[kMaxGridDims];                  // input dimension of each gridded dimension
    double lo[kMaxGridDims];                // origin per gridded dimension
    double inv_w[kMaxGridDims];             // 1 / cell width
    long long g[kMaxGridDims];              // cells per gridded dimension
    unsigned long long stride[kMaxGridDims];  // key strides (1, g0, g0*g1, g0*g1*g2)
};

// Neighbour rows of a cell.  Row r covers the cells at offsets (x in
// [-xr, +xr], o1, o2, o3) in gridded dimensions (0, 1, 2, 3); those cells have
// consecutive keys, hence form one contiguous run of the sorted cell list.
struct Stencil {
    int n_rows;
    int4 rows[kMaxRows];  // (o1, o2, o3, xr), nearest rows first
};

// Per-job parameters of a batched run (independent DBSCAN jobs concatenated into
// one pipeline).  Kernels take a null table in a single-job run.  Cell keys of
// job j are key_base + the job's own cell key, so jobs never share a cell.
struct JobDev {
    long long off;                 // first point of the job in the concatenated input
    long long n;                   // points of the job
    float e2;                      // eps * eps (FP32)
    int min_pts;
    int list_cap;                  // neighbour-list entries recorded (min_pts - 1, 0 = none)
    int linked;                    // same-cell-linked grid (cell units)
    unsigned long long key_base;   // first composite cell key of the job
    long long col_base;            // first entry of the job's columns in the column table
    GridDev g;
    const float *src;              // the job's coordinates (device), gathered into the batch
    int32_t *nn_out;               // caller's outputs (device; may be null)
    int32_t *ci_out;
};

// job of a point in concatenated input order (jobs sorted by offset)
__device__ __forceinline__ int job_of_point(const JobDev *__restrict__ jobs, int n_jobs, long long o) {
    int lo = 0, hi = n_jobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (jobs[mid].off <= o) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

constexpr int kBlock = 256;
constexpr int kMaxRowCells = 5;
constexpr int kMaxListCap = 64;  // largest min_pts - 1 for which neighbour lists are kept
constexpr int kSmemListCap = 16;  // lists up to this length are staged in shared memory  // cells per stencil row looked up together (2*xr+1 <= 5)
constexpr int kWarpsPerBlock = kBlock / kWarp;
// The count runs two warps per block: an item's candidate list can be thousands of
// points long, and small blocks free their slot as soon as both items are done.
constexpr int kCountWarps = 2;

// ---------------------------------------------------------------------------
// point validity: a point takes part in the grid iff all coordinates are finite
// and its first coordinate is not FLT_MAX.  With a finite e2 any other point is in
// range of nothing: NaN/inf coordinates make a squared difference NaN or inf, and
// FLT_MAX in coordinate 0 is the reference's padding marker
// (data_process.cpp:196, :440) whose distance to any other first coordinate
// squares to inf.
// ---------------------------------------------------------------------------
template <int D>
__device__ __forceinline__ bool point_valid(const float *p) {
    if (p[0] == FLT_MAX) return false;
#pragma unroll
    for (int k = 0; k < D; ++k)
        if (!isfinite(p[k])) return false;
    return true;
}

__device__ __forceinline__ int ordered_int(float f) {
    const int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7fffffff;
}

// Also writes the union-find bound of the run (err[1], see uf_limit).
__global__ void bbox_init_kernel(int *lo_hi, int d, unsigned long long *n_invalid, int *err, int uf_limit) {
    const int t = threadIdx.x;
    if (t < d) {
        lo_hi[t] = 0x7fffffff;
        lo_hi[d + t] = (int)0x80000000;
    }
    if (t == 0) {
        *n_invalid = 0ull;
        err[1] = uf_limit;
    }
}

__global__ void set_int_kernel(int *p, int v) { *p = v; }

// lo_hi[0..D) = ordered-int min, lo_hi[D..2D) = ordered-int max.
template <int D>
__global__ void __launch_bounds__(kBlock) bbox_kernel(const float *__restrict__ coords, int64_t n,
                                                      int *lo_hi, unsigned long long *n_invalid) {
    int lo[D], hi[D];
#pragma unroll
    for (int k = 0; k < D; ++k) {
        lo[k] = 0x7fffffff;
        hi[k] = (int)0x80000000;
    }
    unsigned bad = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float *p = coords + i * D;
        float x[D];
#pragma unroll
        for (int k = 0; k < D; ++k) x[k] = p[k];
        bool ok = x[0] != FLT_MAX;
#pragma unroll
        for (int k = 0; k < D; ++k) ok = ok && isfinite(x[k]);
        if (!ok) {
            ++bad;
            continue;
        }
#pragma unroll
        for (int k = 0; k < D; ++k) {
            const int v = ordered_int(x[k]);
            lo[k] = min(lo[k], v);
            hi[k] = max(hi[k], v);
        }
    }
#pragma unroll
    for (int k = 0; k < D; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            lo[k] = min(lo[k], __shfl_xor_sync(kFull, lo[k], o));
            hi[k] = max(hi[k], __shfl_xor_sync(kFull, hi[k], o));
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) bad += __shfl_xor_sync(kFull, bad, o);
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int k = 0; k < D; ++k) {
            if (lo[k] != 0x7fffffff) atomicMin(lo_hi + k, lo[k]);
            if (hi[k] != (int)0x80000000) atomicMax(lo_hi + D + k, hi[k]);
        }
        if (bad) atomicAdd(n_invalid, (unsigned long long)bad);
    }
}

// Cell coordinate along gridded dimension a.  Computed in double: with at most
// 2^30 cells per dimension the result is within 2^-21 cells of the exact value,
// which the host's stencil and same-cell margins absorb.
__device__ __forceinline__ long long cell_coord(const GridDev &g, int a, float x) {
    const double t = ((double)x - g.lo[a]) * g.inv_w[a];
    long long c = (long long)floor(t);
    c = c < 0 ? 0 : c;
    c = c > g.g[a] - 1 ? g.g[a] - 1 : c;
    return c;
}

template <int D, typename K>
__global__ void __launch_bounds__(kBlock) key_kernel(const float *__restrict__ coords, int64_t n,
                                                     GridDev g, K invalid_key, K *__restrict__ keys,
                                                     int32_t *__restrict__ ids) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *p = coords + i * D;
    K key = invalid_key;
    if (point_valid<D>(p)) {
        unsigned long long kk = 0;
#pragma unroll
        for (int a = 0; a < kMaxGridDims; ++a)
            if (a < g.k) kk += (unsigned long long)cell_coord(g, a, p[g.dim[a]]) * g.stride[a];
        key = (K)kk;
    }
    keys[i] = key;
    ids[i] = (int32_t)i;
}

// pos = exclusive scan of "first point of a cell" flags
template <typename K>
__global__ void cell_flag_kernel(const K *__restrict__ keys, int64_t nv, uint32_t *__restrict__ flags) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nv) return;
    flags[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}

template <typename K>
__global__ void cell_write_kernel(const K *__restrict__ keys, int64_t nv, const uint32_t *__restrict__ pos,
                                  const uint32_t *__restrict__ n_cells_dev, int32_t *__restrict__ cell_start,
                                  K *__restrict__ cell_key, int32_t *__restrict__ pcell) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nv) return;
    const bool first = (i == 0 || keys[i] != keys[i - 1]);
    const uint32_t c = first ? pos[i] : pos[i] - 1;
    if (first) {
        cell_start[c] = (int32_t)i;
        cell_key[c] = keys[i];
    }
    pcell[i] = (int32_t)c;
    if (i == nv - 1) cell_start[*n_cells_dev] = (int32_t)nv;
}

template <int D>
__global__ void __launch_bounds__(kBlock) gather_kernel(const float *__restrict__ coords,
                                                        const int32_t *__restrict__ perm, int64_t nv,
                                                        float *__restrict__ xs) {
    constexpr int P = Stride<D>::P;
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nv) return;
    const float *p = coords + (int64_t)perm[s] * D;
    float v[P];
#pragma unroll
    for (int k = 0; k < P; ++k) v[k] = k < D ? p[k] : 0.0f;
    float *q = xs + s * P;
    if constexpr (P % 4 == 0) {
#pragma unroll
        for (int k = 0; k < P / 4; ++k)
            reinterpret_cast<float4 *>(q)[k] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
    } else if constexpr (P == 2) {
        *reinterpret_cast<float2 *>(q) = make_float2(v[0], v[1]);
    } else {
        q[0] = v[0];
    }
}

// Open-addressing hash table of the non-empty cells: key -> cell index.  Empty
// slots hold the all-ones key, which no cell has (it marks invalid points).
__device__ __forceinline__ unsigned long long hash_slot(unsigned long long key, unsigned long long mask) {
    return ((key + 1ull) * 0x9E3779B97F4A7C15ull >> 17) & mask;
}

template <typename K>
__global__ void hash_clear_kernel(K *__restrict__ hkeys, int64_t size) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < size) hkeys[i] = ~(K)0;
}

__device__ __forceinline__ uint32_t key_cas(uint32_t *a, uint32_t cmp, uint32_t val) { return atomicCAS(a, cmp, val); }
__device__ __forceinline__ uint64_t key_cas(uint64_t *a, uint64_t cmp, uint64_t val) {
    return (uint64_t)atomicCAS(reinterpret_cast<unsigned long long *>(a), (unsigned long long)cmp,
                               (unsigned long long)val);
}

template <typename K>
__global__ void hash_insert_kernel(const K *__restrict__ cell_key, int64_t n_cells, K *hkeys,
                                   int32_t *__restrict__ hvals, unsigned long long mask) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_cells) return;
    const K key = cell_key[c];
    unsigned long long h = hash_slot((unsigned long long)key, mask);
    for (unsigned long long probe = 0; probe <= mask; ++probe) {
        const K prev = key_cas(hkeys + h, ~(K)0, key);
        if (prev == ~(K)0 || prev == key) {
            hvals[h] = (int32_t)c;
            return;
        }
        h = (h + 1) & mask;
    }
}

template <typename K>
__device__ __forceinline__ int hash_find(const K *__restrict__ hkeys, const int32_t *__restrict__ hvals,
                                         unsigned long long mask, unsigned long long key) {
    unsigned long long h = hash_slot(key, mask);
    for (unsigned long long probe = 0; probe <= mask; ++probe) {
        const K k = __ldg(hkeys + h);
        if ((unsigned long long)k == key) return __ldg(hvals + h);
        if (k == ~(K)0) return -1;
        h = (h + 1) & mask;
    }
    return -1;
}

// ---------------------------------------------------------------------------
// How cells are found by key.  A column is the run of cells that differ only in
// gridded dimension 0; sorted by key, a column's cells are contiguous and ordered
// by x.  When the grid's columns are few enough (their count depends on the
// bounding box, not on n), a dense table holds each column's [first, end) range
// of cell indices, so a stencil row is one table load plus a search inside one
// short column.  Otherwise the open-addressing hash table of the cell keys is
// probed per x position.
// ---------------------------------------------------------------------------
template <typename K>
struct CellIndex {
    const int2 *col;      // column table (null: use the hash table)
    const K *hkeys;
    const int32_t *hvals;
    unsigned long long mask;
};

// Column of every cell: the table entry of its column gets the first cell (the
// column's first in key order) and the end (one past its last).  The table starts
// zeroed (empty columns read [0, 0)).
template <typename K>
__device__ __forceinline__ long long global_column(const K *__restrict__ cell_key, int64_t c, const GridDev &g_one,
                                                   const JobDev *__restrict__ jobs,
                                                   const int32_t *__restrict__ cell_job) {
    unsigned long long key_base = 0;
    long long col_base = 0, g0 = g_one.g[0];
    if (jobs) {
        const JobDev &J = jobs[cell_job[c]];
        key_base = J.key_base;
        col_base = J.col_base;
        g0 = J.g.g[0];
    }
    const unsigned long long local = (unsigned long long)cell_key[c] - key_base;
    if constexpr (sizeof(K) == 4) return col_base + (long long)((uint32_t)local / (uint32_t)g0);
    else return col_base + (long long)(local / (unsigned long long)g0);
}

template <typename K>
__global__ void col_range_kernel(const K *__restrict__ cell_key, int64_t n_cells, GridDev g_one,
                                 const JobDev *__restrict__ jobs, const int32_t *__restrict__ cell_job,
                                 int2 *__restrict__ col) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_cells) return;
    const long long mine = global_column(cell_key, c, g_one, jobs, cell_job);
    if (c == 0 || global_column(cell_key, c - 1, g_one, jobs, cell_job) != mine) col[mine].x = (int)c;
    if (c == n_cells - 1 || global_column(cell_key, c + 1, g_one, jobs, cell_job) != mine) col[mine].y = (int)(c + 1);
}

// First cell of column range cr whose key is >= rowkey + x (cr.y when none); the
// column's cells have keys rowkey + x' with strictly increasing x'.  A column
// without gaps places it directly: position first + (x - x_first).
template <typename K>
__device__ __forceinline__ int col_lower(const K *__restrict__ cell_key, int2 cr, unsigned long long rowkey,
                                         long long x) {
    if (cr.x >= cr.y) return cr.y;
    const long long xf = (long long)((unsigned long long)__ldg(cell_key + cr.x) - rowkey);
    if (x <= xf) return cr.x;
    const long long p = cr.x + (x - xf);  // keys grow by >= 1 per cell: key[p] >= rowkey + x
    if (p < cr.y && (unsigned long long)__ldg(cell_key + p) == rowkey + (unsigned long long)x) return (int)p;
    int lo = cr.x + 1, hi = (int)(p < cr.y ? p : cr.y);
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if ((unsigned long long)__ldg(cell_key + mid) < rowkey + (unsigned long long)x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Cell index of the cell with key rowkey + x in column ncol, or -1.
template <typename K>
__device__ __forceinline__ int find_cell(const CellIndex<K> &L, const K *__restrict__ cell_key, long long ncol,
                                         unsigned long long rowkey, long long x) {
    const unsigned long long key = rowkey + (unsigned long long)x;
    if (!L.col) return hash_find(L.hkeys, L.hvals, L.mask, key);
    const int2 cr = __ldg(L.col + ncol);
    const int a = col_lower(cell_key, cr, rowkey, x);
    return a < cr.y && (unsigned long long)__ldg(cell_key + a) == key ? a : -1;
}

// nbr[c * n_rows + r] = [first, last) cell index of row r around cell c: the cells
// of a row have consecutive keys, so the existing ones are consecutive in the
// sorted cell list and the range runs from the smallest to the largest found.
// Cell coordinates from a key (x fastest); 32-bit arithmetic for 32-bit keys.
template <typename K>
__device__ __forceinline__ void decode_key(K key, const GridDev &g, long long (&c)[kMaxGridDims]) {
    using U = typename std::conditional<sizeof(K) == 4, uint32_t, unsigned long long>::type;
    U rest = (U)key;
#pragma unroll
    for (int a = 0; a < kMaxGridDims; ++a) {
        if (a < g.k - 1) {
            const U ga = (U)g.g[a];
            const U q = rest / ga;
            c[a] = (long long)(rest - q * ga);
            rest = q;
        } else if (a == g.k - 1) {
            c[a] = (long long)rest;
        } else {
            c[a] = 0;
        }
    }
}

// nbr[c * n_rows + r] = [first, last) cell index of row r around cell c: the cells
// of a row have consecutive keys, so the existing ones are consecutive in the
// sorted cell list and the range runs from the smallest to the largest found.
// Cell coordinates from a key (x fastest); 32-bit arithmetic for 32-bit keys.
template <typename K>
__device__ __forceinline__ void decode_key(K key, const GridDev &g, long long &x, long long &y, long long &z) {
    if constexpr (sizeof(K) == 4) {
        const uint32_t g0 = (uint32_t)g.g[0], g1 = (uint32_t)g.g[1];
        const uint32_t rest = (uint32_t)key / g0;
        x = (long long)((uint32_t)key - rest * g0);
        y = g.k >= 3 ? (long long)(rest % g1) : (long long)rest;
        z = g.k >= 3 ? (long long)(rest / g1) : 0;
    } else {
        const unsigned long long g0 = (unsigned long long)g.g[0], g1 = (unsigned long long)g.g[1];
        const unsigned long long rest = (unsigned long long)key / g0;
        x = (long long)((unsigned long long)key - rest * g0);
        y = g.k >= 3 ? (long long)(rest % g1) : (long long)rest;
        z = g.k >= 3 ? (long long)(rest / g1) : 0;
    }
}

// nbr[c * n_rows + r] = [first, last) cell index of row r around cell c: the cells
// of a row have consecutive keys, so the existing ones are consecutive in the
// sorted cell list and the range runs from the smallest to the largest found.
// One thread per cell (one key decode); the first hash probes of a row's cells
// are issued together.
template <typename K>
__global__ void __launch_bounds__(kBlock) rows_kernel(const K *__restrict__ cell_key, int64_t n_cells,
                                                      GridDev g_one, const int4 *__restrict__ rows, int n_rows,
                                                      int group_log2, CellIndex<K> L, int2 *__restrict__ nbr,
                                                      const JobDev *__restrict__ jobs,
                                                      const int32_t *__restrict__ cell_job) {
    // one lane per (cell, row): 2^group_log2 lanes (>= n_rows) per cell, so
    // a cell's rows are looked up in parallel and its row table is written at once
    __shared__ int4 s_rows[kMaxRows];
    for (int r = threadIdx.x; r < n_rows; r += blockDim.x) s_rows[r] = rows[r];
    __syncthreads();
    const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t c = gid >> group_log2;
    const int r = (int)(gid & ((1 << group_log2) - 1));
    if (c >= n_cells || r >= n_rows) return;
    unsigned long long key_base = 0;
    long long col_base = 0;
    GridDev g = g_one;
    if (jobs) {
        const JobDev &J = jobs[cell_job[c]];
        g = J.g;
        key_base = J.key_base;
        col_base = J.col_base;
    }
    long long cc[kMaxGridDims];
    decode_key<K>((K)((unsigned long long)cell_key[c] - key_base), g, cc);
    const int4 row = s_rows[r];
    const int off[kMaxGridDims] = {0, row.x, row.y, row.z};
    bool in = true;
    unsigned long long base = key_base;
    long long ncol = 0, cstride = 1;  // the row's column: cells differing only in dimension 0
#pragma unroll
    for (int a = 1; a < kMaxGridDims; ++a) {
        if (a < g.k) {
            const long long v = cc[a] + off[a];
            in = in && v >= 0 && v < g.g[a];
            base += (unsigned long long)(v < 0 ? 0 : v) * g.stride[a];
            ncol += (v < 0 ? 0 : v) * cstride;
            cstride *= g.g[a];
        }
    }
    int2 res = make_int2(0, 0);
    if (in) {
        const long long x0 = cc[0] - row.w < 0 ? 0 : cc[0] - row.w;
        const long long x1 = cc[0] + row.w > g.g[0] - 1 ? g.g[0] - 1 : cc[0] + row.w;
        // the row's existing cells are consecutive in the sorted cell list: find the
        // first one (a column-table search, or hashing from x0 on), then count the
        // keys that follow it within the row (independent loads, at most 2 row.w)
        int ca = -1;
        if (L.col) {
            const int2 cr = __ldg(L.col + col_base + ncol);
            const int a = col_lower(cell_key, cr, base, x0);
            if (a < cr.y && (unsigned long long)__ldg(cell_key + a) <= base + (unsigned long long)x1) ca = a;
        } else {
            for (long long xx = x0; xx <= x1 && ca < 0; ++xx)
                ca = hash_find(L.hkeys, L.hvals, L.mask, base + (unsigned long long)xx);
        }
        if (ca >= 0) {
            // keys are sorted and unique: the row's cells after ca are a prefix of the
            // next keys; four independent loads cover rows of up to 5 cells
            const unsigned long long kmax = base + (unsigned long long)x1;
            K nk[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) nk[q] = ca + 1 + q < n_cells ? __ldg(cell_key + ca + 1 + q) : ~(K)0;
            int cb = ca + 1;
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (cb == ca + 1 + q && ca + 1 + q < n_cells && (unsigned long long)nk[q] <= kmax) ++cb;
            if (cb == ca + 5)
                while (cb < n_cells && (unsigned long long)__ldg(cell_key + cb) <= kmax) ++cb;
            res = make_int2(ca, cb);
        }
    }
    nbr[c * n_rows + r] = res;
}

// Items into two lists: those with at least min_cnt points (full tiles: the
// tensor-core count) and the rest (the exact kernel).  Order within a list is
// free; both counts land in device memory.
__global__ void split_items_kernel(const int2 *__restrict__ items, int64_t n_items,
                                   const int32_t *__restrict__ cell_start, int min_cnt, int2 *__restrict__ out_a,
                                   uint32_t *__restrict__ n_a, int2 *__restrict__ out_b, uint32_t *__restrict__ n_b) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < n_items;
    int2 it = make_int2(0, 0);
    bool a = false;
    if (valid) {
        it = items[i];
        a = min(kTile, cell_start[it.x + 1] - it.y) >= min_cnt;
    }
    const unsigned ma = __ballot_sync(kFull, valid && a), mb = __ballot_sync(kFull, valid && !a);
    const int lane = threadIdx.x & 31;
    uint32_t ba = 0, bb = 0;
    if (lane == 0) {
        if (ma) ba = atomicAdd(n_a, (uint32_t)__popc(ma));
        if (mb) bb = atomicAdd(n_b, (uint32_t)__popc(mb));
    }
    ba = __shfl_sync(kFull, ba, 0);
    bb = __shfl_sync(kFull, bb, 0);
    if (valid) {
        if (a) out_a[ba + __popc(ma & lanemask_lt())] = it;
        else out_b[bb + __popc(mb & lanemask_lt())] = it;
    }
}

__global__ void item_count_kernel(const int32_t *__restrict__ cell_start, int64_t n_cells,
                                  uint32_t *__restrict__ cnt) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_cells) return;
    const int32_t size = cell_start[c + 1] - cell_start[c];
    cnt[c] = (uint32_t)((size + kTile - 1) / kTile);
}

__global__ void item_write_kernel(const int32_t *__restrict__ cell_start, int64_t n_cells,
                                  const uint32_t *__restrict__ off, int2 *__restrict__ items) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_cells) return;
    const int32_t s0 = cell_start[c], s1 = cell_start[c + 1];
    uint32_t o = off[c];
    for (int32_t p = s0; p < s1; p += kTile) items[o++] = make_int2((int)c, p);
}

// ---------------------------------------------------------------------------
// Row table: the candidate ranges of one cell's stencil rows, gathered by the
// warp in one round (lane r loads row r) and flattened, so that the lanes walk the
// candidates of all rows 32 at a time instead of row by row.  Host planning keeps
// the number of rows <= 32.
// ---------------------------------------------------------------------------
struct RowTable {
    int start[kWarp];    // first candidate (point index, or cell index for CELLS) of each row
    int off[kWarp + 1];  // exclusive prefix of the row lengths; off[n_rows] = total
};

// Row table from one (start, len) range per lane (lanes >= n_rows hold len 0).
__device__ __forceinline__ int build_rows(int start, int len, int n_rows, RowTable &rt, int lane) {
    int incl = len;
#pragma unroll
    for (int o = 1; o < kWarp; o <<= 1) {
        const int y = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane < n_rows) {
        rt.start[lane] = start;
        rt.off[lane] = incl - len;
    }
    const int total = __shfl_sync(kFull, incl, kWarp - 1);
    if (lane == 0) rt.off[n_rows] = total;
    __syncwarp();
    return total;
}

// CELLS: ranges of cell indices >= min_cell; otherwise ranges of point indices.
template <bool CELLS>
__device__ __forceinline__ int gather_rows(const int2 *__restrict__ nbr_row, int n_rows,
                                           const int32_t *__restrict__ cell_start, int min_cell,
                                           RowTable &rt, int lane) {
    int start = 0, len = 0;
    if (lane < n_rows) {
        const int2 cr = nbr_row[lane];
        if (CELLS) {
            start = max(cr.x, min_cell);
            len = max(cr.y - start, 0);
        } else if (cr.x < cr.y) {
            start = cell_start[cr.x];
            len = cell_start[cr.y] - start;
        }
    }
    return build_rows(start, len, n_rows, rt, lane);
}

// Candidate t (0 <= t < total) of the flattened rows: the last row whose offset is
// <= t.  For rows of cells (at most a few entries each).
__device__ __forceinline__ int row_lookup(const RowTable &rt, int n_rows, int t) {
    int lo = 0, hi = n_rows - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (rt.off[mid] <= t) lo = mid;
        else hi = mid - 1;
    }
    return rt.start[lo] + (t - rt.off[lo]);
}

// Candidate t for a lane whose t only grows (by a warp per step): advance the
// lane's row cursor over the row offsets (empty rows skipped) instead of searching.
__device__ __forceinline__ int row_next(const RowTable &rt, int &row, int t) {
    while (rt.off[row + 1] <= t) ++row;
    return rt.start[row] + (t - rt.off[row]);
}

// ---------------------------------------------------------------------------
// Neighbour count.  One warp per item (up to 32 points i of one cell).  The i
// points sit in shared memory; lanes walk the flattened candidates of the
// stencil rows 32 at a time (coalesced loads), every lane tests its candidate j
// against each i (broadcast reads) and the warp adds popc(ballot) to that i's
// count.  Rows are ordered nearest first.
// EARLY: stop once every i of the item has reached min_pts (exact counts below
// min_pts, so exact core flags).  dense_skip: with same-cell-linked cells a cell
// of >= min_pts points is all cores (every pair inside it is in range), so its
// points need no test at all; they report the cell size.
// ---------------------------------------------------------------------------
//
// GRAM (d >= 8): a pair is first decided from centred FP32 dot products.  With
// a = x_i - o and b = x_j - o (o the item's first point), D~ = |a|^2 + |b|^2 - 2 a.b
// costs d FMAs per pair, against the 3d separately rounded operations of the
// reference's sum.  A pair is a hit when D~ is below e2 by more than a bound on its
// error, a miss when above by more than it; the pairs in between (the guard band)
// are decided by the reference's own FP32 sum.  Counts, lists and core flags are
// therefore the exact kernel's.  Error bound (u = 2^-24, K = d): centring in FP32
// moves |a - b|^2 off |x_i - x_j|^2 by at most 4u (n_a + n_b); the FMA chains give
// |a|^2, |b|^2 and a.b within K u of n_a, n_b and |a||b| <= (n_a + n_b) / 2; forming
// v = n_a - 2 a.b and v + n_b adds 2u (n_a + n_b).  So |D~ - |x_i - x_j|^2| <=
// (3K + 6) u (n_a + n_b), and gram_kappa is twice that.  The reference's sum is
// within (K + 2) u of |x_i - x_j|^2 (gram_gamma covers 2 (K + 8) u), and the
// thresholds carry the rounding of their own arithmetic (kGramSigma e2).
// ---------------------------------------------------------------------------
template <int K>
__host__ __device__ constexpr float gram_kappa() {
    return 2.0f * (3.0f * K + 6.0f) * (1.0f / 16777216.0f);
}
template <int K>
__host__ __device__ constexpr float gram_gamma() {
    return 2.0f * (K + 8) * (1.0f / 16777216.0f);
}
constexpr float kGramSigma = 8.0f / 16777216.0f;

template <int D, bool EARLY, bool GRAM = false>
__global__ void __launch_bounds__(kCountWarps * kWarp) count_kernel(
    const int2 *__restrict__ items, int64_t n_items, const int32_t *__restrict__ cell_start,
    const int2 *__restrict__ nbr, int n_rows, const float *__restrict__ xs, float e2, int min_pts,
    int dense_skip, int32_t *__restrict__ nn_sorted, int32_t *__restrict__ nbr_list, int list_cap,
    int list_stride, unsigned long long *__restrict__ pair_counter, const JobDev *__restrict__ jobs,
    const int32_t *__restrict__ cell_job, const uint32_t *__restrict__ n_items_dev,
    unsigned long long *__restrict__ band_counter) {
    constexpr int P = Stride<D>::P;
    static_assert(!GRAM || D >= 8, "the Gram filter is built for d >= 8");
    // d >= 8: each lane holds two candidates per step (64 per warp), so an owned
    // point is read from shared memory once per two pairs and the two distance sums
    // (each in the reference's order) are independent chains for the scheduler
    constexpr int CH = D >= 8 ? 2 : 1;
    __shared__ __align__(16) float s_i[kCountWarps][kTile * P];
    __shared__ __align__(16) float s_a[kCountWarps][GRAM ? kTile * P : 4];  // centred points
    __shared__ float s_n[kCountWarps][GRAM ? kTile : 1];                     // their squared norms
    __shared__ RowTable s_rows[kCountWarps];
    __shared__ int s_list[kCountWarps][kTile * kSmemListCap];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    if (n_items_dev) n_items = *n_items_dev;  // a list whose length the device wrote
    const int64_t item_id = (int64_t)blockIdx.x * kCountWarps + wib;
    if (item_id >= n_items) return;
    const int2 item = items[item_id];
    const int cell = item.x, p0 = item.y;
    const int cs = cell_start[cell], ce = cell_start[cell + 1];
    const int cnt = min(kTile, ce - p0);
    if (jobs) {
        const JobDev &J = jobs[cell_job[cell]];
        e2 = J.e2;
        min_pts = J.min_pts;
        dense_skip = J.linked;
        list_cap = J.list_cap;
    }
    // lists of up to kSmemListCap entries are gathered in shared memory and written
    // out only for the points that end below min_pts; longer ones go straight out
    const bool smem_list = list_stride <= kSmemListCap;
    int *sl = s_list[wib];
    if (EARLY && dense_skip && ce - cs >= min_pts) {
        if (lane < cnt) nn_sorted[p0 + lane] = ce - cs;
        return;
    }
    float *si = s_i[wib];
    RowTable &rt = s_rows[wib];
    float o[GRAM ? D : 1];  // GRAM: the item's first point, the origin of the centring
    float nmax = 0.0f;      // GRAM: largest |a|^2 of the item
    if constexpr (GRAM) load_point<D>(xs, p0, o);
    if (lane < cnt) {
        float x[D];
        load_point<D>(xs, p0 + lane, x);
        store_point_smem<D>(si + lane * P, x);
        if constexpr (GRAM) {
            float a[D];
            float n = 0.0f;
#pragma unroll
            for (int k = 0; k < D; ++k) {
                a[k] = __fsub_rn(x[k], o[k]);
                n = __fmaf_rn(a[k], a[k], n);
            }
            store_point_smem<D>(s_a[wib] + lane * P, a);
            s_n[wib][lane] = n;
            nmax = n;
        }
    }
    if constexpr (GRAM) {
#pragma unroll
        for (int sft = 16; sft > 0; sft >>= 1) nmax = fmaxf(nmax, __shfl_xor_sync(kFull, nmax, sft));
    }
    const int total = gather_rows<false>(nbr + (int64_t)cell * n_rows, n_rows, cell_start, 0, rt, lane);
    __syncwarp();
    // running counts in registers: lane k holds the count of the item's point k
    int mycnt = 0;
    unsigned long long pairs = 0, band = 0;  // pairs tested; GRAM: pairs rechecked in the guard band
    // points still counting (EARLY: below min_pts), and points whose neighbour list
    // is still filling (count below list_cap): both warp-uniform, updated per chunk
    unsigned act = __ballot_sync(kFull, lane < cnt);
    unsigned lst = nbr_list && list_cap > 0 ? act : 0u;
    int row = 0;  // this lane's stencil row: its candidate index only grows
    for (int tb = 0; tb < total; tb += kWarp * CH) {
        int j[CH];
        float xj[CH][D];  // GRAM: the centred candidate b = x_j - o
        float tlo[CH], thi[CH];
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            const int t = tb + c * kWarp + lane;
            j[c] = t < total ? row_next(rt, row, t) : -1;
            if (j[c] >= 0) load_point<D>(xs, j[c], xj[c]);
            else fill_nan<D>(xj[c]);  // NaN fails the predicate
            if constexpr (GRAM) {
                float nb = 0.0f;
#pragma unroll
                for (int k = 0; k < D; ++k) {
                    xj[c][k] = __fsub_rn(xj[c][k], o[k]);
                    nb = __fmaf_rn(xj[c][k], xj[c][k], nb);
                }
                // hit when v = |a|^2 - 2 a.b <= tlo, miss when v > thi (see the bound above)
                const float slack = __fadd_rn(__fmul_rn(gram_kappa<D>(), __fadd_rn(nmax, nb)),
                                              __fmul_rn(kGramSigma, e2));
                tlo[c] = j[c] >= 0 ? __fsub_rn(__fsub_rn(__fmul_rn(e2, 1.0f - gram_gamma<D>()), nb), slack) : -INFINITY;
                thi[c] = j[c] >= 0 ? __fadd_rn(__fsub_rn(__fmul_rn(e2, 1.0f + gram_gamma<D>()), nb), slack) : -INFINITY;
            }
        }
        int active = 0;
        for (unsigned it = act; it; it &= it - 1) {
            const int k = __ffs(it) - 1;
            bool hit[CH];
            unsigned m[CH];
            if constexpr (GRAM) {
                float a[D];
                load_point_smem<D>(s_a[wib] + k * P, a);
                const float na = s_n[wib][k];
                bool inband[CH];
#pragma unroll
                for (int c = 0; c < CH; ++c) {
                    // four independent FMA chains (the bound holds for any order of
                    // the sum), joined by three additions
                    float g4[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
                    for (int q = 0; q < D; ++q) g4[q & 3] = __fmaf_rn(a[q], xj[c][q], g4[q & 3]);
                    const float g = __fadd_rn(__fadd_rn(g4[0], g4[1]), __fadd_rn(g4[2], g4[3]));
                    const float v = __fmaf_rn(-2.0f, g, na);
                    hit[c] = v <= tlo[c];
                    inband[c] = !hit[c] && v <= thi[c];
                }
                if (inband[0] || (CH > 1 && inband[CH - 1])) {
                    // the guard band (rare): the reference's own sum decides
                    float xi[D];
                    load_point_smem<D>(si + k * P, xi);
#pragma unroll
                    for (int c = 0; c < CH; ++c) {
                        if (!inband[c]) continue;
                        float xr[D];
                        load_point<D>(xs, j[c], xr);
                        hit[c] = in_range<D>(xi, xr, e2);
                        ++band;
                    }
                }
            } else {
                float xi[D];
                load_point_smem<D>(si + k * P, xi);
#pragma unroll
                for (int c = 0; c < CH; ++c) hit[c] = in_range<D>(xi, xj[c], e2);
            }
#pragma unroll
            for (int c = 0; c < CH; ++c) m[c] = __ballot_sync(kFull, hit[c]);
            // the first list_cap neighbours of each point; complete for every point
            // whose count stays below min_pts (list_cap = min_pts - 1)
            if ((lst >> k) & 1u) {
                int base = __shfl_sync(kFull, mycnt, k);
#pragma unroll
                for (int c = 0; c < CH; ++c) {
                    const int slot = base + __popc(m[c] & lanemask_lt());
                    if (hit[c] && slot < list_cap) {
                        if (smem_list) sl[k * kSmemListCap + slot] = j[c];
                        else nbr_list[(int64_t)(p0 + k) * list_stride + slot] = j[c];
                    }
                    base += __popc(m[c]);
                }
            }
            int got = 0;
#pragma unroll
            for (int c = 0; c < CH; ++c) got += __popc(m[c]);
            if (lane == k) mycnt += got;
            ++active;
        }
        pairs += (unsigned long long)active * (unsigned long long)min(kWarp * CH, total - tb);
        if (lst) lst &= __ballot_sync(kFull, mycnt < list_cap);
        if (EARLY) {
            act = __ballot_sync(kFull, lane < cnt && mycnt < min_pts);
            if (!act) break;
        }
    }
    const int mine = lane < cnt ? mycnt : 0;
    if (lane < cnt) nn_sorted[p0 + lane] = mine;
    if (nbr_list && smem_list) {
        __syncwarp();
        // every point's list: the border step reads the non-cores', the union
        // starts from the cores' (for cell units, the items the count ran)
        if (lane < cnt) {
            const int len = min(mine, list_cap);
            for (int q = 0; q < len; ++q) nbr_list[(int64_t)(p0 + lane) * list_stride + q] = sl[lane * kSmemListCap + q];
        }
    }
    if (lane == 0 && pairs) atomicAdd(pair_counter, pairs);
    if constexpr (GRAM) {
        band = __reduce_add_sync(kFull, (unsigned)band);
        if (lane == 0 && band) atomicAdd(band_counter, band);
    }
}

// Core flags: per sorted point (u8), and a bitmap in input order (one bit per
// point, atomicOr; 12.5 MB for 10^8 points, so it stays in L2).  With the
// per-word prefix of its popcounts the bitmap gives every point's rank among the
// cores in input order (data_process.cpp:276-283, :153) without a per-point scan.
__global__ void core_flags_kernel(const int32_t *__restrict__ nn_sorted, int64_t nv, int64_t n, int min_pts,
                                  const int32_t *__restrict__ perm, const int32_t *__restrict__ pcell,
                                  uint8_t *__restrict__ core_sorted, uint8_t *__restrict__ cell_has_core,
                                  uint32_t *__restrict__ core_bits, const JobDev *__restrict__ jobs,
                                  const int32_t *__restrict__ cell_job, int n_jobs) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    if (jobs) min_pts = jobs[s < nv ? cell_job[pcell[s]] : job_of_point(jobs, n_jobs, perm[s])].min_pts;
    bool core;
    if (s < nv) {
        core = nn_sorted[s] >= min_pts;
        core_sorted[s] = core ? 1 : 0;
        if (core) cell_has_core[pcell[s]] = 1;
    } else {
        core = 0 >= min_pts;  // points outside the grid have no neighbour, not even themselves
    }
    if (core) {
        const int32_t o = perm[s];
        atomicOr(core_bits + (o >> 5), 1u << (o & 31));
    }
}

__global__ void popc_words_kernel(const uint32_t *__restrict__ bits, int64_t n_words, uint32_t *__restrict__ cnt) {
    const int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (w < n_words) cnt[w] = (uint32_t)__popc(bits[w]);
}

__device__ __forceinline__ bool is_core_o(const uint32_t *__restrict__ bits, int32_t o) {
    return (bits[o >> 5] >> (o & 31)) & 1u;
}

// rank of point o among the cores, in input order
__device__ __forceinline__ int32_t core_rank(const uint32_t *__restrict__ bits, const uint32_t *__restrict__ prefix,
                                             int32_t o) {
    return (int32_t)(prefix[o >> 5] + __popc(bits[o >> 5] & ((1u << (o & 31)) - 1u)));
}

// nn in input order (the caller's nn output)
// Input-order outputs are random 4-byte writes.  When the output is much larger
// than L2 the host runs the scatter in destination windows [win_lo, win_hi): each
// pass streams the sorted arrays (evict-first loads) and writes only the points
// whose destination falls in its window, so the partial-sector writes stay in L2.
__global__ void scatter_nn_kernel(const int32_t *__restrict__ nn_sorted, int64_t nv, int64_t n,
                                  const int32_t *__restrict__ perm, int32_t *__restrict__ out,
                                  const JobDev *__restrict__ jobs, int n_jobs, int64_t win_lo = 0,
                                  int64_t win_hi = INT64_MAX) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int32_t o = __ldcs(perm + s);
    if (o < win_lo || o >= win_hi) return;
    const int32_t v = s < nv ? __ldcs(nn_sorted + s) : 0;
    if (jobs) {
        const JobDev &J = jobs[job_of_point(jobs, n_jobs, o)];
        if (J.nn_out) J.nn_out[o - J.off] = v;
    } else {
        out[o] = v;
    }
}

__global__ void iota_kernel(int32_t *__restrict__ a, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = (int32_t)i;
}

__global__ void fill_kernel(int32_t *__restrict__ a, int64_t n, int32_t v) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = v;
}

// bytes [0, bytes) of p set to v: n16 16-byte stores (p 16-byte aligned; 0 when it
// is not), then the tail byte by byte
__global__ void fill_bytes_kernel(uint8_t *__restrict__ p, size_t bytes, int64_t n16, uint8_t v) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t w = 0x01010101u * v;
    for (int64_t i = t; i < n16; i += stride) reinterpret_cast<uint4 *>(p)[i] = make_uint4(w, w, w, w);
    for (int64_t i = n16 * 16 + t; i < (int64_t)bytes; i += stride) p[i] = v;
}

// n words from src to dst (either may be mapped host memory)
__global__ void copy_words_kernel(const uint32_t *__restrict__ src, uint32_t *__restrict__ dst, int64_t n) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) dst[i] = src[i];
}

// Loads the core points of an item into shared memory (compacted); returns how many.
template <int D>
__device__ __forceinline__ int load_item_cores(const float *__restrict__ xs, const uint8_t *__restrict__ core_sorted,
                                               int p0, int cnt, bool want_core, float *si, int *sidx, int lane) {
    constexpr int P = Stride<D>::P;
    const bool ok = lane < cnt && ((core_sorted[p0 + lane] != 0) == want_core);
    const unsigned mask = __ballot_sync(kFull, ok);
    if (ok) {
        const int slot = __popc(mask & lanemask_lt());
        float x[D];
        load_point<D>(xs, p0 + lane, x);
        store_point_smem<D>(si + slot * P, x);
        sidx[slot] = p0 + lane;
    }
    __syncwarp();
    return __popc(mask);
}

// Is any core of cell A in range of any core of cell B?  A's cores go through
// shared memory 32 at a time; lanes hold B's points.  Stops at the first hit.
template <int D>
__device__ __forceinline__ bool cells_touch(int A, int B, const int32_t *__restrict__ cell_start,
                                            const float *__restrict__ xs, const uint8_t *__restrict__ core_sorted,
                                            float e2, float *si, int lane, unsigned long long &pairs) {
    constexpr int P = Stride<D>::P;
    const int a0 = cell_start[A], a1 = cell_start[A + 1];
    const int b0 = cell_start[B], b1 = cell_start[B + 1];
    for (int ab = a0; ab < a1; ab += kWarp) {
        const int i = ab + lane;
        const bool ok = i < a1 && core_sorted[i];
        const unsigned mask = __ballot_sync(kFull, ok);
        if (ok) {
            float x[D];
            load_point<D>(xs, i, x);
            store_point_smem<D>(si + __popc(mask & lanemask_lt()) * P, x);
        }
        __syncwarp();
        const int nc = __popc(mask);
        if (nc == 0) continue;
        for (int bb = b0; bb < b1; bb += kWarp) {
            const int j = bb + lane;
            float xj[D];
            if (j < b1 && core_sorted[j]) load_point<D>(xs, j, xj);
            else fill_nan<D>(xj);
            bool hit = false;
            for (int k = 0; k < nc; ++k) {
                float xi[D];
                load_point_smem<D>(si + k * P, xi);
                hit = hit || in_range<D>(xi, xj, e2);
            }
            pairs += (unsigned long long)nc * (unsigned long long)min(kWarp, b1 - bb);
            if (__any_sync(kFull, hit)) return true;
        }
        __syncwarp();
    }
    return false;
}

// ---------------------------------------------------------------------------
// First union pass over cells: one thread per cell A.  It looks at A's three
// forward face neighbours (x+1, y+1, z+1; found through the key order and the cell
// hash table), tests the first kNearProbe cores of A against the first
// kNearProbe cores of each (independent loads, 16 predicates) and links A and B on
// a hit.  Face adjacency already connects every cell of a dense region, so this
// merges dense clusters with one cheap thread per cell; the full pass then sees
// them as one root.
// ---------------------------------------------------------------------------
constexpr int kNearProbe = 4;

template <int D>
__device__ __forceinline__ void load_first_cores(const float *__restrict__ xs, const uint8_t *__restrict__ core_sorted,
                                                 int c0, int c1, float (&x)[kNearProbe][D]) {
#pragma unroll
    for (int q = 0; q < kNearProbe; ++q) {
        const int i = c0 + q;
        if (i < c1 && core_sorted[i]) load_point<D>(xs, i, x[q]);
        else fill_nan<D>(x[q]);
    }
}

template <int D, typename K>
__global__ void __launch_bounds__(kBlock) union_near_kernel(
    int64_t n_cells, GridDev g_one, const K *__restrict__ cell_key, const int32_t *__restrict__ cell_start,
    CellIndex<K> L, const float *__restrict__ xs, float e2, const uint8_t *__restrict__ core_sorted,
    const uint8_t *__restrict__ cell_has_core, int32_t *parent, unsigned long long *__restrict__ pair_counter,
    int *err, const JobDev *__restrict__ jobs, const int32_t *__restrict__ cell_job) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned pairs = 0;
    if (idx < n_cells && cell_has_core[idx]) {
        const int A = (int)idx;
        const unsigned long long key = (unsigned long long)cell_key[A];
        GridDev g = g_one;
        unsigned long long key_base = 0;
        long long col_base = 0;
        if (jobs) {
            const JobDev &J = jobs[cell_job[A]];
            g = J.g;
            e2 = J.e2;
            key_base = J.key_base;
            col_base = J.col_base;
        }
        long long cc[kMaxGridDims];
        decode_key<K>((K)(key - key_base), g, cc);
        // the cell's column, and the keys of x = 0 in the columns one step up in y and z
        const long long col = col_base + cc[1] + (g.k >= 3 ? cc[2] * g.g[1] : 0);
        const unsigned long long row0 = key - (unsigned long long)cc[0];
        int nb[3] = {-1, -1, -1};
        if (cc[0] + 1 < g.g[0] && A + 1 < n_cells && (unsigned long long)cell_key[A + 1] == key + 1ull) nb[0] = A + 1;
        if (g.k >= 2 && cc[1] + 1 < g.g[1]) nb[1] = find_cell(L, cell_key, col + 1, row0 + g.stride[1], cc[0]);
        if (g.k >= 3 && cc[2] + 1 < g.g[2])
            nb[2] = find_cell(L, cell_key, col + g.g[1], row0 + g.stride[2], cc[0]);
        bool any = false;
#pragma unroll
        for (int f = 0; f < 3; ++f) {
            if (nb[f] >= 0 && !cell_has_core[nb[f]]) nb[f] = -1;
            any = any || nb[f] >= 0;
        }
        if (any) {
            float xa[kNearProbe][D];
            load_first_cores<D>(xs, core_sorted, cell_start[A], cell_start[A + 1], xa);
#pragma unroll
            for (int f = 0; f < 3; ++f) {
                if (nb[f] < 0) continue;
                const int B = nb[f];
                float xb[kNearProbe][D];
                load_first_cores<D>(xs, core_sorted, cell_start[B], cell_start[B + 1], xb);
                bool hit = false;
#pragma unroll
                for (int p = 0; p < kNearProbe; ++p)
#pragma unroll
                    for (int q = 0; q < kNearProbe; ++q) hit = hit || in_range<D>(xa[p], xb[q], e2);
                pairs += kNearProbe * kNearProbe;
                if (hit) uf_union(parent, A, B, err);
            }
        }
    }
    pairs = __reduce_add_sync(kFull, pairs);
    if ((threadIdx.x & 31) == 0 && pairs) atomicAdd(pair_counter, (unsigned long long)pairs);
}

// ---------------------------------------------------------------------------
// Union-find over cells (same-cell-linked grids): every pair inside a cell is in
// range, so all cores of a cell belong to one component and the cell is the
// union-find element.  One warp per cell A: the lanes gather A's half stencil
// (cells B > A holding cores), find every B's root in parallel, keep the B whose
// root differs from A's, then link A and B as soon as one core pair is in range.
// ---------------------------------------------------------------------------
constexpr int kMaxCandCells = 128;
constexpr int kProbe = 4;  // points of a candidate cell tested by the probe

//
// Runs after union_near_kernel has linked the adjacent dense cells, so the root
// filter removes most candidates before any point test.
// snap: every cell's root after the near pass (flatten_snap_kernel), -1 for cells
// without cores; one load per candidate tells both.  A root since hooked elsewhere
// only costs a needless probe below, never a missed union.
template <int D>
__global__ void __launch_bounds__(kBlock) union_cells_kernel(
    int64_t n_cells, const int32_t *__restrict__ cell_start, const int2 *__restrict__ nbr, int n_rows,
    const float *__restrict__ xs, float e2, const uint8_t *__restrict__ core_sorted,
    const uint8_t *__restrict__ cell_has_core, int32_t *parent, unsigned long long *__restrict__ pair_counter,
    int *err, const JobDev *__restrict__ jobs, const int32_t *__restrict__ cell_job,
    const int32_t *__restrict__ snap) {
    constexpr int P = Stride<D>::P;
    __shared__ __align__(16) float s_i[kWarpsPerBlock][kTile * P];
    __shared__ RowTable s_rows[kWarpsPerBlock];
    __shared__ int s_b[kWarpsPerBlock][kMaxCandCells];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t A64 = (int64_t)blockIdx.x * kWarpsPerBlock + wib;
    if (A64 >= n_cells) return;
    const int A = (int)A64;
    if (!cell_has_core[A]) return;
    if (jobs) e2 = jobs[cell_job[A]].e2;
    RowTable &rt = s_rows[wib];
    int *sb = s_b[wib];
    const int total = gather_rows<true>(nbr + (int64_t)A * n_rows, n_rows, cell_start, A + 1, rt, lane);
    if (total == 0) return;
    const int rootA = __ldg(snap + A);
    // Candidate cells, four per lane per step so that their loads overlap: a cell with
    // cores whose snapshot root differs from A's is a candidate
    constexpr int U = 4;
    int nb = 0;
    for (int tb = 0; tb < total; tb += kWarp * U) {
        int B[U], p[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int t = tb + u * kWarp + lane;
            B[u] = t < total ? row_lookup(rt, n_rows, t) : -1;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) p[u] = B[u] >= 0 ? __ldg(snap + B[u]) : -1;
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const bool ok = p[u] >= 0 && p[u] != rootA;
            const unsigned mask = __ballot_sync(kFull, ok);
            if (ok) {
                const int slot = nb + __popc(mask & lanemask_lt());
                if (slot < kMaxCandCells) sb[slot] = B[u];
            }
            nb += __popc(mask);
        }
    }
    __syncwarp();
    nb = min(nb, kMaxCandCells);
    unsigned long long pairs = 0;
    // Probe: A's first cores go to shared memory; each lane takes one candidate B
    // and tests B's first kProbe points against them.  Adjacent dense cells are
    // almost always settled here, in one lane-parallel round.
    {
        constexpr int P = Stride<D>::P;
        float *si = s_i[wib];
        const int a0 = cell_start[A], a1 = min(cell_start[A + 1], a0 + kWarp);
        const bool ok = a0 + lane < a1 && core_sorted[a0 + lane];
        const unsigned mask = __ballot_sync(kFull, ok);
        if (ok) {
            float x[D];
            load_point<D>(xs, a0 + lane, x);
            store_point_smem<D>(si + __popc(mask & lanemask_lt()) * P, x);
        }
        __syncwarp();
        const int nc0 = __popc(mask);
        for (int q = lane; q < nb; q += kWarp) {
            const int B = sb[q];
            const int b0 = cell_start[B], b1 = min(cell_start[B + 1], b0 + kProbe);
            bool hit = false;
            for (int j = b0; j < b1 && !hit; ++j) {
                if (!core_sorted[j]) continue;
                float xj[D];
                load_point<D>(xs, j, xj);
                for (int k = 0; k < nc0 && !hit; ++k) {
                    float xi[D];
                    load_point_smem<D>(si + k * P, xi);
                    hit = in_range<D>(xi, xj, e2);
                }
                pairs += (unsigned long long)nc0;
            }
            if (hit) {
                uf_union(parent, A, B, err);
                sb[q] = -1;
            }
        }
        __syncwarp();
    }
    for (int q = 0; q < nb; ++q) {
        const int B = sb[q];
        if (B < 0) continue;
        int same = 0;
        if (lane == 0) same = uf_find(parent, A, err) == uf_find(parent, B, err);
        if (__shfl_sync(kFull, same, 0)) continue;
        if (cells_touch<D>(A, B, cell_start, xs, core_sorted, e2, s_i[wib], lane, pairs) && lane == 0)
            uf_union(parent, A, B, err);
        __syncwarp();
    }
    if (lane == 0 && pairs) atomicAdd(pair_counter, pairs);
}

// ---------------------------------------------------------------------------
// Union-find over core points (general grids).  Pairs are visited once (j > i in
// sorted order); a pair whose j already shares i's root is skipped before the
// predicate.
// ---------------------------------------------------------------------------
template <int D>
__global__ void __launch_bounds__(kCountWarps * kWarp) union_points_kernel(
    const int2 *__restrict__ items, int64_t n_items, const int32_t *__restrict__ cell_start,
    const int2 *__restrict__ nbr, int n_rows, const float *__restrict__ xs, float e2,
    const uint8_t *__restrict__ core_sorted, const uint8_t *__restrict__ cell_has_core,
    int32_t *parent, unsigned long long *__restrict__ pair_counter, int *err, const JobDev *__restrict__ jobs,
    const int32_t *__restrict__ cell_job, const int32_t *__restrict__ cell_root) {
    constexpr int P = Stride<D>::P;
    __shared__ __align__(16) float s_i[kCountWarps][kTile * P];
    __shared__ int s_idx[kCountWarps][kTile];
    __shared__ int s_root[kCountWarps][kTile];
    __shared__ RowTable s_rows[kCountWarps];
    __shared__ RowTable s_cells[kCountWarps];
    __shared__ int s_need[kCountWarps][kWarp];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t item_id = (int64_t)blockIdx.x * kCountWarps + wib;
    if (item_id >= n_items) return;
    const int2 item = items[item_id];
    const int A = item.x, p0 = item.y;
    if (!cell_has_core[A]) return;
    if (jobs) e2 = jobs[cell_job[A]].e2;
    const int cnt = min(kTile, cell_start[A + 1] - p0);
    float *si = s_i[wib];
    int *sidx = s_idx[wib];
    int *sroot = s_root[wib];
    RowTable &rt = s_rows[wib];
    const int nc = load_item_cores<D>(xs, core_sorted, p0, cnt, true, si, sidx, lane);
    if (nc == 0) return;
    // Cell-level pass (cell_root: the one root of each cell's cores, -2 when they
    // differ, -1 without cores; taken after the list unions).  When the item's
    // cores share root r, every candidate cell whose cores all hang under r is
    // already joined to the item and is skipped whole; only the remaining cells'
    // points are scanned.  A stale cell root (a root since hooked elsewhere) only
    // makes a cell scanned, never skipped.
    int total = -1, rows = n_rows;
    if (cell_root) {
        const int myroot = lane < nc ? uf_find(parent, sidx[lane], err) : -1;
        const int root0 = __shfl_sync(kFull, myroot, 0);
        if (__all_sync(kFull, lane >= nc || myroot == root0)) {
            RowTable &rc = s_cells[wib];
            const int tcells = gather_rows<true>(nbr + (int64_t)A * n_rows, n_rows, cell_start, A, rc, lane);
            int n_need = 0;
            bool overflow = false;
            for (int cb = 0; cb < tcells; cb += kWarp) {
                const int t = cb + lane;
                const int c = t < tcells ? row_lookup(rc, n_rows, t) : -1;
                const bool need = c >= 0 && cell_has_core[c] && __ldg(cell_root + c) != root0;
                const unsigned m = __ballot_sync(kFull, need);
                if (n_need + __popc(m) > kWarp) {
                    overflow = true;
                    break;
                }
                if (need) s_need[wib][n_need + __popc(m & lanemask_lt())] = c;
                n_need += __popc(m);
            }
            __syncwarp();
            if (!overflow) {
                if (n_need == 0) return;
                int start = 0, len = 0;
                if (lane < n_need) {
                    const int c = s_need[wib][lane];
                    start = cell_start[c];
                    len = cell_start[c + 1] - start;
                }
                total = build_rows(start, len, n_need, rt, lane);
                rows = n_need;
            }
        }
    }
    if (total < 0) total = gather_rows<false>(nbr + (int64_t)A * n_rows, n_rows, cell_start, 0, rt, lane);
    unsigned long long pairs = 0;
    int cur = 0;  // this lane's stencil row
    // the next step's candidate, its core flag and its parent are loaded one step
    // ahead (independent loads), so their latency overlaps this step's root refresh
    // and tests; a parent read early is still an ancestor, so a stale one can only
    // cost an extra predicate, never a missed union
    int jn = lane < total ? row_next(rt, cur, lane) : -1;
    bool cn = false;
    int pn = -1;
    if (jn >= 0) {
        cn = core_sorted[jn] != 0;
        pn = __ldcg(parent + jn);
    }
    for (int tb = 0; tb < total; tb += kWarp) {
        const int j = jn;
        bool valid = j > p0 && cn;
        int pj = pn;
        {
            const int t = tb + kWarp + lane;
            jn = t < total ? row_next(rt, cur, t) : -1;
            cn = false;
            pn = -1;
            if (jn >= 0) {
                cn = core_sorted[jn] != 0;
                pn = __ldcg(parent + jn);
            }
        }
        // roots of the item's cores, refreshed every chunk so that candidates already
        // joined to them are skipped before the predicate
        int myroot = lane < nc ? uf_find(parent, sidx[lane], err) : -1;
        if (lane < nc) sroot[lane] = myroot;
        // one root for all of the item's cores (the usual case once they are joined)
        const int root0 = __shfl_sync(kFull, myroot, 0);
        const bool uniform = __all_sync(kFull, lane >= nc || myroot == root0);
        __syncwarp();
        float xj[D];
        if (valid) {
            pj = __ldcg(parent + pj);  // second hop: an ancestor of j, usually its root
            if (uniform && pj == root0) valid = false;  // joined to every core of the item already
        }
        if (!__any_sync(kFull, valid)) continue;
        if (valid) load_point<D>(xs, j, xj);
        else fill_nan<D>(xj);
        int tested = 0;
        for (int k = 0; k < nc; ++k) {
            const int ik = sidx[k];
            if constexpr (D >= 8) {
                // as in the count: the second half of the sum only when some lane's
                // first half is still within e2 (exact: partial sums only grow)
                const bool want = valid && j > ik && sroot[k] != pj;
                if (!__any_sync(kFull, want)) continue;
                float xi[D];
                load_point_smem<D>(si + k * P, xi);
                constexpr int H = D / 2;
                const float len = dist_part<D, 0, H>(xi, xj, 0.0f);
                bool hit = false;
                if (__any_sync(kFull, want && len <= e2)) hit = want && dist_part<D, H, D>(xi, xj, len) <= e2;
                tested += want ? 1 : 0;
                // finds from known ancestors: the core's root snapshot and pj; the
                // shared root that comes back is again an ancestor of j
                if (hit) pj = uf_union_root(parent, sroot[k], pj, err);
            } else if (valid && j > ik && sroot[k] != pj) {
                float xi[D];
                load_point_smem<D>(si + k * P, xi);
                ++tested;
                if (in_range<D>(xi, xj, e2)) pj = uf_union_root(parent, sroot[k], pj, err);
            }
        }
        pairs += (unsigned long long)__reduce_add_sync(kFull, (unsigned)tested);
        __syncwarp();
    }
    if (lane == 0 && pairs) atomicAdd(pair_counter, pairs);
}

// comp_min[root] = min core rank in the component.  Runs after flatten_kernel, so
// parent[u] is the root; lanes that share a root combine their minimum first and
// one lane per root issues the atomic (clusters have millions of cores).
__global__ void comp_min_kernel(int64_t nv, const uint8_t *__restrict__ core_sorted,
                                const int32_t *__restrict__ perm, const int32_t *__restrict__ pcell,
                                int cell_units, const uint32_t *__restrict__ core_bits,
                                const uint32_t *__restrict__ core_prefix, const int32_t *__restrict__ parent,
                                int32_t *__restrict__ comp_min) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool ok = s < nv && core_sorted[s];
    int root = -1, r = kNoCluster;
    if (ok) {
        root = parent[cell_units ? pcell[s] : (int)s];
        r = core_rank(core_bits, core_prefix, perm[s]);
    }
    unsigned pending = __ballot_sync(kFull, ok);
    const int lane = threadIdx.x & 31;
    while (pending) {
        const int leader = __ffs(pending) - 1;
        const int lroot = __shfl_sync(kFull, root, leader);
        const bool mine = ok && root == lroot;
        const int m = (int)__reduce_min_sync(kFull, mine ? (unsigned)r : (unsigned)kNoCluster);
        if (lane == leader) atomicMin(comp_min + lroot, m);
        pending &= ~__ballot_sync(kFull, mine);
    }
}

// Cell units: the smallest core rank of a cell is its first core's, because the
// stable radix sort (started from the identity permutation) keeps the points of a
// cell in input order.  One thread per cell instead of one per point: far fewer
// atomics on the roots of large clusters.  Lanes sharing a root combine first.
__global__ void comp_min_cells_kernel(int64_t n_cells, const int32_t *__restrict__ cell_start,
                                      const uint8_t *__restrict__ cell_has_core,
                                      const uint8_t *__restrict__ core_sorted, const int32_t *__restrict__ perm,
                                      const uint32_t *__restrict__ core_bits,
                                      const uint32_t *__restrict__ core_prefix, const int32_t *__restrict__ parent,
                                      int32_t *__restrict__ comp_min) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool ok = c < n_cells && cell_has_core[c];
    int root = -1, r = kNoCluster;
    if (ok) {
        int p = cell_start[c];
        while (!core_sorted[p]) ++p;  // the cell has a core
        root = parent[c];
        r = core_rank(core_bits, core_prefix, perm[p]);
    }
    unsigned pending = __ballot_sync(kFull, ok);
    const int lane = threadIdx.x & 31;
    while (pending) {
        const int leader = __ffs(pending) - 1;
        const int lroot = __shfl_sync(kFull, root, leader);
        const bool mine = ok && root == lroot;
        const int m = (int)__reduce_min_sync(kFull, mine ? (unsigned)r : (unsigned)kNoCluster);
        if (lane == leader) atomicMin(comp_min + lroot, m);
        pending &= ~__ballot_sync(kFull, mine);
    }
}

// The one root of each cell's cores (parent flattened): -1 without cores, -2 when
// they do not all share it.  One thread per point: the first core of a cell to
// arrive installs its root, any core with another root marks the cell mixed; a
// core whose root is already there skips the atomic.  cell_root starts at -1.
__global__ void cell_root_kernel(int64_t nv, const int32_t *__restrict__ pcell,
                                 const uint8_t *__restrict__ core_sorted, const int32_t *__restrict__ parent,
                                 int32_t *cell_root) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nv || !core_sorted[s]) return;
    const int c = pcell[s];
    const int r = parent[s];
    const int cur = __ldcg(cell_root + c);
    if (cur == r || cur == -2) return;
    const int old = cur == -1 ? atomicCAS(cell_root + c, -1, r) : cur;
    if (old != -1 && old != r) atomicExch(cell_root + c, -2);
}

// First step of the union: every core is joined to the cores among the first
// neighbours the count recorded for it (at most kListUnions of them; no distance
// test, each listed point is in range).  Point units join the points, cell units
// their cells.  Clusters are then nearly all linked, and the candidate scans that
// follow skip every candidate already under the same root.  With the early exit, the
// count skips the cells of >= min_pts points of a same-cell-linked grid and records no
// list there (skip_dense): those cells are joined by the near and cell passes.
#ifndef NDB_LIST_UNIONS
#define NDB_LIST_UNIONS 16
#endif
constexpr int kListUnions = NDB_LIST_UNIONS;  // a build-time choice
__global__ void union_lists_kernel(int64_t nv, const int32_t *__restrict__ nn_sorted,
                                   const int32_t *__restrict__ nbr_list, int list_cap, int list_stride,
                                   const uint8_t *__restrict__ core_sorted, int32_t *parent, int *err,
                                   const JobDev *__restrict__ jobs, const int32_t *__restrict__ cell_job,
                                   const int32_t *__restrict__ pcell, int cell_units, int skip_dense,
                                   const int32_t *__restrict__ cell_start, int min_pts) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nv || !core_sorted[s]) return;
    int cap = list_cap;
    if (jobs) {
        const JobDev &J = jobs[cell_job[pcell[s]]];
        cap = J.list_cap;
        min_pts = J.min_pts;
    }
    const int a = cell_units ? pcell[s] : (int)s;
    if (cell_units && skip_dense && cell_start[a + 1] - cell_start[a] >= min_pts) return;
    const int len = min(min(nn_sorted[s], cap), kListUnions);
    const int32_t *l = nbr_list + s * list_stride;
    // every union starts its find from the root the previous one left (an ancestor
    // of a), not from a itself
    int ra = a;
    for (int q = 0; q < len; ++q) {
        const int j = l[q];
        if (j == (int)s || !core_sorted[j]) continue;
        const int b = cell_units ? pcell[j] : j;
        if (a != b) ra = uf_union_root(parent, ra, b, err);
    }
}

// parent[u] = root of u.  Thread u is the only writer of parent[u] here (read-only
// finds), so after the kernel every parent is its root.
__global__ void flatten_kernel(int32_t *parent, int64_t n_units, int *err) {
    const int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n_units) return;
    const int r = uf_find_ro(parent, (int)u, err);
    parent[u] = r;
}

// The same, also recording each cell's root in snap (-1 for a cell without cores)
// for the candidate filter of union_cells_kernel.
__global__ void flatten_snap_kernel(int32_t *parent, int64_t n_units, int *err,
                                    const uint8_t *__restrict__ has_core, int32_t *__restrict__ snap) {
    const int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n_units) return;
    const int r = uf_find_ro(parent, (int)u, err);
    parent[u] = r;
    snap[u] = has_core[u] ? r : -1;
}

// ids of the cores in sorted order; counters[0] += component roots (point units)
__global__ void core_ids_kernel(int64_t nv, const uint8_t *__restrict__ core_sorted,
                                const int32_t *__restrict__ pcell, int cell_units,
                                const int32_t *__restrict__ parent, const int32_t *__restrict__ comp_min,
                                int32_t *__restrict__ ci_sorted, unsigned long long *__restrict__ counters,
                                const int32_t *__restrict__ cell_job, unsigned long long *__restrict__ job_counters) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned roots = 0;
    if (s < nv) {
        if (core_sorted[s]) {
            const int u = cell_units ? pcell[s] : (int)s;
            const int root = parent[u];
            ci_sorted[s] = comp_min[root];
            if (!cell_units && root == (int)s) {
                if (job_counters) atomicAdd(job_counters + 4 * cell_job[pcell[s]], 1ull);
                else roots = 1;
            }
        } else {
            ci_sorted[s] = kNoCluster;
        }
    }
    roots = __reduce_add_sync(kFull, roots);
    if ((threadIdx.x & 31) == 0 && roots) atomicAdd(counters + 0, (unsigned long long)roots);
}

// clusters over cells + the id of every cell's component
__global__ void cell_ids_kernel(int64_t n_cells, const uint8_t *__restrict__ cell_has_core,
                                const int32_t *__restrict__ parent, const int32_t *__restrict__ comp_min,
                                int32_t *__restrict__ cell_cid, unsigned long long *__restrict__ counters,
                                const int32_t *__restrict__ cell_job, unsigned long long *__restrict__ job_counters) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned roots = 0;
    if (c < n_cells) {
        if (cell_has_core[c]) {
            const int root = parent[c];
            cell_cid[c] = comp_min[root];
            if (root == (int)c) {
                if (job_counters) atomicAdd(job_counters + 4 * cell_job[c], 1ull);
                else roots = 1;
            }
        } else {
            cell_cid[c] = kNoCluster;
        }
    }
    roots = __reduce_add_sync(kFull, roots);
    if ((threadIdx.x & 31) == 0 && roots) atomicAdd(counters + 0, (unsigned long long)roots);
}

// ---------------------------------------------------------------------------
// Border points: every non-core point takes the minimum cluster id over the
// cores in range (data_process.cpp:204-209), NO_CLUSTER when there is none.
// Cell units: all cores of a cell share one id, so the warp lists the stencil's
// core cells with their ids, sorts them by id, and walks them in that order; a
// point is settled by the first cell that has a core in range, and the walk ends
// once every point of the item is settled or no cell can lower its minimum.
// Point units: the flattened candidates carry their own ids; the warp takes the
// minimum over the candidates in range.
// ---------------------------------------------------------------------------
template <int D>
__global__ void __launch_bounds__(kBlock) border_kernel(
    const int2 *__restrict__ items, int64_t n_items, const int32_t *__restrict__ cell_start,
    const int2 *__restrict__ nbr, int n_rows, const float *__restrict__ xs, float e2,
    const uint8_t *__restrict__ core_sorted, const uint8_t *__restrict__ cell_has_core, int cell_units,
    const int32_t *__restrict__ cell_cid, int32_t *__restrict__ ci_sorted,
    unsigned long long *__restrict__ pair_counter) {
    constexpr int P = Stride<D>::P;
    __shared__ __align__(16) float s_i[kWarpsPerBlock][kTile * P];
    __shared__ int s_idx[kWarpsPerBlock][kTile];
    __shared__ RowTable s_rows[kWarpsPerBlock];
    __shared__ int2 s_cand[kWarpsPerBlock][kMaxCandCells];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t item_id = (int64_t)blockIdx.x * kWarpsPerBlock + wib;
    if (item_id >= n_items) return;
    const int2 item = items[item_id];
    const int A = item.x, p0 = item.y;
    const int cnt = min(kTile, cell_start[A + 1] - p0);
    float *si = s_i[wib];
    int *sidx = s_idx[wib];
    RowTable &rt = s_rows[wib];
    const int nb = load_item_cores<D>(xs, core_sorted, p0, cnt, false, si, sidx, lane);
    if (nb == 0) return;
    int best[kTile];
#pragma unroll
    for (int k = 0; k < kTile; ++k) best[k] = kNoCluster;
    unsigned long long pairs = 0;
    if (cell_units) {
        int2 *cand = s_cand[wib];
        const int total = gather_rows<true>(nbr + (int64_t)A * n_rows, n_rows, cell_start, 0, rt, lane);
        int nc = 0;
        for (int tb = 0; tb < total; tb += kWarp) {
            const int t = tb + lane;
            int B = 0;
            bool ok = false;
            if (t < total) {
                B = row_lookup(rt, n_rows, t);
                ok = cell_has_core[B] != 0;
            }
            const unsigned mask = __ballot_sync(kFull, ok);
            if (ok) {
                const int slot = nc + __popc(mask & lanemask_lt());
                if (slot < kMaxCandCells) cand[slot] = make_int2(cell_cid[B], B);
            }
            nc += __popc(mask);
        }
        __syncwarp();
        nc = min(nc, kMaxCandCells);
        // Visit the candidate cells in increasing id order, lazily: each round takes
        // the smallest remaining id (warp min), and the walk ends once no pending
        // point can be lowered by it.  Lane l holds candidates l, l+32, ...
        constexpr int kPer = kMaxCandCells / kWarp;
        int lcid[kPer];
#pragma unroll
        for (int q = 0; q < kPer; ++q) {
            const int e = q * kWarp + lane;
            lcid[q] = e < nc ? cand[e].x : kNoCluster;
        }
        while (true) {
            int mloc = kNoCluster, qloc = kPer;
#pragma unroll
            for (int q = 0; q < kPer; ++q)
                if (lcid[q] < mloc) {
                    mloc = lcid[q];
                    qloc = q;
                }
            const int cid = (int)__reduce_min_sync(kFull, (unsigned)mloc);
            if (cid == kNoCluster) break;
            bool useful = false;
#pragma unroll
            for (int k = 0; k < kTile; ++k) useful = useful || (k < nb && cid < best[k]);
            if (!useful) break;  // ids only grow from here
            const int owner = __ffs(__ballot_sync(kFull, mloc == cid)) - 1;
            int B = 0;
            if (lane == owner) {
#pragma unroll
                for (int q = 0; q < kPer; ++q)
                    if (q == qloc) {
                        B = cand[q * kWarp + lane].y;
                        lcid[q] = kNoCluster;
                    }
            }
            B = __shfl_sync(kFull, B, owner);
            const int j0 = cell_start[B], j1 = cell_start[B + 1];
            for (int jb = j0; jb < j1; jb += kWarp) {
                const int j = jb + lane;
                float xj[D];
                if (j < j1 && core_sorted[j]) load_point<D>(xs, j, xj);
                else fill_nan<D>(xj);
                bool pending = false;
#pragma unroll
                for (int k = 0; k < kTile; ++k) {
                    if (k < nb && cid < best[k]) {
                        float xi[D];
                        load_point_smem<D>(si + k * P, xi);
                        if (__any_sync(kFull, in_range<D>(xi, xj, e2))) best[k] = cid;
                        else pending = true;
                    }
                }
                pairs += (unsigned long long)nb * (unsigned long long)min(kWarp, j1 - jb);
                if (!pending) break;
            }
        }
    } else {
        const int total = gather_rows<false>(nbr + (int64_t)A * n_rows, n_rows, cell_start, 0, rt, lane);
        int cur = 0;
        for (int tb = 0; tb < total; tb += kWarp) {
            const int t = tb + lane;
            int j = -1;
            if (t < total) j = row_next(rt, cur, t);
            const bool valid = j >= 0 && core_sorted[j];
            float xj[D];
            int cj = kNoCluster;
            if (valid) {
                load_point<D>(xs, j, xj);
                cj = ci_sorted[j];
            } else {
                fill_nan<D>(xj);
            }
#pragma unroll
            for (int k = 0; k < kTile; ++k) {
                if (k < nb) {
                    float xi[D];
                    load_point_smem<D>(si + k * P, xi);
                    const int v = (cj < best[k] && in_range<D>(xi, xj, e2)) ? cj : kNoCluster;
                    best[k] = min(best[k], (int)__reduce_min_sync(kFull, (unsigned)v));
                }
            }
            pairs += (unsigned long long)nb * (unsigned long long)min(kWarp, total - tb);
        }
    }
    int mine_best = kNoCluster;
#pragma unroll
    for (int k = 0; k < kTile; ++k)
        if (k == lane) mine_best = best[k];
    if (lane < nb) ci_sorted[sidx[lane]] = mine_best;
    if (lane == 0 && pairs) atomicAdd(pair_counter, pairs);
}

// ---------------------------------------------------------------------------
// Border points from the count's neighbour lists: a non-core point has fewer than
// min_pts points in range, all of them recorded by count_kernel, so its id is the
// minimum id over the cores among them -- no second stencil scan.
// ---------------------------------------------------------------------------
__global__ void border_list_kernel(int64_t nv, const int32_t *__restrict__ nn_sorted,
                                   const int32_t *__restrict__ nbr_list, int list_stride,
                                   const uint8_t *__restrict__ core_sorted, int cell_units,
                                   const int32_t *__restrict__ pcell, const int32_t *__restrict__ cell_cid,
                                   int32_t *__restrict__ ci_sorted, unsigned long long *__restrict__ pair_counter) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned looked = 0;
    if (s < nv && !core_sorted[s]) {
        const int cnt = min(nn_sorted[s], list_stride);
        int best = kNoCluster;
        for (int q = 0; q < cnt; ++q) {
            const int j = nbr_list[s * list_stride + q];
            if (core_sorted[j]) best = min(best, cell_units ? cell_cid[pcell[j]] : ci_sorted[j]);
        }
        looked = (unsigned)cnt;
        ci_sorted[s] = best;
    }
    looked = __reduce_add_sync(kFull, looked);
    if ((threadIdx.x & 31) == 0 && looked) atomicAdd(pair_counter, (unsigned long long)looked);
}

// Cluster ids in input order (the caller's output; out may be null) and the
// counts that need them: counters[1] += noise, counters[0] += cores outside the
// grid (possible only with min_pts <= 0: in range of nothing, each is a cluster
// of its own, numbered by its rank).
__global__ void output_ci_kernel(const int32_t *__restrict__ ci_sorted, int64_t nv, int64_t n,
                                 const int32_t *__restrict__ perm, const uint32_t *__restrict__ core_bits,
                                 const uint32_t *__restrict__ core_prefix, int32_t *__restrict__ out,
                                 unsigned long long *__restrict__ counters, const JobDev *__restrict__ jobs,
                                 int n_jobs, unsigned long long *__restrict__ job_counters, int64_t win_lo = 0,
                                 int64_t win_hi = INT64_MAX) {
    // windows as in scatter_nn_kernel; every point is counted in its own window only
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned noise = 0, roots = 0;
    int job = -1;  // batched runs: the point's job, whose counters take its noise and roots
    const int32_t o = s < n ? __ldcs(perm + s) : 0;
    if (s < n && o >= win_lo && o < win_hi) {
        int32_t v;
        if (s < nv) {
            v = __ldcs(ci_sorted + s);
        } else if (is_core_o(core_bits, o)) {
            v = core_rank(core_bits, core_prefix, o);
            roots = 1;
        } else {
            v = kNoCluster;
        }
        noise = v == kNoCluster;
        if (jobs) {
            // ids are ranks among all cores of the batch: make them ranks within the job
            job = job_of_point(jobs, n_jobs, o);
            const JobDev &J = jobs[job];
            if (v != kNoCluster) v -= core_rank(core_bits, core_prefix, (int32_t)J.off);
            if (J.ci_out) J.ci_out[o - J.off] = v;
        } else if (out) {
            out[o] = v;
        }
    }
    if (jobs) {
        // per-job counters: the lanes of one job (sorted points are grouped by job,
        // so usually the whole warp) add their noise and roots with one atomic each
        const unsigned peers = __match_any_sync(kFull, job);
        const unsigned nm = __ballot_sync(kFull, noise != 0) & peers, rm = __ballot_sync(kFull, roots != 0) & peers;
        if (job >= 0 && (int)(threadIdx.x & 31) == __ffs(peers) - 1) {
            if (nm) atomicAdd(job_counters + 4 * job + 1, (unsigned long long)__popc(nm));
            if (rm) atomicAdd(job_counters + 4 * job, (unsigned long long)__popc(rm));
        }
        noise = 0;
        roots = 0;
    }
    noise = __reduce_add_sync(kFull, noise);
    roots = __reduce_add_sync(kFull, roots);
    if ((threadIdx.x & 31) == 0) {
        if (noise) atomicAdd(counters + 1, (unsigned long long)noise);
        if (roots) atomicAdd(counters + 0, (unsigned long long)roots);
    }
}

// ndb_b200_assign_border: the caller's id of every core (input order) into the
// sorted ids and the cells' ids, which the border kernels read; non-cores start
// over at NO_CLUSTER.  The cores of one cell are one component, so they carry one id.
__global__ void set_core_ids_kernel(int64_t nv, const uint8_t *__restrict__ core_sorted,
                                    const int32_t *__restrict__ perm, const int32_t *__restrict__ ids,
                                    const int32_t *__restrict__ pcell, int cell_units, int32_t *__restrict__ ci_sorted,
                                    int32_t *__restrict__ cell_cid) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nv) return;
    if (core_sorted[s]) {
        const int32_t v = ids[perm[s]];
        ci_sorted[s] = v;
        if (cell_units) cell_cid[pcell[s]] = v;
    } else {
        ci_sorted[s] = kNoCluster;
    }
}

// Ids in input order after ndb_b200_assign_border: the border pass's ids, and the
// caller's for cores outside the grid.
__global__ void output_ids_kernel(const int32_t *__restrict__ ci_sorted, int64_t nv, int64_t n,
                                  const int32_t *__restrict__ perm, const uint32_t *__restrict__ core_bits,
                                  const int32_t *__restrict__ ids, int32_t *__restrict__ out) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int32_t o = perm[s];
    out[o] = s < nv ? ci_sorted[s] : (is_core_o(core_bits, o) ? ids[o] : kNoCluster);
}

// v_cluster_label in canonical form, on request: labels[rank(o)] = id of core o.
__global__ void labels_kernel(const int32_t *__restrict__ ci_sorted, int64_t nv, int64_t n,
                              const int32_t *__restrict__ perm, const uint32_t *__restrict__ core_bits,
                              const uint32_t *__restrict__ core_prefix, int32_t *__restrict__ labels) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int32_t o = perm[s];
    if (!is_core_o(core_bits, o)) return;
    const int32_t r = core_rank(core_bits, core_prefix, o);
    labels[r] = s < nv ? ci_sorted[s] : r;
}


// ---------------------------------------------------------------------------
// Batched runs: per-job bounding boxes, the concatenation of the jobs'
// coordinates, composite cell keys and the cell -> job map.  blockIdx.y is the job.
// ---------------------------------------------------------------------------
template <int D>
__global__ void __launch_bounds__(kBlock) gather_jobs_kernel(const JobDev *__restrict__ jobs,
                                                             float *__restrict__ coords) {
    const JobDev &J = jobs[blockIdx.y];
    const int64_t total = J.n * D;
    float *dst = coords + J.off * D;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = J.src[i];
}

__global__ void bbox_batch_init_kernel(int *lo_hi, int d, int n_jobs, unsigned long long *n_invalid) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < (int64_t)n_jobs * d) {
        const int64_t j = i / d, k = i - j * d;
        lo_hi[j * 2 * d + k] = 0x7fffffff;
        lo_hi[j * 2 * d + d + k] = (int)0x80000000;
    }
    if (i < n_jobs) n_invalid[i] = 0ull;
}

// One point's coordinates: 16-byte vector loads when a point's row is a multiple of
// 16 bytes (d % 4 == 0; rows then start 16-byte aligned), 8-byte ones at d = 2.
template <int D>
__device__ __forceinline__ void load_row(const float *__restrict__ p, float (&x)[D]) {
    if constexpr (D % 4 == 0) {
#pragma unroll
        for (int q = 0; q < D / 4; ++q) {
            const float4 v = __ldg(reinterpret_cast<const float4 *>(p) + q);
            x[4 * q + 0] = v.x;
            x[4 * q + 1] = v.y;
            x[4 * q + 2] = v.z;
            x[4 * q + 3] = v.w;
        }
    } else if constexpr (D == 2) {
        const float2 v = __ldg(reinterpret_cast<const float2 *>(p));
        x[0] = v.x;
        x[1] = v.y;
    } else {
#pragma unroll
        for (int k = 0; k < D; ++k) x[k] = __ldg(p + k);
    }
}

// Per-job bounding boxes (ordered-int min/max per dimension) and invalid-point counts
// of a batch: blocks (x, job).  Warps reduce by shuffles, the block through shared
// memory, and one lane per dimension and bound issues the block's atomic.
template <int D>
__global__ void __launch_bounds__(kBlock) bbox_batch_kernel(const float *__restrict__ coords,
                                                            const JobDev *__restrict__ jobs, int *lo_hi,
                                                            unsigned long long *n_invalid) {
    constexpr int W = kBlock / 32;
    __shared__ int s_lh[W][2 * D];
    __shared__ unsigned s_bad[W];
    const int j = blockIdx.y;
    const JobDev &J = jobs[j];
    int lo[D], hi[D];
#pragma unroll
    for (int k = 0; k < D; ++k) {
        lo[k] = 0x7fffffff;
        hi[k] = (int)0x80000000;
    }
    unsigned bad = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < J.n; i += (int64_t)gridDim.x * blockDim.x) {
        float x[D];
        load_row<D>(coords + (J.off + i) * D, x);
        bool ok = x[0] != FLT_MAX;
#pragma unroll
        for (int k = 0; k < D; ++k) ok = ok && isfinite(x[k]);
        if (!ok) {
            ++bad;
            continue;
        }
#pragma unroll
        for (int k = 0; k < D; ++k) {
            const int v = ordered_int(x[k]);
            lo[k] = min(lo[k], v);
            hi[k] = max(hi[k], v);
        }
    }
#pragma unroll
    for (int k = 0; k < D; ++k) {
        lo[k] = __reduce_min_sync(kFull, lo[k]);
        hi[k] = __reduce_max_sync(kFull, hi[k]);
    }
    bad = __reduce_add_sync(kFull, bad);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < D; ++k) {
            s_lh[w][k] = lo[k];
            s_lh[w][D + k] = hi[k];
        }
        s_bad[w] = bad;
    }
    __syncthreads();
    if (threadIdx.x < 2 * D) {
        const int t = threadIdx.x;
        int v = s_lh[0][t];
        for (int q = 1; q < W; ++q) v = t < D ? min(v, s_lh[q][t]) : max(v, s_lh[q][t]);
        int *lh = lo_hi + (int64_t)j * 2 * D;
        if (t < D) {
            if (v != 0x7fffffff) atomicMin(lh + t, v);
        } else {
            if (v != (int)0x80000000) atomicMax(lh + t, v);
        }
    }
    if (threadIdx.x == 0) {
        unsigned b = 0;
        for (int q = 0; q < W; ++q) b += s_bad[q];
        if (b) atomicAdd(n_invalid + j, (unsigned long long)b);
    }
}

template <int D, typename K>
__global__ void __launch_bounds__(kBlock) key_batch_kernel(const float *__restrict__ coords,
                                                           const JobDev *__restrict__ jobs, K invalid_key,
                                                           K *__restrict__ keys, int32_t *__restrict__ ids) {
    const JobDev &J = jobs[blockIdx.y];
    const GridDev g = J.g;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < J.n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t o = J.off + i;
        const float *p = coords + o * D;
        K key = invalid_key;
        float x[D];  // validity from one vector load of the row; the gridded coordinates are re-read (L1)
        load_row<D>(p, x);
        bool ok = x[0] != FLT_MAX;
#pragma unroll
        for (int k = 0; k < D; ++k) ok = ok && isfinite(x[k]);
        if (ok) {
            unsigned long long kk = J.key_base;
#pragma unroll
            for (int a = 0; a < kMaxGridDims; ++a)
                if (a < g.k) kk += (unsigned long long)cell_coord(g, a, p[g.dim[a]]) * g.stride[a];
            key = (K)kk;
        }
        keys[o] = key;
        ids[o] = (int32_t)o;
    }
}

// job of every cell: the last job whose key range starts at or below the cell key
// (every job of a pipeline owns a non-empty key range, so the bases increase)
template <typename K>
__global__ void cell_job_kernel(const K *__restrict__ cell_key, int64_t n_cells, const JobDev *__restrict__ jobs,
                                int n_jobs, int32_t *__restrict__ cell_job) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_cells) return;
    const unsigned long long key = (unsigned long long)cell_key[c];
    int lo = 0, hi = n_jobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (jobs[mid].key_base <= key) lo = mid;
        else hi = mid - 1;
    }
    cell_job[c] = lo;
}

// cores of every job: rank of the job's end minus rank of its start
__global__ void job_cores_kernel(const JobDev *__restrict__ jobs, int n_jobs, const uint32_t *__restrict__ core_bits,
                                 const uint32_t *__restrict__ core_prefix, int64_t n_total,
                                 unsigned long long *__restrict__ job_counters) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n_jobs) return;
    const JobDev &J = jobs[j];
    const int64_t end = J.off + J.n;
    const int32_t r0 = core_rank(core_bits, core_prefix, (int32_t)J.off);
    const int32_t r1 = end < n_total ? core_rank(core_bits, core_prefix, (int32_t)end)
                                     : (int32_t)(core_prefix[(n_total - 1) >> 5] +
                                                 __popc(core_bits[(n_total - 1) >> 5] &
                                                        (0xffffffffu >> (31 - ((n_total - 1) & 31)))));
    job_counters[4 * j + 2] = (unsigned long long)(r1 - r0);
}

}  // namespace ndb
