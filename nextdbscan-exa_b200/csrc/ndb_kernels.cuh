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

#include "ndb_common.cuh"

namespace ndb {

// Grid description passed by value to the kernels.
struct GridDev {
    int k;                   // gridded dimensions (1..3)
    int dim[3];              // input dimension of each gridded dimension
    double lo[3];            // origin per gridded dimension
    double inv_w[3];         // 1 / cell width
    long long g[3];          // cells per gridded dimension
    unsigned long long stride[3];  // key strides (1, g0, g0*g1)
};

// Neighbour rows of a cell.  Row r covers the cells at offsets (x in
// [-xr, +xr], o1, o2) in gridded dimensions (0, 1, 2); those cells have
// consecutive keys, hence form one contiguous run of the sorted cell list.
struct Stencil {
    int n_rows;
    int4 rows[kMaxRows];  // (o1, o2, xr, unused), nearest rows first
};

constexpr int kBlock = 256;
constexpr int kWarpsPerBlock = kBlock / kWarp;

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

__global__ void bbox_init_kernel(int *lo_hi, int d, unsigned long long *n_invalid) {
    const int t = threadIdx.x;
    if (t < d) {
        lo_hi[t] = 0x7fffffff;
        lo_hi[d + t] = (int)0x80000000;
    }
    if (t == 0) *n_invalid = 0ull;
}

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
        for (int a = 0; a < g.k; ++a)
            kk += (unsigned long long)cell_coord(g, a, p[g.dim[a]]) * g.stride[a];
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

template <typename K>
__device__ __forceinline__ int64_t lower_bound_key(const K *__restrict__ a, int64_t n, unsigned long long key) {
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if ((unsigned long long)__ldg(a + mid) < key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// nbr[c * n_rows + r] = [first, last) cell index of row r around cell c.
template <typename K>
__global__ void __launch_bounds__(kBlock) rows_kernel(const K *__restrict__ cell_key, int64_t n_cells,
                                                      GridDev g, Stencil st, int2 *__restrict__ nbr) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n_cells * st.n_rows) return;
    const int64_t c = idx / st.n_rows;
    const int r = (int)(idx - c * st.n_rows);
    const unsigned long long key = (unsigned long long)cell_key[c];
    long long cc[3] = {0, 0, 0};
    unsigned long long rest = key;
    for (int a = 0; a < g.k; ++a) {
        if (a == g.k - 1) {
            cc[a] = (long long)rest;
        } else {
            cc[a] = (long long)(rest % (unsigned long long)g.g[a]);
            rest /= (unsigned long long)g.g[a];
        }
    }
    const int4 row = st.rows[r];
    const long long y = cc[1] + row.x, z = cc[2] + row.y;
    int2 out = make_int2(0, 0);
    const bool in = (g.k < 2 || (y >= 0 && y < g.g[1])) && (g.k < 3 || (z >= 0 && z < g.g[2]));
    if (in) {
        const long long x0 = cc[0] - row.z < 0 ? 0 : cc[0] - row.z;
        const long long x1 = cc[0] + row.z > g.g[0] - 1 ? g.g[0] - 1 : cc[0] + row.z;
        unsigned long long base = 0;
        if (g.k >= 2) base += (unsigned long long)y * g.stride[1];
        if (g.k >= 3) base += (unsigned long long)z * g.stride[2];
        const int64_t ca = lower_bound_key(cell_key, n_cells, base + (unsigned long long)x0);
        const int64_t cb = lower_bound_key(cell_key, n_cells, base + (unsigned long long)x1 + 1ull);
        out = make_int2((int)ca, (int)cb);
    }
    nbr[idx] = out;
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
// Neighbour count.  One warp per item (up to 32 points i of one cell).  The i
// points sit in shared memory; lanes walk the candidate points j of the
// stencil rows 32 at a time (coalesced loads), every lane tests its j against
// each i (broadcast reads) and the warp adds popc(ballot) to that i's count.
// EARLY: stop once every i of the item has reached min_pts (exact counts below
// min_pts, so exact core flags).  dense_skip: with same-cell-linked cells a cell
// of >= min_pts points is all cores (every pair inside it is in range), so its
// points need no test at all; they report the cell size.
// ---------------------------------------------------------------------------
template <int D, bool EARLY>
__global__ void __launch_bounds__(kBlock) count_kernel(
    const int2 *__restrict__ items, int64_t n_items, const int32_t *__restrict__ cell_start,
    const int2 *__restrict__ nbr, int n_rows, const float *__restrict__ xs, float e2, int min_pts,
    int dense_skip, int32_t *__restrict__ nn_sorted, unsigned long long *__restrict__ pair_counter) {
    constexpr int P = Stride<D>::P;
    __shared__ __align__(16) float s_i[kWarpsPerBlock][kTile * P];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t item_id = (int64_t)blockIdx.x * kWarpsPerBlock + wib;
    if (item_id >= n_items) return;
    const int2 item = items[item_id];
    const int cell = item.x, p0 = item.y;
    const int cs = cell_start[cell], ce = cell_start[cell + 1];
    const int cnt = min(kTile, ce - p0);
    if (EARLY && dense_skip && ce - cs >= min_pts) {
        if (lane < cnt) nn_sorted[p0 + lane] = ce - cs;
        return;
    }
    float *si = s_i[wib];
    if (lane < cnt) {
        float x[D];
        load_point<D>(xs, p0 + lane, x);
        store_point_smem<D>(si + lane * P, x);
    }
    __syncwarp();
    int c[kTile];
#pragma unroll
    for (int k = 0; k < kTile; ++k) c[k] = 0;
    unsigned long long pairs = 0;
    const int2 *cr = nbr + (int64_t)cell * n_rows;
    for (int r = 0; r < n_rows; ++r) {
        const int2 range = cr[r];
        if (range.x >= range.y) continue;
        const int j0 = cell_start[range.x], j1 = cell_start[range.y];
        bool done = false;
        for (int jb = j0; jb < j1; jb += kWarp) {
            const int j = jb + lane;
            float xj[D];
            if (j < j1) load_point<D>(xs, j, xj);
            else fill_nan<D>(xj);  // NaN fails the predicate
#pragma unroll
            for (int k = 0; k < kTile; ++k) {
                if (k < cnt) {
                    float xi[D];
                    load_point_smem<D>(si + k * P, xi);
                    c[k] += __popc(__ballot_sync(kFull, in_range<D>(xi, xj, e2)));
                }
            }
            pairs += (unsigned long long)cnt * (unsigned long long)min(kWarp, j1 - jb);
            if (EARLY) {
                bool all = true;
#pragma unroll
                for (int k = 0; k < kTile; ++k) all = all && (k >= cnt || c[k] >= min_pts);
                if (all) {
                    done = true;
                    break;
                }
            }
        }
        if (done) break;
    }
    int mine = 0;
#pragma unroll
    for (int k = 0; k < kTile; ++k)
        if (k == lane) mine = c[k];
    if (lane < cnt) nn_sorted[p0 + lane] = mine;
    if (lane == 0 && pairs) atomicAdd(pair_counter, pairs);
}

// core flags in sorted and in input order; nn in input order
__global__ void core_flags_kernel(const int32_t *__restrict__ nn_sorted, int64_t nv, int64_t n, int min_pts,
                                  const int32_t *__restrict__ perm, const int32_t *__restrict__ pcell,
                                  uint8_t *__restrict__ core_sorted, uint8_t *__restrict__ cell_has_core,
                                  int32_t *__restrict__ nn_orig, uint32_t *__restrict__ core_orig) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int32_t o = perm[s];
    if (s < nv) {
        const int32_t v = nn_sorted[s];
        const bool core = v >= min_pts;
        core_sorted[s] = core ? 1 : 0;
        if (core) cell_has_core[pcell[s]] = 1;
        nn_orig[o] = v;
        core_orig[o] = core ? 1u : 0u;
    } else {
        nn_orig[o] = 0;
        core_orig[o] = (0 >= min_pts) ? 1u : 0u;
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

// ---------------------------------------------------------------------------
// Union-find over cells (same-cell-linked grids): every pair inside a cell is in
// range, so all cores of a cell belong to one component and the cell is the
// union-find element.  Each item (cores of one chunk of cell A) looks at the
// cells B > A of its stencil rows that hold cores and whose root differs from
// A's, and links A and B as soon as one core pair is in range.
// ---------------------------------------------------------------------------
template <int D>
__global__ void __launch_bounds__(kBlock) union_cells_kernel(
    const int2 *__restrict__ items, int64_t n_items, const int32_t *__restrict__ cell_start,
    const int2 *__restrict__ nbr, int n_rows, const float *__restrict__ xs, float e2,
    const uint8_t *__restrict__ core_sorted, const uint8_t *__restrict__ cell_has_core,
    int32_t *parent, unsigned long long *__restrict__ pair_counter, int *err) {
    constexpr int P = Stride<D>::P;
    __shared__ __align__(16) float s_i[kWarpsPerBlock][kTile * P];
    __shared__ int s_idx[kWarpsPerBlock][kTile];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t item_id = (int64_t)blockIdx.x * kWarpsPerBlock + wib;
    if (item_id >= n_items) return;
    const int2 item = items[item_id];
    const int A = item.x, p0 = item.y;
    if (!cell_has_core[A]) return;
    const int cnt = min(kTile, cell_start[A + 1] - p0);
    float *si = s_i[wib];
    const int nc = load_item_cores<D>(xs, core_sorted, p0, cnt, true, si, s_idx[wib], lane);
    if (nc == 0) return;
    unsigned long long pairs = 0;
    const int2 *cr = nbr + (int64_t)A * n_rows;
    for (int r = 0; r < n_rows; ++r) {
        const int2 range = cr[r];
        for (int B = max(range.x, A + 1); B < range.y; ++B) {
            if (!cell_has_core[B]) continue;
            int same = 0;
            if (lane == 0) same = uf_find(parent, A, err) == uf_find(parent, B, err);
            if (__shfl_sync(kFull, same, 0)) continue;
            const int j0 = cell_start[B], j1 = cell_start[B + 1];
            bool found = false;
            for (int jb = j0; jb < j1 && !found; jb += kWarp) {
                const int j = jb + lane;
                float xj[D];
                if (j < j1 && core_sorted[j]) load_point<D>(xs, j, xj);
                else fill_nan<D>(xj);
                bool hit = false;
                for (int k = 0; k < nc; ++k) {
                    float xi[D];
                    load_point_smem<D>(si + k * P, xi);
                    hit = hit || in_range<D>(xi, xj, e2);
                }
                pairs += (unsigned long long)nc * (unsigned long long)min(kWarp, j1 - jb);
                found = __any_sync(kFull, hit);
            }
            if (found && lane == 0) uf_union(parent, A, B, err);
        }
    }
    if (lane == 0 && pairs) atomicAdd(pair_counter, pairs);
}

// ---------------------------------------------------------------------------
// Union-find over core points (general grids).  Pairs are visited once
// (j > i in sorted order); a pair whose j already shares i's root is skipped
// before the predicate.
// ---------------------------------------------------------------------------
template <int D>
__global__ void __launch_bounds__(kBlock) union_points_kernel(
    const int2 *__restrict__ items, int64_t n_items, const int32_t *__restrict__ cell_start,
    const int2 *__restrict__ nbr, int n_rows, const float *__restrict__ xs, float e2,
    const uint8_t *__restrict__ core_sorted, const uint8_t *__restrict__ cell_has_core,
    int32_t *parent, unsigned long long *__restrict__ pair_counter, int *err) {
    constexpr int P = Stride<D>::P;
    __shared__ __align__(16) float s_i[kWarpsPerBlock][kTile * P];
    __shared__ int s_idx[kWarpsPerBlock][kTile];
    __shared__ int s_root[kWarpsPerBlock][kTile];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t item_id = (int64_t)blockIdx.x * kWarpsPerBlock + wib;
    if (item_id >= n_items) return;
    const int2 item = items[item_id];
    const int A = item.x, p0 = item.y;
    if (!cell_has_core[A]) return;
    const int cnt = min(kTile, cell_start[A + 1] - p0);
    float *si = s_i[wib];
    int *sidx = s_idx[wib];
    int *sroot = s_root[wib];
    const int nc = load_item_cores<D>(xs, core_sorted, p0, cnt, true, si, sidx, lane);
    if (nc == 0) return;
    unsigned long long pairs = 0;
    const int2 *cr = nbr + (int64_t)A * n_rows;
    for (int r = 0; r < n_rows; ++r) {
        const int2 range = cr[r];
        if (range.x >= range.y) continue;
        const int j0 = max(cell_start[range.x], p0 + 1), j1 = cell_start[range.y];
        if (lane < nc) sroot[lane] = uf_find(parent, sidx[lane], err);
        __syncwarp();
        for (int jb = j0; jb < j1; jb += kWarp) {
            const int j = jb + lane;
            const bool valid = j < j1 && core_sorted[j];
            float xj[D];
            int pj = -1;
            if (valid) {
                load_point<D>(xs, j, xj);
                pj = __ldcg(parent + j);
            } else {
                fill_nan<D>(xj);
            }
            for (int k = 0; k < nc; ++k) {
                const int ik = sidx[k];
                if (valid && j > ik && sroot[k] != pj) {
                    float xi[D];
                    load_point_smem<D>(si + k * P, xi);
                    if (in_range<D>(xi, xj, e2)) {
                        uf_union(parent, ik, j, err);
                        pj = uf_find(parent, j, err);
                    }
                }
            }
            pairs += (unsigned long long)nc * (unsigned long long)min(kWarp, j1 - jb);
        }
        __syncwarp();
    }
    if (lane == 0 && pairs) atomicAdd(pair_counter, pairs);
}

// comp_min[root] = min core rank in the component
__global__ void comp_min_kernel(int64_t nv, const uint8_t *__restrict__ core_sorted,
                                const int32_t *__restrict__ perm, const int32_t *__restrict__ pcell,
                                int cell_units, const uint32_t *__restrict__ rank, int32_t *parent,
                                int32_t *__restrict__ comp_min, int *err) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nv || !core_sorted[s]) return;
    const int u = cell_units ? pcell[s] : (int)s;
    const int root = uf_find(parent, u, err);
    atomicMin(comp_min + root, (int32_t)rank[perm[s]]);
}

__global__ void flatten_kernel(int32_t *parent, int64_t n_units, int *err) {
    const int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n_units) return;
    const int r = uf_find(parent, (int)u, err);
    parent[u] = r;
}

// counters[0] = clusters (roots), counters[1] = noise
__global__ void core_ids_kernel(int64_t nv, int64_t n, const uint8_t *__restrict__ core_sorted,
                                const int32_t *__restrict__ perm, const int32_t *__restrict__ pcell,
                                int cell_units, const int32_t *__restrict__ parent,
                                const int32_t *__restrict__ comp_min, const uint32_t *__restrict__ rank,
                                const uint32_t *__restrict__ core_orig, int32_t *__restrict__ ci_sorted,
                                int32_t *__restrict__ ci_orig, unsigned long long *__restrict__ counters) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned roots = 0;
    if (s < nv) {
        if (core_sorted[s]) {
            const int u = cell_units ? pcell[s] : (int)s;
            const int root = parent[u];
            const int32_t cid = comp_min[root];
            ci_sorted[s] = cid;
            ci_orig[perm[s]] = cid;
            if (!cell_units && root == (int)s) roots = 1;
        } else {
            ci_sorted[s] = kNoCluster;
        }
    } else if (s < n) {
        // points outside the grid: in range of nothing, so a core among them (only
        // possible with min_pts <= 0) is a cluster of its own
        const int32_t o = perm[s];
        if (core_orig[o]) {
            ci_orig[o] = (int32_t)rank[o];
            roots = 1;
        } else {
            ci_orig[o] = kNoCluster;
        }
    }
    roots = __reduce_add_sync(kFull, roots);
    if ((threadIdx.x & 31) == 0 && roots) atomicAdd(counters + 0, (unsigned long long)roots);
}

// clusters over cells + the id of every cell's component
__global__ void cell_ids_kernel(int64_t n_cells, const uint8_t *__restrict__ cell_has_core,
                                const int32_t *__restrict__ parent, const int32_t *__restrict__ comp_min,
                                int32_t *__restrict__ cell_cid, unsigned long long *__restrict__ counters) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned roots = 0;
    if (c < n_cells) {
        if (cell_has_core[c]) {
            const int root = parent[c];
            cell_cid[c] = comp_min[root];
            if (root == (int)c) roots = 1;
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
// With cell units all cores of a cell share one id, so a cell is skipped when
// its id cannot lower any pending minimum, and its scan stops at the first hit.
// ---------------------------------------------------------------------------
template <int D>
__global__ void __launch_bounds__(kBlock) border_kernel(
    const int2 *__restrict__ items, int64_t n_items, const int32_t *__restrict__ cell_start,
    const int2 *__restrict__ nbr, int n_rows, const float *__restrict__ xs, float e2,
    const uint8_t *__restrict__ core_sorted, const uint8_t *__restrict__ cell_has_core, int cell_units,
    const int32_t *__restrict__ cell_cid, const int32_t *__restrict__ perm, int32_t *__restrict__ ci_sorted,
    int32_t *__restrict__ ci_orig, unsigned long long *__restrict__ pair_counter) {
    constexpr int P = Stride<D>::P;
    __shared__ __align__(16) float s_i[kWarpsPerBlock][kTile * P];
    __shared__ int s_idx[kWarpsPerBlock][kTile];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t item_id = (int64_t)blockIdx.x * kWarpsPerBlock + wib;
    if (item_id >= n_items) return;
    const int2 item = items[item_id];
    const int A = item.x, p0 = item.y;
    const int cnt = min(kTile, cell_start[A + 1] - p0);
    float *si = s_i[wib];
    int *sidx = s_idx[wib];
    const int nb = load_item_cores<D>(xs, core_sorted, p0, cnt, false, si, sidx, lane);
    if (nb == 0) return;
    int best[kTile];
#pragma unroll
    for (int k = 0; k < kTile; ++k) best[k] = kNoCluster;
    unsigned long long pairs = 0;
    const int2 *cr = nbr + (int64_t)A * n_rows;
    for (int r = 0; r < n_rows; ++r) {
        const int2 range = cr[r];
        if (range.x >= range.y) continue;
        if (cell_units) {
            for (int B = range.x; B < range.y; ++B) {
                if (!cell_has_core[B]) continue;
                const int cid = cell_cid[B];
                bool useful = false;
#pragma unroll
                for (int k = 0; k < kTile; ++k) useful = useful || (k < nb && cid < best[k]);
                if (!useful) continue;
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
            const int j0 = cell_start[range.x], j1 = cell_start[range.y];
            for (int jb = j0; jb < j1; jb += kWarp) {
                const int j = jb + lane;
                const bool valid = j < j1 && core_sorted[j];
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
                pairs += (unsigned long long)nb * (unsigned long long)min(kWarp, j1 - jb);
            }
        }
    }
    int mine = kNoCluster;
#pragma unroll
    for (int k = 0; k < kTile; ++k)
        if (k == lane) mine = best[k];
    if (lane < nb) {
        const int s = sidx[lane];
        ci_sorted[s] = mine;
        ci_orig[perm[s]] = mine;
    }
    if (lane == 0 && pairs) atomicAdd(pair_counter, pairs);
}

// counters[1] += noise points; labels[rank[o]] = ci[o] for cores
__global__ void meta_kernel(int64_t n, const int32_t *__restrict__ ci_orig, const uint32_t *__restrict__ core_orig,
                            const uint32_t *__restrict__ rank, int32_t *__restrict__ labels,
                            unsigned long long *__restrict__ counters) {
    const int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned noise = 0;
    if (o < n) {
        const int32_t c = ci_orig[o];
        if (c == kNoCluster) noise = 1;
        if (core_orig[o]) labels[rank[o]] = c;
    }
    noise = __reduce_add_sync(kFull, noise);
    if ((threadIdx.x & 31) == 0 && noise) atomicAdd(counters + 1, (unsigned long long)noise);
}

}  // namespace ndb
