// ndb_api.cu -- context, grid planning and the extern "C" entry points of
// libndb_b200.so (declared in include/ndb_b200.h).
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <condition_variable>
#include <deque>
#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/ndb_b200.h"
#include "ndb_internal.h"
#include "ndb_kernels.cuh"
#include "ndb_tc.cuh"

using namespace ndb;

#define NDB_VERSION "0.1.0"

struct ndb_ctx {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    // ndb_b200_run with host outputs: the counts go back to the host on this stream
    // while the label phase runs on `stream`
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_nn = nullptr;
    bool in_run = false;     // classify is the first half of ndb_b200_run
    bool nn_pending = false; // a count copy on copy_stream not yet waited for
    bool stats_pending = false; // classify's counters are read by the label phase
    std::string last_cuda_error;

    // inputs / per-point arrays
    DevBuf coords, keys0, keys1, ids0, ids1, flags, pos, pcell, xs;
    DevBuf nn_sorted, nn_orig, core_sorted, core_bits, core_prefix, ci_sorted, ci_orig, labels;
    // per-cell arrays
    DevBuf cell_start, cell_key, nbr, item_cnt, items, cell_has_core, cell_cid, hash_keys, hash_vals;
    // column table of the grid (CellIndex): one [first, end) cell range per column
    DevBuf col_range;
    size_t col_budget = size_t(1) << 27;  // largest column table (entries) a run may build, else the hash table
    bool use_cols = false;                // the current job's cells are found through the column table
    // union-find
    DevBuf parent, comp_min;
    // neighbour lists of the points whose count stays below min_pts (border step)
    DevBuf nbr_list;
    size_t list_budget = size_t(8) << 30;  // largest list buffer the context may use (else: scan border)
    int list_cap = 0;                 // entries per point, 0 when the lists are off
    bool tc_count = false;            // neighbour count on the tensor-core filter
    bool gram_count = false;          // CUDA-core count with the Gram filter (d >= 8)
    int sm_count = 148;
    // scratch
    DevBuf sort_hist, scan_scratch, small;  // small: counters, bbox, scalars
    // batched runs: job table, per-job bounding boxes, cell -> job, per-job counters
    DevBuf jobs_dev, batch_bbox, cell_job, job_counters;
    // items split between the tensor-core count (full items) and the exact one, and
    // the tensor count's per-item records
    DevBuf items_split, tc_rec;
    // caller's core ids of ndb_b200_assign_border (host inputs)
    DevBuf ids_in;
    // batched runs on host buffers: every job's coordinates and outputs on the device
    DevBuf batch_in, batch_nn, batch_ci;
    cudaEvent_t ev_grp[NDB_MAX_DIM + 1] = {};   // a group's inputs are on the device
    cudaEvent_t ev_done[NDB_MAX_DIM + 2] = {};  // a group's outputs are ready (last: the solo jobs')
    // batched runs: the pipelines' small host <-> device transfers (job tables,
    // bounding boxes, sizes, counters) go through this mapped pinned buffer with copy
    // kernels, so they never queue behind the copy engines' transfers of the other
    // groups' inputs and outputs
    char *mail = nullptr;      // host address; the device reads and writes it (mapped)
    char *mail_dev = nullptr;  // its device address
    size_t mail_bytes = 0, mail_used = 0;
    // ndb_b200_load_bin: two pinned staging chunks, the loaded job (its coordinates in
    // `coords`) and its bounding box, reduced chunk by chunk while it arrived
    void *pin[2] = {nullptr, nullptr};
    size_t pin_bytes = 0;
    cudaEvent_t ev_pin[2] = {nullptr, nullptr};
    DevBuf load_box;
    bool loaded = false;
    int64_t loaded_n = 0;
    int loaded_d = 0;
    // largest device footprint the context may hold (bytes); 0 = no cap
    size_t mem_limit = 0;
    // count-kernel thresholds set by ndb_b200_set_tuning (0: the library's defaults)
    ndb_tuning tuning{0, 0, 0};
    // bound of the device-side union-find loops (ndb_b200_set_debug_limits; 0: kUfMaxSteps)
    int uf_max_steps = 0;

    template <typename F>
    void for_each_buf(F f) {
        DevBuf *bufs[] = {&coords,      &keys0,       &keys1,       &ids0,        &ids1,        &flags,
                          &pos,         &pcell,       &xs,          &nn_sorted,   &nn_orig,     &core_sorted,
                          &core_bits,   &core_prefix, &ci_sorted,   &ci_orig,     &labels,      &cell_start,
                          &cell_key,    &nbr,         &item_cnt,    &items,       &cell_has_core, &cell_cid,
                          &parent,      &comp_min,    &sort_hist,   &scan_scratch, &small,      &hash_keys,
                          &hash_vals,   &nbr_list,    &jobs_dev,    &batch_bbox,  &cell_job,    &job_counters,
                          &items_split, &col_range,   &ids_in,      &batch_in,    &batch_nn,    &batch_ci,
                          &load_box,    &tc_rec};
        for (DevBuf *b : bufs) f(*b);
    }
    size_t held_bytes() {
        size_t total = 0;
        for_each_buf([&](DevBuf &b) { total += b.bytes; });
        return total;
    }

    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    // kernel-level events: sort, count, union, border (begin, end)
    cudaEvent_t kev[8] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};

    // state kept between classify and assign_labels
    bool have_state = false;
    int64_t n = 0, nv = 0, n_cells = 0, n_items = 0;
    int d = 0;
    float e2 = 0.0f;
    int min_pts = 0;
    uint32_t flags_run = 0;
    bool key64 = false;
    int cell_units = 0;
    int n_rows = 0;
    unsigned long long hash_mask = 0;
    int32_t *ci_user = nullptr;  // caller's cluster_index buffer of the current assign_labels call
    const float *coords_dev = nullptr;  // device coordinates of the current job
    GridDev grid{};
    Stencil stencil{};
    int64_t n_cores = 0;
    ndb_result result{};
    bool have_labels = false;
    ndb_stats stats{};
};

namespace {

// layout of ctx->small
constexpr size_t kSmallBboxOff = 0;          // int[2*kMaxDim]
constexpr size_t kSmallInvalidOff = 256;     // u64
constexpr size_t kSmallCountersOff = 512;    // u64[12]: 0 clusters 1 noise 2 count pairs 3 union pairs 4 border pairs
                                             // 5 band pairs 6 work counter of the persistent count kernel
                                             // 8..11 filter audit (tc::audit_tile)
constexpr int kCounters = 12;
constexpr size_t kSmallScalarOff = 1024;     // u32[8]: 0 n_cells 1 n_items 2 n_cores
constexpr size_t kSmallErrOff = 1536;        // int
constexpr size_t kSmallStencilOff = 2048;    // int4[kMaxRows]: stencil rows of the current job
constexpr size_t kSmallBytes = 4096;

// Destination window of the input-order output scatters: 24M int32 (96 MB) stays
// within the 126 MB L2, so outputs larger than that are written in several passes.
constexpr int64_t kScatterWindow = int64_t(24) << 20;

inline unsigned blocks_for(int64_t n, int threads = kBlock) {
    int64_t b = (n + threads - 1) / threads;
    return (unsigned)(b < 1 ? 1 : b);
}

struct Fail {
    ndb_status st;
};

constexpr uint32_t kAllFlags = NDB_FLAG_APPROXIMATE | NDB_FLAG_FULL_COUNT | NDB_FLAG_DEVICE_PTRS |
                               NDB_FLAG_EXACT_COUNT | NDB_FLAG_TENSOR_FILTER | NDB_FLAG_FILTER_AUDIT |
                               NDB_FLAG_GRAM_FILTER;
// internal: the job is the context's loaded copy (ndb_b200_run_loaded); never a caller's flag
constexpr uint32_t kFlagLoaded = 0x80000000u;

// load_box layout: lo_hi ints, then the invalid-point count, then two error words
constexpr size_t kLoadBoxInvalidOff = 2 * kMaxDim * sizeof(int);
constexpr size_t kLoadBoxErrOff = kLoadBoxInvalidOff + 8;
constexpr size_t kLoadBoxBytes = kLoadBoxErrOff + 8;
constexpr size_t kPinChunk = size_t(32) << 20;  // bytes of one pinned staging chunk

inline void ck(ndb_ctx *ctx, cudaError_t e) {
    if (e == cudaSuccess) return;
    ctx->last_cuda_error = cudaGetErrorString(e);
    throw Fail{e == cudaErrorMemoryAllocation ? NDB_ERR_OUT_OF_MEMORY : NDB_ERR_CUDA};
}

// Grows b to at least `bytes`, refusing (as an allocation failure, before any
// cudaMalloc) when the context's footprint would pass its memory cap.
inline cudaError_t grow(ndb_ctx *ctx, DevBuf &b, size_t bytes) {
    if (bytes < 16) bytes = 16;
    if (ctx->mem_limit && bytes > b.bytes) {
        const size_t rounded = (bytes + 4095) & ~size_t(4095);
        if (ctx->held_bytes() - b.bytes + rounded > ctx->mem_limit) return cudaErrorMemoryAllocation;
    }
    return b.ensure(bytes);
}

inline void ensure(ndb_ctx *ctx, DevBuf &b, size_t bytes) { ck(ctx, grow(ctx, b, bytes)); }

template <typename T>
T *small_at(ndb_ctx *ctx, size_t off) {
    return reinterpret_cast<T *>(static_cast<char *>(ctx->small.ptr) + off);
}

// An event of the context, created on first use.
inline cudaEvent_t lazy_event(ndb_ctx *ctx, cudaEvent_t &e) {
    if (!e) ck(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    return e;
}

// Sets `bytes` bytes at p to v with a kernel (a memset that never waits for a copy
// engine).
inline void fill_bytes(ndb_ctx *ctx, void *p, int v, size_t bytes, cudaStream_t st) {
    if (bytes == 0) return;
    const int64_t n16 = ((uintptr_t)p & 15) ? 0 : (int64_t)(bytes / 16);
    const unsigned blocks = (unsigned)std::min<int64_t>(std::max<int64_t>((n16 + kBlock - 1) / kBlock, 1),
                                                        int64_t(ctx->sm_count) * 8);
    ++launch_counter(), fill_bytes_kernel<<<blocks, kBlock, 0, st>>>(static_cast<uint8_t *>(p), bytes, n16,
                                                                   (uint8_t)v);
    ck(ctx, cudaGetLastError());
}

// The mailbox holds at least `bytes`; grown only between runs (nothing of the
// context in flight).
inline void ensure_mail(ndb_ctx *ctx, size_t bytes) {
    if (bytes <= ctx->mail_bytes) return;
    bytes = (bytes + (size_t(1) << 20) - 1) & ~((size_t(1) << 20) - 1);
    if (ctx->mail) {
        cudaFreeHost(ctx->mail);
        ctx->mail = ctx->mail_dev = nullptr;
        ctx->mail_bytes = 0;
    }
    void *h = nullptr, *d = nullptr;
    ck(ctx, cudaHostAlloc(&h, bytes, cudaHostAllocMapped));
    if (cudaHostGetDevicePointer(&d, h, 0) != cudaSuccess) {
        cudaFreeHost(h);
        ck(ctx, cudaErrorInvalidValue);
    }
    ctx->mail = static_cast<char *>(h);
    ctx->mail_dev = static_cast<char *>(d);
    ctx->mail_bytes = bytes;
}

// A 16-byte aligned slice of the mailbox; slices are handed out in order and
// released together (mail_used = 0) once the stream has drained.
inline char *mail_slice(ndb_ctx *ctx, size_t bytes) {
    const size_t off = (ctx->mail_used + 15) & ~size_t(15);
    if (!ctx->mail || off + bytes > ctx->mail_bytes) ck(ctx, cudaErrorInvalidValue);
    ctx->mail_used = off + bytes;
    return ctx->mail + off;
}

inline void copy_words(ndb_ctx *ctx, const void *src, void *dst, size_t bytes, cudaStream_t st) {
    const int64_t n = (int64_t)(bytes / 4);
    if (n == 0) return;
    const unsigned blocks = (unsigned)std::min<int64_t>((n + kBlock - 1) / kBlock, int64_t(ctx->sm_count) * 4);
    ++launch_counter(), copy_words_kernel<<<blocks, kBlock, 0, st>>>(static_cast<const uint32_t *>(src),
                                                                   static_cast<uint32_t *>(dst), n);
    ck(ctx, cudaGetLastError());
}

// Device -> host through the mailbox: a copy kernel in stream order; the returned
// host copy is valid once the stream is synchronized.
template <typename T>
const T *mail_from_device(ndb_ctx *ctx, const T *src, size_t count, cudaStream_t st) {
    static_assert(sizeof(T) % 4 == 0, "mailbox transfers are whole words");
    char *h = mail_slice(ctx, count * sizeof(T));
    copy_words(ctx, src, ctx->mail_dev + (h - ctx->mail), count * sizeof(T), st);
    return reinterpret_cast<const T *>(h);
}

// Host -> device through the mailbox: the data is copied into the mailbox now and
// moved by a copy kernel in stream order.
template <typename T>
void mail_to_device(ndb_ctx *ctx, T *dst, const T *src, size_t count, cudaStream_t st) {
    static_assert(sizeof(T) % 4 == 0, "mailbox transfers are whole words");
    char *h = mail_slice(ctx, count * sizeof(T));
    memcpy(h, src, count * sizeof(T));
    copy_words(ctx, ctx->mail_dev + (h - ctx->mail), dst, count * sizeof(T), st);
}

// ---------------------------------------------------------------------------
// Grid planning (host).
//
// r bounds |a_k - b_k| for every dimension k of every pair the FP32 predicate
// accepts: the rounded square of the rounded difference is <= e2, so the real
// difference is at most max(sqrt(e2), 2^-63) * (1 + 2^-20).
//
// Same-cell-linked grid (d <= 3, e2 >= 2^-100): cubic cells of width
// w = sqrt(e2 / d * (1 - 2^-10)).  Two points of one cell differ by less than
// w * (1 + 2^-20) per dimension, so their FP32 length is below
// d * w^2 * (1 + 2^-19) * (1 + 2^-24)^5 < e2: every pair inside a cell is in range.
// Otherwise (or when a dimension would need more than the per-dimension cell cap)
// up to four dimensions are gridded with cells of at least r * (1 + 2^-12).
//
// Stencil: cell coordinates of an accepted pair differ by at most
// R = ceil(r / w + 2^-18) per dimension (the 2^-18 covers the cell-coordinate
// rounding, < 2^-21 cells); a row of offsets is dropped only when even the
// closest points of the two cells, min |delta| >= (|o| - 1 - 2^-18) * w per
// dimension, are further apart than r.
// ---------------------------------------------------------------------------
struct Plan {
    GridDev g{};
    Stencil st{};
    bool cell_units = false;
    int key_bits = 0;
};

Plan plan_grid(int d, float e2, const double *lo, const double *hi) {
    Plan pl;
    double r = sqrt((double)e2);
    if (r < ldexp(1.0, -63)) r = ldexp(1.0, -63);
    r *= 1.0 + ldexp(1.0, -20);
    const double slack = ldexp(1.0, -18);

    // cells per gridded dimension: keys stay below 2^62 and cell coordinates exact in double
    auto cap_for = [](int k) { return k >= 4 ? ldexp(1.0, 15) : k == 3 ? ldexp(1.0, 20) : ldexp(1.0, 30); };

    int k = 0;
    int dims[kMaxGridDims] = {0, 0, 0, 0};
    double w[kMaxGridDims] = {1, 1, 1, 1};
    bool linked = false;
    if (d <= 3 && (double)e2 >= ldexp(1.0, -100)) {
        const double wl = sqrt((double)e2 / d * (1.0 - ldexp(1.0, -10)));
        bool fits = wl > 0;
        for (int a = 0; a < d && fits; ++a) fits = (hi[a] - lo[a]) / wl + 1.0 < cap_for(d);
        if (fits) {
            k = d;
            for (int a = 0; a < d; ++a) {
                dims[a] = a;
                w[a] = wl;
            }
            linked = true;
        }
    }
    if (!linked) {
        // up to four dimensions, the widest ones (input order kept among them)
        k = d < kMaxGridDims ? d : kMaxGridDims;
        std::vector<int> order(d);
        for (int a = 0; a < d; ++a) order[a] = a;
        std::stable_sort(order.begin(), order.end(),
                         [&](int x, int y) { return (hi[x] - lo[x]) > (hi[y] - lo[y]); });
        std::sort(order.begin(), order.begin() + k);
        for (int a = 0; a < k; ++a) {
            dims[a] = order[a];
            const double span = hi[dims[a]] - lo[dims[a]];
            w[a] = r * (1.0 + ldexp(1.0, -12));
            if (span / w[a] + 1.0 >= cap_for(k)) w[a] = span / (cap_for(k) - 2.0);
        }
    }
    pl.cell_units = linked;
    pl.g.k = k;
    unsigned long long stride = 1;
    double total = 1;
    for (int a = 0; a < kMaxGridDims; ++a) {
        if (a < k) {
            const double span = hi[dims[a]] - lo[dims[a]];
            pl.g.dim[a] = dims[a];
            pl.g.lo[a] = lo[dims[a]];
            pl.g.inv_w[a] = 1.0 / w[a];
            pl.g.g[a] = (long long)floor(span / w[a]) + 1;
            pl.g.stride[a] = stride;
            stride *= (unsigned long long)pl.g.g[a];
            total *= (double)pl.g.g[a];
        } else {
            pl.g.dim[a] = 0;
            pl.g.lo[a] = 0;
            pl.g.inv_w[a] = 0;
            pl.g.g[a] = 1;
            pl.g.stride[a] = stride;
        }
    }
    // key bits: every valid key <= total - 1 < 2^bits - 1 (the all-ones key marks invalid points)
    int bits = 1;
    while (bits < 64 && ldexp(1.0, bits) - 1.0 < total) ++bits;
    pl.key_bits = bits;

    int R[kMaxGridDims] = {0, 0, 0, 0};
    for (int a = 0; a < k; ++a) R[a] = (int)ceil(r / w[a] + slack);
    struct Row {
        int o1, o2, o3, xr;
        double dist2;
    };
    std::vector<Row> rows;
    auto gap = [&](int o, int a) {
        double q = (double)(o < 0 ? -o : o) - 1.0 - slack;
        return q > 0 ? q * w[a] : 0.0;
    };
    const double r2 = r * r;
    for (int o3 = -R[3]; o3 <= R[3]; ++o3) {
        for (int o2 = -R[2]; o2 <= R[2]; ++o2) {
            for (int o1 = -R[1]; o1 <= R[1]; ++o1) {
                const double g1 = k >= 2 ? gap(o1, 1) : 0.0, g2 = k >= 3 ? gap(o2, 2) : 0.0,
                             g3 = k >= 4 ? gap(o3, 3) : 0.0;
                const double base = g1 * g1 + g2 * g2 + g3 * g3;
                if (base > r2) continue;
                int xr = 0;
                for (int o0 = 1; o0 <= R[0]; ++o0) {
                    const double g0 = gap(o0, 0);
                    if (base + g0 * g0 <= r2) xr = o0;
                }
                rows.push_back({o1, o2, o3, xr, base});
            }
        }
    }
    std::stable_sort(rows.begin(), rows.end(), [](const Row &x, const Row &y) {
        if (x.dist2 != y.dist2) return x.dist2 < y.dist2;
        return std::abs(x.o1) + std::abs(x.o2) + std::abs(x.o3) < std::abs(y.o1) + std::abs(y.o2) + std::abs(y.o3);
    });
    pl.st.n_rows = (int)rows.size();
    for (size_t i = 0; i < rows.size() && i < (size_t)kMaxRows; ++i)
        pl.st.rows[i] = make_int4(rows[i].o1, rows[i].o2, rows[i].o3, rows[i].xr);
    return pl;
}

float elapsed(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) ms = 0.0f;
    return ms;
}

// ---------------------------------------------------------------------------
// phase 1
// ---------------------------------------------------------------------------
// Lanes per cell of the row lookup, as log2: the stencil's row count rounded up to a
// power of two (25 rows: one warp per cell; 5 rows: four cells per warp).
inline int row_group_log2(int n_rows) {
    int l = 0;
    while ((1 << l) < n_rows) ++l;
    return l;
}

// Columns of a grid: cells that differ only in gridded dimension 0.
inline double grid_columns(const GridDev &g) {
    double c = 1;
    for (int a = 1; a < g.k; ++a) c *= (double)g.g[a];
    return c;
}

// The cell lookup of a pipeline: the dense column table when the columns of all
// its jobs fit the context's budget, else a hash table of the cell keys (load
// factor <= 1/4, so most probes settle at the first slot).
template <typename K>
CellIndex<K> build_cell_index(ndb_ctx *ctx, int64_t n_cells, double columns, const GridDev &g_one,
                              const JobDev *jobs, const int32_t *cell_job) {
    cudaStream_t st = ctx->stream;
    CellIndex<K> L{nullptr, nullptr, nullptr, 0};
    ctx->use_cols = columns >= 1 && columns <= (double)ctx->col_budget;
    if (ctx->use_cols) {
        const size_t cols = (size_t)columns;
        ensure(ctx, ctx->col_range, (cols + 1) * sizeof(int2));
        fill_bytes(ctx, ctx->col_range.ptr, 0, (size_t)(cols + 1) * sizeof(int2), st);
        ++launch_counter(), col_range_kernel<K><<<blocks_for(n_cells), kBlock, 0, st>>>(
            ctx->cell_key.as<K>(), n_cells, g_one, jobs, cell_job, ctx->col_range.as<int2>());
        ck(ctx, cudaGetLastError());
        L.col = ctx->col_range.as<int2>();
        return L;
    }
    int64_t hsize = 1024;
    while (hsize < 4 * n_cells) hsize <<= 1;
    ctx->hash_mask = (unsigned long long)(hsize - 1);
    ensure(ctx, ctx->hash_keys, hsize * sizeof(K));
    ensure(ctx, ctx->hash_vals, hsize * sizeof(int32_t));
    ++launch_counter(), hash_clear_kernel<K><<<blocks_for(hsize), kBlock, 0, st>>>(ctx->hash_keys.as<K>(), hsize);
    ++launch_counter(), hash_insert_kernel<K><<<blocks_for(n_cells), kBlock, 0, st>>>(
        ctx->cell_key.as<K>(), n_cells, ctx->hash_keys.as<K>(), ctx->hash_vals.as<int32_t>(), ctx->hash_mask);
    ck(ctx, cudaGetLastError());
    L.hkeys = ctx->hash_keys.as<K>();
    L.hvals = ctx->hash_vals.as<int32_t>();
    L.mask = ctx->hash_mask;
    return L;
}

// The lookup built by build_cell_index, for kernels of the label phase.
template <typename K>
CellIndex<K> cell_index(ndb_ctx *ctx) {
    if (ctx->use_cols) return CellIndex<K>{ctx->col_range.as<int2>(), nullptr, nullptr, 0};
    return CellIndex<K>{nullptr, ctx->hash_keys.as<K>(), ctx->hash_vals.as<int32_t>(), ctx->hash_mask};
}

template <int D, typename K>
void classify_grid(ndb_ctx *ctx, const Plan &pl) {
    cudaStream_t st = ctx->stream;
    const int64_t n = ctx->n;
    const int64_t nv = ctx->nv;
    constexpr int P = Stride<D>::P;

    ensure(ctx, ctx->keys0, n * sizeof(K));
    ensure(ctx, ctx->keys1, n * sizeof(K));
    ensure(ctx, ctx->ids0, n * sizeof(int32_t));
    ensure(ctx, ctx->ids1, n * sizeof(int32_t));
    ensure(ctx, ctx->sort_hist, sort_hist_words(n) * sizeof(uint32_t));
    const size_t scan_words = std::max(scan_scratch_words(n + 1), scan_scratch_words((int64_t)sort_hist_words(n)));
    ensure(ctx, ctx->scan_scratch, (scan_words + 64) * sizeof(uint32_t));

    K invalid_key = (K)(pl.key_bits >= (int)(8 * sizeof(K)) ? ~(K)0 : (((K)1 << pl.key_bits) - 1));
    ++launch_counter(), key_kernel<D, K><<<blocks_for(n), kBlock, 0, st>>>(ctx->coords_dev, n, pl.g, invalid_key,
                                                        ctx->keys0.as<K>(), ctx->ids0.as<int32_t>());
    ck(ctx, cudaGetLastError());
    bool in_first = true;
    cudaEventRecord(ctx->kev[0], st);
    if (sizeof(K) == 4)
        ck(ctx, radix_sort_pairs_u32(reinterpret_cast<uint32_t *>(ctx->keys0.ptr), ctx->ids0.as<int32_t>(),
                                     reinterpret_cast<uint32_t *>(ctx->keys1.ptr), ctx->ids1.as<int32_t>(), n,
                                     pl.key_bits, ctx->sort_hist.as<uint32_t>(), ctx->scan_scratch.as<uint32_t>(),
                                     &in_first, st));
    else
        ck(ctx, radix_sort_pairs_u64(reinterpret_cast<uint64_t *>(ctx->keys0.ptr), ctx->ids0.as<int32_t>(),
                                     reinterpret_cast<uint64_t *>(ctx->keys1.ptr), ctx->ids1.as<int32_t>(), n,
                                     pl.key_bits, ctx->sort_hist.as<uint32_t>(), ctx->scan_scratch.as<uint32_t>(),
                                     &in_first, st));
    cudaEventRecord(ctx->kev[1], st);
    ctx->stats.sort_passes = (pl.key_bits + 7) / 8;
    ctx->stats.key_bytes = (int32_t)sizeof(K);
    if (!in_first) {
        std::swap(ctx->keys0, ctx->keys1);
        std::swap(ctx->ids0, ctx->ids1);
    }
    const K *keys = ctx->keys0.as<K>();
    const int32_t *perm = ctx->ids0.as<int32_t>();

    // cells
    ensure(ctx, ctx->flags, (n + 1) * sizeof(uint32_t));
    ensure(ctx, ctx->pos, (n + 1) * sizeof(uint32_t));
    ensure(ctx, ctx->pcell, (n + 1) * sizeof(int32_t));
    ensure(ctx, ctx->cell_start, (n + 2) * sizeof(int32_t));
    ensure(ctx, ctx->cell_key, (n + 1) * sizeof(K));
    uint32_t *scal = small_at<uint32_t>(ctx, kSmallScalarOff);
    ++launch_counter(), cell_flag_kernel<K><<<blocks_for(nv), kBlock, 0, st>>>(keys, nv, ctx->flags.as<uint32_t>());
    ck(ctx, cudaGetLastError());
    ck(ctx, scan_exclusive_u32(ctx->flags.as<uint32_t>(), ctx->pos.as<uint32_t>(), nv, scal + 0,
                               ctx->scan_scratch.as<uint32_t>(), st));
    ++launch_counter(), cell_write_kernel<K><<<blocks_for(nv), kBlock, 0, st>>>(keys, nv, ctx->pos.as<uint32_t>(), scal + 0,
                                                            ctx->cell_start.as<int32_t>(), ctx->cell_key.as<K>(),
                                                            ctx->pcell.as<int32_t>());
    ck(ctx, cudaGetLastError());
    ensure(ctx, ctx->xs, (nv + 1) * P * sizeof(float));
    ++launch_counter(), gather_kernel<D><<<blocks_for(nv), kBlock, 0, st>>>(ctx->coords_dev, perm, nv, ctx->xs.as<float>());
    ck(ctx, cudaGetLastError());
    uint32_t n_cells32 = 0;
    ck(ctx, cudaMemcpyAsync(&n_cells32, scal + 0, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    ck(ctx, cudaStreamSynchronize(st));
    const int64_t n_cells = n_cells32;
    ctx->n_cells = n_cells;

    // neighbour rows, through the column table (or a hash table) of the cells
    const int n_rows = pl.st.n_rows;
    const CellIndex<K> L = build_cell_index<K>(ctx, n_cells, grid_columns(pl.g), pl.g, nullptr, nullptr);
    ensure(ctx, ctx->nbr, (size_t)(n_cells * n_rows + 1) * sizeof(int2));
    int4 *rows_dev = small_at<int4>(ctx, kSmallStencilOff);
    ck(ctx, cudaMemcpyAsync(rows_dev, pl.st.rows, n_rows * sizeof(int4), cudaMemcpyHostToDevice, st));
    const int rlog = row_group_log2(n_rows);
    ++launch_counter(), rows_kernel<K><<<blocks_for(n_cells << rlog), kBlock, 0, st>>>(
        ctx->cell_key.as<K>(), n_cells, pl.g, rows_dev, n_rows, rlog, L, ctx->nbr.as<int2>(), nullptr, nullptr);
    ck(ctx, cudaGetLastError());

    // work items
    ensure(ctx, ctx->item_cnt, (n_cells + 1) * sizeof(uint32_t));
    ++launch_counter(), item_count_kernel<<<blocks_for(n_cells), kBlock, 0, st>>>(ctx->cell_start.as<int32_t>(), n_cells,
                                                              ctx->item_cnt.as<uint32_t>());
    ck(ctx, cudaGetLastError());
    ck(ctx, scan_exclusive_u32(ctx->item_cnt.as<uint32_t>(), ctx->item_cnt.as<uint32_t>(), n_cells, scal + 1,
                               ctx->scan_scratch.as<uint32_t>(), st));
    uint32_t n_items32 = 0;
    ck(ctx, cudaMemcpyAsync(&n_items32, scal + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    ck(ctx, cudaStreamSynchronize(st));
    ctx->n_items = n_items32;
    ensure(ctx, ctx->items, (ctx->n_items + 1) * sizeof(int2));
    ++launch_counter(), item_write_kernel<<<blocks_for(n_cells), kBlock, 0, st>>>(ctx->cell_start.as<int32_t>(), n_cells,
                                                              ctx->item_cnt.as<uint32_t>(), ctx->items.as<int2>());
    ck(ctx, cudaGetLastError());
}

template <int D>
void count_phase(ndb_ctx *ctx);

// The tensor-core filter's preconditions: d >= 8 (and, unless NDB_FLAG_TENSOR_FILTER
// asks for it or counts are full, d at or above the automatic threshold: 12 by
// measurement on B200, where with early exit the filter beats the exact kernel on
// full items at d = 16 but not at d = 8; NDB_TC_MIN_DIM overrides), the eps grid (row tables of <= 32 rows), eps^2 a
// normal float far from under- and overflow, and coordinates within +-2^60 so that
// no centred difference or squared norm overflows.  Results never depend on it.
inline int default_tc_min_dim() {
    static const int v = [] {
        const char *s = getenv("NDB_TC_MIN_DIM");
        const int x = s ? atoi(s) : 12;
        return x < tc::kMinDim ? tc::kMinDim : x;
    }();
    return v;
}

inline bool tc_eligible(const ndb_ctx *ctx, int d, float e2, const double *lo, const double *hi, bool linked,
                        int n_rows, uint32_t flags) {
    // a context's own tuning (ndb_b200_set_tuning) applies to both count modes; by
    // default full counts start at d = 8: they scan every candidate of every point,
    // so the tiles stay full, and there the filter measured 1.17x the exact kernel
    const int tuned = ctx->tuning.tc_min_dim;
    const int min_dim = (flags & NDB_FLAG_TENSOR_FILTER) ? tc::kMinDim
                        : tuned > 0                        ? std::max(tuned, tc::kMinDim)
                        : (flags & NDB_FLAG_FULL_COUNT)    ? tc::kMinDim
                                                           : default_tc_min_dim();
    if (d < min_dim || (flags & NDB_FLAG_EXACT_COUNT) || linked || n_rows > kWarp) return false;
    if (!(e2 >= 0x1p-100f && e2 <= 0x1p100f)) return false;
    for (int a = 0; a < d; ++a)
        if (!(fabs(lo[a]) <= 0x1p60 && fabs(hi[a]) <= 0x1p60)) return false;
    return true;
}

// The Gram-filtered count on CUDA cores (count_kernel<D, E, true>), when asked for
// (NDB_FLAG_GRAM_FILTER or the context's tuning; measured on B200 it does not beat
// the exact sum, whose cost there is latency rather than FP32 issue): d >= 8, not the
// plain form (NDB_FLAG_EXACT_COUNT), eps^2 a normal float far from under- and
// overflow, and coordinates within +-2^60 so that no centred square or norm
// overflows.  Results never depend on it.
inline bool gram_eligible(const ndb_ctx *ctx, int d, float e2, const double *lo, const double *hi, uint32_t flags) {
    if (!((flags & NDB_FLAG_GRAM_FILTER) || ctx->tuning.gram_filter > 0)) return false;
    if (d < 8 || (flags & NDB_FLAG_EXACT_COUNT)) return false;
    if (!(e2 >= 0x1p-100f && e2 <= 0x1p100f)) return false;
    for (int a = 0; a < d; ++a)
        if (!(fabs(lo[a]) <= 0x1p60 && fabs(hi[a]) <= 0x1p60)) return false;
    return true;
}

// Which items the tensor kernel takes: it stages every candidate row once per item
// and most of its per-tile epilogue is fixed, so it pays only for full items (many
// points of one cell).  Measured on B200: with about 11 points per item the exact
// kernel is faster even at d = 16.  Items with at least this many points go to the
// tensor-core count, the rest to the exact kernel (NDB_TC_MIN_ITEM overrides it;
// NDB_FLAG_TENSOR_FILTER sends every item).
inline int default_tc_min_item() {
    static const int v = [] {
        const char *s = getenv("NDB_TC_MIN_ITEM");
        const int x = s ? atoi(s) : 16;
        return x < 1 ? 1 : x;
    }();
    return v;
}

inline int ctx_tc_min_item(const ndb_ctx *ctx) {
    const int v = ctx->tuning.tc_min_item;
    return v <= 0 ? default_tc_min_item() : v;
}

template <int D>
void launch_count_tc(ndb_ctx *ctx, int64_t n_items, const int2 *items, const int32_t *cell_start, const int2 *nbr,
                     int n_rows, const float *xs, float e2, int min_pts, bool early, int32_t *nn_sorted,
                     int32_t *list, int list_cap, int list_stride, const JobDev *jobs, const int32_t *cell_job,
                     const uint32_t *n_items_dev, bool audit) {
    if constexpr (D >= tc::kMinDim) {
        cudaStream_t st = ctx->stream;
        unsigned long long *counters = small_at<unsigned long long>(ctx, kSmallCountersOff);
        unsigned int *work = reinterpret_cast<unsigned int *>(counters + 6);
        fill_bytes(ctx, work, 0, sizeof(unsigned long long), st);
        // the items' records (stencil rows as point ranges), which the kernel fetches
        // one item ahead by bulk copies; without room for them (a memory cap, the
        // allocation-free entry point) the kernel gathers the rows itself
        int2 *rec = nullptr;
        if (n_items_dev && grow(ctx, ctx->tc_rec, (size_t)n_items * tc::kRecBytes) == cudaSuccess) {
            rec = ctx->tc_rec.as<int2>();
            ++launch_counter(), tc::tc_records_kernel<<<blocks_for(n_items * kWarp), kBlock, 0, st>>>(
                items, n_items_dev, cell_start, nbr, n_rows, cell_job, rec);
            ck(ctx, cudaGetLastError());
        } else {
            cudaGetLastError();  // a refused or failed allocation leaves no error behind
        }
        const unsigned grid = (unsigned)std::min<int64_t>(n_items, (int64_t)ctx->sm_count * tc::TcBlocks<D>::v);
        if (audit)
            ++launch_counter(), tc::count_tc_kernel<D, true><<<grid, tc::kThreads, 0, st>>>(
                items, n_items, cell_start, nbr, n_rows, xs, e2, min_pts, early ? 1 : 0, nn_sorted, list, list_cap,
                list_stride, counters + 2, counters + 5, work, small_at<int>(ctx, kSmallErrOff), jobs, cell_job,
                n_items_dev, counters + 8, rec);
        else
            ++launch_counter(), tc::count_tc_kernel<D><<<grid, tc::kThreads, 0, st>>>(
                items, n_items, cell_start, nbr, n_rows, xs, e2, min_pts, early ? 1 : 0, nn_sorted, list, list_cap,
                list_stride, counters + 2, counters + 5, work, small_at<int>(ctx, kSmallErrOff), jobs, cell_job,
                n_items_dev, nullptr, rec);
        ck(ctx, cudaGetLastError());
    } else {
        throw Fail{NDB_ERR_INVALID_ARGUMENT};
    }
}

// The neighbour count of one pipeline.  tc: the tensor-core filter may run (input
// eligible); then the items are split by size and each list goes to its kernel,
// both launched at the upper bound and reading their list length on the device.
template <int D>
void count_items(ndb_ctx *ctx, bool tc, bool force_tc, bool gram, bool early, int64_t n_items, const int2 *items,
                 const int32_t *cell_start, const int2 *nbr, int n_rows, const float *xs, float e2, int min_pts,
                 int dense_skip, int32_t *nn_sorted, int32_t *list, int list_cap, int list_stride,
                 const JobDev *jobs, const int32_t *cell_job, bool audit) {
    if (n_items <= 0) return;
    cudaStream_t st = ctx->stream;
    unsigned long long *counters = small_at<unsigned long long>(ctx, kSmallCountersOff);
    const int2 *ex_items = items;
    const uint32_t *ex_n = nullptr;
    if (tc) {
        uint32_t *scal = small_at<uint32_t>(ctx, kSmallScalarOff);
        ensure(ctx, ctx->items_split, (size_t)(2 * n_items + 2) * sizeof(int2));
        int2 *tc_items = ctx->items_split.as<int2>();
        int2 *rest = tc_items + n_items + 1;
        fill_bytes(ctx, scal + 4, 0, 2 * sizeof(uint32_t), st);
        ++launch_counter(), split_items_kernel<<<blocks_for(n_items), kBlock, 0, st>>>(
            items, n_items, cell_start, force_tc ? 1 : ctx_tc_min_item(ctx), tc_items, scal + 4, rest, scal + 5);
        ck(ctx, cudaGetLastError());
        launch_count_tc<D>(ctx, n_items, tc_items, cell_start, nbr, n_rows, xs, e2, min_pts, early, nn_sorted, list,
                           list_cap, list_stride, jobs, cell_job, scal + 4, audit);
        ex_items = rest;
        ex_n = scal + 5;
    }
    const unsigned grid = (unsigned)((n_items + kCountWarps - 1) / kCountWarps);
    // the counts on CUDA cores: the Gram-filtered kernel (d >= 8) or the exact one
    auto launch = [&](auto early_c, auto gram_c) {
        constexpr bool E = decltype(early_c)::value, G = decltype(gram_c)::value;
        ++launch_counter(), count_kernel<D, E, G><<<grid, kCountWarps * kWarp, 0, st>>>(
            ex_items, n_items, cell_start, nbr, n_rows, xs, e2, min_pts, dense_skip, nn_sorted, list, list_cap,
            list_stride, counters + 2, jobs, cell_job, ex_n, counters + 5);
    };
    using T = std::true_type;
    using F = std::false_type;
    if constexpr (D >= 8) {
        if (gram) {
            if (early) launch(T{}, T{});
            else launch(F{}, T{});
            ck(ctx, cudaGetLastError());
            return;
        }
    }
    if (early) launch(T{}, F{});
    else launch(F{}, F{});
    ck(ctx, cudaGetLastError());
}

template <int D>
void count_phase(ndb_ctx *ctx) {
    cudaStream_t st = ctx->stream;
    unsigned long long *counters = small_at<unsigned long long>(ctx, kSmallCountersOff);
    ensure(ctx, ctx->nn_sorted, (ctx->n + 1) * sizeof(int32_t));
    const bool early = (ctx->flags_run & NDB_FLAG_FULL_COUNT) == 0;
    // neighbour lists for the border step: min_pts - 1 entries per point
    ctx->list_cap = 0;
    const int64_t cap = (int64_t)ctx->min_pts - 1;
    if (cap >= 1 && cap <= kMaxListCap && (size_t)(ctx->nv * cap) * sizeof(int32_t) <= ctx->list_budget) {
        ensure(ctx, ctx->nbr_list, (size_t)(ctx->nv * cap + 1) * sizeof(int32_t));
        ctx->list_cap = (int)cap;
    }
    int32_t *list = ctx->list_cap ? ctx->nbr_list.as<int32_t>() : nullptr;
    cudaEventRecord(ctx->kev[2], st);
    count_items<D>(ctx, ctx->tc_count, (ctx->flags_run & NDB_FLAG_TENSOR_FILTER) != 0, ctx->gram_count, early,
                   ctx->n_items,
                   ctx->items.as<int2>(), ctx->cell_start.as<int32_t>(), ctx->nbr.as<int2>(), ctx->n_rows,
                   ctx->xs.as<float>(), ctx->e2, ctx->min_pts, ctx->cell_units, ctx->nn_sorted.as<int32_t>(), list,
                   ctx->list_cap, ctx->list_cap, nullptr, nullptr, (ctx->flags_run & NDB_FLAG_FILTER_AUDIT) != 0);
    cudaEventRecord(ctx->kev[3], st);
}

void core_flags_phase(ndb_ctx *ctx) {
    cudaStream_t st = ctx->stream;
    const int64_t n = ctx->n;
    const int64_t n_words = (n + 31) / 32;
    uint32_t *scal = small_at<uint32_t>(ctx, kSmallScalarOff);
    ensure(ctx, ctx->core_sorted, n + 1);
    ensure(ctx, ctx->cell_has_core, ctx->n_cells + 1);
    ensure(ctx, ctx->core_bits, (n_words + 1) * sizeof(uint32_t));
    ensure(ctx, ctx->core_prefix, (n_words + 1) * sizeof(uint32_t));
    fill_bytes(ctx, ctx->cell_has_core.ptr, 0, (size_t)ctx->n_cells + 1, st);
    fill_bytes(ctx, ctx->core_bits.ptr, 0, (size_t)(n_words + 1) * sizeof(uint32_t), st);
    ++launch_counter(), core_flags_kernel<<<blocks_for(n), kBlock, 0, st>>>(
        ctx->nn_sorted.as<int32_t>(), ctx->nv, n, ctx->min_pts, ctx->ids0.as<int32_t>(), ctx->pcell.as<int32_t>(),
        ctx->core_sorted.as<uint8_t>(), ctx->cell_has_core.as<uint8_t>(), ctx->core_bits.as<uint32_t>(), nullptr,
        nullptr, 0);
    // ranks among cores in input order (data_process.cpp:276-283, :153): per-word prefix of the bitmap
    ++launch_counter(), popc_words_kernel<<<blocks_for(n_words), kBlock, 0, st>>>(
        ctx->core_bits.as<uint32_t>(), n_words, ctx->core_prefix.as<uint32_t>());
    ck(ctx, cudaGetLastError());
    ck(ctx, scan_exclusive_u32(ctx->core_prefix.as<uint32_t>(), ctx->core_prefix.as<uint32_t>(), n_words, scal + 2,
                               ctx->scan_scratch.as<uint32_t>(), st));
}

template <int D>
void classify_dispatch(ndb_ctx *ctx, const Plan &pl) {
    if (pl.key_bits <= 32) {
        ctx->key64 = false;
        classify_grid<D, uint32_t>(ctx, pl);
    } else {
        ctx->key64 = true;
        classify_grid<D, uint64_t>(ctx, pl);
    }
    cudaEventRecord(ctx->ev[1], ctx->stream);
    count_phase<D>(ctx);
    core_flags_phase(ctx);
    cudaEventRecord(ctx->ev[2], ctx->stream);
}

// ---------------------------------------------------------------------------
// phase 2
// ---------------------------------------------------------------------------
// Border points: the minimum id over the cores in range, from the count's
// neighbour lists when there are lists, else by a stencil scan.  Reads the core ids
// in ci_sorted (point units) or cell_cid (cell units).
template <int D>
void border_phase(ndb_ctx *ctx) {
    cudaStream_t st = ctx->stream;
    const int64_t nv = ctx->nv;
    unsigned long long *counters = small_at<unsigned long long>(ctx, kSmallCountersOff);
    if (ctx->list_cap > 0) {
        ++launch_counter(), border_list_kernel<<<blocks_for(nv), kBlock, 0, st>>>(
            nv, ctx->nn_sorted.as<int32_t>(), ctx->nbr_list.as<int32_t>(), ctx->list_cap,
            ctx->core_sorted.as<uint8_t>(), ctx->cell_units, ctx->pcell.as<int32_t>(), ctx->cell_cid.as<int32_t>(),
            ctx->ci_sorted.as<int32_t>(), counters + 4);
        ck(ctx, cudaGetLastError());
    } else if (ctx->n_items > 0) {
        const unsigned grid = (unsigned)((ctx->n_items + kWarpsPerBlock - 1) / kWarpsPerBlock);
        ++launch_counter(), border_kernel<D><<<grid, kBlock, 0, st>>>(
            ctx->items.as<int2>(), ctx->n_items, ctx->cell_start.as<int32_t>(), ctx->nbr.as<int2>(), ctx->n_rows,
            ctx->xs.as<float>(), ctx->e2, ctx->core_sorted.as<uint8_t>(), ctx->cell_has_core.as<uint8_t>(),
            ctx->cell_units, ctx->cell_cid.as<int32_t>(), ctx->ci_sorted.as<int32_t>(), counters + 4);
        ck(ctx, cudaGetLastError());
    }
}

template <int D>
void labels_phase(ndb_ctx *ctx) {
    cudaStream_t st = ctx->stream;
    const int64_t n = ctx->n, nv = ctx->nv, n_cells = ctx->n_cells;
    unsigned long long *counters = small_at<unsigned long long>(ctx, kSmallCountersOff);
    int *err = small_at<int>(ctx, kSmallErrOff);
    uint32_t *scal = small_at<uint32_t>(ctx, kSmallScalarOff);

    const int64_t n_units = ctx->cell_units ? n_cells : nv;
    ensure(ctx, ctx->parent, (n_units + 1) * sizeof(int32_t));
    ensure(ctx, ctx->comp_min, (n_units + 1) * sizeof(int32_t));
    ensure(ctx, ctx->ci_sorted, (n + 1) * sizeof(int32_t));
    ensure(ctx, ctx->cell_cid, (n_cells + 1) * sizeof(int32_t));
    ++launch_counter(), iota_kernel<<<blocks_for(n_units), kBlock, 0, st>>>(ctx->parent.as<int32_t>(), n_units);
    ++launch_counter(), fill_kernel<<<blocks_for(n_units), kBlock, 0, st>>>(ctx->comp_min.as<int32_t>(), n_units, kNoCluster);
    ck(ctx, cudaGetLastError());

    cudaEventRecord(ctx->kev[4], st);  // moved to the main union kernel below when there is one
    if (ctx->n_items > 0) {
        if (ctx->cell_units) {
            if (ctx->list_cap > 0)
                ++launch_counter(), union_lists_kernel<<<blocks_for(nv), kBlock, 0, st>>>(
                    nv, ctx->nn_sorted.as<int32_t>(), ctx->nbr_list.as<int32_t>(), ctx->list_cap, ctx->list_cap,
                    ctx->core_sorted.as<uint8_t>(), ctx->parent.as<int32_t>(), err, nullptr, nullptr,
                    ctx->pcell.as<int32_t>(), 1, (ctx->flags_run & NDB_FLAG_FULL_COUNT) == 0,
                    ctx->cell_start.as<int32_t>(), ctx->min_pts);
            if (ctx->key64)
                ++launch_counter(), union_near_kernel<D, uint64_t><<<blocks_for(n_cells), kBlock, 0, st>>>(
                    n_cells, ctx->grid, ctx->cell_key.as<uint64_t>(), ctx->cell_start.as<int32_t>(),
                    cell_index<uint64_t>(ctx), ctx->xs.as<float>(),
                    ctx->e2, ctx->core_sorted.as<uint8_t>(), ctx->cell_has_core.as<uint8_t>(),
                    ctx->parent.as<int32_t>(), counters + 3, err, nullptr, nullptr);
            else
                ++launch_counter(), union_near_kernel<D, uint32_t><<<blocks_for(n_cells), kBlock, 0, st>>>(
                    n_cells, ctx->grid, ctx->cell_key.as<uint32_t>(), ctx->cell_start.as<int32_t>(),
                    cell_index<uint32_t>(ctx), ctx->xs.as<float>(),
                    ctx->e2, ctx->core_sorted.as<uint8_t>(), ctx->cell_has_core.as<uint8_t>(),
                    ctx->parent.as<int32_t>(), counters + 3, err, nullptr, nullptr);
            // comp_min holds the cells' root snapshot until the union is done
            ++launch_counter(), flatten_snap_kernel<<<blocks_for(n_units), kBlock, 0, st>>>(
                ctx->parent.as<int32_t>(), n_units, err, ctx->cell_has_core.as<uint8_t>(), ctx->comp_min.as<int32_t>());
            cudaEventRecord(ctx->kev[4], st);
            ++launch_counter(), union_cells_kernel<D><<<blocks_for(n_cells * kWarp), kBlock, 0, st>>>(
                n_cells, ctx->cell_start.as<int32_t>(), ctx->nbr.as<int2>(), ctx->n_rows, ctx->xs.as<float>(),
                ctx->e2, ctx->core_sorted.as<uint8_t>(), ctx->cell_has_core.as<uint8_t>(), ctx->parent.as<int32_t>(),
                counters + 3, err, nullptr, nullptr, ctx->comp_min.as<int32_t>());
            ++launch_counter(), fill_kernel<<<blocks_for(n_units), kBlock, 0, st>>>(ctx->comp_min.as<int32_t>(), n_units,
                                                                                   kNoCluster);
        }
        else {
            if (ctx->list_cap > 0) {
                ++launch_counter(), union_lists_kernel<<<blocks_for(nv), kBlock, 0, st>>>(
                    nv, ctx->nn_sorted.as<int32_t>(), ctx->nbr_list.as<int32_t>(), ctx->list_cap, ctx->list_cap,
                    ctx->core_sorted.as<uint8_t>(), ctx->parent.as<int32_t>(), err, nullptr, nullptr,
                    ctx->pcell.as<int32_t>(), 0, 0, ctx->cell_start.as<int32_t>(), ctx->min_pts);
                ++launch_counter(), flatten_kernel<<<blocks_for(n_units), kBlock, 0, st>>>(ctx->parent.as<int32_t>(),
                                                                                          n_units, err);
            }
            fill_bytes(ctx, ctx->cell_cid.ptr, 0xff, (size_t)n_cells * sizeof(int32_t), st);  // -1
            ++launch_counter(), cell_root_kernel<<<blocks_for(nv), kBlock, 0, st>>>(
                nv, ctx->pcell.as<int32_t>(), ctx->core_sorted.as<uint8_t>(), ctx->parent.as<int32_t>(),
                ctx->cell_cid.as<int32_t>());
            cudaEventRecord(ctx->kev[4], st);
            const unsigned pgrid = (unsigned)((ctx->n_items + kCountWarps - 1) / kCountWarps);
            ++launch_counter(), union_points_kernel<D><<<pgrid, kCountWarps * kWarp, 0, st>>>(
                ctx->items.as<int2>(), ctx->n_items, ctx->cell_start.as<int32_t>(), ctx->nbr.as<int2>(), ctx->n_rows,
                ctx->xs.as<float>(), ctx->e2, ctx->core_sorted.as<uint8_t>(), ctx->cell_has_core.as<uint8_t>(),
                ctx->parent.as<int32_t>(), counters + 3, err, nullptr, nullptr, ctx->cell_cid.as<int32_t>());
        }
        ck(ctx, cudaGetLastError());
    }
    cudaEventRecord(ctx->kev[5], st);
    ++launch_counter(), flatten_kernel<<<blocks_for(n_units), kBlock, 0, st>>>(ctx->parent.as<int32_t>(), n_units, err);
    if (ctx->cell_units)
        ++launch_counter(), comp_min_cells_kernel<<<blocks_for(n_cells), kBlock, 0, st>>>(
            n_cells, ctx->cell_start.as<int32_t>(), ctx->cell_has_core.as<uint8_t>(), ctx->core_sorted.as<uint8_t>(),
            ctx->ids0.as<int32_t>(), ctx->core_bits.as<uint32_t>(), ctx->core_prefix.as<uint32_t>(),
            ctx->parent.as<int32_t>(), ctx->comp_min.as<int32_t>());
    else
        ++launch_counter(), comp_min_kernel<<<blocks_for(nv), kBlock, 0, st>>>(
            nv, ctx->core_sorted.as<uint8_t>(), ctx->ids0.as<int32_t>(), ctx->pcell.as<int32_t>(), ctx->cell_units,
            ctx->core_bits.as<uint32_t>(), ctx->core_prefix.as<uint32_t>(), ctx->parent.as<int32_t>(),
            ctx->comp_min.as<int32_t>());
    ++launch_counter(), core_ids_kernel<<<blocks_for(nv), kBlock, 0, st>>>(
        nv, ctx->core_sorted.as<uint8_t>(), ctx->pcell.as<int32_t>(), ctx->cell_units, ctx->parent.as<int32_t>(),
        ctx->comp_min.as<int32_t>(), ctx->ci_sorted.as<int32_t>(), counters, nullptr, nullptr);
    if (ctx->cell_units)
        ++launch_counter(), cell_ids_kernel<<<blocks_for(n_cells), kBlock, 0, st>>>(n_cells, ctx->cell_has_core.as<uint8_t>(),
                                                                ctx->parent.as<int32_t>(), ctx->comp_min.as<int32_t>(),
                                                                ctx->cell_cid.as<int32_t>(), counters, nullptr, nullptr);
    ck(ctx, cudaGetLastError());
    cudaEventRecord(ctx->ev[3], st);
    cudaEventRecord(ctx->kev[6], st);
    border_phase<D>(ctx);
    cudaEventRecord(ctx->kev[7], st);
    // ids in input order, straight into the caller's device buffer when there is one
    int32_t *target = nullptr;
    if (ctx->ci_user && (ctx->flags_run & NDB_FLAG_DEVICE_PTRS)) {
        target = ctx->ci_user;
    } else if (ctx->ci_user) {
        ensure(ctx, ctx->ci_orig, (n + 1) * sizeof(int32_t));
        target = ctx->ci_orig.as<int32_t>();
    }
    const int64_t wci = target ? kScatterWindow : n;  // no output: one pass counts
    for (int64_t lo = 0; lo < n; lo += wci)
        ++launch_counter(), output_ci_kernel<<<blocks_for(n), kBlock, 0, st>>>(
            ctx->ci_sorted.as<int32_t>(), nv, n, ctx->ids0.as<int32_t>(), ctx->core_bits.as<uint32_t>(),
            ctx->core_prefix.as<uint32_t>(), target, counters, nullptr, 0, nullptr, lo,
            wci >= n ? INT64_MAX : lo + wci);
    ck(ctx, cudaGetLastError());
    cudaEventRecord(ctx->ev[4], st);
}

ndb_status check_ctx(ndb_ctx *ctx) {
    if (!ctx) return NDB_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return NDB_ERR_NO_DEVICE;
    return NDB_OK;
}

bool is_device_ptr(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// The filter audit's counters (tc::audit_tile) into the stats.
inline void audit_stats(ndb_stats &S, const unsigned long long *a) {
    double mx, mr;
    memcpy(&mx, &a[0], sizeof(double));
    memcpy(&mr, &a[1], sizeof(double));
    S.filter_max_abs_err = mx;
    S.filter_max_err_over_bound = mr;
    S.filter_audited_pairs = (int64_t)a[2];
    S.filter_misclassified_pairs = (int64_t)a[3];
}

// Counters and times of phase 1, once its work on the context's stream is done.
template <int D>
void classify_stats(ndb_ctx *ctx) {
    unsigned long long h_counters[kCounters];
    uint32_t h_tc_items = 0;
    ck(ctx, cudaMemcpyAsync(h_counters, small_at<unsigned long long>(ctx, kSmallCountersOff), sizeof(h_counters),
                            cudaMemcpyDeviceToHost, ctx->stream));
    ck(ctx, cudaMemcpyAsync(&h_tc_items, small_at<uint32_t>(ctx, kSmallScalarOff) + 4, sizeof(uint32_t),
                            cudaMemcpyDeviceToHost, ctx->stream));
    ck(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->stats.tensor_items = ctx->tc_count ? h_tc_items : 0;
    ctx->stats.count_pairs = (int64_t)h_counters[2];
    ctx->stats.count_pair_dims = (int64_t)h_counters[2] * D;
    ctx->stats.count_fp32_ops = (int64_t)h_counters[2] * (ctx->gram_count ? D + 3 : 3 * D);
    ctx->stats.gram_filter = ctx->gram_count ? 1 : 0;
    ctx->stats.band_pairs = (int64_t)h_counters[5];
    audit_stats(ctx->stats, h_counters + 8);
    ctx->stats.ms_grid = elapsed(ctx->ev[0], ctx->ev[1]);
    ctx->stats.ms_count = elapsed(ctx->ev[1], ctx->ev[2]);
    ctx->stats.ms_sort_kernels = elapsed(ctx->kev[0], ctx->kev[1]);
    ctx->stats.ms_count_kernel = elapsed(ctx->kev[2], ctx->kev[3]);
}

template <int D>
ndb_status classify_impl(ndb_ctx *ctx, const float *coords, int64_t n, float eps, int32_t min_pts, uint32_t flags,
                         int32_t *nn_out) {
    cudaStream_t st = ctx->stream;
    ctx->have_state = false;
    ctx->have_labels = false;
    ctx->n = n;
    ctx->d = D;
    ctx->e2 = eps * eps;  // data_process.h:73, FP32 product
    ctx->min_pts = min_pts;
    ctx->flags_run = flags;
    ctx->stats = ndb_stats{};
    ctx->stats_pending = false;
    launch_counter() = 0;
    ensure(ctx, ctx->small, kSmallBytes);
    ck(ctx, cudaMemsetAsync(ctx->small.ptr, 0, kSmallBytes, st));
    cudaEventRecord(ctx->ev[0], st);

    if (flags & kFlagLoaded) {
        ctx->coords_dev = ctx->coords.as<float>();
    } else if (flags & NDB_FLAG_DEVICE_PTRS) {
        ctx->coords_dev = coords;
    } else {
        ctx->loaded = false;  // the loaded copy is overwritten
        ensure(ctx, ctx->coords, (size_t)n * D * sizeof(float));
        ck(ctx, cudaMemcpyAsync(ctx->coords.ptr, coords, (size_t)n * D * sizeof(float), cudaMemcpyHostToDevice, st));
        ctx->coords_dev = ctx->coords.as<float>();
    }

    // bounding box of the grid-eligible points (a loaded job's was reduced while it arrived)
    int *lo_hi = small_at<int>(ctx, kSmallBboxOff);
    unsigned long long *n_invalid = small_at<unsigned long long>(ctx, kSmallInvalidOff);
    if (flags & kFlagLoaded) {
        ck(ctx, cudaMemcpyAsync(lo_hi, ctx->load_box.ptr, 2 * D * sizeof(int), cudaMemcpyDeviceToDevice, st));
        ck(ctx, cudaMemcpyAsync(n_invalid, ctx->load_box.as<char>() + kLoadBoxInvalidOff, sizeof(unsigned long long),
                                cudaMemcpyDeviceToDevice, st));
        ++launch_counter(), set_int_kernel<<<1, 1, 0, st>>>(small_at<int>(ctx, kSmallErrOff) + 1, ctx->uf_max_steps);
    } else {
        ++launch_counter(), bbox_init_kernel<<<1, 32, 0, st>>>(lo_hi, D, n_invalid, small_at<int>(ctx, kSmallErrOff),
                                                               ctx->uf_max_steps);
        ++launch_counter(), bbox_kernel<D><<<std::min<unsigned>(blocks_for(n), 148 * 8), kBlock, 0, st>>>(
            ctx->coords_dev, n, lo_hi, n_invalid);
    }
    ck(ctx, cudaGetLastError());
    int h_lo_hi[2 * kMaxDim];
    unsigned long long h_invalid = 0;
    ck(ctx, cudaMemcpyAsync(h_lo_hi, lo_hi, 2 * D * sizeof(int), cudaMemcpyDeviceToHost, st));
    ck(ctx, cudaMemcpyAsync(&h_invalid, n_invalid, sizeof(h_invalid), cudaMemcpyDeviceToHost, st));
    ck(ctx, cudaStreamSynchronize(st));
    ctx->nv = n - (int64_t)h_invalid;
    double lo[kMaxDim], hi[kMaxDim];
    for (int a = 0; a < D; ++a) {
        auto dec = [](int v) {
            const int i = v >= 0 ? v : v ^ 0x7fffffff;
            float f;
            memcpy(&f, &i, sizeof(f));
            return (double)f;
        };
        lo[a] = ctx->nv > 0 ? dec(h_lo_hi[a]) : 0.0;
        hi[a] = ctx->nv > 0 ? dec(h_lo_hi[D + a]) : 0.0;
    }
    const Plan pl = plan_grid(D, ctx->e2, lo, hi);
    ctx->grid = pl.g;
    ctx->stencil = pl.st;
    ctx->n_rows = pl.st.n_rows;
    ctx->cell_units = pl.cell_units ? 1 : 0;
    if (pl.st.n_rows > kWarp) return NDB_ERR_INVALID_ARGUMENT;  // row tables hold one row per lane
    ctx->tc_count = tc_eligible(ctx, D, ctx->e2, lo, hi, pl.cell_units, pl.st.n_rows, flags);
    ctx->gram_count = gram_eligible(ctx, D, ctx->e2, lo, hi, flags);

    classify_dispatch<D>(ctx, pl);

    if (nn_out) {
        // counts in input order, straight into the caller's device buffer when there is one
        int32_t *target = nn_out;
        if (!(flags & NDB_FLAG_DEVICE_PTRS)) {
            ensure(ctx, ctx->nn_orig, (n + 1) * sizeof(int32_t));
            target = ctx->nn_orig.as<int32_t>();
        }
        for (int64_t lo = 0; lo < n; lo += kScatterWindow)
            ++launch_counter(), scatter_nn_kernel<<<blocks_for(n), kBlock, 0, st>>>(
                ctx->nn_sorted.as<int32_t>(), ctx->nv, n, ctx->ids0.as<int32_t>(), target, nullptr, 0, lo,
                n <= kScatterWindow ? INT64_MAX : lo + kScatterWindow);
        ck(ctx, cudaGetLastError());
        if (!(flags & NDB_FLAG_DEVICE_PTRS)) {
            if (ctx->in_run && ctx->copy_stream) {
                // nothing later in the job writes nn_orig: the copy overlaps the label phase
                ck(ctx, cudaEventRecord(ctx->ev_nn, st));
                ck(ctx, cudaStreamWaitEvent(ctx->copy_stream, ctx->ev_nn, 0));
                ck(ctx, cudaMemcpyAsync(nn_out, ctx->nn_orig.ptr, n * sizeof(int32_t), cudaMemcpyDeviceToHost,
                                        ctx->copy_stream));
                ctx->nn_pending = true;
            } else {
                ck(ctx, cudaMemcpyAsync(nn_out, ctx->nn_orig.ptr, n * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
            }
        }
    }
    ctx->stats.n_valid = ctx->nv;
    ctx->stats.n_cells = ctx->n_cells;
    ctx->stats.n_tiles = ctx->n_items;
    ctx->stats.grid_dims = pl.g.k;
    ctx->stats.stencil_rows = pl.st.n_rows;
    ctx->stats.same_cell_linked = ctx->cell_units;
    ctx->stats.key_bits = pl.key_bits;
    ctx->stats.tensor_filter = ctx->tc_count ? 1 : 0;
    ctx->have_state = true;
    if (ctx->in_run) {
        // ndb_b200_run goes on with the label phase, which reads these counters with
        // its own: no host round trip between the phases, and no host read queued
        // behind the count copy on the copy engine
        ctx->stats_pending = true;
        return NDB_OK;
    }
    ck(ctx, cudaStreamSynchronize(st));
    classify_stats<D>(ctx);
    return NDB_OK;
}

template <int D>
ndb_status labels_impl(ndb_ctx *ctx, int32_t *ci_out, ndb_result *result) {
    cudaStream_t st = ctx->stream;
    ctx->ci_user = ci_out;
    labels_phase<D>(ctx);
    ctx->ci_user = nullptr;
    const int64_t n = ctx->n;
    if (ci_out && !(ctx->flags_run & NDB_FLAG_DEVICE_PTRS))
        ck(ctx, cudaMemcpyAsync(ci_out, ctx->ci_orig.ptr, n * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    unsigned long long h_counters[kCounters];
    uint32_t h_scal[8];
    int h_err = 0;
    ck(ctx, cudaMemcpyAsync(h_counters, small_at<unsigned long long>(ctx, kSmallCountersOff), sizeof(h_counters),
                            cudaMemcpyDeviceToHost, st));
    ck(ctx, cudaMemcpyAsync(h_scal, small_at<uint32_t>(ctx, kSmallScalarOff), sizeof(h_scal), cudaMemcpyDeviceToHost,
                            st));
    ck(ctx, cudaMemcpyAsync(&h_err, small_at<int>(ctx, kSmallErrOff), sizeof(int), cudaMemcpyDeviceToHost, st));
    ck(ctx, cudaStreamSynchronize(st));
    if (ctx->stats_pending) {
        // classify_stats without its own copies: the label phase leaves counters 2 and 5
        // and scalar 4 as phase 1 wrote them
        ctx->stats_pending = false;
        ctx->stats.tensor_items = ctx->tc_count ? h_scal[4] : 0;
        ctx->stats.count_pairs = (int64_t)h_counters[2];
        ctx->stats.count_pair_dims = (int64_t)h_counters[2] * D;
        ctx->stats.count_fp32_ops = (int64_t)h_counters[2] * (ctx->gram_count ? D + 3 : 3 * D);
        ctx->stats.gram_filter = ctx->gram_count ? 1 : 0;
        ctx->stats.band_pairs = (int64_t)h_counters[5];
        audit_stats(ctx->stats, h_counters + 8);
        ctx->stats.ms_grid = elapsed(ctx->ev[0], ctx->ev[1]);
        ctx->stats.ms_count = elapsed(ctx->ev[1], ctx->ev[2]);
        ctx->stats.ms_sort_kernels = elapsed(ctx->kev[0], ctx->kev[1]);
        ctx->stats.ms_count_kernel = elapsed(ctx->kev[2], ctx->kev[3]);
    }
    if (h_err) return NDB_ERR_DEVICE_LIMIT;
    ctx->n_cores = h_scal[2];
    ctx->result.clusters = (int32_t)h_counters[0];
    ctx->result.noise = (int32_t)h_counters[1];
    ctx->result.core_count = (int32_t)ctx->n_cores;
    ctx->result.n = (int32_t)n;
    ctx->stats.union_pairs = (int64_t)h_counters[3];
    ctx->stats.border_pairs = (int64_t)h_counters[4];
    ctx->stats.union_pair_dims = (int64_t)h_counters[3] * D;
    ctx->stats.border_pair_dims = (int64_t)h_counters[4] * D;
    ctx->stats.ms_union = elapsed(ctx->ev[2], ctx->ev[3]);
    ctx->stats.ms_border = elapsed(ctx->ev[3], ctx->ev[4]);
    ctx->stats.ms_union_kernel = elapsed(ctx->kev[4], ctx->kev[5]);
    ctx->stats.ms_border_kernel = elapsed(ctx->kev[6], ctx->kev[7]);
    ctx->stats.kernel_launches = launch_counter();
    ctx->have_labels = true;
    if (result) *result = ctx->result;
    return NDB_OK;
}

template <int D>
ndb_status classify_entry(ndb_ctx *ctx, const float *coords, int64_t n, float eps, int32_t m, uint32_t flags,
                          int32_t *nn_out) {
    try {
        return classify_impl<D>(ctx, coords, n, eps, m, flags, nn_out);
    } catch (const Fail &f) {
        ctx->have_state = false;
        return f.st;
    }
}

template <int D>
ndb_status labels_entry(ndb_ctx *ctx, int32_t *ci_out, ndb_result *result) {
    try {
        return labels_impl<D>(ctx, ci_out, result);
    } catch (const Fail &f) {
        return f.st;
    }
}

// The reference's binary input (magma_input.h:113-125): int32 n, int32 d, then
// n*d float32 row-major.  Read in chunks into two pinned buffers; chunk k's copy to
// the device runs on the copy stream while chunk k+1 is read from the file, and the
// bounding-box kernel reduces chunk k on the context's stream as soon as it landed.
template <int D>
void bbox_chunk(ndb_ctx *ctx, const float *p, int64_t cnt) {
    int *lo_hi = ctx->load_box.as<int>();
    auto *inval = reinterpret_cast<unsigned long long *>(ctx->load_box.as<char>() + kLoadBoxInvalidOff);
    ++launch_counter(), bbox_kernel<D><<<std::min<unsigned>(blocks_for(cnt), 148 * 8), kBlock, 0, ctx->stream>>>(
        p, cnt, lo_hi, inval);
    ck(ctx, cudaGetLastError());
}

ndb_status load_bin_impl(ndb_ctx *ctx, FILE *f, int64_t *n_out, int32_t *d_out) {
    int32_t hdr[2];
    if (fread(hdr, sizeof(int32_t), 2, f) != 2) return NDB_ERR_IO;
    const int64_t n = hdr[0];
    const int d = hdr[1];
    if (n < 0) return NDB_ERR_IO;
    if (d < 1 || d > NDB_MAX_DIM) return NDB_ERR_UNSUPPORTED_DIM;
    if (fseeko(f, 0, SEEK_END) != 0) return NDB_ERR_IO;
    const off_t size = ftello(f);
    if (size < (off_t)(8 + n * d * (int64_t)sizeof(float)) || fseeko(f, 8, SEEK_SET) != 0) return NDB_ERR_IO;
    cudaStream_t st = ctx->stream;
    ensure(ctx, ctx->coords, (size_t)(n * d + 1) * sizeof(float));
    ensure(ctx, ctx->load_box, kLoadBoxBytes);
    if (ctx->pin_bytes < kPinChunk) {
        for (int b = 0; b < 2; ++b) {
            if (ctx->pin[b]) cudaFreeHost(ctx->pin[b]);
            ctx->pin[b] = nullptr;
        }
        ctx->pin_bytes = 0;
        for (int b = 0; b < 2; ++b) ck(ctx, cudaHostAlloc(&ctx->pin[b], kPinChunk, cudaHostAllocDefault));
        ctx->pin_bytes = kPinChunk;
    }
    for (int b = 0; b < 2; ++b) lazy_event(ctx, ctx->ev_pin[b]);
    ++launch_counter(), bbox_init_kernel<<<1, 32, 0, st>>>(
        ctx->load_box.as<int>(), d, reinterpret_cast<unsigned long long *>(ctx->load_box.as<char>() + kLoadBoxInvalidOff),
        reinterpret_cast<int *>(ctx->load_box.as<char>() + kLoadBoxErrOff), 0);
    ck(ctx, cudaGetLastError());
    const int64_t per = (int64_t)(ctx->pin_bytes / (sizeof(float) * d));
    int k = 0;
    for (int64_t off = 0; off < n; off += per, ++k) {
        const int b = k & 1;
        const int64_t cnt = std::min(per, n - off);
        if (k >= 2) ck(ctx, cudaEventSynchronize(ctx->ev_pin[b]));  // the buffer's previous copy is done
        if (fread(ctx->pin[b], sizeof(float) * d, (size_t)cnt, f) != (size_t)cnt) {
            cudaStreamSynchronize(ctx->copy_stream);
            return NDB_ERR_IO;
        }
        float *dst = ctx->coords.as<float>() + off * d;
        ck(ctx, cudaMemcpyAsync(dst, ctx->pin[b], (size_t)cnt * d * sizeof(float), cudaMemcpyHostToDevice,
                                ctx->copy_stream));
        ck(ctx, cudaEventRecord(ctx->ev_pin[b], ctx->copy_stream));
        ck(ctx, cudaStreamWaitEvent(st, ctx->ev_pin[b], 0));
        switch (d) {
            case 1: bbox_chunk<1>(ctx, dst, cnt); break;
            case 2: bbox_chunk<2>(ctx, dst, cnt); break;
            case 3: bbox_chunk<3>(ctx, dst, cnt); break;
            case 4: bbox_chunk<4>(ctx, dst, cnt); break;
            case 5: bbox_chunk<5>(ctx, dst, cnt); break;
            case 6: bbox_chunk<6>(ctx, dst, cnt); break;
            case 7: bbox_chunk<7>(ctx, dst, cnt); break;
            case 8: bbox_chunk<8>(ctx, dst, cnt); break;
            case 9: bbox_chunk<9>(ctx, dst, cnt); break;
            case 10: bbox_chunk<10>(ctx, dst, cnt); break;
            case 11: bbox_chunk<11>(ctx, dst, cnt); break;
            case 12: bbox_chunk<12>(ctx, dst, cnt); break;
            case 13: bbox_chunk<13>(ctx, dst, cnt); break;
            case 14: bbox_chunk<14>(ctx, dst, cnt); break;
            case 15: bbox_chunk<15>(ctx, dst, cnt); break;
            default: bbox_chunk<16>(ctx, dst, cnt); break;
        }
    }
    // the pinned buffers are reused by the next load: its first reads wait on these copies
    ctx->loaded = true;
    ctx->loaded_n = n;
    ctx->loaded_d = d;
    *n_out = n;
    *d_out = d;
    return NDB_OK;
}

ndb_status load_bin_file(ndb_ctx *ctx, FILE *f, int64_t *n_out, int32_t *d_out) {
    try {
        return load_bin_impl(ctx, f, n_out, d_out);
    } catch (const Fail &fl) {
        cudaStreamSynchronize(ctx->copy_stream);
        return fl.st;
    }
}

// ndb_b200_assign_border: the border pass again, with the caller's ids for the cores.
template <int D>
ndb_status border_ids_impl(ndb_ctx *ctx, const int32_t *core_ids, int32_t *ci_out) {
    cudaStream_t st = ctx->stream;
    const int64_t n = ctx->n, nv = ctx->nv;
    const bool dev = (ctx->flags_run & NDB_FLAG_DEVICE_PTRS) != 0;
    const int32_t *ids = core_ids;
    if (!dev) {
        ensure(ctx, ctx->ids_in, (size_t)(n + 1) * sizeof(int32_t));
        ck(ctx, cudaMemcpyAsync(ctx->ids_in.ptr, core_ids, n * sizeof(int32_t), cudaMemcpyHostToDevice, st));
        ids = ctx->ids_in.as<int32_t>();
    }
    ++launch_counter(), set_core_ids_kernel<<<blocks_for(nv), kBlock, 0, st>>>(
        nv, ctx->core_sorted.as<uint8_t>(), ctx->ids0.as<int32_t>(), ids, ctx->pcell.as<int32_t>(), ctx->cell_units,
        ctx->ci_sorted.as<int32_t>(), ctx->cell_cid.as<int32_t>());
    ck(ctx, cudaGetLastError());
    border_phase<D>(ctx);
    if (ci_out) {
        int32_t *target = ci_out;
        if (!dev) {
            ensure(ctx, ctx->ci_orig, (n + 1) * sizeof(int32_t));
            target = ctx->ci_orig.as<int32_t>();
        }
        ++launch_counter(), output_ids_kernel<<<blocks_for(n), kBlock, 0, st>>>(
            ctx->ci_sorted.as<int32_t>(), nv, n, ctx->ids0.as<int32_t>(), ctx->core_bits.as<uint32_t>(), ids, target);
        ck(ctx, cudaGetLastError());
        if (!dev) ck(ctx, cudaMemcpyAsync(ci_out, target, n * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    }
    ck(ctx, cudaStreamSynchronize(st));
    return NDB_OK;
}

template <int D>
ndb_status border_ids_entry(ndb_ctx *ctx, const int32_t *core_ids, int32_t *ci_out) {
    try {
        return border_ids_impl<D>(ctx, core_ids, ci_out);
    } catch (const Fail &f) {
        return f.st;
    }
}

#define NDB_DISPATCH_D(d, CALL)  \
    switch (d) {                 \
        case 1: return CALL(1);  \
        case 2: return CALL(2);  \
        case 3: return CALL(3);  \
        case 4: return CALL(4);  \
        case 5: return CALL(5);  \
        case 6: return CALL(6);  \
        case 7: return CALL(7);  \
        case 8: return CALL(8);  \
        case 9: return CALL(9);  \
        case 10: return CALL(10); \
        case 11: return CALL(11); \
        case 12: return CALL(12); \
        case 13: return CALL(13); \
        case 14: return CALL(14); \
        case 15: return CALL(15); \
        case 16: return CALL(16); \
        default: return NDB_ERR_UNSUPPORTED_DIM; \
    }

}  // namespace

extern "C" {

ndb_status ndb_b200_create(ndb_ctx **out, int32_t device) {
    if (!out) return NDB_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
        cudaGetLastError();
        return NDB_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= count) return NDB_ERR_NO_DEVICE;
    if (cudaSetDevice(device) != cudaSuccess) return NDB_ERR_NO_DEVICE;
    ndb_ctx *ctx = new ndb_ctx();
    ctx->device = device;
    if (cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        ctx->sm_count <= 0)
        ctx->sm_count = 148;
    if (cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return NDB_ERR_CUDA;
    }
    ctx->stream = ctx->own_stream;
    if (cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->ev_nn, cudaEventDisableTiming) != cudaSuccess) {
        ndb_b200_destroy(ctx);
        return NDB_ERR_CUDA;
    }
    for (auto &e : ctx->ev) {
        if (cudaEventCreate(&e) != cudaSuccess) {
            ndb_b200_destroy(ctx);  // frees the stream and the events made so far
            return NDB_ERR_CUDA;
        }
    }
    for (auto &e : ctx->kev) {
        if (cudaEventCreate(&e) != cudaSuccess) {
            ndb_b200_destroy(ctx);
            return NDB_ERR_CUDA;
        }
    }
    *out = ctx;
    return NDB_OK;
}

ndb_status ndb_b200_destroy(ndb_ctx *ctx) {
    if (!ctx) return NDB_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
    ctx->for_each_buf([](DevBuf &b) { b.release(); });
    for (auto &e : ctx->ev)
        if (e) cudaEventDestroy(e);
    for (auto &e : ctx->kev)
        if (e) cudaEventDestroy(e);
    if (ctx->ev_nn) cudaEventDestroy(ctx->ev_nn);
    for (auto &e : ctx->ev_grp)
        if (e) cudaEventDestroy(e);
    for (auto &e : ctx->ev_done)
        if (e) cudaEventDestroy(e);
    for (int b = 0; b < 2; ++b) {
        if (ctx->ev_pin[b]) cudaEventDestroy(ctx->ev_pin[b]);
        if (ctx->pin[b]) cudaFreeHost(ctx->pin[b]);
    }
    if (ctx->mail) cudaFreeHost(ctx->mail);
    if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return NDB_OK;
}

ndb_status ndb_b200_set_memory_limit(ndb_ctx *ctx, int64_t max_bytes) {
    if (!ctx || max_bytes < 0) return NDB_ERR_INVALID_ARGUMENT;
    ctx->mem_limit = (size_t)max_bytes;
    if (ctx->mem_limit && ctx->held_bytes() > ctx->mem_limit) {
        // drop every buffer; the next run allocates what it needs under the new cap
        cudaSetDevice(ctx->device);
        if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return NDB_ERR_CUDA;
        ctx->for_each_buf([](DevBuf &b) { b.release(); });
        ctx->have_state = false;
        ctx->have_labels = false;
    }
    return NDB_OK;
}

ndb_status ndb_b200_set_tuning(ndb_ctx *ctx, const ndb_tuning *tuning) {
    if (!ctx) return NDB_ERR_INVALID_ARGUMENT;
    if (!tuning) {
        ctx->tuning = ndb_tuning{0, 0, 0};
        return NDB_OK;
    }
    if (tuning->tc_min_dim < 0 || tuning->tc_min_item < 0 || tuning->gram_filter < 0) return NDB_ERR_INVALID_ARGUMENT;
    ctx->tuning = *tuning;
    return NDB_OK;
}

ndb_status ndb_b200_set_debug_limits(ndb_ctx *ctx, int64_t uf_max_steps) {
    if (!ctx || uf_max_steps < 0 || uf_max_steps > INT32_MAX) return NDB_ERR_INVALID_ARGUMENT;
    ctx->uf_max_steps = (int)uf_max_steps;
    return NDB_OK;
}

ndb_status ndb_b200_get_tuning(ndb_ctx *ctx, ndb_tuning *tuning) {
    if (!ctx || !tuning) return NDB_ERR_INVALID_ARGUMENT;
    *tuning = ctx->tuning;
    return NDB_OK;
}

ndb_status ndb_b200_device_bytes(ndb_ctx *ctx, int64_t *bytes) {
    if (!ctx || !bytes) return NDB_ERR_INVALID_ARGUMENT;
    *bytes = (int64_t)ctx->held_bytes();
    return NDB_OK;
}

ndb_status ndb_b200_set_stream(ndb_ctx *ctx, void *stream) {
    if (!ctx) return NDB_ERR_INVALID_ARGUMENT;
    ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
    return NDB_OK;
}

// ndb_b200_classify with the internal flag allowed (the loaded job).
static ndb_status classify_checked(ndb_ctx *ctx, const float *coords, int64_t n, int32_t d, float eps,
                                   int32_t min_pts, uint32_t flags, int32_t *nn_out) {
    ndb_status s = check_ctx(ctx);
    if (s != NDB_OK) return s;
    if (flags & ~(kAllFlags | kFlagLoaded)) return NDB_ERR_INVALID_ARGUMENT;
    if (n < 0) return NDB_ERR_INVALID_ARGUMENT;
    if (n > NDB_MAX_POINTS) return NDB_ERR_TOO_MANY_POINTS;
    if (d < 1 || d > NDB_MAX_DIM) return NDB_ERR_UNSUPPORTED_DIM;
    if (n > 0 && !coords && !(flags & kFlagLoaded)) return NDB_ERR_INVALID_ARGUMENT;
    const float e2 = eps * eps;
    if (!isfinite(e2)) return NDB_ERR_INVALID_EPS;
    if ((flags & NDB_FLAG_DEVICE_PTRS) && n > 0) {
        if (!(flags & kFlagLoaded) && !is_device_ptr(coords)) return NDB_ERR_INVALID_ARGUMENT;
        if (nn_out && !is_device_ptr(nn_out)) return NDB_ERR_INVALID_ARGUMENT;
    }
    if (n == 0) {
        ctx->have_state = true;
        ctx->have_labels = false;
        ctx->n = 0;
        ctx->nv = 0;
        ctx->n_cells = 0;
        ctx->n_items = 0;
        ctx->d = d;
        ctx->min_pts = min_pts;
        ctx->flags_run = flags;
        ctx->stats = ndb_stats{};
        return NDB_OK;
    }
#define NDB_CLASSIFY(D) classify_entry<D>(ctx, coords, n, eps, min_pts, flags, nn_out)
    NDB_DISPATCH_D(d, NDB_CLASSIFY)
#undef NDB_CLASSIFY
}

ndb_status ndb_b200_classify(ndb_ctx *ctx, const float *coords, int64_t n, int32_t d, float eps, int32_t min_pts,
                             uint32_t flags, int32_t *nn_out) {
    if (flags & kFlagLoaded) return NDB_ERR_INVALID_ARGUMENT;
    return classify_checked(ctx, coords, n, d, eps, min_pts, flags, nn_out);
}

ndb_status ndb_b200_assign_labels(ndb_ctx *ctx, int32_t *cluster_index_out, ndb_result *result) {
    ndb_status s = check_ctx(ctx);
    if (s != NDB_OK) return s;
    if (!ctx->have_state) return NDB_ERR_NO_STATE;
    if (ctx->n == 0) {
        ctx->result = ndb_result{0, 0, 0, 0};
        ctx->n_cores = 0;
        ctx->have_labels = true;
        if (result) *result = ctx->result;
        return NDB_OK;
    }
    if ((ctx->flags_run & NDB_FLAG_DEVICE_PTRS) && cluster_index_out && !is_device_ptr(cluster_index_out))
        return NDB_ERR_INVALID_ARGUMENT;
#define NDB_LABELS(D) labels_entry<D>(ctx, cluster_index_out, result)
    NDB_DISPATCH_D(ctx->d, NDB_LABELS)
#undef NDB_LABELS
}

static ndb_status run_checked(ndb_ctx *ctx, const float *coords, int64_t n, int32_t d, float eps, int32_t min_pts,
                              uint32_t flags, int32_t *nn_out, int32_t *cluster_index_out, ndb_result *result) {
    if (!ctx) return NDB_ERR_INVALID_ARGUMENT;
    ctx->in_run = true;
    ndb_status s = classify_checked(ctx, coords, n, d, eps, min_pts, flags, nn_out);
    ctx->in_run = false;
    if (s == NDB_OK) s = ndb_b200_assign_labels(ctx, cluster_index_out, result);
    if (ctx->nn_pending) {
        // the counts are in the caller's buffer only once their copy is done
        ctx->nn_pending = false;
        cudaSetDevice(ctx->device);
        if (cudaStreamSynchronize(ctx->copy_stream) != cudaSuccess && s == NDB_OK) s = NDB_ERR_CUDA;
    }
    return s;
}

ndb_status ndb_b200_run(ndb_ctx *ctx, const float *coords, int64_t n, int32_t d, float eps, int32_t min_pts,
                        uint32_t flags, int32_t *nn_out, int32_t *cluster_index_out, ndb_result *result) {
    if (flags & kFlagLoaded) return NDB_ERR_INVALID_ARGUMENT;
    return run_checked(ctx, coords, n, d, eps, min_pts, flags, nn_out, cluster_index_out, result);
}

ndb_status ndb_b200_load_bin(ndb_ctx *ctx, const char *path, int64_t *n_out, int32_t *d_out) {
    ndb_status s = check_ctx(ctx);
    if (s != NDB_OK) return s;
    if (!path || !n_out || !d_out) return NDB_ERR_INVALID_ARGUMENT;
    ctx->loaded = false;
    ctx->have_state = false;
    ctx->have_labels = false;
    FILE *f = fopen(path, "rb");
    if (!f) return NDB_ERR_IO;
    s = load_bin_file(ctx, f, n_out, d_out);
    fclose(f);
    return s;
}

ndb_status ndb_b200_run_loaded(ndb_ctx *ctx, float eps, int32_t min_pts, uint32_t flags, int32_t *nn_out,
                               int32_t *cluster_index_out, ndb_result *result) {
    if (!ctx) return NDB_ERR_INVALID_ARGUMENT;
    if (!ctx->loaded) return NDB_ERR_NO_STATE;
    if (flags & ~kAllFlags) return NDB_ERR_INVALID_ARGUMENT;
    return run_checked(ctx, ctx->coords.as<float>(), ctx->loaded_n, ctx->loaded_d, eps, min_pts, flags | kFlagLoaded,
                       nn_out, cluster_index_out, result);
}

ndb_status ndb_b200_cluster_label(ndb_ctx *ctx, int32_t *label_out, int64_t capacity) {
    ndb_status s = check_ctx(ctx);
    if (s != NDB_OK) return s;
    if (!ctx->have_labels) return NDB_ERR_NO_STATE;
    if (capacity < ctx->n_cores || (ctx->n_cores > 0 && !label_out)) return NDB_ERR_INVALID_ARGUMENT;
    if (ctx->n_cores == 0) return NDB_OK;
    if (grow(ctx, ctx->labels, (size_t)(ctx->n_cores + 1) * sizeof(int32_t)) != cudaSuccess)
        return NDB_ERR_OUT_OF_MEMORY;
    ++launch_counter(), labels_kernel<<<blocks_for(ctx->n), kBlock, 0, ctx->stream>>>(
        ctx->ci_sorted.as<int32_t>(), ctx->nv, ctx->n, ctx->ids0.as<int32_t>(), ctx->core_bits.as<uint32_t>(),
        ctx->core_prefix.as<uint32_t>(), ctx->labels.as<int32_t>());
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyAsync(label_out, ctx->labels.ptr, ctx->n_cores * sizeof(int32_t), cudaMemcpyDeviceToHost,
                        ctx->stream) != cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess)
        return NDB_ERR_CUDA;
    return NDB_OK;
}

ndb_status ndb_b200_assign_border(ndb_ctx *ctx, const int32_t *core_ids, int32_t *cluster_index_out) {
    ndb_status s = check_ctx(ctx);
    if (s != NDB_OK) return s;
    if (!ctx->have_labels) return NDB_ERR_NO_STATE;
    if (ctx->n == 0) return NDB_OK;
    if (!core_ids) return NDB_ERR_INVALID_ARGUMENT;
    if (ctx->flags_run & NDB_FLAG_DEVICE_PTRS) {
        if (!is_device_ptr(core_ids) || (cluster_index_out && !is_device_ptr(cluster_index_out)))
            return NDB_ERR_INVALID_ARGUMENT;
    }
    // the pass replaces the library's own ids: ndb_b200_cluster_label would now report the caller's
    ctx->have_labels = false;
#define NDB_BORDER(D) border_ids_entry<D>(ctx, core_ids, cluster_index_out)
    NDB_DISPATCH_D(ctx->d, NDB_BORDER)
#undef NDB_BORDER
}

ndb_status ndb_b200_get_stats(ndb_ctx *ctx, ndb_stats *stats) {
    if (!ctx || !stats) return NDB_ERR_INVALID_ARGUMENT;
    *stats = ctx->stats;
    return NDB_OK;
}

const char *ndb_b200_strerror(ndb_status s) {
    switch (s) {
        case NDB_OK: return "ok";
        case NDB_ERR_INVALID_ARGUMENT: return "invalid argument";
        case NDB_ERR_UNSUPPORTED_DIM: return "unsupported dimensionality (1..16)";
        case NDB_ERR_INVALID_EPS: return "eps*eps is not a finite float";
        case NDB_ERR_TOO_MANY_POINTS: return "too many points for int32 indices";
        case NDB_ERR_OUT_OF_MEMORY: return "device out of memory";
        case NDB_ERR_CUDA: return "CUDA error";
        case NDB_ERR_NO_DEVICE: return "no CUDA device";
        case NDB_ERR_DEVICE_LIMIT: return "device-side iteration bound reached";
        case NDB_ERR_NO_STATE: return "no classified job in this context";
        case NDB_ERR_BAD_JOB: return "invalid batched job descriptor";
        case NDB_ERR_IO: return "cannot read the input file (missing, short, or a bad header)";
    }
    return "unknown status";
}

const char *ndb_b200_last_cuda_error(ndb_ctx *ctx) { return ctx ? ctx->last_cuda_error.c_str() : ""; }

const char *ndb_b200_version(void) { return NDB_VERSION; }

}  // extern "C"

// ---------------------------------------------------------------------------
// Batched runs (ndb_b200_run_batched)
// ---------------------------------------------------------------------------
namespace {

constexpr int64_t kMaxBatchPoints = int64_t(1) << 30;  // points of one pipeline (int32 indices, headroom)

struct BatchPlan {
    std::vector<JobDev> jd;  // per member, in member order
    Stencil st{};
    int key_bits = 0;
    int linked = 0;
    int list_stride = 0;
    bool tc = false;  // neighbour count on the tensor-core filter (every job eligible)
    bool gram = true; // CUDA-core count with the Gram filter (every job eligible)
    int64_t total_n = 0, nv = 0;
    double columns = 0;  // entries of the pipeline's column table (sum over its jobs)
};

template <int D, typename K>
void run_group_keys(ndb_ctx *ctx, ndb_job *jobs, const std::vector<int> &members, BatchPlan &bp, uint32_t flags) {
    cudaStream_t st = ctx->stream;
    constexpr int P = Stride<D>::P;
    const int nj = (int)members.size();
    const int64_t n = bp.total_n, nv = bp.nv;
    const JobDev *jobs_dev = ctx->jobs_dev.as<JobDev>();
    unsigned long long *counters = small_at<unsigned long long>(ctx, kSmallCountersOff);
    int *err = small_at<int>(ctx, kSmallErrOff);
    uint32_t *scal = small_at<uint32_t>(ctx, kSmallScalarOff);
    int64_t max_n = 1;
    for (auto &j : bp.jd) max_n = std::max<int64_t>(max_n, j.n);
    const unsigned gx = (unsigned)std::min<int64_t>((max_n + kBlock - 1) / kBlock, 64);

    cudaEventRecord(ctx->ev[0], st);
    // composite keys and the sort
    ensure(ctx, ctx->keys0, n * sizeof(K));
    ensure(ctx, ctx->keys1, n * sizeof(K));
    ensure(ctx, ctx->ids0, n * sizeof(int32_t));
    ensure(ctx, ctx->ids1, n * sizeof(int32_t));
    ensure(ctx, ctx->sort_hist, sort_hist_words(n) * sizeof(uint32_t));
    const size_t scan_words = std::max(scan_scratch_words(n + 1), scan_scratch_words((int64_t)sort_hist_words(n)));
    ensure(ctx, ctx->scan_scratch, (scan_words + 64) * sizeof(uint32_t));
    const K invalid_key = (K)(bp.key_bits >= (int)(8 * sizeof(K)) ? ~(K)0 : (((K)1 << bp.key_bits) - 1));
    ++launch_counter(), key_batch_kernel<D, K><<<dim3(gx, nj), kBlock, 0, st>>>(
        ctx->coords.as<float>(), jobs_dev, invalid_key, ctx->keys0.as<K>(), ctx->ids0.as<int32_t>());
    ck(ctx, cudaGetLastError());
    bool in_first = true;
    cudaEventRecord(ctx->kev[0], st);
    if (sizeof(K) == 4)
        ck(ctx, radix_sort_pairs_u32(reinterpret_cast<uint32_t *>(ctx->keys0.ptr), ctx->ids0.as<int32_t>(),
                                     reinterpret_cast<uint32_t *>(ctx->keys1.ptr), ctx->ids1.as<int32_t>(), n,
                                     bp.key_bits, ctx->sort_hist.as<uint32_t>(), ctx->scan_scratch.as<uint32_t>(),
                                     &in_first, st));
    else
        ck(ctx, radix_sort_pairs_u64(reinterpret_cast<uint64_t *>(ctx->keys0.ptr), ctx->ids0.as<int32_t>(),
                                     reinterpret_cast<uint64_t *>(ctx->keys1.ptr), ctx->ids1.as<int32_t>(), n,
                                     bp.key_bits, ctx->sort_hist.as<uint32_t>(), ctx->scan_scratch.as<uint32_t>(),
                                     &in_first, st));
    cudaEventRecord(ctx->kev[1], st);
    if (!in_first) {
        std::swap(ctx->keys0, ctx->keys1);
        std::swap(ctx->ids0, ctx->ids1);
    }
    const K *keys = ctx->keys0.as<K>();
    const int32_t *perm = ctx->ids0.as<int32_t>();

    // cells
    ensure(ctx, ctx->flags, (n + 1) * sizeof(uint32_t));
    ensure(ctx, ctx->pos, (n + 1) * sizeof(uint32_t));
    ensure(ctx, ctx->pcell, (n + 1) * sizeof(int32_t));
    ensure(ctx, ctx->cell_start, (n + 2) * sizeof(int32_t));
    ensure(ctx, ctx->cell_key, (n + 1) * sizeof(K));
    ++launch_counter(), cell_flag_kernel<K><<<blocks_for(nv), kBlock, 0, st>>>(keys, nv, ctx->flags.as<uint32_t>());
    ck(ctx, scan_exclusive_u32(ctx->flags.as<uint32_t>(), ctx->pos.as<uint32_t>(), nv, scal + 0,
                               ctx->scan_scratch.as<uint32_t>(), st));
    ++launch_counter(), cell_write_kernel<K><<<blocks_for(nv), kBlock, 0, st>>>(
        keys, nv, ctx->pos.as<uint32_t>(), scal + 0, ctx->cell_start.as<int32_t>(), ctx->cell_key.as<K>(),
        ctx->pcell.as<int32_t>());
    ensure(ctx, ctx->xs, (nv + 1) * P * sizeof(float));
    ++launch_counter(), gather_kernel<D><<<blocks_for(nv), kBlock, 0, st>>>(ctx->coords.as<float>(), perm, nv,
                                                                           ctx->xs.as<float>());
    ck(ctx, cudaGetLastError());
    const uint32_t *m_cells = mail_from_device(ctx, scal + 0, 1, st);
    ck(ctx, cudaStreamSynchronize(st));
    const int64_t n_cells = nv > 0 ? *m_cells : 0;
    ensure(ctx, ctx->cell_job, (n_cells + 1) * sizeof(int32_t));
    ++launch_counter(), cell_job_kernel<K><<<blocks_for(n_cells), kBlock, 0, st>>>(
        ctx->cell_key.as<K>(), n_cells, jobs_dev, nj, ctx->cell_job.as<int32_t>());
    const int32_t *cell_job = ctx->cell_job.as<int32_t>();

    // neighbour rows through the column table (or the hash table) of the cells
    const int n_rows = bp.st.n_rows;
    const CellIndex<K> L = build_cell_index<K>(ctx, n_cells, (double)bp.columns, bp.jd[0].g, jobs_dev, cell_job);
    ensure(ctx, ctx->nbr, (size_t)(n_cells * n_rows + 1) * sizeof(int2));
    int4 *rows_dev = small_at<int4>(ctx, kSmallStencilOff);
    mail_to_device(ctx, rows_dev, bp.st.rows, (size_t)n_rows, st);
    const int rlog = row_group_log2(n_rows);
    ++launch_counter(), rows_kernel<K><<<blocks_for(n_cells << rlog), kBlock, 0, st>>>(
        ctx->cell_key.as<K>(), n_cells, bp.jd[0].g, rows_dev, n_rows, rlog, L, ctx->nbr.as<int2>(), jobs_dev,
        cell_job);
    ck(ctx, cudaGetLastError());

    // work items
    ensure(ctx, ctx->item_cnt, (n_cells + 1) * sizeof(uint32_t));
    ++launch_counter(), item_count_kernel<<<blocks_for(n_cells), kBlock, 0, st>>>(
        ctx->cell_start.as<int32_t>(), n_cells, ctx->item_cnt.as<uint32_t>());
    ck(ctx, scan_exclusive_u32(ctx->item_cnt.as<uint32_t>(), ctx->item_cnt.as<uint32_t>(), n_cells, scal + 1,
                               ctx->scan_scratch.as<uint32_t>(), st));
    const uint32_t *m_items = mail_from_device(ctx, scal + 1, 1, st);
    ck(ctx, cudaStreamSynchronize(st));
    const int64_t n_items = n_cells > 0 ? *m_items : 0;
    ensure(ctx, ctx->items, (n_items + 1) * sizeof(int2));
    ++launch_counter(), item_write_kernel<<<blocks_for(n_cells), kBlock, 0, st>>>(
        ctx->cell_start.as<int32_t>(), n_cells, ctx->item_cnt.as<uint32_t>(), ctx->items.as<int2>());

    // neighbour counts and core flags
    ensure(ctx, ctx->nn_sorted, (n + 1) * sizeof(int32_t));
    int32_t *list = nullptr;
    if (bp.list_stride > 0) {
        ensure(ctx, ctx->nbr_list, (size_t)(nv * bp.list_stride + 1) * sizeof(int32_t));
        list = ctx->nbr_list.as<int32_t>();
    }
    const bool early = (flags & NDB_FLAG_FULL_COUNT) == 0;
    cudaEventRecord(ctx->ev[1], st);
    cudaEventRecord(ctx->kev[2], st);
    count_items<D>(ctx, bp.tc, (flags & NDB_FLAG_TENSOR_FILTER) != 0, bp.gram, early, n_items,
                   ctx->items.as<int2>(),
                   ctx->cell_start.as<int32_t>(), ctx->nbr.as<int2>(), n_rows, ctx->xs.as<float>(), 0.0f, 0, 0,
                   ctx->nn_sorted.as<int32_t>(), list, 0, bp.list_stride, jobs_dev, cell_job,
                   (flags & NDB_FLAG_FILTER_AUDIT) != 0);
    cudaEventRecord(ctx->kev[3], st);
    const int64_t n_words = (n + 31) / 32;
    ensure(ctx, ctx->core_sorted, n + 1);
    ensure(ctx, ctx->cell_has_core, n_cells + 1);
    ensure(ctx, ctx->core_bits, (n_words + 1) * sizeof(uint32_t));
    ensure(ctx, ctx->core_prefix, (n_words + 1) * sizeof(uint32_t));
    fill_bytes(ctx, ctx->cell_has_core.ptr, 0, (size_t)n_cells + 1, st);
    fill_bytes(ctx, ctx->core_bits.ptr, 0, (size_t)(n_words + 1) * sizeof(uint32_t), st);
    ++launch_counter(), core_flags_kernel<<<blocks_for(n), kBlock, 0, st>>>(
        ctx->nn_sorted.as<int32_t>(), nv, n, 0, perm, ctx->pcell.as<int32_t>(), ctx->core_sorted.as<uint8_t>(),
        ctx->cell_has_core.as<uint8_t>(), ctx->core_bits.as<uint32_t>(), jobs_dev, cell_job, nj);
    ++launch_counter(), popc_words_kernel<<<blocks_for(n_words), kBlock, 0, st>>>(
        ctx->core_bits.as<uint32_t>(), n_words, ctx->core_prefix.as<uint32_t>());
    ck(ctx, cudaGetLastError());
    ck(ctx, scan_exclusive_u32(ctx->core_prefix.as<uint32_t>(), ctx->core_prefix.as<uint32_t>(), n_words, scal + 2,
                               ctx->scan_scratch.as<uint32_t>(), st));
    cudaEventRecord(ctx->ev[2], st);

    // union-find, canonical ids, border points
    const int64_t n_units = bp.linked ? n_cells : nv;
    ensure(ctx, ctx->parent, (n_units + 1) * sizeof(int32_t));
    ensure(ctx, ctx->comp_min, (n_units + 1) * sizeof(int32_t));
    ensure(ctx, ctx->ci_sorted, (n + 1) * sizeof(int32_t));
    ensure(ctx, ctx->cell_cid, (n_cells + 1) * sizeof(int32_t));
    ensure(ctx, ctx->job_counters, (size_t)(4 * nj + 4) * sizeof(unsigned long long));
    unsigned long long *jc = ctx->job_counters.as<unsigned long long>();
    fill_bytes(ctx, jc, 0, (size_t)(4 * nj + 4) * sizeof(unsigned long long), st);
    ++launch_counter(), iota_kernel<<<blocks_for(n_units), kBlock, 0, st>>>(ctx->parent.as<int32_t>(), n_units);
    ++launch_counter(), fill_kernel<<<blocks_for(n_units), kBlock, 0, st>>>(ctx->comp_min.as<int32_t>(), n_units,
                                                                           kNoCluster);
    cudaEventRecord(ctx->kev[4], st);
    if (n_items > 0) {
        if (bp.linked) {
            if (bp.list_stride > 0)
                ++launch_counter(), union_lists_kernel<<<blocks_for(nv), kBlock, 0, st>>>(
                    nv, ctx->nn_sorted.as<int32_t>(), list, 0, bp.list_stride, ctx->core_sorted.as<uint8_t>(),
                    ctx->parent.as<int32_t>(), err, jobs_dev, cell_job, ctx->pcell.as<int32_t>(), 1,
                    (flags & NDB_FLAG_FULL_COUNT) == 0, ctx->cell_start.as<int32_t>(), 0);
            ++launch_counter(), union_near_kernel<D, K><<<blocks_for(n_cells), kBlock, 0, st>>>(
                n_cells, bp.jd[0].g, ctx->cell_key.as<K>(), ctx->cell_start.as<int32_t>(), L,
                ctx->xs.as<float>(), 0.0f, ctx->core_sorted.as<uint8_t>(),
                ctx->cell_has_core.as<uint8_t>(), ctx->parent.as<int32_t>(), counters + 3, err, jobs_dev, cell_job);
            ++launch_counter(), flatten_snap_kernel<<<blocks_for(n_units), kBlock, 0, st>>>(
                ctx->parent.as<int32_t>(), n_units, err, ctx->cell_has_core.as<uint8_t>(), ctx->comp_min.as<int32_t>());
            ++launch_counter(), union_cells_kernel<D><<<blocks_for(n_cells * kWarp), kBlock, 0, st>>>(
                n_cells, ctx->cell_start.as<int32_t>(), ctx->nbr.as<int2>(), n_rows, ctx->xs.as<float>(), 0.0f,
                ctx->core_sorted.as<uint8_t>(), ctx->cell_has_core.as<uint8_t>(), ctx->parent.as<int32_t>(),
                counters + 3, err, jobs_dev, cell_job, ctx->comp_min.as<int32_t>());
            ++launch_counter(), fill_kernel<<<blocks_for(n_units), kBlock, 0, st>>>(ctx->comp_min.as<int32_t>(), n_units,
                                                                                   kNoCluster);
        } else {
            if (bp.list_stride > 0) {
                ++launch_counter(), union_lists_kernel<<<blocks_for(nv), kBlock, 0, st>>>(
                    nv, ctx->nn_sorted.as<int32_t>(), list, 0, bp.list_stride, ctx->core_sorted.as<uint8_t>(),
                    ctx->parent.as<int32_t>(), err, jobs_dev, cell_job, ctx->pcell.as<int32_t>(), 0, 0,
                    ctx->cell_start.as<int32_t>(), 0);
                ++launch_counter(), flatten_kernel<<<blocks_for(n_units), kBlock, 0, st>>>(ctx->parent.as<int32_t>(),
                                                                                          n_units, err);
            }
            fill_bytes(ctx, ctx->cell_cid.ptr, 0xff, (size_t)n_cells * sizeof(int32_t), st);  // -1
            ++launch_counter(), cell_root_kernel<<<blocks_for(nv), kBlock, 0, st>>>(
                nv, ctx->pcell.as<int32_t>(), ctx->core_sorted.as<uint8_t>(), ctx->parent.as<int32_t>(),
                ctx->cell_cid.as<int32_t>());
            const unsigned pgrid = (unsigned)((n_items + kCountWarps - 1) / kCountWarps);
            ++launch_counter(), union_points_kernel<D><<<pgrid, kCountWarps * kWarp, 0, st>>>(
                ctx->items.as<int2>(), n_items, ctx->cell_start.as<int32_t>(), ctx->nbr.as<int2>(), n_rows,
                ctx->xs.as<float>(), 0.0f, ctx->core_sorted.as<uint8_t>(), ctx->cell_has_core.as<uint8_t>(),
                ctx->parent.as<int32_t>(), counters + 3, err, jobs_dev, cell_job, ctx->cell_cid.as<int32_t>());
        }
        ck(ctx, cudaGetLastError());
    }
    cudaEventRecord(ctx->kev[5], st);
    ++launch_counter(), flatten_kernel<<<blocks_for(n_units), kBlock, 0, st>>>(ctx->parent.as<int32_t>(), n_units, err);
    if (bp.linked)
        ++launch_counter(), comp_min_cells_kernel<<<blocks_for(n_cells), kBlock, 0, st>>>(
            n_cells, ctx->cell_start.as<int32_t>(), ctx->cell_has_core.as<uint8_t>(), ctx->core_sorted.as<uint8_t>(),
            perm, ctx->core_bits.as<uint32_t>(), ctx->core_prefix.as<uint32_t>(), ctx->parent.as<int32_t>(),
            ctx->comp_min.as<int32_t>());
    else
        ++launch_counter(), comp_min_kernel<<<blocks_for(nv), kBlock, 0, st>>>(
            nv, ctx->core_sorted.as<uint8_t>(), perm, ctx->pcell.as<int32_t>(), bp.linked,
            ctx->core_bits.as<uint32_t>(), ctx->core_prefix.as<uint32_t>(), ctx->parent.as<int32_t>(),
            ctx->comp_min.as<int32_t>());
    ++launch_counter(), core_ids_kernel<<<blocks_for(nv), kBlock, 0, st>>>(
        nv, ctx->core_sorted.as<uint8_t>(), ctx->pcell.as<int32_t>(), bp.linked, ctx->parent.as<int32_t>(),
        ctx->comp_min.as<int32_t>(), ctx->ci_sorted.as<int32_t>(), counters, cell_job, jc);
    if (bp.linked)
        ++launch_counter(), cell_ids_kernel<<<blocks_for(n_cells), kBlock, 0, st>>>(
            n_cells, ctx->cell_has_core.as<uint8_t>(), ctx->parent.as<int32_t>(), ctx->comp_min.as<int32_t>(),
            ctx->cell_cid.as<int32_t>(), counters, cell_job, jc);
    cudaEventRecord(ctx->ev[3], st);
    cudaEventRecord(ctx->kev[6], st);
    if (bp.list_stride > 0)
        ++launch_counter(), border_list_kernel<<<blocks_for(nv), kBlock, 0, st>>>(
            nv, ctx->nn_sorted.as<int32_t>(), list, bp.list_stride, ctx->core_sorted.as<uint8_t>(), bp.linked,
            ctx->pcell.as<int32_t>(), ctx->cell_cid.as<int32_t>(), ctx->ci_sorted.as<int32_t>(), counters + 4);
    ck(ctx, cudaGetLastError());
    cudaEventRecord(ctx->kev[7], st);

    // outputs straight into each job's buffers, per-job meta
    ++launch_counter(), scatter_nn_kernel<<<blocks_for(n), kBlock, 0, st>>>(ctx->nn_sorted.as<int32_t>(), nv, n, perm,
                                                                           nullptr, jobs_dev, nj);
    ++launch_counter(), output_ci_kernel<<<blocks_for(n), kBlock, 0, st>>>(
        ctx->ci_sorted.as<int32_t>(), nv, n, perm, ctx->core_bits.as<uint32_t>(), ctx->core_prefix.as<uint32_t>(),
        nullptr, counters, jobs_dev, nj, jc);
    ++launch_counter(), job_cores_kernel<<<blocks_for(nj), kBlock, 0, st>>>(
        jobs_dev, nj, ctx->core_bits.as<uint32_t>(), ctx->core_prefix.as<uint32_t>(), n, jc);
    ck(ctx, cudaGetLastError());
    cudaEventRecord(ctx->ev[4], st);
    // count, union, border, band pairs (running totals), then the filter audit
    // (running over the call's pipelines)
    const unsigned long long *m_pairs = mail_from_device(ctx, counters + 2, 4, st);
    const unsigned long long *m_audit = mail_from_device(ctx, counters + 8, 4, st);
    const unsigned long long *m_jc = mail_from_device(ctx, jc, (size_t)4 * nj, st);
    const uint32_t *m_tc = mail_from_device(ctx, scal + 4, 1, st);
    const int *m_err = mail_from_device(ctx, err, 1, st);
    if (!(flags & NDB_FLAG_DEVICE_PTRS)) {
        for (int m = 0; m < nj; ++m) {
            ndb_job &J = jobs[members[m]];
            const int64_t off = bp.jd[m].off;
            if (J.nn_out)
                ck(ctx, cudaMemcpyAsync(J.nn_out, ctx->nn_orig.as<int32_t>() + off, J.n * sizeof(int32_t),
                                        cudaMemcpyDeviceToHost, st));
            if (J.cluster_index_out)
                ck(ctx, cudaMemcpyAsync(J.cluster_index_out, ctx->ci_orig.as<int32_t>() + off, J.n * sizeof(int32_t),
                                        cudaMemcpyDeviceToHost, st));
        }
    }
    ck(ctx, cudaStreamSynchronize(st));
    unsigned long long h_pairs[4], h_audit[4];
    memcpy(h_pairs, m_pairs, sizeof(h_pairs));
    memcpy(h_audit, m_audit, sizeof(h_audit));
    const std::vector<unsigned long long> h_jc(m_jc, m_jc + (size_t)4 * nj);
    const uint32_t h_tc_items = bp.tc ? *m_tc : 0;
    const int h_err = *m_err;
    // statistics summed over the pipelines of one batched call
    ndb_stats &S = ctx->stats;
    S.pipelines += 1;
    // pair counters run on over the pipelines of a call: this pipeline's share
    const int64_t dc = (int64_t)h_pairs[0] - S.count_pairs, du = (int64_t)h_pairs[1] - S.union_pairs,
                  db = (int64_t)h_pairs[2] - S.border_pairs;
    S.band_pairs = (int64_t)h_pairs[3];
    audit_stats(S, h_audit);
    S.tensor_items += h_tc_items;
    S.tensor_filter |= bp.tc ? 1 : 0;
    S.count_pairs += dc;
    S.union_pairs += du;
    S.border_pairs += db;
    S.count_pair_dims += dc * D;
    S.count_fp32_ops += dc * (bp.gram ? D + 3 : 3 * D);
    S.gram_filter |= bp.gram ? 1 : 0;
    S.union_pair_dims += du * D;
    S.border_pair_dims += db * D;
    S.n_valid += nv;
    S.n_cells += n_cells;
    S.n_tiles += n_items;
    S.grid_dims = std::max(S.grid_dims, bp.jd[0].g.k);
    S.stencil_rows = std::max(S.stencil_rows, n_rows);
    S.same_cell_linked |= bp.linked;
    S.key_bits = std::max(S.key_bits, bp.key_bits);
    S.sort_passes += (bp.key_bits + 7) / 8;
    S.key_bytes = std::max(S.key_bytes, (int32_t)sizeof(K));
    S.ms_grid += elapsed(ctx->ev[0], ctx->ev[1]);
    S.ms_count += elapsed(ctx->ev[1], ctx->ev[2]);
    S.ms_union += elapsed(ctx->ev[2], ctx->ev[3]);
    S.ms_border += elapsed(ctx->ev[3], ctx->ev[4]);
    S.ms_sort_kernels += elapsed(ctx->kev[0], ctx->kev[1]);
    S.ms_count_kernel += elapsed(ctx->kev[2], ctx->kev[3]);
    S.ms_union_kernel += elapsed(ctx->kev[4], ctx->kev[5]);
    S.ms_border_kernel += elapsed(ctx->kev[6], ctx->kev[7]);
    for (int m = 0; m < nj; ++m) {
        ndb_job &J = jobs[members[m]];
        J.result.clusters = (int32_t)h_jc[4 * m + 0];
        J.result.noise = (int32_t)h_jc[4 * m + 1];
        J.result.core_count = (int32_t)h_jc[4 * m + 2];
        J.result.n = (int32_t)J.n;
        J.status = h_err ? NDB_ERR_DEVICE_LIMIT : NDB_OK;
    }
}

// One pipeline over jobs of dimensionality D (members: indices into jobs).  Jobs
// the pipeline cannot take (a grid of another kind, min_pts beyond the neighbour-
// list cap, key space exhausted) are moved to `solo` and the pipeline is rebuilt
// over the rest, so it only ever holds jobs it runs.
template <int D>
void run_group(ndb_ctx *ctx, ndb_job *jobs, const std::vector<int> &members, uint32_t flags,
               std::vector<int> &solo) {
    if (members.empty()) return;
    cudaStream_t st = ctx->stream;
    ctx->mail_used = 0;  // the stream has drained: every earlier mailbox slice is consumed
    const int nj = (int)members.size();
    BatchPlan bp;
    bp.jd.resize(nj);
    int64_t off = 0, max_n = 1;
    for (int m = 0; m < nj; ++m) {
        const ndb_job &J = jobs[members[m]];
        JobDev &jd = bp.jd[m];
        memset(&jd, 0, sizeof(jd));
        jd.off = off;
        jd.n = J.n;
        jd.e2 = J.eps * J.eps;  // data_process.h:73
        jd.min_pts = J.min_pts;
        jd.src = J.coords;
        off += J.n;
        max_n = std::max<int64_t>(max_n, J.n);
    }
    bp.total_n = off;
    const int64_t n = off;
    ensure(ctx, ctx->coords, (size_t)n * D * sizeof(float));
    ensure(ctx, ctx->jobs_dev, (size_t)nj * sizeof(JobDev));
    mail_to_device(ctx, ctx->jobs_dev.as<JobDev>(), bp.jd.data(), (size_t)nj, st);
    const unsigned gx = (unsigned)std::min<int64_t>((max_n + kBlock - 1) / kBlock, 64);
    if (flags & NDB_FLAG_DEVICE_PTRS) {
        ++launch_counter(), gather_jobs_kernel<D><<<dim3(gx, nj), kBlock, 0, st>>>(ctx->jobs_dev.as<JobDev>(),
                                                                                  ctx->coords.as<float>());
        ck(ctx, cudaGetLastError());
    } else {
        for (int m = 0; m < nj; ++m)
            if (jobs[members[m]].n > 0)
                ck(ctx, cudaMemcpyAsync(ctx->coords.as<float>() + bp.jd[m].off * D, jobs[members[m]].coords,
                                        (size_t)jobs[members[m]].n * D * sizeof(float), cudaMemcpyHostToDevice, st));
    }

    // per-job bounding boxes, then every job's grid planned on the host (one sync)
    const size_t lh_bytes = ((size_t)nj * 2 * D * sizeof(int) + 15) & ~size_t(15);
    ensure(ctx, ctx->batch_bbox, lh_bytes + (size_t)nj * sizeof(unsigned long long) + 64);
    int *lo_hi = ctx->batch_bbox.as<int>();
    unsigned long long *inval = reinterpret_cast<unsigned long long *>(ctx->batch_bbox.as<char>() + lh_bytes);
    ++launch_counter(), bbox_batch_init_kernel<<<blocks_for((int64_t)nj * D), kBlock, 0, st>>>(lo_hi, D, nj, inval);
    ++launch_counter(), bbox_batch_kernel<D><<<dim3(gx, nj), kBlock, 0, st>>>(ctx->coords.as<float>(),
                                                                             ctx->jobs_dev.as<JobDev>(), lo_hi, inval);
    ck(ctx, cudaGetLastError());
    const int *m_lo_hi = mail_from_device(ctx, lo_hi, (size_t)nj * 2 * D, st);
    const unsigned long long *m_inval = mail_from_device(ctx, inval, (size_t)nj, st);
    ck(ctx, cudaStreamSynchronize(st));
    const std::vector<int> h_lo_hi(m_lo_hi, m_lo_hi + (size_t)nj * 2 * D);
    const std::vector<unsigned long long> h_inval(m_inval, m_inval + nj);

    auto dec = [](int v) {
        const int i = v >= 0 ? v : v ^ 0x7fffffff;
        float f;
        memcpy(&f, &i, sizeof(f));
        return (double)f;
    };
    unsigned long long key_base = 0;
    bool have_stencil = false;
    bp.linked = D <= 3 ? 1 : 0;
    int64_t nv = 0;
    std::vector<int> kept;
    for (int m = 0; m < nj; ++m) {
        JobDev &jd = bp.jd[m];
        const int64_t jnv = jd.n - (int64_t)h_inval[m];
        double lo[kMaxDim], hi[kMaxDim];
        for (int a = 0; a < D; ++a) {
            lo[a] = jnv > 0 ? dec(h_lo_hi[(size_t)m * 2 * D + a]) : 0.0;
            hi[a] = jnv > 0 ? dec(h_lo_hi[(size_t)m * 2 * D + D + a]) : 0.0;
        }
        const Plan pl = plan_grid(D, jd.e2, lo, hi);
        const bool job_tc = tc_eligible(ctx, D, jd.e2, lo, hi, pl.cell_units, pl.st.n_rows, flags);
        const bool job_gram = gram_eligible(ctx, D, jd.e2, lo, hi, flags);
        double cells = 1;
        for (int a = 0; a < pl.g.k; ++a) cells *= (double)pl.g.g[a];
        bool keep = (pl.cell_units ? 1 : 0) == bp.linked && jd.min_pts - 1 <= kMaxListCap &&
                    (double)key_base + cells < ldexp(1.0, 62);
        if (keep && have_stencil) keep = pl.st.n_rows == bp.st.n_rows && job_tc == bp.tc;  // one count kernel
        if (!keep) {
            solo.push_back(members[m]);
            continue;
        }
        kept.push_back(members[m]);
        bp.gram = bp.gram && job_gram;
        if (!have_stencil) {
            bp.st = pl.st;
            bp.tc = job_tc;
            have_stencil = true;
        }
        jd.g = pl.g;
        jd.linked = bp.linked;
        jd.list_cap = std::max(0, jd.min_pts - 1);
        jd.key_base = key_base;  // every job owns >= 1 key, so the bases increase
        key_base += (unsigned long long)cells;
        jd.col_base = (long long)std::min(bp.columns, 9e18);  // used only when the table fits its budget
        bp.columns += grid_columns(pl.g);
        bp.list_stride = std::max(bp.list_stride, jd.list_cap);
        nv += jnv;
    }
    if ((int)kept.size() != nj) {
        run_group<D>(ctx, jobs, kept, flags, solo);  // the pipeline over the jobs it can run
        return;
    }
    bp.nv = nv;
    // the all-ones key of invalid points must exceed every composite key
    int bits = 1;
    while (bits < 64 && ldexp(1.0, bits) - 1.0 < (double)key_base) ++bits;
    bp.key_bits = bits;
    // keys past 32 bits: split into pipelines whose cells fit 32-bit keys (one sort
    // pass fewer, half the hash table) as long as every part keeps more than one job
    if (bits > 32 && nj > 1) {
        const unsigned long long limit = (1ull << 32) - 1;  // room for the invalid key
        std::vector<int> part;
        unsigned long long acc = 0;
        bool split_ok = true;
        std::vector<std::vector<int>> parts;
        for (int m = 0; m < nj; ++m) {
            const unsigned long long cells = (m + 1 < nj ? bp.jd[m + 1].key_base : key_base) - bp.jd[m].key_base;
            if (cells >= limit) split_ok = false;
            if (!part.empty() && acc + cells >= limit) {
                parts.push_back(part);
                part.clear();
                acc = 0;
            }
            part.push_back(members[m]);
            acc += cells;
        }
        parts.push_back(part);
        if (split_ok && parts.size() > 1) {
            for (auto &pm : parts) run_group<D>(ctx, jobs, pm, flags, solo);
            return;
        }
    }
    // outputs: device pointers go straight to the kernels; host ones through staging
    if (flags & NDB_FLAG_DEVICE_PTRS) {
        for (int m = 0; m < nj; ++m) {
            bp.jd[m].nn_out = jobs[members[m]].nn_out;
            bp.jd[m].ci_out = jobs[members[m]].cluster_index_out;
        }
    } else {
        ensure(ctx, ctx->nn_orig, (n + 1) * sizeof(int32_t));
        ensure(ctx, ctx->ci_orig, (n + 1) * sizeof(int32_t));
        for (int m = 0; m < nj; ++m) {
            bp.jd[m].nn_out = jobs[members[m]].nn_out ? ctx->nn_orig.as<int32_t>() + bp.jd[m].off : nullptr;
            bp.jd[m].ci_out = jobs[members[m]].cluster_index_out ? ctx->ci_orig.as<int32_t>() + bp.jd[m].off : nullptr;
        }
    }
    mail_to_device(ctx, ctx->jobs_dev.as<JobDev>(), bp.jd.data(), (size_t)nj, st);
    if (bits <= 32) run_group_keys<D, uint32_t>(ctx, jobs, members, bp, flags);
    else run_group_keys<D, uint64_t>(ctx, jobs, members, bp, flags);
}

template <int D>
ndb_status run_group_entry(ndb_ctx *ctx, ndb_job *jobs, const std::vector<int> &members, uint32_t flags,
                           std::vector<int> &solo) {
    try {
        run_group<D>(ctx, jobs, members, flags, solo);
        return NDB_OK;
    } catch (const Fail &f) {
        for (int m : members)
            if (jobs[m].status == NDB_OK) jobs[m].status = f.st;
        return f.st;
    }
}

// Host buffers of a batched run: the device copies of every job's coordinates and
// output slots, group after group in the order the groups run; the jobs the
// pipelines see (dj) point at them.  Allocation happens here, on the calling
// thread, before any copy is issued.
void plan_stage(ndb_ctx *ctx, const ndb_job *jobs, int64_t n_jobs, const std::vector<std::vector<int>> &groups,
                std::vector<ndb_job> &dj) {
    size_t nf = 0, np = 0;
    bool want_nn = false, want_ci = false;
    for (int d = 1; d <= NDB_MAX_DIM; ++d)
        for (int i : groups[d]) {
            nf += (size_t)jobs[i].n * d;
            np += (size_t)jobs[i].n;
            want_nn |= jobs[i].nn_out != nullptr;
            want_ci |= jobs[i].cluster_index_out != nullptr;
        }
    ensure(ctx, ctx->batch_in, (nf + 4) * sizeof(float));
    if (want_nn) ensure(ctx, ctx->batch_nn, (np + 1) * sizeof(int32_t));
    if (want_ci) ensure(ctx, ctx->batch_ci, (np + 1) * sizeof(int32_t));
    dj.assign(jobs, jobs + n_jobs);
    size_t f = 0, p = 0;
    for (int d = 1; d <= NDB_MAX_DIM; ++d) {
        if (groups[d].empty()) continue;
        for (int i : groups[d]) {
            const ndb_job &J = jobs[i];
            dj[i].coords = ctx->batch_in.as<float>() + f;
            dj[i].nn_out = J.nn_out ? ctx->batch_nn.as<int32_t>() + p : nullptr;
            dj[i].cluster_index_out = J.cluster_index_out ? ctx->batch_ci.as<int32_t>() + p : nullptr;
            f += (size_t)J.n * d;
            p += (size_t)J.n;
        }
        lazy_event(ctx, ctx->ev_grp[d]);
        lazy_event(ctx, ctx->ev_done[d]);
    }
    lazy_event(ctx, ctx->ev_done[NDB_MAX_DIM + 1]);
}

// Issues a batched call's host copies from a second host thread, in order, on the
// copy stream.  A batch of thousands of jobs needs thousands of copy calls; issued
// there they run while the calling thread drives the pipelines, so the device does
// not idle between groups while the host queues one group's output copies or the
// next groups' input copies.  Marks let the calling thread wait until a group's
// input copies (and the event after them) are queued.
class CopyIssuer {
  public:
    explicit CopyIssuer(int device) : device_(device), th_([this] { loop(); }) {}
    ~CopyIssuer() { finish(); }
    void push(std::function<cudaError_t()> task) {
        {
            std::lock_guard<std::mutex> lk(mu_);
            tasks_.push_back(std::move(task));
        }
        cv_.notify_all();
    }
    // a task that records mark m as reached
    void mark(int m) {
        push([this, m] {
            std::lock_guard<std::mutex> lk(mu_);
            marks_.push_back(m);
            cv_.notify_all();
            return cudaSuccess;
        });
    }
    // blocks until mark m is reached (true) or a task failed (false)
    bool wait_mark(int m) {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] {
            return err_ != cudaSuccess || std::find(marks_.begin(), marks_.end(), m) != marks_.end();
        });
        return err_ == cudaSuccess;
    }
    // runs the remaining tasks and joins; the first failure
    cudaError_t finish() {
        if (th_.joinable()) {
            {
                std::lock_guard<std::mutex> lk(mu_);
                done_ = true;
            }
            cv_.notify_all();
            th_.join();
        }
        return err_;
    }

  private:
    void loop() {
        cudaError_t e = cudaSetDevice(device_);
        for (;;) {
            std::function<cudaError_t()> task;
            {
                std::unique_lock<std::mutex> lk(mu_);
                if (e != cudaSuccess && err_ == cudaSuccess) {
                    err_ = e;  // later tasks are dropped; waiters see the failure
                    cv_.notify_all();
                }
                cv_.wait(lk, [&] { return done_ || !tasks_.empty(); });
                if (tasks_.empty()) return;
                task = std::move(tasks_.front());
                tasks_.pop_front();
                if (err_ != cudaSuccess) continue;
            }
            e = task();
        }
    }
    int device_;
    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<std::function<cudaError_t()>> tasks_;
    std::vector<int> marks_;
    bool done_ = false;
    cudaError_t err_ = cudaSuccess;
    std::thread th_;
};

// Input copies of group d, then its event (issued by the copy thread).
cudaError_t issue_stage_group(ndb_ctx *ctx, const ndb_job *jobs, const std::vector<ndb_job> &dj,
                              const std::vector<int> &members, int d) {
    for (int i : members) {
        const cudaError_t e = cudaMemcpyAsync(const_cast<float *>(dj[i].coords), jobs[i].coords,
                                              (size_t)jobs[i].n * d * sizeof(float), cudaMemcpyHostToDevice,
                                              ctx->copy_stream);
        if (e != cudaSuccess) return e;
    }
    return cudaEventRecord(ctx->ev_grp[d], ctx->copy_stream);
}

// Output copies of finished jobs, after the event `done` the calling thread
// recorded on the context's stream (issued by the copy thread).
cudaError_t issue_unstage(ndb_ctx *ctx, const ndb_job *jobs, const std::vector<ndb_job> &dj,
                          const std::vector<int> &which, cudaEvent_t done) {
    cudaError_t e = cudaStreamWaitEvent(ctx->copy_stream, done, 0);
    for (size_t q = 0; q < which.size() && e == cudaSuccess; ++q) {
        const int i = which[q];
        const ndb_job &J = jobs[i];
        if (J.nn_out)
            e = cudaMemcpyAsync(J.nn_out, dj[i].nn_out, (size_t)J.n * sizeof(int32_t), cudaMemcpyDeviceToHost,
                                ctx->copy_stream);
        if (e == cudaSuccess && J.cluster_index_out)
            e = cudaMemcpyAsync(J.cluster_index_out, dj[i].cluster_index_out, (size_t)J.n * sizeof(int32_t),
                                cudaMemcpyDeviceToHost, ctx->copy_stream);
    }
    return e;
}

}  // namespace

extern "C" ndb_status ndb_b200_run_batched(ndb_ctx *ctx, ndb_job *jobs, int64_t n_jobs, uint32_t flags) {
    ndb_status s = check_ctx(ctx);
    if (s != NDB_OK) return s;
    if (n_jobs < 0 || (n_jobs > 0 && !jobs)) return NDB_ERR_INVALID_ARGUMENT;
    if (flags & ~kAllFlags) return NDB_ERR_INVALID_ARGUMENT;
    ctx->have_state = false;
    ctx->have_labels = false;
    ctx->stats = ndb_stats{};
    launch_counter() = 0;
    if (grow(ctx, ctx->small, kSmallBytes) != cudaSuccess) return NDB_ERR_OUT_OF_MEMORY;
    try {
        fill_bytes(ctx, ctx->small.ptr, 0, kSmallBytes, ctx->stream);
    } catch (const Fail &f) {
        return f.st;
    }
    ++launch_counter(), set_int_kernel<<<1, 1, 0, ctx->stream>>>(small_at<int>(ctx, kSmallErrOff) + 1,
                                                                 ctx->uf_max_steps);
    if (cudaGetLastError() != cudaSuccess) return NDB_ERR_CUDA;
    ndb_status first = NDB_OK;
    // validate, and group by dimensionality
    std::vector<std::vector<int>> groups(NDB_MAX_DIM + 1);
    for (int64_t i = 0; i < n_jobs; ++i) {
        ndb_job &J = jobs[i];
        J.result = ndb_result{0, 0, 0, (int32_t)(J.n > 0 ? J.n : 0)};
        J.status = NDB_OK;
        const float e2 = J.eps * J.eps;
        if (J.d < 1 || J.d > NDB_MAX_DIM) J.status = NDB_ERR_UNSUPPORTED_DIM;
        else if (J.n < 0 || (J.n > 0 && !J.coords)) J.status = NDB_ERR_INVALID_ARGUMENT;
        else if (J.n > NDB_MAX_POINTS) J.status = NDB_ERR_TOO_MANY_POINTS;
        else if (!isfinite(e2)) J.status = NDB_ERR_INVALID_EPS;
        if (J.status != NDB_OK) {
            if (first == NDB_OK) first = (ndb_status)J.status;
            continue;
        }
        if (J.n == 0) continue;
        groups[J.d].push_back((int)i);
    }
    // the pipelines' small transfers: per job two job-table entries, a bounding box,
    // its invalid count and four counters; per pipeline the stencil and some scalars
    try {
        ensure_mail(ctx, (size_t)n_jobs * (2 * sizeof(JobDev) + 2 * NDB_MAX_DIM * sizeof(int) + 5 * 8) +
                             kMaxRows * sizeof(int4) + 16 * 1024);
    } catch (const Fail &f) {
        return f.st;
    }
    // host buffers: inputs staged group by group on the copy stream, outputs back
    // group by group; the pipelines run on the device copies
    const bool host_io = !(flags & NDB_FLAG_DEVICE_PTRS) && ctx->copy_stream;
    std::vector<ndb_job> dj;
    ndb_job *work = jobs;
    uint32_t wflags = flags;
    std::unique_ptr<CopyIssuer> io;  // issues the host copies from its own thread
    if (host_io) {
        try {
            plan_stage(ctx, jobs, n_jobs, groups, dj);
        } catch (const Fail &f) {
            for (int d = 1; d <= NDB_MAX_DIM; ++d)  // every job that was to run carries the failure
                for (int i : groups[d]) jobs[i].status = f.st;
            return f.st;
        }
        work = dj.data();
        wflags |= NDB_FLAG_DEVICE_PTRS;
        io.reset(new CopyIssuer(ctx->device));
        for (int d = 1; d <= NDB_MAX_DIM; ++d) {
            if (groups[d].empty()) continue;
            const std::vector<int> &members = groups[d];
            io->push([ctx, jobs, &dj, &members, d] { return issue_stage_group(ctx, jobs, dj, members, d); });
            io->mark(d);
        }
    }
    std::vector<int> solo;
    for (int d = 1; d <= NDB_MAX_DIM; ++d) {
        if (host_io && !groups[d].empty()) {
            // the group's input copies and their event are queued before the stream waits on it
            if (!io->wait_mark(d) || cudaStreamWaitEvent(ctx->stream, ctx->ev_grp[d], 0) != cudaSuccess) {
                if (first == NDB_OK) first = NDB_ERR_CUDA;
                for (int i : groups[d]) dj[i].status = NDB_ERR_CUDA;
                continue;
            }
        }
        const size_t solo_before = solo.size();
        // pipelines of at most kMaxBatchPoints points
        size_t b = 0;
        while (b < groups[d].size()) {
            std::vector<int> members;
            int64_t pts = 0;
            while (b < groups[d].size() && (members.empty() || pts + jobs[groups[d][b]].n <= kMaxBatchPoints)) {
                pts += jobs[groups[d][b]].n;
                members.push_back(groups[d][b++]);
            }
#define NDB_GROUP(D) run_group_entry<D>(ctx, work, members, wflags, solo)
            ndb_status gs;
            switch (d) {
                case 1: gs = NDB_GROUP(1); break;
                case 2: gs = NDB_GROUP(2); break;
                case 3: gs = NDB_GROUP(3); break;
                case 4: gs = NDB_GROUP(4); break;
                case 5: gs = NDB_GROUP(5); break;
                case 6: gs = NDB_GROUP(6); break;
                case 7: gs = NDB_GROUP(7); break;
                case 8: gs = NDB_GROUP(8); break;
                case 9: gs = NDB_GROUP(9); break;
                case 10: gs = NDB_GROUP(10); break;
                case 11: gs = NDB_GROUP(11); break;
                case 12: gs = NDB_GROUP(12); break;
                case 13: gs = NDB_GROUP(13); break;
                case 14: gs = NDB_GROUP(14); break;
                case 15: gs = NDB_GROUP(15); break;
                default: gs = NDB_GROUP(16); break;
            }
#undef NDB_GROUP
            if (gs != NDB_OK && first == NDB_OK) first = gs;
        }
        if (host_io && !groups[d].empty()) {
            auto done = std::make_shared<std::vector<int>>();
            for (int i : groups[d])
                if (std::find(solo.begin() + solo_before, solo.end(), i) == solo.end()) done->push_back(i);
            if (cudaEventRecord(ctx->ev_done[d], ctx->stream) != cudaSuccess) {
                if (first == NDB_OK) first = NDB_ERR_CUDA;
            } else if (!done->empty()) {
                cudaEvent_t ev = ctx->ev_done[d];
                io->push([ctx, jobs, &dj, done, ev] { return issue_unstage(ctx, jobs, dj, *done, ev); });
            }
        }
    }
    // statistics of the pipelines, then of the jobs the pipelines could not take,
    // which run one call each
    ndb_stats acc = ctx->stats;
    acc.kernel_launches = launch_counter();
    for (int i : solo) {
        ndb_job &J = work[i];
        ndb_result r{};
        const ndb_status js = ndb_b200_run(ctx, J.coords, J.n, J.d, J.eps, J.min_pts, wflags, J.nn_out,
                                           J.cluster_index_out, &r);
        J.status = js;
        if (js == NDB_OK) J.result = r;
        else if (first == NDB_OK) first = js;
        const ndb_stats &s1 = ctx->stats;
        acc.n_valid += s1.n_valid;
        acc.n_cells += s1.n_cells;
        acc.n_tiles += s1.n_tiles;
        acc.count_pairs += s1.count_pairs;
        acc.union_pairs += s1.union_pairs;
        acc.border_pairs += s1.border_pairs;
        acc.band_pairs += s1.band_pairs;
        acc.tensor_items += s1.tensor_items;
        acc.tensor_filter |= s1.tensor_filter;
        acc.count_pair_dims += s1.count_pair_dims;
        acc.count_fp32_ops += s1.count_fp32_ops;
        acc.gram_filter |= s1.gram_filter;
        acc.union_pair_dims += s1.union_pair_dims;
        acc.border_pair_dims += s1.border_pair_dims;
        acc.ms_grid += s1.ms_grid;
        acc.ms_count += s1.ms_count;
        acc.ms_union += s1.ms_union;
        acc.ms_border += s1.ms_border;
        acc.ms_sort_kernels += s1.ms_sort_kernels;
        acc.ms_count_kernel += s1.ms_count_kernel;
        acc.ms_union_kernel += s1.ms_union_kernel;
        acc.ms_border_kernel += s1.ms_border_kernel;
        acc.sort_passes += s1.sort_passes;
        acc.kernel_launches += s1.kernel_launches;
    }
    acc.solo_jobs = (int32_t)solo.size();
    ctx->stats = acc;
    if (host_io) {
        if (!solo.empty()) {
            cudaEvent_t ev = ctx->ev_done[NDB_MAX_DIM + 1];
            if (cudaEventRecord(ev, ctx->stream) != cudaSuccess) {
                if (first == NDB_OK) first = NDB_ERR_CUDA;
            } else {
                io->push([ctx, jobs, &dj, &solo, ev] { return issue_unstage(ctx, jobs, dj, solo, ev); });
            }
        }
        const cudaError_t ioe = io->finish();
        if (ioe != cudaSuccess) {
            ctx->last_cuda_error = cudaGetErrorString(ioe);
            if (first == NDB_OK) first = ioe == cudaErrorMemoryAllocation ? NDB_ERR_OUT_OF_MEMORY : NDB_ERR_CUDA;
        }
        if (cudaStreamSynchronize(ctx->copy_stream) != cudaSuccess && first == NDB_OK) first = NDB_ERR_CUDA;
        for (int64_t i = 0; i < n_jobs; ++i) {
            jobs[i].status = dj[i].status;
            jobs[i].result = dj[i].result;
        }
    }
    // a pipeline reports a device-side failure through its jobs' statuses
    for (int64_t i = 0; i < n_jobs && first == NDB_OK; ++i)
        if (jobs[i].status != NDB_OK) first = (ndb_status)jobs[i].status;
    ctx->have_state = false;
    ctx->have_labels = false;
    return first;
}

// ---------------------------------------------------------------------------
// Allocation-free entry point (ndb_b200_run_noalloc).
//
// Some callers cannot allocate device memory: a service that reserves its GPU
// memory once at start-up and forbids cudaMalloc afterwards (so a late request can
// never fail or fragment the pool), code running where an allocation would
// synchronise the device at the wrong moment, or a plugin host that hands out
// only the buffers it owns.  For them this entry point runs the same pipeline as
// ndb_b200_run with every scratch buffer carved out of one file-scope device
// array of fixed size, so no call allocates.
//
// The array lives in the library image: every GPU that loads the library holds
// it until the process exits.  All calls share it and it keeps the last call's
// contents; the pipeline clears what must start at zero itself.  Calls are
// serialised on the host per device and each returns only after its work is
// done; work the caller enqueues on the GPU around a call must not overlap it,
// since two overlapping users of the array would race.
// ---------------------------------------------------------------------------
namespace {

constexpr size_t na_align(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kNaN = NDB_NOALLOC_MAX_POINTS;

// Capacity of each buffer for jobs of up to kNaN points (upper bounds of the
// requests the pipeline makes: keys may be 64-bit, coordinates padded to 16).
enum NaBuf {
    NA_KEYS0, NA_KEYS1, NA_IDS0, NA_IDS1, NA_FLAGS, NA_POS, NA_PCELL, NA_XS, NA_NN_SORTED, NA_NN_ORIG,
    NA_CORE_SORTED, NA_CORE_BITS, NA_CORE_PREFIX, NA_CI_SORTED, NA_CI_ORIG, NA_LABELS, NA_CELL_START, NA_CELL_KEY,
    NA_NBR, NA_ITEM_CNT, NA_ITEMS, NA_CELL_HAS_CORE, NA_CELL_CID, NA_PARENT, NA_COMP_MIN, NA_SORT_HIST,
    NA_SCAN, NA_SMALL, NA_HASH_KEYS, NA_HASH_VALS, NA_NBR_LIST, NA_ITEMS_SPLIT, NA_COUNT
};

constexpr size_t na_cap(int b) {
    return b == NA_KEYS0 || b == NA_KEYS1 ? 8 * kNaN
         : b == NA_IDS0 || b == NA_IDS1 ? 4 * kNaN
         : b == NA_XS ? 4 * 16 * (kNaN + 1)
         : b == NA_CELL_START ? 4 * (kNaN + 2)
         : b == NA_CELL_KEY || b == NA_ITEMS ? 8 * (kNaN + 1)
         : b == NA_NBR ? 8 * kWarp * kNaN + 8  // classify refuses stencils of more than kWarp rows
         : b == NA_CORE_SORTED || b == NA_CELL_HAS_CORE ? kNaN + 1
         : b == NA_SORT_HIST ? 4 * 256 * ((kNaN + kSortTile - 1) / kSortTile)
         : b == NA_SCAN ? 4 * 4096
         : b == NA_SMALL ? kSmallBytes
         : b == NA_HASH_KEYS ? 8 * 4 * kNaN
         : b == NA_HASH_VALS ? 4 * 4 * kNaN
         : b == NA_NBR_LIST ? 4 * 16 * kNaN
         : b == NA_ITEMS_SPLIT ? 16 * (kNaN + 1)  // both item lists of the tensor-core count (items <= n)
         : 4 * (kNaN + 1);
}

constexpr size_t na_offset(int b) { return b == 0 ? 0 : na_offset(b - 1) + na_align(na_cap(b - 1)); }
constexpr size_t kNaBytes = na_offset(NA_COUNT);

struct NoAllocState {
    std::mutex mu;
    bool ready = false;
    unsigned char *base = nullptr;
    ndb_ctx ctx;
};

constexpr int kNaMaxDevices = 64;
NoAllocState g_na_state[kNaMaxDevices];

DevBuf *na_buf(ndb_ctx &c, int b) {
    DevBuf *bufs[NA_COUNT] = {&c.keys0,       &c.keys1,     &c.ids0,      &c.ids1,         &c.flags,
                              &c.pos,         &c.pcell,     &c.xs,        &c.nn_sorted,    &c.nn_orig,
                              &c.core_sorted, &c.core_bits, &c.core_prefix, &c.ci_sorted,  &c.ci_orig,
                              &c.labels,      &c.cell_start, &c.cell_key, &c.nbr,          &c.item_cnt,
                              &c.items,       &c.cell_has_core, &c.cell_cid, &c.parent,    &c.comp_min,
                              &c.sort_hist,   &c.scan_scratch, &c.small,     &c.hash_keys, &c.hash_vals,
                              &c.nbr_list,    &c.items_split};
    return bufs[b];
}

// Points every buffer of the shared context back at its slice of the array
// (the pipeline swaps the ping-pong sort buffers between calls).
void na_carve(NoAllocState &s) {
    for (int b = 0; b < NA_COUNT; ++b) {
        DevBuf *d = na_buf(s.ctx, b);
        d->ptr = s.base + na_offset(b);
        d->bytes = na_cap(b);
    }
}

bool na_inside(const NoAllocState &s, const ndb_ctx &c) {
    for (int b = 0; b < NA_COUNT; ++b) {
        const DevBuf *d = na_buf(const_cast<ndb_ctx &>(c), b);
        const unsigned char *p = static_cast<const unsigned char *>(d->ptr);
        if (p < s.base || p + d->bytes > s.base + kNaBytes) return false;
    }
    return c.coords.ptr == nullptr;
}

}  // namespace

// The scratch of ndb_b200_run_noalloc: file scope, fixed size, no allocation.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

extern "C" ndb_status ndb_b200_run_noalloc(const float *coords, int64_t n, int32_t d, float eps, int32_t min_pts,
                                           uint32_t flags, int32_t *nn_out, int32_t *cluster_index_out,
                                           ndb_result *result, void *cuda_stream) {
    if (n < 0 || d < 1) return d < 1 ? NDB_ERR_UNSUPPORTED_DIM : NDB_ERR_INVALID_ARGUMENT;
    if (n > (int64_t)kNaN) return NDB_ERR_TOO_MANY_POINTS;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNaMaxDevices) {
        cudaGetLastError();
        return NDB_ERR_NO_DEVICE;
    }
    NoAllocState &s = g_na_state[dev];
    std::lock_guard<std::mutex> lock(s.mu);
    if (!s.ready) {
        // once per device, with that device current: the host-side name of the array
        // is not a device address, so look the address up
        void *addr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
        if (e != cudaSuccess || addr == nullptr) {
            s.ctx.last_cuda_error = cudaGetErrorString(e);
            cudaGetLastError();
            return NDB_ERR_CUDA;
        }
        // the timing events, kept only once all of them exist (a failed attempt
        // leaves nothing behind, so a retry starts clean)
        constexpr int kNev = sizeof(s.ctx.ev) / sizeof(s.ctx.ev[0]), kNkev = sizeof(s.ctx.kev) / sizeof(s.ctx.kev[0]);
        cudaEvent_t evs[kNev + kNkev] = {};
        for (int i = 0; i < kNev + kNkev; ++i) {
            e = cudaEventCreate(&evs[i]);
            if (e != cudaSuccess) {
                s.ctx.last_cuda_error = cudaGetErrorString(e);
                for (int k = 0; k < i; ++k) cudaEventDestroy(evs[k]);
                cudaGetLastError();
                return NDB_ERR_CUDA;
            }
        }
        for (int i = 0; i < kNev; ++i) s.ctx.ev[i] = evs[i];
        for (int i = 0; i < kNkev; ++i) s.ctx.kev[i] = evs[kNev + i];
        s.base = static_cast<unsigned char *>(addr);
        s.ctx.device = dev;
        s.ready = true;
    }
    na_carve(s);
    // cap the footprint at the slices themselves: a request that would outgrow its
    // slice is refused before any cudaFree/cudaMalloc instead of reallocating
    s.ctx.mem_limit = s.ctx.held_bytes();
    s.ctx.list_budget = na_cap(NA_NBR_LIST) - 4;  // lists only where they fit the slice
    s.ctx.col_budget = 0;  // a column table's size follows the bounding box, not n: cells hashed instead
    s.ctx.own_stream = nullptr;
    s.ctx.stream = static_cast<cudaStream_t>(cuda_stream);
    ndb_status st = ndb_b200_classify(&s.ctx, coords, n, d, eps, min_pts, flags | NDB_FLAG_DEVICE_PTRS, nn_out);
    if (st == NDB_OK) st = ndb_b200_assign_labels(&s.ctx, cluster_index_out, result);
    if (!na_inside(s, s.ctx)) st = NDB_ERR_OUT_OF_MEMORY;  // a request outgrew its slice
    if (st != NDB_OK) {
        // a failure can return with kernels still queued on the array: wait for
        // them, so that every call is complete on return and the next one (from
        // any stream) finds the array idle
        cudaStreamSynchronize(s.ctx.stream);
        cudaGetLastError();
    }
    return st;
}
