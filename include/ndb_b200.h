/*
 * ndb_b200.h -- C ABI of the B200 DBSCAN hot path (libndb_b200.so).
 *
 * Drop-in for nextdbscan-exa's algorithm layer, the class data_process
 * (data_process.h:45-102, data_process.cpp:50-458), which the reference selects at
 * compile time (data_process.cpp:24-30) and calls from nextdbscan::start
 * (nextdbscan.cpp:46-58).  Each entry point below names the reference interface it
 * replaces.  Plain pointers and sizes only; no C++ or CUDA types cross this boundary.
 *
 * Conventions
 *   - Every call returns an ndb_status; the library never exits the process (the
 *     reference is noexcept everywhere and calls exit() on hard errors).
 *   - Output buffers are owned by the caller.  Host pointers unless
 *     NDB_FLAG_DEVICE_PTRS is set, in which case coords and every output array
 *     are device pointers on the context's device.
 *   - A context is used by one host thread at a time.  Work is queued on the
 *     context's stream; calls return after their results are in the caller's
 *     buffers.
 *   - Coordinates are FP32, row-major (point-major), n x d, exactly the
 *     reference's v_coord layout (data_process.h:55, magma_input.h:113-125).
 *
 * Result semantics (bit-identical to the reference OpenMP implementation):
 *   nn[i]             points j (i included) with dist2(i,j) <= eps*eps, where
 *                     dist2 = 0; dist2 += (a-b)*(a-b) per dimension, every FP32
 *                     operation separately rounded (data_process.cpp:443-447).
 *                     Without NDB_FLAG_FULL_COUNT the count of a core point stops
 *                     early once it reaches min_pts: nn[i] is exact whenever it is
 *                     below min_pts and is some value >= min_pts otherwise, so the
 *                     core flags are exact either way.
 *   cluster_index[i]  NDB_NO_CLUSTER (INT32_MAX, data_process.h:26) for noise; else
 *                     the rank among core points (index order) of the smallest-index
 *                     core of the core-connected component; a border point takes the
 *                     minimum such id over the cores within eps
 *                     (data_process.cpp:93-266 after convergence).
 */
#ifndef NDB_B200_H
#define NDB_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NDB_NO_CLUSTER INT32_MAX

/* Largest supported dimensionality. */
#define NDB_MAX_DIM 16

typedef enum ndb_status {
    NDB_OK = 0,
    NDB_ERR_INVALID_ARGUMENT = 1, /* null pointer, n < 0, bad flags, ... */
    NDB_ERR_UNSUPPORTED_DIM = 2,  /* d outside 1..NDB_MAX_DIM */
    NDB_ERR_INVALID_EPS = 3,      /* eps*eps (FP32) is NaN or infinite */
    NDB_ERR_TOO_MANY_POINTS = 4,  /* n > NDB_MAX_POINTS */
    NDB_ERR_OUT_OF_MEMORY = 5,    /* device allocation failed */
    NDB_ERR_CUDA = 6,             /* a CUDA runtime call failed; see ndb_b200_last_cuda_error */
    NDB_ERR_NO_DEVICE = 7,        /* no CUDA device / bad device ordinal */
    NDB_ERR_DEVICE_LIMIT = 8,     /* a device-side loop hit its iteration bound */
    NDB_ERR_NO_STATE = 9,         /* ndb_b200_assign_labels before ndb_b200_classify */
    NDB_ERR_BAD_JOB = 10,         /* a batched job descriptor is invalid */
    NDB_ERR_IO = 11               /* ndb_b200_load_bin: the file is missing, short, or has a bad header */
} ndb_status;

/* Largest n per job: indices are int32, as in the reference (data_process.h:47-59). */
#define NDB_MAX_POINTS 2147483000LL

/* flags */
#define NDB_FLAG_APPROXIMATE 0x1u  /* reference -a 1 (main.cpp:45, data_process.cpp:215-217).
                                      Accepted for drop-in compatibility; the union-find
                                      result is already exact, which is a valid (tight)
                                      upper bound on the cluster count. */
#define NDB_FLAG_FULL_COUNT  0x2u  /* exact nn for every point (no early exit at min_pts) */
#define NDB_FLAG_DEVICE_PTRS 0x4u  /* coords and outputs are device pointers */
#define NDB_FLAG_EXACT_COUNT 0x8u  /* count with the exact FP32 kernel only, never the tensor-core or the
                                    * FP32 Gram filter (results are identical either way; this is the plain form) */
#define NDB_FLAG_TENSOR_FILTER 0x10u /* d >= 8: count on the tensor-core filter whenever the input allows
                                      * it, whatever the tile-fill heuristic would pick (results identical) */
#define NDB_FLAG_GRAM_FILTER  0x40u  /* d >= 8: the CUDA-core count decides pairs from FP32 Gram dot products
                                      * first, with a guard band and the exact sum inside it (results identical) */
#define NDB_FLAG_FILTER_AUDIT 0x20u  /* diagnostic: when the tensor-core filter runs, measure every pair it
                                      * classifies against its FP64 distance and the exact FP32 predicate
                                      * (ndb_stats.filter_*); slower, results identical */

/* Mirrors nextdbscan::result (nextdbscan.h:43-48). */
typedef struct ndb_result {
    int32_t clusters;
    int32_t noise;
    int32_t core_count;
    int32_t n;
} ndb_result;

/* Counters of the last run, for measurement (no reference counterpart; the
 * reference prints phase times from magma_util::measure_duration, magma_util.h:51-64). */
typedef struct ndb_stats {
    int64_t n_valid;          /* points that took part in the grid */
    int64_t n_cells;          /* non-empty grid cells */
    int64_t n_tiles;          /* work items (cell chunks of up to 32 points) */
    int32_t grid_dims;        /* gridded dimensions (1..4) */
    int32_t stencil_rows;     /* neighbour rows per cell */
    int32_t same_cell_linked; /* 1 when all points of a cell are provably within eps */
    int32_t key_bits;         /* radix-sort key width actually sorted */
    int64_t count_pairs;      /* pair predicates evaluated by the neighbour count */
    int64_t union_pairs;      /* pair predicates evaluated by the union-find */
    int64_t border_pairs;     /* pair predicates evaluated by the border assignment */
    float ms_grid;            /* device time of bbox + keys + sort + cells + gather + rows */
    float ms_count;           /* device time of the neighbour count / core flags */
    float ms_union;           /* device time of the union-find + canonical ids */
    float ms_border;          /* device time of the border assignment + meta */
    float ms_sort_kernels;    /* device time of the radix sort (all passes) */
    float ms_count_kernel;    /* device time of the neighbour-count kernel */
    float ms_union_kernel;    /* device time of the main union kernel (cells, or points after the list unions) */
    float ms_border_kernel;   /* device time of the border kernel */
    int32_t sort_passes;      /* radix passes (8 bits each) */
    int32_t key_bytes;        /* 4 or 8 */
    int32_t kernel_launches;  /* kernels launched by the last classify + assign_labels */
    int32_t pipelines;        /* batched runs: pipelines built (one per d and chunk of jobs) */
    int64_t count_pair_dims;  /* sum over pipelines of count_pairs x d */
    int64_t union_pair_dims;  /* the same for the union-find */
    int64_t border_pair_dims; /* the same for the border assignment */
    int32_t solo_jobs;        /* batched runs: jobs the pipelines could not take, run one call each */
    int32_t tensor_filter;    /* 1 when the neighbour count ran on the tensor-core filter (d >= 8) */
    int64_t band_pairs;       /* pairs inside the filter's guard band, rechecked with the exact predicate */
    int64_t tensor_items;     /* items (points of one cell, up to 32) counted on the tensor-core filter */
    /* NDB_FLAG_FILTER_AUDIT only (0 otherwise): the filter's squared distance D~ against the FP64
     * distance of the same FP32 points, over every pair it classified */
    double filter_max_abs_err;        /* largest |D~ - d64| */
    double filter_max_err_over_bound; /* largest |D~ - d64| over the error bound the guard band is built from */
    int64_t filter_audited_pairs;     /* pairs measured */
    int64_t filter_misclassified_pairs; /* pairs decided outside the band that the exact predicate decides otherwise */
    int64_t count_fp32_ops;           /* FP32 pipe operations of the CUDA-core count: 3d per pair for the exact
                                       * sum, d + 3 per pair with the Gram filter (one FMA per dimension) */
    int32_t gram_filter;              /* 1 when the CUDA-core count ran with the Gram filter (d >= 8) */
} ndb_stats;

typedef struct ndb_ctx ndb_ctx;

/* Creates a context on CUDA device `device` with its own non-blocking stream.
 * Replaces the construction of data_process (data_process.h:60-77). */
ndb_status ndb_b200_create(ndb_ctx **ctx, int32_t device);

/* Frees every device buffer of the context. */
ndb_status ndb_b200_destroy(ndb_ctx *ctx);

/* Use an existing cudaStream_t (passed as void*) instead of the context's own
 * stream; NULL restores the context's stream. */
ndb_status ndb_b200_set_stream(ndb_ctx *ctx, void *cuda_stream);

/* Phase 1: epsilon grid, neighbour counting and core flags.
 * Replaces data_process::select_and_process (data_process.cpp:334-392) and
 * process_points (data_process.cpp:395-458).  nn_out (n int32) may be NULL.
 * The grid and the counts stay in the context for ndb_b200_assign_labels. */
ndb_status ndb_b200_classify(ndb_ctx *ctx, const float *coords, int64_t n, int32_t d,
                             float eps, int32_t min_pts, uint32_t flags, int32_t *nn_out);

/* Phase 2: union-find over core points, canonical cluster ids, border points and
 * the result meta.  Replaces data_process::select_cores_and_process
 * (data_process.cpp:268-332), process_cores (:93-266) and get_result_meta (:50-91).
 * cluster_index_out (n int32) may be NULL; result may be NULL. */
ndb_status ndb_b200_assign_labels(ndb_ctx *ctx, int32_t *cluster_index_out, ndb_result *result);

/* Both phases in one call: the body of nextdbscan::start without the file read
 * (nextdbscan.cpp:46-58). */
ndb_status ndb_b200_run(ndb_ctx *ctx, const float *coords, int64_t n, int32_t d, float eps,
                        int32_t min_pts, uint32_t flags, int32_t *nn_out,
                        int32_t *cluster_index_out, ndb_result *result);

/* The reference's binary input file (magma_input.h:113-125: int32 n, int32 d, then
 * n*d float32 row-major) read straight into the context's device memory: the file
 * is read in chunks into two pinned staging buffers, each chunk's copy to the device
 * runs while the next chunk is read, and the bounding box of the grid is reduced
 * chunk by chunk as the chunks land.  Replaces magma_input::read_input for .bin
 * files (magma_input.h:144-167) and the host-to-device copy of the data_process
 * constructor (data_process.h:62).  n and d of the file are returned; the job stays
 * loaded until the next run or load on the context that is not
 * ndb_b200_run_loaded.  A missing or short file, or a bad header, is NDB_ERR_IO
 * (d outside 1..NDB_MAX_DIM is NDB_ERR_UNSUPPORTED_DIM). */
ndb_status ndb_b200_load_bin(ndb_ctx *ctx, const char *path, int64_t *n, int32_t *d);

/* ndb_b200_run on the job ndb_b200_load_bin loaded (any number of times, with any
 * eps, min_pts and flags).  Outputs are host pointers, or device pointers with
 * NDB_FLAG_DEVICE_PTRS; NDB_ERR_NO_STATE when nothing is loaded. */
ndb_status ndb_b200_run_loaded(ndb_ctx *ctx, float eps, int32_t min_pts, uint32_t flags, int32_t *nn_out,
                               int32_t *cluster_index_out, ndb_result *result);

/* One job of a batched run: an independent DBSCAN problem with its own
 * coordinates, dimensionality, eps and min_pts (the arguments of one
 * ndb_b200_run call).  result and status are written by ndb_b200_run_batched. */
typedef struct ndb_job {
    const float *coords;        /* n x d FP32, row-major; device memory with NDB_FLAG_DEVICE_PTRS */
    int64_t n;
    int32_t d;
    float eps;
    int32_t min_pts;
    int32_t *nn_out;            /* n int32 or NULL */
    int32_t *cluster_index_out; /* n int32 or NULL */
    ndb_result result;          /* out */
    int32_t status;             /* out: ndb_status of this job */
} ndb_job;

/* Runs many independent jobs as one pipeline: jobs of the same dimensionality
 * are concatenated, every phase is one launch over all of them (per-job eps,
 * min_pts and grid are looked up per cell), and results land in each job's own
 * buffers.  Results are identical to one ndb_b200_run per job.  No counterpart
 * in the reference, which clusters one input per process (nextdbscan.cpp:28-68).
 * Returns the first failing job's status (each job also carries its own). */
ndb_status ndb_b200_run_batched(ndb_ctx *ctx, ndb_job *jobs, int64_t n_jobs, uint32_t flags);

/* The border pass of the last run again, with the caller's cluster ids for the core
 * points: core_ids (n int32, input order; read for core points only) replaces the
 * library's ids, every non-core point takes the minimum of those ids over the cores
 * within eps (the reference's tie rule, data_process.cpp:204-209), and
 * cluster_index_out (n int32, may be NULL) receives the result in input order.
 * Host or device pointers as the run's NDB_FLAG_DEVICE_PTRS says.  The cores of one
 * component must carry one id.  For the sharded form: there a component spans ranks,
 * its final id is known only after the ranks' merge, and a border point's minimum
 * over the local ids would not survive that merge -- the step that replaces the
 * reference's allreduce-min of labels across ranks (data_process.cpp:232-233).
 * Afterwards ndb_b200_cluster_label returns NDB_ERR_NO_STATE. */
ndb_status ndb_b200_assign_border(ndb_ctx *ctx, const int32_t *core_ids, int32_t *cluster_index_out);

/* Per-core label array of the last run, the reference's v_cluster_label
 * (data_process.h:58, filled at data_process.cpp:141-260): entry k is the cluster id
 * of the k-th core point, so label[k] == k exactly for the reference's roots
 * (data_process.cpp:79-88).  Host buffer of at least core_count entries. */
ndb_status ndb_b200_cluster_label(ndb_ctx *ctx, int32_t *label_out, int64_t capacity);

/* Caps the device memory the context may hold, in bytes (0 = no cap, the default).
 * A run whose buffers would grow past the cap fails with NDB_ERR_OUT_OF_MEMORY before
 * it allocates anything, and the context stays usable for the next run.  A cap below
 * what the context holds now releases all its buffers (after the context's stream
 * drains); a pending ndb_b200_assign_labels then returns NDB_ERR_NO_STATE.  Lets a
 * caller share one GPU with other work at a known footprint, and injects allocation
 * failures in tests.  No counterpart in the reference, which only tracks its host
 * footprint (allocated_bytes, data_process.h:54,63,75,79-85) and exits on failure. */
ndb_status ndb_b200_set_memory_limit(ndb_ctx *ctx, int64_t max_bytes);

/* Count-kernel thresholds of a context, picked by measurement (the autotuner of
 * the Python package times the candidates on a sample of the caller's data).  They
 * choose which kernel counts neighbours; results never depend on them.  0 = the
 * library's default.  No counterpart in the reference, whose count has one form.
 *   tc_min_dim   smallest d at which the count may run on the tensor-core filter
 *                (clamped to >= 8).  Default: 8 with NDB_FLAG_FULL_COUNT, 12 with the
 *                early exit (or the NDB_TC_MIN_DIM environment variable); a value
 *                above 16 keeps every count on the exact kernel.
 *   tc_min_item  smallest item (points of one cell, up to 32) the tensor-core filter
 *                takes; smaller items go to the exact kernel.  Default 16 (or
 *                NDB_TC_MIN_ITEM); above 32 sends every item to the exact kernel.
 * NDB_FLAG_EXACT_COUNT and NDB_FLAG_TENSOR_FILTER on a call override both. */
typedef struct ndb_tuning {
    int32_t tc_min_dim;
    int32_t tc_min_item;
    int32_t gram_filter;  /* 1: the CUDA-core count uses the FP32 Gram filter at d >= 8 (as
                           * NDB_FLAG_GRAM_FILTER); 0: the library's default (the exact sum) */
} ndb_tuning;

/* Sets the context's thresholds (NULL: back to the defaults); negative values are
 * NDB_ERR_INVALID_ARGUMENT. */
ndb_status ndb_b200_set_tuning(ndb_ctx *ctx, const ndb_tuning *tuning);

/* The context's thresholds as set (0 where the default applies). */
ndb_status ndb_b200_get_tuning(ndb_ctx *ctx, ndb_tuning *tuning);

/* Bound of the device-side union-find loops of the context's runs: steps of one
 * find and attempts of one union (0 = the default, 2^26).  A loop that reaches it
 * ends, and the run returns NDB_ERR_DEVICE_LIMIT instead of spinning; its outputs
 * are then undefined, and the context stays usable.  The default is far above any
 * depth lock-free hooking reaches; small values exist so that tests can make the
 * bound run out on purpose.  No counterpart in the reference, whose propagation
 * loop (data_process.cpp:183) has no bound. */
ndb_status ndb_b200_set_debug_limits(ndb_ctx *ctx, int64_t uf_max_steps);

/* Device bytes the context holds now (its buffers grow to the largest job run and
 * are kept until ndb_b200_destroy or a lower memory cap). */
ndb_status ndb_b200_device_bytes(ndb_ctx *ctx, int64_t *bytes);

/* Counters and phase times of the last run. */
ndb_status ndb_b200_get_stats(ndb_ctx *ctx, ndb_stats *stats);

/* Human-readable text of a status. */
const char *ndb_b200_strerror(ndb_status status);

/* Text of the last CUDA error seen by this context (empty when none). */
const char *ndb_b200_last_cuda_error(ndb_ctx *ctx);

/* Library version string. */
const char *ndb_b200_version(void);

/* Largest job ndb_b200_run_noalloc accepts. */
#define NDB_NOALLOC_MAX_POINTS 32768

/* ndb_b200_run for callers that may not allocate device memory -- a service that
 * reserves its GPU memory once at start-up and forbids cudaMalloc later, or a host
 * program that only lends out buffers it owns.  No counterpart in the reference.
 * Every scratch buffer comes from one fixed device array inside the library (about
 * 16 MiB, held by every GPU that loads the library until the process exits); the
 * call makes no cudaMalloc or cudaFree.  coords, nn_out and cluster_index_out are
 * device pointers on the current device (outputs may be NULL); the work runs on
 * cuda_stream (NULL: the legacy default stream) and is complete when the call
 * returns.  n above NDB_NOALLOC_MAX_POINTS returns NDB_ERR_TOO_MANY_POINTS; a
 * buffer request beyond its slice of the array returns NDB_ERR_OUT_OF_MEMORY (the
 * slices are sized for the largest request of any job within the limit).
 * The first call on a device does the set-up (it looks up the array's device
 * address and creates the shared state's timing events), so make it before any
 * stream capture.  Calls share the array: they are serialised per device, and GPU
 * work that overlaps a call and touches the same array would race. */
ndb_status ndb_b200_run_noalloc(const float *coords, int64_t n, int32_t d, float eps, int32_t min_pts,
                                uint32_t flags, int32_t *nn_out, int32_t *cluster_index_out,
                                ndb_result *result, void *cuda_stream);

#ifdef __cplusplus
}
#endif

#endif /* NDB_B200_H */
