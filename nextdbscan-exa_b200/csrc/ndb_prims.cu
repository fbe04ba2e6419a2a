// ndb_prims.cu -- device-wide exclusive scan and stable LSD radix sort (key, value).
//
// These replace the reference's generic parallel primitives on the hot path
// (exa::exclusive_scan magma_exa_omp.h:92-129, exa::copy_if :131-162, and the
// sample sort :282-364 that the reference ships but never calls) with
// purpose-built histogram / scan / scatter kernels.  Both are HBM-bound:
// a scan moves 8 bytes per element (read + write) plus a 4-byte reduce pass, a
// sort pass moves 2 x (key + value) bytes per element plus the histogram read.
#include "ndb_common.cuh"
#include "ndb_internal.h"

namespace ndb {

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = kScanTile / kScanThreads;  // 8

__device__ __forceinline__ int pad32(int e) { return e + (e >> 5); }

__global__ void __launch_bounds__(kScanThreads) scan_reduce_kernel(const uint32_t *__restrict__ in,
                                                                   int64_t n,
                                                                   uint32_t *__restrict__ partials) {
    const int t = threadIdx.x;
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        const int64_t e = base + i * kScanThreads + t;
        if (e < n) s += in[e];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
    __shared__ uint32_t s_w[kScanThreads / kWarp];
    if ((t & 31) == 0) s_w[t >> 5] = s;
    __syncthreads();
    if (t == 0) {
        uint32_t tot = 0;
#pragma unroll
        for (int w = 0; w < kScanThreads / kWarp; ++w) tot += s_w[w];
        partials[blockIdx.x] = tot;
    }
}

__global__ void __launch_bounds__(kScanThreads) scan_down_kernel(const uint32_t *in, uint32_t *out,
                                                                 int64_t n,
                                                                 const uint32_t *__restrict__ offsets,
                                                                 uint32_t *__restrict__ total_dev) {
    __shared__ uint32_t s[kScanTile + kScanTile / 32];
    __shared__ uint32_t s_w[kScanThreads / kWarp];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        const int e = i * kScanThreads + t;
        s[pad32(e)] = (base + e < n) ? in[base + e] : 0u;
    }
    __syncthreads();
    uint32_t v[kScanItems];
    uint32_t sum = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        v[i] = s[pad32(t * kScanItems + i)];
        sum += v[i];
    }
    uint32_t x = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(kFull, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_w[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kScanThreads / kWarp ? s_w[lane] : 0u;
#pragma unroll
        for (int o = 1; o < kScanThreads / kWarp; o <<= 1) {
            const uint32_t y = __shfl_up_sync(kFull, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kScanThreads / kWarp) s_w[lane] = w;
    }
    __syncthreads();
    const uint32_t block_off = offsets ? offsets[blockIdx.x] : 0u;
    uint32_t run = block_off + (warp > 0 ? s_w[warp - 1] : 0u) + x - sum;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        s[pad32(t * kScanItems + i)] = run;
        run += v[i];
    }
    if (total_dev && blockIdx.x == gridDim.x - 1 && t == 0)
        *total_dev = block_off + s_w[kScanThreads / kWarp - 1];
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        const int e = i * kScanThreads + t;
        if (base + e < n) out[base + e] = s[pad32(e)];
    }
}

// ---------------------------------------------------------------------------
// radix sort
// ---------------------------------------------------------------------------
constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / kWarp;           // 8
constexpr int kSortItems = kSortTile / kSortThreads;       // 8 per lane
constexpr int kRadix = 256;

template <typename K>
__global__ void __launch_bounds__(kSortThreads) sort_upsweep_kernel(const K *__restrict__ keys, int64_t n,
                                                                    int shift, uint32_t *__restrict__ hist,
                                                                    int nblocks) {
    __shared__ uint32_t s_h[kSortWarps][kRadix];
    const int t = threadIdx.x, warp = t >> 5;
    for (int i = t; i < kSortWarps * kRadix; i += kSortThreads) (&s_h[0][0])[i] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kSortTile;
#pragma unroll
    for (int i = 0; i < kSortItems; ++i) {
        const int64_t e = base + i * kSortThreads + t;
        if (e < n) atomicAdd(&s_h[warp][(uint32_t)(keys[e] >> shift) & 0xffu], 1u);
    }
    __syncthreads();
    uint32_t c = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) c += s_h[w][t];
    hist[(int64_t)t * nblocks + blockIdx.x] = c;
}

// Stable scatter.  Element order inside a block: warp w owns elements
// [w*256, w*256+256), item j of lane l is element w*256 + j*32 + l.  Ranks follow
// that order (items in order, lanes in order within an item), warps follow each
// other, and blocks follow each other through the digit-major histogram scan.
// The tile is first reordered by digit in shared memory, so the global writes go
// out as contiguous runs per digit instead of 32 scattered words per warp.
template <typename K>
__global__ void __launch_bounds__(kSortThreads) sort_downsweep_kernel(
    const K *__restrict__ kin, const int32_t *__restrict__ vin, K *__restrict__ kout,
    int32_t *__restrict__ vout, int64_t n, int shift, const uint32_t *__restrict__ hist_scanned,
    int nblocks) {
    __shared__ uint32_t s_cnt[kSortWarps][kRadix];
    __shared__ uint32_t s_base[kRadix];     // global position of the block's first element of each digit
    __shared__ uint32_t s_local[kRadix];    // first tile position of each digit
    __shared__ K s_key[kSortTile];
    __shared__ int32_t s_val[kSortTile];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    for (int i = t; i < kSortWarps * kRadix; i += kSortThreads) (&s_cnt[0][0])[i] = 0;
    s_base[t] = hist_scanned[(int64_t)t * nblocks + blockIdx.x];
    __syncthreads();

    const int64_t tile0 = (int64_t)blockIdx.x * kSortTile;
    const int64_t base = tile0 + warp * (kSortItems * kWarp);
    const unsigned lt = lanemask_lt();
    K key[kSortItems];
    int32_t val[kSortItems];
    uint32_t dig[kSortItems], rank[kSortItems];
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        const int64_t e = base + j * kWarp + lane;
        const bool valid = e < n;
        dig[j] = 0;
        rank[j] = 0;
        if (valid) {
            key[j] = kin[e];
            val[j] = vin[e];
            dig[j] = (uint32_t)(key[j] >> shift) & 0xffu;
        }
        const unsigned active = __ballot_sync(kFull, valid);
        if (valid) {
            const unsigned peers = __match_any_sync(active, dig[j]);
            const int leader = __ffs(peers) - 1;
            uint32_t old = 0;
            if (lane == leader) {
                old = s_cnt[warp][dig[j]];
                s_cnt[warp][dig[j]] = old + __popc(peers);
            }
            old = __shfl_sync(active, old, leader);
            rank[j] = old + __popc(peers & lt);
        }
        __syncwarp();
    }
    __syncthreads();
    // per digit: exclusive prefix over warps, and the digit's total in the tile
    uint32_t tot = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) {
        const uint32_t c = s_cnt[w][t];
        s_cnt[w][t] = tot;
        tot += c;
    }
    // exclusive scan of the digit totals over the 256 digits (one digit per thread)
    {
        uint32_t x = tot;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(kFull, x, o);
            if (lane >= o) x += y;
        }
        __shared__ uint32_t s_w[kSortWarps];
        if (lane == 31) s_w[warp] = x;
        __syncthreads();
        uint32_t wp = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w)
            if (w < warp) wp += s_w[w];
        s_local[t] = wp + x - tot;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        const int64_t e = base + j * kWarp + lane;
        if (e < n) {
            const uint32_t lp = s_local[dig[j]] + s_cnt[warp][dig[j]] + rank[j];
            s_key[lp] = key[j];
            s_val[lp] = val[j];
        }
    }
    __syncthreads();
    const int valid_in_tile = (int)min((int64_t)kSortTile, n - tile0);
#pragma unroll
    for (int i = 0; i < kSortItems; ++i) {
        const int e = i * kSortThreads + t;
        if (e < valid_in_tile) {
            const K k = s_key[e];
            const uint32_t d = (uint32_t)(k >> shift) & 0xffu;
            const uint32_t pos = s_base[d] + (uint32_t)e - s_local[d];
            kout[pos] = k;
            vout[pos] = s_val[e];
        }
    }
}

template <typename K>
cudaError_t radix_sort_pairs(K *k0, int32_t *v0, K *k1, int32_t *v1, int64_t n, int bits,
                             uint32_t *hist, uint32_t *scan_scratch, bool *result_in_first,
                             cudaStream_t st) {
    *result_in_first = true;
    if (n <= 1 || bits <= 0) return cudaSuccess;
    const int nblocks = (int)((n + kSortTile - 1) / kSortTile);
    K *ka = k0, *kb = k1;
    int32_t *va = v0, *vb = v1;
    for (int shift = 0; shift < bits; shift += 8) {
        ++launch_counter(), sort_upsweep_kernel<K><<<nblocks, kSortThreads, 0, st>>>(ka, n, shift, hist, nblocks);
        cudaError_t e = scan_exclusive_u32(hist, hist, (int64_t)kRadix * nblocks, nullptr,
                                           scan_scratch, st);
        if (e != cudaSuccess) return e;
        ++launch_counter(), sort_downsweep_kernel<K><<<nblocks, kSortThreads, 0, st>>>(ka, va, kb, vb, n, shift, hist,
                                                                   nblocks);
        K *tk = ka;
        ka = kb;
        kb = tk;
        int32_t *tv = va;
        va = vb;
        vb = tv;
        *result_in_first = !*result_in_first;
    }
    return cudaGetLastError();
}

}  // namespace

int &launch_counter() {
    static thread_local int count = 0;
    return count;
}

size_t scan_scratch_words(int64_t n) {
    const int64_t nb = (n + kScanTile - 1) / kScanTile;
    if (nb <= 1) return 0;
    return (size_t)((nb + 63) & ~int64_t(63)) + scan_scratch_words(nb);
}

cudaError_t scan_exclusive_u32(const uint32_t *in, uint32_t *out, int64_t n, uint32_t *total_dev,
                               uint32_t *scratch, cudaStream_t st) {
    if (n <= 0) {
        if (total_dev) return cudaMemsetAsync(total_dev, 0, sizeof(uint32_t), st);
        return cudaSuccess;
    }
    const int64_t nb = (n + kScanTile - 1) / kScanTile;
    if (nb == 1) {
        ++launch_counter(), scan_down_kernel<<<1, kScanThreads, 0, st>>>(in, out, n, nullptr, total_dev);
        return cudaGetLastError();
    }
    uint32_t *partials = scratch;
    uint32_t *rest = scratch + ((nb + 63) & ~int64_t(63));
    ++launch_counter(), scan_reduce_kernel<<<(unsigned)nb, kScanThreads, 0, st>>>(in, n, partials);
    cudaError_t e = scan_exclusive_u32(partials, partials, nb, nullptr, rest, st);
    if (e != cudaSuccess) return e;
    ++launch_counter(), scan_down_kernel<<<(unsigned)nb, kScanThreads, 0, st>>>(in, out, n, partials, total_dev);
    return cudaGetLastError();
}

size_t sort_hist_words(int64_t n) {
    const int64_t nblocks = (n + kSortTile - 1) / kSortTile;
    return (size_t)(kRadix * (nblocks > 0 ? nblocks : 1));
}

cudaError_t radix_sort_pairs_u32(uint32_t *k0, int32_t *v0, uint32_t *k1, int32_t *v1, int64_t n,
                                 int bits, uint32_t *hist, uint32_t *scan_scratch,
                                 bool *result_in_first, cudaStream_t st) {
    return radix_sort_pairs<uint32_t>(k0, v0, k1, v1, n, bits, hist, scan_scratch, result_in_first,
                                      st);
}

cudaError_t radix_sort_pairs_u64(uint64_t *k0, int32_t *v0, uint64_t *k1, int32_t *v1, int64_t n,
                                 int bits, uint32_t *hist, uint32_t *scan_scratch,
                                 bool *result_in_first, cudaStream_t st) {
    return radix_sort_pairs<uint64_t>(k0, v0, k1, v1, n, bits, hist, scan_scratch, result_in_first,
                                      st);
}

}  // namespace ndb
