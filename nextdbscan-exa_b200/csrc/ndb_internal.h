// ndb_internal.h -- host-side declarations shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

namespace ndb {

// A device buffer that only grows.
struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    cudaError_t ensure(size_t want) {
        if (want <= bytes) return cudaSuccess;
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
        size_t rounded = (want + 4095) & ~size_t(4095);
        cudaError_t e = cudaMalloc(&ptr, rounded);
        if (e == cudaSuccess) bytes = rounded;
        return e;
    }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
    template <typename T>
    T *as() const { return static_cast<T *>(ptr); }
};

// Kernels launched by the calling thread since the last reset (a context is used
// by one host thread at a time, so this counts the launches of one job).
int &launch_counter();

// ---- primitives (ndb_prims.cu) ----
constexpr int kScanTile = 2048;
// Scratch (in uint32 words) that scan_exclusive_u32 needs for n elements.
size_t scan_scratch_words(int64_t n);
// out[i] = sum(in[0..i)); *total_dev (if not null) = sum(in[0..n)).  in may equal out.
cudaError_t scan_exclusive_u32(const uint32_t *in, uint32_t *out, int64_t n, uint32_t *total_dev,
                               uint32_t *scratch, cudaStream_t st);

constexpr int kSortTile = 2048;
size_t sort_hist_words(int64_t n);
// Stable LSD radix sort of (key, value) pairs on the low `bits` bits of the keys.
// Sorts between (k0, v0) and (k1, v1); returns via *result_in_first whether the
// sorted data ended in (k0, v0).
cudaError_t radix_sort_pairs_u32(uint32_t *k0, int32_t *v0, uint32_t *k1, int32_t *v1, int64_t n,
                                 int bits, uint32_t *hist, uint32_t *scan_scratch,
                                 bool *result_in_first, cudaStream_t st);
cudaError_t radix_sort_pairs_u64(uint64_t *k0, int32_t *v0, uint64_t *k1, int32_t *v1, int64_t n,
                                 int bits, uint32_t *hist, uint32_t *scan_scratch,
                                 bool *result_in_first, cudaStream_t st);

}  // namespace ndb
