// ndb_common.cuh -- device helpers shared by the DBSCAN kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ndb {

constexpr int kWarp = 32;
constexpr unsigned kFull = 0xffffffffu;
constexpr int kNoCluster = 0x7fffffff;
constexpr int kMaxDim = 16;
constexpr int kMaxRows = 64;        // stencil rows (3-D same-cell grid: 25, 3-D eps grid: 9)
constexpr int kTile = 32;           // points of one cell handled by one warp item

// Sorted coordinates are stored point-major with a padded stride so that one
// point is one (or a few) 8/16-byte vector loads.
template <int D>
struct Stride {
    static constexpr int P = (D <= 2) ? D : ((D + 3) / 4) * 4;
};

// The reference's predicate (data_process.cpp:443-447): length starts at 0 and
// accumulates (a-b)*(a-b) dimension by dimension; every operation is separately
// rounded (no FMA contraction), and the pair is in range iff length <= e2.
template <int D>
__device__ __forceinline__ bool in_range(const float (&a)[D], const float (&b)[D], float e2) {
    float len = 0.0f;
#pragma unroll
    for (int k = 0; k < D; ++k) {
        const float t = __fsub_rn(a[k], b[k]);
        len = __fadd_rn(len, __fmul_rn(t, t));
    }
    return len <= e2;
}

// The same sum in two parts: dimensions [K0, K1) added to len.  Every term is
// non-negative, and rounding to nearest is monotone, so a partial sum above e2 already
// decides the pair (out of range) -- the kernels use that to skip the remaining
// dimensions; continuing the sum gives exactly in_range's length.
template <int D, int K0, int K1>
__device__ __forceinline__ float dist_part(const float (&a)[D], const float (&b)[D], float len) {
#pragma unroll
    for (int k = K0; k < K1; ++k) {
        const float t = __fsub_rn(a[k], b[k]);
        len = __fadd_rn(len, __fmul_rn(t, t));
    }
    return len;
}

template <int D>
__device__ __forceinline__ void load_point(const float *__restrict__ xs, int64_t idx, float (&x)[D]) {
    constexpr int P = Stride<D>::P;
    const float *p = xs + idx * P;
    if constexpr (P == 1) {
        x[0] = __ldg(p);
    } else if constexpr (P == 2) {
        const float2 v = __ldg(reinterpret_cast<const float2 *>(p));
        x[0] = v.x;
        x[1] = v.y;
    } else {
#pragma unroll
        for (int q = 0; q < P / 4; ++q) {
            const float4 v = __ldg(reinterpret_cast<const float4 *>(p) + q);
            if (4 * q + 0 < D) x[4 * q + 0] = v.x;
            if (4 * q + 1 < D) x[4 * q + 1] = v.y;
            if (4 * q + 2 < D) x[4 * q + 2] = v.z;
            if (4 * q + 3 < D) x[4 * q + 3] = v.w;
        }
    }
}

// Point from shared memory (same padded stride), read as a warp-wide broadcast.
template <int D>
__device__ __forceinline__ void load_point_smem(const float *p, float (&x)[D]) {
    constexpr int P = Stride<D>::P;
    if constexpr (P == 1) {
        x[0] = p[0];
    } else if constexpr (P == 2) {
        const float2 v = *reinterpret_cast<const float2 *>(p);
        x[0] = v.x;
        x[1] = v.y;
    } else {
#pragma unroll
        for (int q = 0; q < P / 4; ++q) {
            const float4 v = reinterpret_cast<const float4 *>(p)[q];
            if (4 * q + 0 < D) x[4 * q + 0] = v.x;
            if (4 * q + 1 < D) x[4 * q + 1] = v.y;
            if (4 * q + 2 < D) x[4 * q + 2] = v.z;
            if (4 * q + 3 < D) x[4 * q + 3] = v.w;
        }
    }
}

template <int D>
__device__ __forceinline__ void store_point_smem(float *p, const float (&x)[D]) {
    constexpr int P = Stride<D>::P;
#pragma unroll
    for (int k = 0; k < P; ++k) p[k] = (k < D) ? x[k] : 0.0f;
}

template <int D>
__device__ __forceinline__ void fill_nan(float (&x)[D]) {
#pragma unroll
    for (int k = 0; k < D; ++k) x[k] = __int_as_float(0x7fc00000);
}

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// ---------------------------------------------------------------------------
// Lock-free union-find over int32 ids.  parent[x] <= x always (the larger root
// is hooked under the smaller), so every find terminates.  Reads go through L2
// (ld.cg) because other SMs rewrite parents concurrently.
//
// Every loop is bounded.  err[0] is the run's error flag; err[1] holds the bound
// (steps of one find, attempts of one union), written by the host before the run
// (0 means the default kUfMaxSteps).  A loop that reaches it sets err[0] and
// returns, so the host reports NDB_ERR_DEVICE_LIMIT instead of a hung kernel.  The
// bound is never written while a kernel runs, so it is read through the
// read-only path.
// ---------------------------------------------------------------------------
constexpr int kUfMaxSteps = 1 << 26;

__device__ __forceinline__ int uf_limit(const int *err) {
    const int v = __ldg(err + 1);
    return v > 0 ? v : kUfMaxSteps;
}

__device__ __forceinline__ int uf_find(int *parent, int x, int *err) {
    int p = __ldcg(parent + x);
    const int lim = uf_limit(err);
    int steps = 0;
    while (p != x) {
        const int gp = __ldcg(parent + p);
        if (gp != p) __stcg(parent + x, gp);  // path halving: gp is an ancestor of x
        x = p;
        p = gp;
        if (++steps > lim) {
            atomicExch(err, 1);
            break;
        }
    }
    return x;
}

// Find without path halving: no stores.  A flatten pass must use it.  There each
// thread stores its unit's root, and a halving store by another thread (which read
// the unit's old parent before that store) could land after it and leave an
// intermediate ancestor behind, where the kernels that follow expect the root.
__device__ __forceinline__ int uf_find_ro(const int *parent, int x, int *err) {
    int p = __ldcg(parent + x);
    const int lim = uf_limit(err);
    int steps = 0;
    while (p != x) {
        x = p;
        p = __ldcg(parent + x);
        if (++steps > lim) {
            atomicExch(err, 1);
            break;
        }
    }
    return x;
}

// Union of the components of a and b; returns the root they share afterwards (as
// of the hook: later unions may hang it under a smaller root, so it stays an
// ancestor of both, and a later find from it is a shortcut from a or b).
__device__ __forceinline__ int uf_union_root(int *parent, int a, int b, int *err) {
    const int lim = uf_limit(err);
    for (int it = 0; it < lim; ++it) {
        a = uf_find(parent, a, err);
        b = uf_find(parent, b, err);
        if (a == b) return a;
        if (a > b) {
            const int t = a;
            a = b;
            b = t;
        }
        const int old = atomicCAS(parent + b, b, a);
        if (old == b) return a;
    }
    atomicExch(err, 1);
    return a;
}

__device__ __forceinline__ void uf_union(int *parent, int a, int b, int *err) {
    const int lim = uf_limit(err);
    for (int it = 0; it < lim; ++it) {
        a = uf_find(parent, a, err);
        b = uf_find(parent, b, err);
        if (a == b) return;
        if (a > b) {
            const int t = a;
            a = b;
            b = t;
        }
        const int old = atomicCAS(parent + b, b, a);
        if (old == b) return;
    }
    atomicExch(err, 1);
}

}  // namespace ndb
