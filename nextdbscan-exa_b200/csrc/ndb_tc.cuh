// ndb_tc.cuh -- tensor-core filtered neighbour count for d >= 8 (sm_100a).
//
// The exact predicate (data_process.cpp:443-447) costs 3d separately rounded FP32
// operations per pair.  For d >= 8 the count runs instead on Gram tiles from the
// 5th-generation tensor cores: for an item (up to 32 points i of one cell) and a
// tile of 128 candidates j, one CTA computes
//
//     D~(i,j) = |a_i|^2 + |b_j|^2 - 2 a_i.b_j,   a = x_i - o, b = x_j - o,
//
// with o the item's first point, a.b from three TF32 products (hi.hi + hi.lo +
// lo.hi of the split a = hi + lo) accumulated in FP32 in tensor memory.  A pair is
// a hit when D~ is below eps^2 by more than a rigorous bound on the filter's error,
// a miss when above by more than it, and otherwise (the guard band) it is rechecked
// with the reference's own FP32 arithmetic.  Counts, core flags and neighbour lists
// are therefore identical to the exact kernel's.
//
// Error bound (per pair, u = 2^-24, t = 2^-11 the TF32 rounding unit, K the padded
// dimension):  |D~ - |x_i - x_j|^2| <= kappa (n_i + n_j) with n = |a|^2, from
//   the split (3 t^2 |a||b|), the FP32 accumulation of 3K exact TF32 products
//   (assumed no worse than 4u per addition of the running magnitude), the FP32
//   norms (K u n), the centring x - o (4u (n_i + n_j)) and the rounding of the
//   comparison value; kappa = (10 + 8K) 2^-22 is about twice their sum.
// The reference's FP32 sum itself differs from the exact distance by at most
// (d + 2) u relatively; gamma = 2 (K + 8) u covers it.
#pragma once
#include "ndb_kernels.cuh"

namespace ndb {
namespace tc {

constexpr int kM = 128;              // candidates per tile: MMA M, TMEM lanes
constexpr int kN = 32;               // points of one item: MMA N, TMEM columns per buffer
constexpr int kThreads = 128;        // four warps, one per TMEM lane quadrant
constexpr uint32_t kTmemCols = 64;   // two accumulator buffers
constexpr uint32_t kWaitLimit = 1u << 22;
constexpr int kMinDim = 8;           // the kernel is built for d >= 8 (K padded to 8 or 16)
// resident CTAs per SM the register allocation is sized for (a build-time choice):
// d > 8 (42 KB of shared memory per CTA; 5 measured 2 % faster than 4 on the 16-D
// batch, at 96 registers) and d = 8 (23 KB)
#ifndef NDB_TC_MIN_BLOCKS
#define NDB_TC_MIN_BLOCKS 5
#endif
#ifndef NDB_TC_MIN_BLOCKS_8
#define NDB_TC_MIN_BLOCKS_8 5
#endif
template <int D>
struct TcBlocks {
    static constexpr int v = D <= 8 ? NDB_TC_MIN_BLOCKS_8 : NDB_TC_MIN_BLOCKS;
};

// Per-item record of the tensor count (tc_records_kernel), fetched one item ahead
// by a bulk copy: int2 slot 0 = (cell, first point), slot 1 + r = (first point,
// length) of stencil row r (r < 32), slot 33 = (points of the item, job or -1).
// 34 slots = 272 bytes, a multiple of 16.
constexpr int kRecSlots = 34;
constexpr uint32_t kRecBytes = kRecSlots * 8;

template <int D>
struct KPad {
    static constexpr int v = D <= 8 ? 8 : 16;
};

template <int KP>
__host__ __device__ constexpr float kappa() {
    return (10.0f + 8.0f * KP) * (1.0f / 4194304.0f);  // 2^-22
}
template <int KP>
__host__ __device__ constexpr float gamma_rel() {
    return 2.0f * (KP + 8) * (1.0f / 16777216.0f);  // 2^-24
}
constexpr float kSigma = 8.0f / 16777216.0f;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint32_t tf32_rna(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

// Shared-memory matrix descriptor, K-major, no swizzle: 8-row core matrices of
// 16-byte rows, the next 16-byte K chunk lbo bytes away, the next 8 rows sbo bytes
// away; bits 46-47 = 1 (the sm_100 descriptor version).
__device__ __forceinline__ uint64_t desc_kmajor(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::tf32: FP32 accumulator (bits 4-5 = 1), A and B
// TF32 (bits 7-9, 10-12 = 2), both K-major, N >> 3 at bits 17-22, M >> 4 at 24-28.
// N is 32 (a whole item) or 16 (its still-active points, packed; M = 128 allows N
// in steps of 16).
__host__ __device__ constexpr uint32_t idesc_tf32(int n) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kM >> 4) << 24);
}
constexpr uint32_t kIdesc = idesc_tf32(kN);
constexpr uint32_t kIdescNarrow = idesc_tf32(kN / 2);

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for the phase of the given parity; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    for (uint32_t i = 0; i < kWaitLimit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// One bulk copy (the TMA's untiled form) of `bytes` (a multiple of 16; both addresses
// 16-byte aligned) from this GPU's global memory into this CTA's shared memory,
// completing on the mbarrier with a transaction count.  No multicast.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tc_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate,
                                         uint32_t idesc = kIdesc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
// 32 consecutive accumulator columns of this thread's TMEM lane.  The load and
// its wait are one asm statement: the destination registers are undefined until
// tcgen05.wait::ld, so no use of them may be scheduled in between.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
        "tcgen05.wait::ld.sync.aligned;\n"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr)
        : "memory");
}
// The first 16 of them (the packed form, N = 16).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        "tcgen05.wait::ld.sync.aligned;\n"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr)
        : "memory");
}

// (acc << 1) | sign bit of x: one funnel shift appends a sign bit to a mask built
// from the last column down, so that column c ends at bit c
__device__ __forceinline__ unsigned push_sign(unsigned acc, float x) {
    unsigned r;
    asm("shf.l.wrap.b32 %0, %1, %2, 1;" : "=r"(r) : "r"(__float_as_uint(x)), "r"(acc));
    return r;
}

// Classification of the first NC accumulator columns of this thread's TMEM lane (one
// candidate j) against its bounds tlo, thi of the comparison value v_c = n_c - 2 g_c.
// v is formed negated, two columns per packed FMA: w_c = 2 g_c + (-n_c) is -v_c
// exactly (one rounding to nearest, which is symmetric); tlo + w_c = RN(tlo - v_c),
// two columns per packed add.  With finite operands the sum is >= +0 exactly when
// v_c <= tlo (neither bound is ever -0), so bit c of mlo (mhi) is set when v_c > tlo
// (v_c > thi); one funnel shift per bound appends the sign bit, last column first.
// Bits at and above NC are 0.  s_nneg holds -n_c.
template <int NC>
__device__ __forceinline__ void classify(const uint32_t (&g)[32], const float *s_nneg, float tlo, float thi,
                                         unsigned &mlo, unsigned &mhi) {
    const float2 two = make_float2(2.0f, 2.0f), lo2 = make_float2(tlo, tlo), hi2 = make_float2(thi, thi);
    unsigned ml = 0, mh = 0;
#pragma unroll
    for (int q = NC / 4 - 1; q >= 0; --q) {
        const float4 n4 = reinterpret_cast<const float4 *>(s_nneg)[q];
        const float2 w1 = __ffma2_rn(make_float2(__uint_as_float(g[4 * q + 2]), __uint_as_float(g[4 * q + 3])), two,
                                     make_float2(n4.z, n4.w));
        const float2 w0 = __ffma2_rn(make_float2(__uint_as_float(g[4 * q + 0]), __uint_as_float(g[4 * q + 1])), two,
                                     make_float2(n4.x, n4.y));
        const float2 l1 = __fadd2_rn(lo2, w1), h1 = __fadd2_rn(hi2, w1);
        const float2 l0 = __fadd2_rn(lo2, w0), h0 = __fadd2_rn(hi2, w0);
        ml = push_sign(ml, l1.y);
        mh = push_sign(mh, h1.y);
        ml = push_sign(ml, l1.x);
        mh = push_sign(mh, h1.x);
        ml = push_sign(ml, l0.y);
        mh = push_sign(mh, h0.y);
        ml = push_sign(ml, l0.x);
        mh = push_sign(mh, h0.x);
    }
    mlo = ml;
    mhi = mh;
}

// 32x32 bit-matrix transpose across a warp: lane l holds row l (bit c = column
// c) on entry and column l (bit r = row r) on return.
__device__ __forceinline__ unsigned transpose32(unsigned x, int lane) {
    const unsigned masks[5] = {0x0000FFFFu, 0x00FF00FFu, 0x0F0F0F0Fu, 0x33333333u, 0x55555555u};
#pragma unroll
    for (int s = 0; s < 5; ++s) {
        const int j = 16 >> s;
        const unsigned m = masks[s];
        const unsigned y = __shfl_xor_sync(kFull, x, j);
        x = (lane & j) ? ((x & ~m) | ((y >> j) & m)) : ((x & m) | ((y << j) & ~m));
    }
    return x;
}

// Operand tile in shared memory: element (row r, k) of an R-row tile at
// ((k / 4) * R + r) * 16 + (k % 4) * 4 bytes (LBO = 16 R, SBO = 128).
template <int KP>
__device__ __forceinline__ void store_row(uint32_t *tile, int rows, int r, const uint32_t (&v)[KP]) {
#pragma unroll
    for (int q = 0; q < KP / 4; ++q)
        *reinterpret_cast<uint4 *>(tile + ((size_t)q * rows + r) * 4) =
            make_uint4(v[4 * q + 0], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
}

// a = x - o, split into TF32 hi + lo, and |a|^2 (FP32), two dimensions per packed
// instruction; no = -o.  a = RN(x + (-o)) and lo = tf32(RN(a - hi)) (exact: a - hi
// fits in FP32) are the scalar values; the norm is two interleaved FMA chains added
// at the end, within the K u |a|^2 the error bound allows for it.  Padded dimensions
// (k >= D) are zero.
template <int D, int KP>
__device__ __forceinline__ float centre_split(const float (&x)[D], const float (&no)[D], uint32_t (&hi)[KP],
                                              uint32_t (&lo)[KP]) {
    float2 n2 = make_float2(0.0f, 0.0f);
#pragma unroll
    for (int k = 0; k < KP; k += 2) {
        if (k >= D) {
            hi[k] = lo[k] = hi[k + 1] = lo[k + 1] = 0u;
            continue;
        }
        const float2 a = k + 1 < D ? __fadd2_rn(make_float2(x[k], x[k + 1]), make_float2(no[k], no[k + 1]))
                                   : make_float2(__fadd_rn(x[k], no[k]), 0.0f);
        hi[k] = tf32_rna(a.x);
        hi[k + 1] = k + 1 < D ? tf32_rna(a.y) : 0u;
        const float2 l = __ffma2_rn(make_float2(__uint_as_float(hi[k]), __uint_as_float(hi[k + 1])),
                                    make_float2(-1.0f, -1.0f), a);
        lo[k] = tf32_rna(l.x);
        lo[k + 1] = k + 1 < D ? tf32_rna(l.y) : 0u;
        n2 = __ffma2_rn(a, a, n2);
    }
    return __fadd_rn(n2.x, n2.y);
}

// ---------------------------------------------------------------------------
// The count kernel.  Persistent CTAs take items from a work counter.  Per item:
// warp 0 gathers the stencil rows, warp 1 stages the item's points (the MMA's B
// operand, N = 32); then candidate tiles of 128 are staged by all threads (one
// row each: load, centre, split, store) while the tensor core runs the previous
// tile's three MMAs per K step into the other TMEM buffer.  Each thread owns one
// TMEM lane = one candidate; it classifies its 32 columns, rechecks band pairs
// exactly, and a warp transpose turns the row masks into per-column hit masks.
// EARLY: columns leave the active set once their count reaches min_pts.
// Neighbour lists: the first list_cap hits of each column (complete for every
// point that stays below min_pts), slots reserved by shared-memory atomics.
// ---------------------------------------------------------------------------
// Audit of the filter (AUDIT, a diagnostic run, never the timed one): every pair the
// filter classifies is also measured against its FP64 distance and the reference's
// FP32 predicate.  audit[0] = largest |D~ - d64| (bits of a non-negative double),
// audit[1] = largest |D~ - d64| / (kappa (n_i + n_j)), the error over the bound the
// guard band is built from, audit[2] = pairs audited, audit[3] = pairs decided
// outside the band (hit or miss without a recheck) whose decision differs from the
// reference's predicate.  D~ = v + |b_j|^2 is the filter's squared distance.
template <int D>
__device__ __forceinline__ void audit_tile(const float *s_x, const float *s_ni, const uint32_t (&g)[32], unsigned act,
                                           unsigned hit, unsigned band, int j, float nj, const float *__restrict__ xs,
                                           float e2, float kap, unsigned long long *audit) {
    constexpr int P = Stride<D>::P;
    double mx = 0.0, mr = 0.0;
    unsigned cnt = 0, mis = 0;
    if (j >= 0) {
        float xj[D];
        load_point<D>(xs, j, xj);
#pragma unroll
        for (int c = 0; c < 32; ++c) {
            if (!((act >> c) & 1u)) continue;
            float xi[D];
            load_point_smem<D>(s_x + c * P, xi);
            double d64 = 0.0;
#pragma unroll
            for (int k = 0; k < D; ++k) {
                const double t = (double)xi[k] - (double)xj[k];
                d64 = fma(t, t, d64);
            }
            const float v = __fmaf_rn(-2.0f, __uint_as_float(g[c]), s_ni[c]);
            const double err = fabs(((double)v + (double)nj) - d64);
            const double bound = (double)kap * ((double)s_ni[c] + (double)nj);
            mx = fmax(mx, err);
            if (bound > 0.0) mr = fmax(mr, err / bound);
            ++cnt;
            const bool exact = in_range<D>(xi, xj, e2);
            if (!((band >> c) & 1u) && (((hit >> c) & 1u) != 0) != exact) ++mis;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mx = fmax(mx, __shfl_xor_sync(kFull, mx, o));
        mr = fmax(mr, __shfl_xor_sync(kFull, mr, o));
        cnt += __shfl_xor_sync(kFull, cnt, o);
        mis += __shfl_xor_sync(kFull, mis, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (mx > 0.0) atomicMax(audit + 0, (unsigned long long)__double_as_longlong(mx));
        if (mr > 0.0) atomicMax(audit + 1, (unsigned long long)__double_as_longlong(mr));
        if (cnt) atomicAdd(audit + 2, (unsigned long long)cnt);
        if (mis) atomicAdd(audit + 3, (unsigned long long)mis);
    }
}

// Position of the (k+1)-th set bit of m (k < popc(m)): binary search on popcounts.
__device__ __forceinline__ int nth_set_bit(unsigned m, int k) {
    int pos = 0;
#pragma unroll
    for (int w = 16; w > 0; w >>= 1) {
        const int c = __popc(m & ((1u << w) - 1u));
        if (k >= c) {
            k -= c;
            m >>= w;
            pos += w;
        }
    }
    return pos;
}

// The records of the items in items[0, *n_items): one warp per item.
__global__ void tc_records_kernel(const int2 *__restrict__ items, const uint32_t *__restrict__ n_items,
                                  const int32_t *__restrict__ cell_start, const int2 *__restrict__ nbr, int n_rows,
                                  const int32_t *__restrict__ cell_job, int2 *__restrict__ rec) {
    const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= (int64_t)*n_items) return;
    const int2 it = items[w];
    int2 *r = rec + w * kRecSlots;
    if (lane < n_rows) {
        const int2 cr = nbr[(int64_t)it.x * n_rows + lane];
        int2 v = make_int2(0, 0);
        if (cr.x < cr.y) {
            const int a = cell_start[cr.x];
            v = make_int2(a, cell_start[cr.y] - a);
        }
        r[1 + lane] = v;
    }
    if (lane == 0) {
        r[0] = it;
        r[33] = make_int2(min(kN, cell_start[it.x + 1] - it.y), cell_job ? cell_job[it.x] : -1);
    }
}

template <int D, bool AUDIT = false>
__global__ void __launch_bounds__(kThreads, TcBlocks<D>::v) count_tc_kernel(
    const int2 *__restrict__ items, int64_t n_items, const int32_t *__restrict__ cell_start,
    const int2 *__restrict__ nbr, int n_rows, const float *__restrict__ xs, float e2, int min_pts, int early,
    int32_t *__restrict__ nn_sorted, int32_t *__restrict__ nbr_list, int list_cap, int list_stride,
    unsigned long long *__restrict__ pair_counter, unsigned long long *__restrict__ band_counter,
    unsigned int *__restrict__ work, int *__restrict__ err, const JobDev *__restrict__ jobs,
    const int32_t *__restrict__ cell_job, const uint32_t *__restrict__ n_items_dev = nullptr,
    unsigned long long *__restrict__ audit = nullptr, const int2 *__restrict__ rec = nullptr) {
    constexpr int KP = KPad<D>::v, P = Stride<D>::P, KC = KP / 4;
    static_assert(P % 4 == 0, "point rows are copied as float4");
    __shared__ __align__(1024) uint32_t s_a[2][2][KC * kM * 4];  // [buffer][hi, lo] candidate tiles
    __shared__ __align__(128) uint32_t s_b[2][KC * kN * 4];      // [hi, lo] the item's points
    __shared__ __align__(16) float s_x[kN * P];                   // the item's points as stored
    __shared__ __align__(16) float s_ni[kN];                      // |x_c - o|^2
    __shared__ __align__(16) float s_nneg[kN];                    // -|x_c - o|^2
    __shared__ int s_j[2][kM];
    __shared__ int s_part[2][4][kN];
    __shared__ int s_listn[kN];
    __shared__ RowTable s_rt;
    __shared__ __align__(16) int2 s_rec[2][kRecSlots];  // [slot] the records of this item and the next
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ __align__(8) uint64_t s_rbar[2];  // [slot] record copy complete
    __shared__ uint32_t s_tmem;
    __shared__ int s_item, s_abort;
    __shared__ float s_nmax;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (warp == 0) {
        tmem_alloc(&s_tmem, kTmemCols);
        tmem_relinquish();
    }
    if (tid == 0) {
        mbar_init(&s_bar[0], 1);
        mbar_init(&s_bar[1], 1);
        mbar_init(&s_rbar[0], 1);
        mbar_init(&s_rbar[1], 1);
        fence_mbar_init();
        s_abort = 0;
    }
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tmem = s_tmem;
    if (n_items_dev) n_items = *n_items_dev;  // a list whose length the device wrote
    uint32_t phase = 0, pending = 0;  // per buffer: parity of its next completion; MMAs not yet waited for
    unsigned long long pairs = 0, band = 0;
    const float kap = kappa<KP>();

    // Items are claimed one ahead (tid 0): the claim of the next item and, with
    // records, the bulk copy of its record are issued when this item starts, so
    // neither the work counter's round trip nor the record's dependent loads lie on
    // the item's critical path.  Slot k & 1 holds item k's record.
    int64_t cur = 0, nxt = 0;
    uint32_t rphase = 0, rpend = 0;  // per slot: parity of its next completion; copies not yet waited for
    if (tid == 0) {
        cur = (int64_t)atomicAdd(work, 1u);
        if (rec && cur < n_items) {
            bulk_load(s_rec[0], rec + cur * kRecSlots, kRecBytes, &s_rbar[0]);
            rpend |= 1u;
        }
        nxt = (int64_t)atomicAdd(work, 1u);
    }
    for (int k_item = 0;; ++k_item) {
        const int slot = k_item & 1;
        if (tid == 0) {
            s_item = (int)(cur < n_items ? cur : n_items);
            if (rec && nxt < n_items) {
                // the other slot was last read before the previous item's setup barrier
                fence_async_smem();
                bulk_load(s_rec[slot ^ 1], rec + nxt * kRecSlots, kRecBytes, &s_rbar[slot ^ 1]);
                rpend |= 1u << (slot ^ 1);
            }
            cur = nxt;
            nxt = (int64_t)atomicAdd(work, 1u);
        }
        __syncthreads();
        const int64_t item_id = s_item;
        if (item_id >= n_items || s_abort) break;
        int2 item;
        int cnt, jb = -1;
        if (rec) {
            const bool ok = mbar_wait(&s_rbar[slot], (rphase >> slot) & 1u);
            if (ok) {  // else the copy may still be in flight: the exit waits for it
                rphase ^= 1u << slot;
                rpend &= ~(1u << slot);
            }
            if (__syncthreads_or(!ok)) {
                if (tid == 0) {
                    s_abort = 1;
                    atomicExch(err, 2);
                }
                break;
            }
            item = s_rec[slot][0];
            const int2 t = s_rec[slot][33];
            cnt = t.x;
            jb = t.y;
        } else {
            item = items[item_id];
            cnt = min(kN, cell_start[item.x + 1] - item.y);
            if (jobs) jb = cell_job[item.x];
        }
        const int cell = item.x, p0 = item.y;
        float e2j = e2;
        int mp = min_pts, lc = list_cap;
        if (jobs) {
            const JobDev &J = jobs[jb];
            e2j = J.e2;
            mp = J.min_pts;
            lc = J.list_cap;
        }
        float o[D];  // the item's first point, negated: the centre of its Gram tiles
        load_point<D>(xs, p0, o);
#pragma unroll
        for (int k = 0; k < D; ++k) o[k] = -o[k];
        if (warp == 0) {
            if (rec) {
                const int2 rw = lane < n_rows ? s_rec[slot][1 + lane] : make_int2(0, 0);
                build_rows(rw.x, rw.y, n_rows, s_rt, lane);
            } else {
                gather_rows<false>(nbr + (int64_t)cell * n_rows, n_rows, cell_start, 0, s_rt, lane);
            }
            s_listn[lane] = 0;
        } else if (warp == 1) {
            float x[D];
            load_point<D>(xs, p0 + min(lane, cnt - 1), x);
            store_point_smem<D>(s_x + lane * P, x);
            uint32_t hi[KP], lo[KP];
            const float n = centre_split<D, KP>(x, o, hi, lo);
            store_row<KP>(s_b[0], kN, lane, hi);
            store_row<KP>(s_b[1], kN, lane, lo);
            s_ni[lane] = n;
            s_nneg[lane] = -n;
            float nm = lane < cnt ? n : 0.0f;
#pragma unroll
            for (int s = 16; s > 0; s >>= 1) nm = fmaxf(nm, __shfl_xor_sync(kFull, nm, s));
            if (lane == 0) s_nmax = nm;
            fence_async_smem();
        }
        __syncthreads();
        const int total = s_rt.off[n_rows];
        const float nmax = s_nmax;
        const float e2lo = e2j * (1.0f - gamma_rel<KP>()), e2hi = e2j * (1.0f + gamma_rel<KP>());
        const int n_tiles = (total + kM - 1) / kM;
        unsigned act = cnt >= kN ? kFull : ((1u << cnt) - 1u);
        int run = 0, totals = 0;  // lane c: this warp's hits of column c; all warps' hits after the last tile
        // Columns: column c (row c of s_b, s_x, s_ni) holds item point pcol (of lane c); ncols
        // columns hold points.  narrow: the MMA computes 16 columns (N = 16).
        int ncols = cnt, pcol = lane;
        bool narrow = false;

        // One candidate row per thread.  fetch: the row's point index (a cursor over
        // the stencil rows, advanced as the tile index grows) and its coordinates,
        // loaded into registers before the previous tile is processed so that the
        // load latency hides behind that work.  stage: centre, split, store, and the
        // thresholds of the comparison value v = n_i - 2 g (hit if v <= tlo, miss if
        // v > thi).
        int row = 0;
        auto fetch = [&](int t, int &jrow, float (&x)[D]) {
            const int v = t * kM + tid;
            jrow = -1;
            if (v < total) {
                while (s_rt.off[row + 1] <= v) ++row;
                jrow = s_rt.start[row] + (v - s_rt.off[row]);
                load_point<D>(xs, jrow, x);
            }
        };
        auto stage = [&](int buf, int jrow, const float (&x)[D], float &tlo, float &thi, float &nj) {
            uint32_t hi[KP], lo[KP];
            float n = 0.0f;
            if (jrow >= 0) {
                n = centre_split<D, KP>(x, o, hi, lo);
            } else {
#pragma unroll
                for (int k = 0; k < KP; ++k) hi[k] = lo[k] = 0u;
            }
            store_row<KP>(s_a[buf][0], kM, tid, hi);
            store_row<KP>(s_a[buf][1], kM, tid, lo);
            s_j[buf][tid] = jrow;
            const float slack = __fadd_rn(__fmul_rn(kap, __fadd_rn(nmax, n)), __fmul_rn(kSigma, e2j));
            nj = n;
            tlo = jrow >= 0 ? __fsub_rn(__fsub_rn(e2lo, n), slack) : -INFINITY;
            thi = jrow >= 0 ? __fadd_rn(__fsub_rn(e2hi, n), slack) : -INFINITY;
        };
        auto issue = [&](int t) {
            const int b = t & 1;
            const uint32_t d = tmem + (uint32_t)(b * kN);
            const uint32_t ah = smem_u32(s_a[b][0]), al = smem_u32(s_a[b][1]);
            const uint32_t bh = smem_u32(s_b[0]), bl = smem_u32(s_b[1]);
            const uint32_t id = narrow ? kIdescNarrow : kIdesc;
#pragma unroll
            for (int s = 0; s < KP / 8; ++s) {
                const uint32_t ao = (uint32_t)(s * 2 * kM * 16), bo = (uint32_t)(s * 2 * kN * 16);
                const uint64_t dah = desc_kmajor(ah + ao, kM * 16, 128), dal = desc_kmajor(al + ao, kM * 16, 128);
                const uint64_t dbh = desc_kmajor(bh + bo, kN * 16, 128), dbl = desc_kmajor(bl + bo, kN * 16, 128);
                mma_tf32(d, dah, dbh, s > 0 ? 1u : 0u, id);
                mma_tf32(d, dah, dbl, 1u, id);
                mma_tf32(d, dal, dbh, 1u, id);
            }
            mma_commit(&s_bar[b]);
        };

        int j_cur = -1, j_nxt = -1;
        float tlo_cur = -INFINITY, thi_cur = -INFINITY, tlo_nxt = -INFINITY, thi_nxt = -INFINITY;
        float nj_cur = 0.0f, nj_nxt = 0.0f;
        float x_nxt[D];
        fetch(0, j_cur, x_nxt);
        stage(0, j_cur, x_nxt, tlo_cur, thi_cur, nj_cur);
        fence_async_smem();
        tc_before_sync();
        __syncthreads();
        tc_after_sync();
        if (tid == 0) issue(0);
        pending |= 1u;
        for (int t = 1; t <= n_tiles; ++t) {
            const int pb = (t - 1) & 1;
            if (t < n_tiles) fetch(t, j_nxt, x_nxt);
            const bool ok = mbar_wait(&s_bar[pb], (phase >> pb) & 1u);
            if (ok) {
                phase ^= 1u << pb;
                pending &= ~(1u << pb);
                tc_after_sync();
                uint32_t g[32];
                const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(pb * kN);
                // Every column is classified (no per-column branch; inactive ones are
                // masked out afterwards): 16 columns once the item is packed, else 32.
                unsigned mlo, mhi;  // bit c: v_c > tlo, v_c > thi
                if (narrow) {
                    tmem_ld16(taddr, g);
                    classify<kN / 2>(g, s_nneg, tlo_cur, thi_cur, mlo, mhi);
                } else {
                    tmem_ld32(taddr, g);
                    classify<kN>(g, s_nneg, tlo_cur, thi_cur, mlo, mhi);
                }
                const float *sx = s_x;
                unsigned hb = ~mlo & act;
                unsigned bb = ~mhi & mlo & act;
                if constexpr (AUDIT)
                    audit_tile<D>(sx, s_ni, g, act, hb, bb, j_cur, nj_cur, xs, e2j, kap, audit);
                if (__any_sync(kFull, bb != 0)) {
                    if (bb) {
                        float xj[D];
                        load_point<D>(xs, j_cur, xj);
                        band += (unsigned long long)__popc(bb);
                        for (unsigned m = bb; m; m &= m - 1) {
                            const int c = __ffs(m) - 1;
                            float xi[D];
                            load_point_smem<D>(sx + c * P, xi);
                            if (in_range<D>(xi, xj, e2j)) hb |= 1u << c;
                        }
                    }
                }
                const unsigned cm = transpose32(hb, lane);  // rows of this warp that hit column `lane`
                if ((act >> lane) & 1u) {
                    const int h = __popc(cm);
                    run += h;
                    if (nbr_list && h && totals < lc) {
                        int slot = atomicAdd(&s_listn[lane], h);
                        for (unsigned m = cm; m && slot < lc; m &= m - 1, ++slot)
                            nbr_list[(int64_t)(p0 + pcol) * list_stride + slot] = s_j[pb][warp * 32 + __ffs(m) - 1];
                    }
                }
                s_part[t & 1][warp][lane] = run;
                if (tid == 0) pairs += (unsigned long long)__popc(act) * (unsigned long long)min(kM, total - (t - 1) * kM);
            } else {
                s_abort = 1;
                atomicExch(err, 2);
            }
            if (t < n_tiles) stage(t & 1, j_nxt, x_nxt, tlo_nxt, thi_nxt, nj_nxt);
            fence_async_smem();
            tc_before_sync();
            __syncthreads();
            tc_after_sync();
            if (s_abort) break;
            totals = s_part[t & 1][0][lane] + s_part[t & 1][1][lane] + s_part[t & 1][2][lane] + s_part[t & 1][3][lane];
            if (early) act = __ballot_sync(kFull, lane < ncols && totals < mp);
            if (early && !act) break;
            if (t < n_tiles) {
                // Packing (early exit only, once per item): when at most 16 columns are
                // still active, they move to the first 16 rows of the item's operand and
                // the MMAs compute N = 16 from then on, halving the classification.  A
                // finished column's count is final: it is written out here.  No MMA is in
                // flight (the last one was waited for above), so the operand may be
                // rewritten; warp 1 moves the rows through the candidate buffer of the
                // tile before this one (its MMA is complete, and it is next staged after
                // the following barrier), so only warp 1 touches them meanwhile.
                if (early && !narrow && __popc(act) <= kN / 2) {
                    const int nk = __popc(act);
                    if (warp == 0 && lane < ncols && !((act >> lane) & 1u)) nn_sorted[p0 + pcol] = totals;
                    const int src = lane < nk ? nth_set_bit(act, lane) : lane;
                    run = __shfl_sync(kFull, run, src);
                    totals = __shfl_sync(kFull, totals, src);
                    pcol = __shfl_sync(kFull, pcol, src);
                    if (warp == 0) {
                        const int ln = s_listn[src];
                        __syncwarp();
                        s_listn[lane] = ln;
                    } else if (warp == 1) {
                        constexpr int TS = 2 * KC * 4 + P + 4;  // words per row in the buffer (16-byte multiple)
                        uint32_t *tmp = &s_a[(t + 1) & 1][0][0] + lane * TS;
                        if (lane < nk) {
#pragma unroll
                            for (int h = 0; h < 2; ++h)
#pragma unroll
                                for (int q = 0; q < KC; ++q)
                                    *reinterpret_cast<uint4 *>(tmp + (h * KC + q) * 4) =
                                        *reinterpret_cast<const uint4 *>(&s_b[h][(q * kN + src) * 4]);
#pragma unroll
                            for (int q = 0; q < P / 4; ++q)
                                *reinterpret_cast<float4 *>(tmp + 2 * KC * 4 + 4 * q) =
                                    *reinterpret_cast<const float4 *>(&s_x[src * P + 4 * q]);
                            tmp[2 * KC * 4 + P] = __float_as_uint(s_ni[src]);
                            tmp[2 * KC * 4 + P + 1] = __float_as_uint(s_nneg[src]);
                        }
                        __syncwarp();
                        if (lane < nk) {
#pragma unroll
                            for (int h = 0; h < 2; ++h)
#pragma unroll
                                for (int q = 0; q < KC; ++q)
                                    *reinterpret_cast<uint4 *>(&s_b[h][(q * kN + lane) * 4]) =
                                        *reinterpret_cast<const uint4 *>(tmp + (h * KC + q) * 4);
#pragma unroll
                            for (int q = 0; q < P / 4; ++q)
                                *reinterpret_cast<float4 *>(&s_x[lane * P + 4 * q]) =
                                    *reinterpret_cast<const float4 *>(tmp + 2 * KC * 4 + 4 * q);
                            s_ni[lane] = __uint_as_float(tmp[2 * KC * 4 + P]);
                            s_nneg[lane] = __uint_as_float(tmp[2 * KC * 4 + P + 1]);
                            fence_async_smem();
                        }
                    }
                    narrow = true;
                    ncols = nk;
                    act = (1u << nk) - 1u;
                    __syncthreads();
                }
                if (tid == 0) issue(t);
                pending |= 1u << (t & 1);
                j_cur = j_nxt;
                tlo_cur = tlo_nxt;
                nj_cur = nj_nxt;
                thi_cur = thi_nxt;
            }
        }
        if (s_abort) break;
        if (warp == 0 && lane < ncols) nn_sorted[p0 + pcol] = totals;
    }
    // MMAs still in flight after an abort: wait for them (bounded) before freeing TMEM;
    // record copies still in flight (issued by tid 0): wait for them before exiting
    for (int b = 0; b < 2; ++b)
        if ((pending >> b) & 1u) mbar_wait(&s_bar[b], (phase >> b) & 1u);
    if (tid == 0)
        for (int b = 0; b < 2; ++b)
            if ((rpend >> b) & 1u) mbar_wait(&s_rbar[b], (rphase >> b) & 1u);
    tc_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc_after_sync();
        tmem_dealloc(tmem, kTmemCols);
    }
    if (tid == 0 && pairs) atomicAdd(pair_counter, pairs);
    if (band) atomicAdd(band_counter, band);
}

}  // namespace tc
}  // namespace ndb
