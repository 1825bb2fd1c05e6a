// Shared device building blocks for the ANQI RkNN kernels (sm_100a).
//
// Bit-exact FP32 distances.  The reference computes every distance with
// AVX-512 intrinsics (include/distance.h:22-161): 16 lane accumulators, lane l
// accumulating elements j = l (mod 16) with a fused multiply-add in increasing
// j; the 16 lanes are folded by _mm512_reduce_add_ps (upper 256 bits onto the
// lower, upper 128 onto the lower, lanes {2,3} onto {0,1}, lane 1 onto lane 0);
// a masked tail (dim mod 16 elements) is multiplied without FMA, folded by the
// same tree and added last.  Here a group of four consecutive threads owns one
// vector pair: thread t of the group holds AVX lanes 4t..4t+3, loaded as one
// float4 per 16-element chunk, so rows are read with 16-byte coalesced loads.
// Every operation uses the _rn intrinsics so nvcc cannot contract or reorder.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace anqi {

constexpr uint32_t kEmpty = 0xFFFFFFFFu;
constexpr uint32_t kExpanded = 0x80000000u;
constexpr uint32_t kIdMask = 0x7FFFFFFFu;
constexpr float kSplitEps = 1e-6f;  // distance.h:14

// Device-side error word codes (first error wins; the host maps them to status codes).
enum DeviceError : uint32_t {
    kDevOk = 0,
    kDevCandOverflow = 1,   // per-query candidate list capacity
    kDevOutOverflow = 2,    // batch output buffer capacity
    kDevPoolOverflow = 3,   // gather pool capacity
    kDevBadId = 4,          // an id read from a graph or list is out of range
    kDevWaitTimeout = 5,    // a bounded wait ran out
    kDevSortOverflow = 6,
};

__host__ __device__ __forceinline__ uint64_t min_u64(uint64_t a, uint64_t b) { return a < b ? a : b; }

__device__ __forceinline__ void set_error(uint32_t* err, uint32_t code) {
    if (err) atomicCAS(err, 0u, code);
}

// ------------------------------------------------------------ AVX order

// _mm512_reduce_add_ps on a 16-lane value spread over a 4-thread group: thread
// t holds lanes a[0..3] = A[4t..4t+3].  The result is valid in all 4 threads.
__device__ __forceinline__ float group_reduce16(float a0, float a1, float a2, float a3, unsigned mask) {
    // T3[i] = A[i+8] + A[i]: threads 0,1 take the lanes of threads 2,3.
    float u0 = __shfl_down_sync(mask, a0, 2, 4);
    float u1 = __shfl_down_sync(mask, a1, 2, 4);
    float u2 = __shfl_down_sync(mask, a2, 2, 4);
    float u3 = __shfl_down_sync(mask, a3, 2, 4);
    float t0 = __fadd_rn(u0, a0), t1 = __fadd_rn(u1, a1), t2 = __fadd_rn(u2, a2), t3 = __fadd_rn(u3, a3);
    // T6[j] = T3[j+4] + T3[j]: thread 0 takes thread 1's T3[4..7].
    float v0 = __shfl_down_sync(mask, t0, 1, 4);
    float v1 = __shfl_down_sync(mask, t1, 1, 4);
    float v2 = __shfl_down_sync(mask, t2, 1, 4);
    float v3 = __shfl_down_sync(mask, t3, 1, 4);
    float s0 = __fadd_rn(v0, t0), s1 = __fadd_rn(v1, t1), s2 = __fadd_rn(v2, t2), s3 = __fadd_rn(v3, t3);
    // T8 = T6 + shuffle(T6, {2,3,0,1}); result = T8[0] + T8[1]
    float r = __fadd_rn(__fadd_rn(s0, s2), __fadd_rn(s1, s3));
    return __shfl_sync(mask, r, 0, 4);
}

// Squared L2 (distance.h:58-86).  a, b: 16-byte aligned rows whose allocation
// extends to a multiple of 4 floats past dim.  gt = thread index in the group.
__device__ __forceinline__ float group_l2sqr(const float* __restrict__ a, const float* __restrict__ b,
                                             uint32_t dim, uint32_t gt, unsigned mask) {
    const uint32_t q16 = dim >> 4, rem = dim & 15u;
    float c0 = 0.f, c1 = 0.f, c2 = 0.f, c3 = 0.f;
#pragma unroll 4
    for (uint32_t c = 0; c < q16; c++) {
        float4 x = *reinterpret_cast<const float4*>(a + 16 * c + 4 * gt);
        float4 y = *reinterpret_cast<const float4*>(b + 16 * c + 4 * gt);
        float d0 = __fsub_rn(x.x, y.x), d1 = __fsub_rn(x.y, y.y), d2 = __fsub_rn(x.z, y.z), d3 = __fsub_rn(x.w, y.w);
        c0 = __fmaf_rn(d0, d0, c0);
        c1 = __fmaf_rn(d1, d1, c1);
        c2 = __fmaf_rn(d2, d2, c2);
        c3 = __fmaf_rn(d3, d3, c3);
    }
    float res = group_reduce16(c0, c1, c2, c3, mask);
    if (rem) {
        float p0 = 0.f, p1 = 0.f, p2 = 0.f, p3 = 0.f;
        const uint32_t base = 16 * q16 + 4 * gt;
        if (4 * gt < rem) {
            float4 x = *reinterpret_cast<const float4*>(a + base);
            float4 y = *reinterpret_cast<const float4*>(b + base);
            float d0 = __fsub_rn(x.x, y.x), d1 = __fsub_rn(x.y, y.y), d2 = __fsub_rn(x.z, y.z), d3 = __fsub_rn(x.w, y.w);
            p0 = __fmul_rn(d0, d0);
            p1 = (4 * gt + 1 < rem) ? __fmul_rn(d1, d1) : 0.f;
            p2 = (4 * gt + 2 < rem) ? __fmul_rn(d2, d2) : 0.f;
            p3 = (4 * gt + 3 < rem) ? __fmul_rn(d3, d3) : 0.f;
        }
        res = __fadd_rn(res, group_reduce16(p0, p1, p2, p3, mask));
    }
    return res;
}

// Inner product (distance.h:89-116; NormSIMD16ExtAVX512__ is ip(a, a)).
__device__ __forceinline__ float group_ip(const float* __restrict__ a, const float* __restrict__ b,
                                          uint32_t dim, uint32_t gt, unsigned mask) {
    const uint32_t q16 = dim >> 4, rem = dim & 15u;
    float c0 = 0.f, c1 = 0.f, c2 = 0.f, c3 = 0.f;
#pragma unroll 4
    for (uint32_t c = 0; c < q16; c++) {
        float4 x = *reinterpret_cast<const float4*>(a + 16 * c + 4 * gt);
        float4 y = *reinterpret_cast<const float4*>(b + 16 * c + 4 * gt);
        c0 = __fmaf_rn(x.x, y.x, c0);
        c1 = __fmaf_rn(x.y, y.y, c1);
        c2 = __fmaf_rn(x.z, y.z, c2);
        c3 = __fmaf_rn(x.w, y.w, c3);
    }
    float res = group_reduce16(c0, c1, c2, c3, mask);
    if (rem) {
        float p0 = 0.f, p1 = 0.f, p2 = 0.f, p3 = 0.f;
        const uint32_t base = 16 * q16 + 4 * gt;
        if (4 * gt < rem) {
            float4 x = *reinterpret_cast<const float4*>(a + base);
            float4 y = *reinterpret_cast<const float4*>(b + base);
            p0 = __fmul_rn(x.x, y.x);
            p1 = (4 * gt + 1 < rem) ? __fmul_rn(x.y, y.y) : 0.f;
            p2 = (4 * gt + 2 < rem) ? __fmul_rn(x.z, y.z) : 0.f;
            p3 = (4 * gt + 3 < rem) ? __fmul_rn(x.w, y.w) : 0.f;
        }
        res = __fadd_rn(res, group_reduce16(p0, p1, p2, p3, mask));
    }
    return res;
}

// ------------------------------------------- wider groups (same arithmetic)
// A group of G = 8 or 16 threads per vector pair: thread t holds AVX lanes
// (16 / G) t .. (16 / G) t + 16 / G - 1.  Every lane accumulates the same
// FMAs in the same order as in the 4-thread form and the fold is the same
// tree, so the result has the same bits; fewer rows per round, fewer
// instructions per row.  Used when a batch has few rows, and for long rows
// (large dimensions), where fewer rows fit the staging buffer.

// _mm512_reduce_add_ps over a G-thread group (G = 8: a0, a1 = lanes 2t, 2t+1;
// G = 16: a0 = lane t).  The result is valid in all G threads.
template <int G>
__device__ __forceinline__ float group_reduce16_w(float a0, float a1, unsigned mask) {
    if constexpr (G == 8) {
        // T3[i] = A[i+8] + A[i]: threads 0..3 take threads 4..7
        const float t0 = __fadd_rn(__shfl_down_sync(mask, a0, 4, 8), a0);
        const float t1 = __fadd_rn(__shfl_down_sync(mask, a1, 4, 8), a1);
        // T6[i] = T3[i+4] + T3[i]: threads 0, 1 take threads 2, 3
        const float s0 = __fadd_rn(__shfl_down_sync(mask, t0, 2, 8), t0);
        const float s1 = __fadd_rn(__shfl_down_sync(mask, t1, 2, 8), t1);
        // (T6[0] + T6[2]) + (T6[1] + T6[3]): thread 0 holds T6[0..1], thread 1 T6[2..3]
        const float w0 = __shfl_down_sync(mask, s0, 1, 8), w1 = __shfl_down_sync(mask, s1, 1, 8);
        return __shfl_sync(mask, __fadd_rn(__fadd_rn(s0, w0), __fadd_rn(s1, w1)), 0, 8);
    } else {
        const float t0 = __fadd_rn(__shfl_down_sync(mask, a0, 8, 16), a0);
        const float s0 = __fadd_rn(__shfl_down_sync(mask, t0, 4, 16), t0);
        const float x = __fadd_rn(s0, __shfl_down_sync(mask, s0, 2, 16));  // T6[0]+T6[2] | T6[1]+T6[3]
        return __shfl_sync(mask, __fadd_rn(x, __shfl_down_sync(mask, x, 1, 16)), 0, 16);
    }
}

// Squared L2 (distance.h:58-86) by a group of G = 8 or 16 threads.
template <int G>
__device__ __forceinline__ float group_l2sqr_w(const float* __restrict__ a, const float* __restrict__ b,
                                               uint32_t dim, uint32_t gt, unsigned mask) {
    const uint32_t q16 = dim >> 4, rem = dim & 15u;
    constexpr uint32_t NL = 16 / G;
    float c0 = 0.f, c1 = 0.f;
#pragma unroll 4
    for (uint32_t c = 0; c < q16; c++) {
        if constexpr (NL == 2) {
            const float2 x = *reinterpret_cast<const float2*>(a + 16 * c + 2 * gt);
            const float2 y = *reinterpret_cast<const float2*>(b + 16 * c + 2 * gt);
            const float d0 = __fsub_rn(x.x, y.x), d1 = __fsub_rn(x.y, y.y);
            c0 = __fmaf_rn(d0, d0, c0);
            c1 = __fmaf_rn(d1, d1, c1);
        } else {
            const float d0 = __fsub_rn(a[16 * c + gt], b[16 * c + gt]);
            c0 = __fmaf_rn(d0, d0, c0);
        }
    }
    float res = group_reduce16_w<G>(c0, c1, mask);
    if (rem) {
        const uint32_t base = 16 * q16 + NL * gt;
        float p0 = 0.f, p1 = 0.f;
        if (NL * gt < rem) {
            const float d0 = __fsub_rn(a[base], b[base]);
            p0 = __fmul_rn(d0, d0);
        }
        if (NL == 2 && NL * gt + 1 < rem) {
            const float d1 = __fsub_rn(a[base + 1], b[base + 1]);
            p1 = __fmul_rn(d1, d1);
        }
        res = __fadd_rn(res, group_reduce16_w<G>(p0, p1, mask));
    }
    return res;
}

// Inner product (distance.h:89-116) by a group of G = 8 or 16 threads.
template <int G>
__device__ __forceinline__ float group_ip_w(const float* __restrict__ a, const float* __restrict__ b, uint32_t dim,
                                            uint32_t gt, unsigned mask) {
    const uint32_t q16 = dim >> 4, rem = dim & 15u;
    constexpr uint32_t NL = 16 / G;
    float c0 = 0.f, c1 = 0.f;
#pragma unroll 4
    for (uint32_t c = 0; c < q16; c++) {
        if constexpr (NL == 2) {
            const float2 x = *reinterpret_cast<const float2*>(a + 16 * c + 2 * gt);
            const float2 y = *reinterpret_cast<const float2*>(b + 16 * c + 2 * gt);
            c0 = __fmaf_rn(x.x, y.x, c0);
            c1 = __fmaf_rn(x.y, y.y, c1);
        } else {
            c0 = __fmaf_rn(a[16 * c + gt], b[16 * c + gt], c0);
        }
    }
    float res = group_reduce16_w<G>(c0, c1, mask);
    if (rem) {
        const uint32_t base = 16 * q16 + NL * gt;
        float p0 = 0.f, p1 = 0.f;
        if (NL * gt < rem) p0 = __fmul_rn(a[base], b[base]);
        if (NL == 2 && NL * gt + 1 < rem) p1 = __fmul_rn(a[base + 1], b[base + 1]);
        res = __fadd_rn(res, group_reduce16_w<G>(p0, p1, mask));
    }
    return res;
}

// ------------------------------------------------ chunk column order
// A row layout for 4-thread groups: within each full 16-float chunk, position
// 4t + k holds element t + 4k, so thread t of the group loads AVX lanes t,
// t + 4, t + 8, t + 12 as one float4 and the first two fold steps (lane i + 8
// onto i, then i + 4 onto i) stay in its registers.  Elements from `full` on
// (the tail) keep their places.  The map is its own inverse.
__host__ __device__ __forceinline__ uint32_t chunk_col_pos(uint32_t j, uint32_t full) {
    return j < full ? (j & ~15u) | ((j & 3u) << 2) | ((j >> 2) & 3u) : j;
}

// Inner product (distance.h:89-116) of two rows in chunk column order,
// dimension kDim (a multiple of 16) known at compile time: thread gt holds
// AVX lanes gt, gt + 4, gt + 8, gt + 12 of every chunk, folds lane i + 8 onto
// i and i + 4 onto i in registers and finishes the reference's tree with two
// shuffles.  The accumulators and the tree are group_ip's, so the bits are
// the same; the result is valid in all 4 threads.
template <uint32_t kDim>
__device__ __forceinline__ float group_ip_cols(const float* __restrict__ a, const float* __restrict__ b, uint32_t gt,
                                               unsigned mask) {
    static_assert(kDim % 16 == 0, "whole chunks only");
    float c0 = 0.f, c1 = 0.f, c2 = 0.f, c3 = 0.f;  // AVX lanes gt, gt + 4, gt + 8, gt + 12
#pragma unroll
    for (uint32_t c = 0; c < kDim / 16; c++) {
        const float4 x = *reinterpret_cast<const float4*>(a + 16 * c + 4 * gt);
        const float4 y = *reinterpret_cast<const float4*>(b + 16 * c + 4 * gt);
        c0 = __fmaf_rn(x.x, y.x, c0);
        c1 = __fmaf_rn(x.y, y.y, c1);
        c2 = __fmaf_rn(x.z, y.z, c2);
        c3 = __fmaf_rn(x.w, y.w, c3);
    }
    const float t6 = __fadd_rn(__fadd_rn(c3, c1), __fadd_rn(c2, c0));
    const float t8 = __fadd_rn(__shfl_xor_sync(mask, t6, 2, 4), t6);
    return __fadd_rn(__shfl_xor_sync(mask, t8, 1, 4), t8);
}

// Squared L2 (distance.h:58-86) of two rows in chunk column order, dimension
// kDim known at compile time with a tail of at most 4 elements.  The lane
// accumulators, the fold tree and the tail are those of group_l2sqr, so the
// bits are the same; the result is valid in all 4 threads.
template <uint32_t kDim>
__device__ __forceinline__ float group_l2sqr_cols(const float* __restrict__ a, const float* __restrict__ b,
                                                  uint32_t gt, unsigned mask) {
    constexpr uint32_t q16 = kDim / 16, rem = kDim % 16;
    static_assert(rem <= 4, "the tail must fit one float4");
    float c0 = 0.f, c1 = 0.f, c2 = 0.f, c3 = 0.f;  // AVX lanes gt, gt + 4, gt + 8, gt + 12
#pragma unroll
    for (uint32_t c = 0; c < q16; c++) {
        const float4 x = *reinterpret_cast<const float4*>(a + 16 * c + 4 * gt);
        const float4 y = *reinterpret_cast<const float4*>(b + 16 * c + 4 * gt);
        const float d0 = __fsub_rn(x.x, y.x), d1 = __fsub_rn(x.y, y.y), d2 = __fsub_rn(x.z, y.z),
                    d3 = __fsub_rn(x.w, y.w);
        c0 = __fmaf_rn(d0, d0, c0);
        c1 = __fmaf_rn(d1, d1, c1);
        c2 = __fmaf_rn(d2, d2, c2);
        c3 = __fmaf_rn(d3, d3, c3);
    }
    // T3[i] = A[i + 8] + A[i]; T6[gt] = T3[gt + 4] + T3[gt]
    const float t6 = __fadd_rn(__fadd_rn(c3, c1), __fadd_rn(c2, c0));
    // T8[k] = T6[k + 2] + T6[k]; T8[0] + T8[1] (xor partners: every thread
    // forms the same sums, addition being commutative)
    const float t8 = __fadd_rn(__shfl_xor_sync(mask, t6, 2, 4), t6);
    float res = __fadd_rn(__shfl_xor_sync(mask, t8, 1, 4), t8);
    if constexpr (rem != 0) {
        // masked tail, lanes 0..rem-1, products without FMA, same fold:
        // (p0 + p2) + (p1 + p3) with absent lanes zero (x + 0 = x for the
        // non-negative squares)
        const float4 x = *reinterpret_cast<const float4*>(a + 16 * q16);
        const float4 y = *reinterpret_cast<const float4*>(b + 16 * q16);
        const float e0 = __fsub_rn(x.x, y.x), p0 = __fmul_rn(e0, e0);
        float tail = p0;
        if constexpr (rem >= 2) {
            const float e1 = __fsub_rn(x.y, y.y), p1 = __fmul_rn(e1, e1);
            float lo = p0;
            if constexpr (rem >= 3) {
                const float e2 = __fsub_rn(x.z, y.z);
                lo = __fadd_rn(p0, __fmul_rn(e2, e2));
            }
            float hi = p1;
            if constexpr (rem == 4) {
                const float e3 = __fsub_rn(x.w, y.w);
                hi = __fadd_rn(p1, __fmul_rn(e3, e3));
            }
            tail = __fadd_rn(lo, hi);
        }
        res = __fadd_rn(res, tail);
    }
    return res;
}

// ------------------------------------------------------- row staging
// Global -> shared copies of whole rows with cp.async (16 bytes per
// instruction, no registers held while in flight): a row costs one memory
// round trip however long it is.  Rows are `stride` floats, 16-byte aligned,
// stride a multiple of 4.

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}

// Waits for this thread's outstanding cp.async copies.
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// The `nthreads` threads starting at `t0` of a warp copy one row; the caller
// waits (cp_async_wait_all + __syncwarp) before reading it.
__device__ __forceinline__ void stage_row_async(float* dst, const float* __restrict__ src, uint32_t stride,
                                                uint32_t t, uint32_t nthreads) {
    for (uint32_t c = t; c < stride / 4; c += nthreads) cp_async16(dst + 4 * c, src + 4 * c);
}

// nndindex::d2 (index.h:172-176): (na + nb) - 2 * ip(a, b)
__device__ __forceinline__ float norm_d2(float na, float nb, float ip) {
    return __fsub_rn(__fadd_rn(na, nb), __fmul_rn(2.0f, ip));
}

// The ip metric's distance 1 - sum a_i b_i (include/distance.h:170-174), by
// one thread, in the order the reference's compiled binary evaluates it (GCC
// 13 at -O3 on AVX-512 hosts): index order, the first 8 floor(dim / 8)
// products rounded and then added, the remaining dim mod 8 accumulated by
// fused multiply-adds.  Rows are 16-byte aligned (strides multiples of 4).
__device__ __forceinline__ float ip_dist_seq(const float* __restrict__ a, const float* __restrict__ b, uint32_t dim) {
    const uint32_t d8 = dim & ~7u;
    float p = 0.f;
    for (uint32_t i = 0; i < d8; i += 4) {
        const float4 x = *reinterpret_cast<const float4*>(a + i), y = *reinterpret_cast<const float4*>(b + i);
        p = __fadd_rn(p, __fmul_rn(x.x, y.x));
        p = __fadd_rn(p, __fmul_rn(x.y, y.y));
        p = __fadd_rn(p, __fmul_rn(x.z, y.z));
        p = __fadd_rn(p, __fmul_rn(x.w, y.w));
    }
    for (uint32_t i = d8; i < dim; i++) p = __fmaf_rn(a[i], b[i], p);
    return __fsub_rn(1.0f, p);
}

// --------------------------------------------------------- ordering

// (dist, id) total order of neighbor.h:22-24 (id without the expanded bit).
__device__ __forceinline__ bool nb_less(float da, uint32_t ia, float db, uint32_t ib) {
    return da < db || (da == db && (ia & kIdMask) < (ib & kIdMask));
}

// The (dist, id) order as a functor: ids compared directly ...
struct IdOrder {
    __device__ __forceinline__ bool operator()(float da, uint32_t ia, float db, uint32_t ib) const {
        return nb_less(da, ia, db, ib);
    }
};

// ... or, for objects renumbered for locality, through their original ids
// (perm: new id -> original id), so ties break exactly as in the original
// numbering.  The lookup happens only on equal distances.
struct PermOrder {
    const uint32_t* perm;  // null: the ids are original ids
    __device__ __forceinline__ bool operator()(float da, uint32_t ia, float db, uint32_t ib) const {
        if (da != db) return da < db;
        const uint32_t a = ia & kIdMask, b = ib & kIdMask;
        // equal ids, or a pad / idle-lane value (kEmpty; never an object id):
        // no lookup
        if (a == b || !perm || a == kIdMask || b == kIdMask) return a < b;
        return perm[a] < perm[b];
    }
};

// Plain (key, id) lexicographic order on full 32-bit ids (std::pair order).
__device__ __forceinline__ bool kv_less(float da, uint32_t ia, float db, uint32_t ib) {
    return da < db || (da == db && ia < ib);
}

// One compare-exchange step (stage k, distance j) of the 64-entry bitonic
// network below.
template <class Ord>
__device__ __forceinline__ void bitonic64_step(uint32_t k, uint32_t j, float& d0, uint32_t& i0, float& d1,
                                               uint32_t& i1, Ord ord) {
    const uint32_t lane = threadIdx.x & 31u;
    if (j == 32) {
        // partner of slot 0 is slot 1 of the same lane
        bool up = ((lane & k) == 0);  // k == 64 here -> always ascending
        bool sw = up ? ord(d1, i1, d0, i0) : ord(d0, i0, d1, i1);
        if (sw) {
            float td = d0; d0 = d1; d1 = td;
            uint32_t ti = i0; i0 = i1; i1 = ti;
        }
    } else {
#pragma unroll
        for (int s = 0; s < 2; s++) {
            float& d = s ? d1 : d0;
            uint32_t& id = s ? i1 : i0;
            const uint32_t e = lane + 32u * s;
            float od = __shfl_xor_sync(0xFFFFFFFFu, d, j);
            uint32_t oi = __shfl_xor_sync(0xFFFFFFFFu, id, j);
            const bool lower = (e & j) == 0;
            const bool up = (e & k) == 0;
            // keep the smaller if (lower == up); ties cannot occur between
            // distinct entries (total order)
            bool other_less = ord(od, oi, d, id);
            bool take = (lower == up) ? other_less : !other_less;
            if (take) {
                d = od;
                id = oi;
            }
        }
    }
}

// Bitonic sort of 64 (d, id) pairs held two per lane (index lane and lane+32),
// ascending in the order ord (nb_less by default).  Pads must be (+inf, kEmpty).
// kCompact keeps the network as loops (small code, for kernels whose speed
// depends on instruction fetch and that sort 64 entries rarely).
template <class Ord = IdOrder, bool kCompact = false>
__device__ __forceinline__ void warp_sort64(float& d0, uint32_t& i0, float& d1, uint32_t& i1, Ord ord = Ord()) {
    if constexpr (kCompact) {
#pragma unroll 1
        for (uint32_t k = 2; k <= 64; k <<= 1)
#pragma unroll 1
            for (uint32_t j = k >> 1; j > 0; j >>= 1) bitonic64_step(k, j, d0, i0, d1, i1, ord);
    } else {
#pragma unroll
        for (uint32_t k = 2; k <= 64; k <<= 1)
#pragma unroll
            for (uint32_t j = k >> 1; j > 0; j >>= 1) bitonic64_step(k, j, d0, i0, d1, i1, ord);
    }
}

// Number of entries in sorted a[0..n) strictly less than (d, id).
template <class Ord = IdOrder>
__device__ __forceinline__ uint32_t lower_rank(const float* ad, const uint32_t* ai, uint32_t n, float d, uint32_t id,
                                               Ord ord = Ord()) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (ord(ad[mid], ai[mid], d, id)) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// ----------------------------------------------------- visited bitmap

// A per-slot bitmap over all n objects plus a log of set bits, so the slot can
// be cleared in O(visited) at the end of a query/row (or wholesale on overflow).
struct VisitSlot {
    uint32_t* bits;      // ceil(n/32) words
    uint32_t* log;       // log_cap entries
    uint32_t log_cap;
    uint32_t words;
};

// Returns true when id was not yet visited (and marks it).
__device__ __forceinline__ bool visit_first(uint32_t* bits, uint32_t id) {
    const uint32_t m = 1u << (id & 31u);
    return (atomicOr(bits + (id >> 5), m) & m) == 0u;
}

// Warp-cooperative clear at the end of a query: either replay the log or wipe.
__device__ __forceinline__ void visit_clear(const VisitSlot& s, uint32_t logged) {
    const uint32_t lane = threadIdx.x & 31u;
    if (logged <= s.log_cap) {
        for (uint32_t i = lane; i < logged; i += 32) s.bits[s.log[i] >> 5] = 0u;
    } else {
        for (uint32_t w = lane; w < s.words; w += 32) s.bits[w] = 0u;
    }
    __syncwarp();
}

}  // namespace anqi
