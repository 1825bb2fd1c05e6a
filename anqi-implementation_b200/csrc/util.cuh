// Warp-level sorting / merging / heap primitives shared by the build kernels.
#pragma once

#include <cstdint>

#include "common.cuh"

namespace anqi {

constexpr unsigned kAll = 0xFFFFFFFFu;

__device__ __forceinline__ uint32_t lane_lt_mask() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ uint32_t next_pow2(uint32_t x) {
    return x <= 1 ? 1u : 1u << (32 - __clz(x - 1));
}

// In-memory bitonic sort by one warp of (d, id) pairs, ascending nb_less order.
// n is padded internally to a power of two by the caller (pads: +inf, kEmpty).
static __device__ void warp_sort_pairs(float* d, uint32_t* id, uint32_t n_pow2) {
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t k = 2; k <= n_pow2; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = lane; i < n_pow2; i += 32) {
                const uint32_t p = i ^ j;
                if (p > i) {
                    const bool up = (i & k) == 0;
                    const float di = d[i], dp = d[p];
                    const uint32_t ii = id[i], ip = id[p];
                    const bool gt = nb_less(dp, ip, di, ii);  // element i greater than p
                    if (gt == up) {
                        d[i] = dp;
                        d[p] = di;
                        id[i] = ip;
                        id[p] = ii;
                    }
                }
            }
            __syncwarp();
        }
    }
}

static __device__ void warp_sort_u64(uint64_t* a, uint32_t n_pow2) {
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t k = 2; k <= n_pow2; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = lane; i < n_pow2; i += 32) {
                const uint32_t p = i ^ j;
                if (p > i) {
                    const bool up = (i & k) == 0;
                    const uint64_t x = a[i], y = a[p];
                    if ((x > y) == up) {
                        a[i] = y;
                        a[p] = x;
                    }
                }
            }
            __syncwarp();
        }
    }
}

// Merge m sorted new entries (nd/ni, distinct from each other) into a sorted
// list of `size` entries (ld/li) with capacity cap, writing od/oi.  When dedupe
// is set, new entries equal (same id, same distance) to a list entry are dropped
// first.  Returns the new size.  All 32 lanes must call it.
static __device__ uint32_t warp_merge(const float* ld, const uint32_t* li, uint32_t size, float* nd, uint32_t* ni, uint32_t m,
                               uint32_t cap, float* od, uint32_t* oi, bool dedupe) {
    const uint32_t lane = threadIdx.x & 31u;
    if (dedupe) {
        // compact away duplicates of list entries (order preserving)
        uint32_t kept = 0;
        for (uint32_t r0 = 0; r0 < m; r0 += 32) {
            const uint32_t r = r0 + lane;
            bool keep = false;
            float dv = 0;
            uint32_t iv = 0;
            if (r < m) {
                dv = nd[r];
                iv = ni[r];
                const uint32_t pos = lower_rank(ld, li, size, dv, iv);
                keep = !(pos < size && (li[pos] & kIdMask) == (iv & kIdMask));
            }
            const unsigned b = __ballot_sync(kAll, keep);
            __syncwarp();
            if (keep) {
                const uint32_t w = kept + __popc(b & lane_lt_mask());
                nd[w] = dv;
                ni[w] = iv;
            }
            kept += __popc(b);
            __syncwarp();
        }
        m = kept;
    }
    const uint32_t ns = min(cap, size + m);
    for (uint32_t p0 = lane; p0 < size; p0 += 32) {
        const float dv = ld[p0];
        const uint32_t iv = li[p0];
        const uint32_t pos = p0 + lower_rank(nd, ni, m, dv, iv);
        if (pos < ns) {
            od[pos] = dv;
            oi[pos] = iv;
        }
    }
    for (uint32_t r = lane; r < m; r += 32) {
        const uint32_t pos = r + lower_rank(ld, li, size, nd[r], ni[r]);
        if (pos < ns) {
            od[pos] = nd[r];
            oi[pos] = ni[r];
        }
    }
    __syncwarp();
    return ns;
}

// Sorts up to 64 (d, id) entries held in nd/ni[0..m) (pads filled here).
__device__ __forceinline__ void warp_sort_batch64(float* nd, uint32_t* ni, uint32_t m) {
    const uint32_t lane = threadIdx.x & 31u;
    const float inf = __int_as_float(0x7f800000);
    float d0 = lane < m ? nd[lane] : inf;
    uint32_t i0 = lane < m ? ni[lane] : kEmpty;
    float d1 = lane + 32 < m ? nd[lane + 32] : inf;
    uint32_t i1 = lane + 32 < m ? ni[lane + 32] : kEmpty;
    warp_sort64(d0, i0, d1, i1);
    __syncwarp();
    nd[lane] = d0;
    ni[lane] = i0;
    nd[lane + 32] = d1;
    ni[lane + 32] = i1;
    __syncwarp();
}

// heap.h:162-186 push_nolock / check_push (no reverse edges), by one lane.
__device__ __forceinline__ bool heap_push(uint32_t* ids, float* vals, uint32_t K, uint32_t node, float value) {
    if (value > vals[0]) return false;
    for (uint32_t i = 0; i < K; i++)
        if (ids[i] == node) return false;
    uint32_t cur = 0, sw;
    for (;;) {
        const uint32_t l = 2 * cur + 1, r = l + 1;
        if (l >= K) break;
        if (r >= K) {
            if (vals[l] > value) sw = l;
            else break;
        } else if (vals[l] >= vals[r]) {
            if (vals[l] > value) sw = l;
            else break;
        } else {
            if (vals[r] > value) sw = r;
            else break;
        }
        ids[cur] = ids[sw];
        vals[cur] = vals[sw];
        cur = sw;
    }
    ids[cur] = node;
    vals[cur] = value;
    return true;
}

__device__ __forceinline__ uint64_t hash64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

}  // namespace anqi
