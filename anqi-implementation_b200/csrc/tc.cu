// BF16 tensor-core (tcgen05) tiles for the brute-force distance work: the
// exact ground truth (tools/dataset_gt.cpp:206-313) in the precision form.
//
// Rows are converted once to bf16 (padded to a multiple of 16).  A CTA of 4
// warps owns a 128-row query tile resident in shared memory and streams
// 128-row base tiles through a two-stage shared-memory ring; one thread
// issues the K = 16 tcgen05.mma steps into one of two 128-column TMEM
// accumulators while the four warps run the epilogue of the previous tile
// (tcgen05.ld: thread = query row, 32 columns per load).
//
// Epilogue: key~ = |q|^2 + |x|^2 - 2 <q~, x~> with the reference's FP32
// norms.  A pair is a candidate when key~ - eps <= threshold, where eps bounds
// |key~ - key32| (key32 = the reference's FP32 key):
//   eps = 2 (|dq| |x| + |q| |dx| + |dq| |dx|)      bf16 rounding of the rows
//       + 4 g (|q~| |x~| + |q| |x|)                 FP32 accumulation, g = 2 d 2^-24
//       + 4 u (|q|^2 + |x|^2 + 2 |q| |x|)           the key's own roundings, u = 2^-24
// (|dq| = |q - bf16(q)|).  The ip metric's keys (1 - <q, x> for the AKNN
// source, -<q, x> for the ground truth) hold the product once: half the
// first two terms, and 4 u (1 + |q| |x|) for the rounding of the key.
// Candidates are recomputed in the reference's FP32
// order, so accept decisions and keys equal the FP32 path.  When both rows
// hold integers of magnitude <= 256 and d <= 128, bf16 and every partial
// sum are exact and key~ == key32: eps = 0 and no recheck is needed.
#include <cuda_bf16.h>

#include <algorithm>
#include <vector>

#include "internal.h"
#include "tc.cuh"
#include "util.cuh"

namespace anqi {
namespace {

constexpr uint32_t kTile = 128;     // M = N = 128
constexpr uint32_t kMaxDp = 256;    // padded dimension limit of the tensor path
constexpr uint32_t kWaitPolls = 1u << 24;

// ------------------------------------------------------------ row prep
// Per row: bf16 copy padded to dp (zeros), |x| (rounded up), |x - bf16(x)|
// (rounded up), and whether the row is exact-int (integers, |v| <= 256).
__global__ void bf16_rows_kernel(const float* __restrict__ x, uint64_t n, uint32_t xs, uint32_t d, uint32_t dp,
                                 __nv_bfloat16* __restrict__ xb, float* __restrict__ xnorm,
                                 float* __restrict__ xerr, uint8_t* __restrict__ exact_int) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t r = w; r < n; r += nw) {
        double s = 0.0, e = 0.0;
        bool ok = true;
        for (uint32_t k = lane; k < dp; k += 32) {
            const float v = k < d ? x[r * xs + k] : 0.0f;
            const __nv_bfloat16 b = __float2bfloat16_rn(v);
            xb[r * dp + k] = b;
            const double dv = (double)v - (double)__bfloat162float(b);
            s += (double)v * v;
            e += dv * dv;
            ok = ok && v == rintf(v) && fabsf(v) <= 256.0f;
        }
        for (int o = 16; o > 0; o >>= 1) {
            s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
            e += __shfl_xor_sync(0xFFFFFFFFu, e, o);
        }
        ok = __all_sync(0xFFFFFFFFu, ok);
        if (lane == 0) {
            xnorm[r] = __double2float_ru(sqrt(s) * (1.0 + 1e-12));
            xerr[r] = __double2float_ru(sqrt(e) * (1.0 + 1e-12));
            exact_int[r] = ok ? 1 : 0;
        }
    }
}

// Stages rows [r0, r0 + 128) of a bf16 matrix (dp wide) into the interleaved
// K-major layout; rows at or past nrows are zero-filled.  All threads of the
// CTA take part; completion via cp.async.wait.
__device__ __forceinline__ void stage_tile(unsigned char* dst, const __nv_bfloat16* __restrict__ src, uint64_t r0,
                                           uint64_t nrows, uint32_t dp) {
    const uint32_t chunks = dp / 8;
    for (uint32_t t = threadIdx.x; t < kTile * chunks; t += blockDim.x) {
        const uint32_t r = t % kTile, c = t / kTile;
        const uint64_t row = r0 + r;
        const bool ok = row < nrows;
        const __nv_bfloat16* s = src + (ok ? row : 0) * dp + 8 * c;
        tc::cp_async16_zfill(dst + (size_t)c * kTile * 16 + r * 16, s, ok ? 16u : 0u);
    }
}

__device__ __forceinline__ void cp_async_wait_all_() {
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// Issues the dp/16 MMA steps of one 128 x 128 tile (K = dp elements staged
// at a and b); the first step accumulates onto TMEM when `accumulate`.
__device__ __forceinline__ void issue_tile_mma(uint32_t tmem_d, const unsigned char* a, const unsigned char* b,
                                               uint32_t dp, bool accumulate = false) {
    constexpr uint32_t idesc = tc::idesc_bf16_f32(kTile, kTile);
    const uint32_t sa = tc::smem_u32(a), sb = tc::smem_u32(b);
    for (uint32_t s = 0; s < dp / 16; s++) {
        const uint64_t ad = tc::smem_desc(sa + 2 * s * kTile * 16, kTile * 16, 128);
        const uint64_t bd = tc::smem_desc(sb + 2 * s * kTile * 16, kTile * 16, 128);
        tc::mma_bf16(tmem_d, ad, bd, idesc, (s > 0 || accumulate) ? 1u : 0u);
    }
}

// ------------------------------------------------------------------ Gram
// out[i, j] = <bf16(a_i), bf16(b_j)> in FP32 for one 128 x 128 tile per CTA.
__global__ void __launch_bounds__(128) gram_kernel(const __nv_bfloat16* __restrict__ a, uint64_t na,
                                                   const __nv_bfloat16* __restrict__ b, uint64_t nb, uint32_t dp,
                                                   float* __restrict__ out, uint32_t* __restrict__ err) {
    extern __shared__ __align__(128) unsigned char sm[];
    unsigned char* sa = sm;
    unsigned char* sb = sm + (size_t)kTile * dp * 2;
    __shared__ uint64_t bar;
    __shared__ uint32_t tslot;
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint64_t i0 = (uint64_t)blockIdx.x * kTile, j0 = (uint64_t)blockIdx.y * kTile;
    if (warp == 0) tc::tmem_alloc(&tslot, 128);
    if (threadIdx.x == 0) {
        tc::mbar_init(&bar, 1);
        tc::fence_mbar_init();
    }
    stage_tile(sa, a, i0, na, dp);
    stage_tile(sb, b, j0, nb, dp);
    cp_async_wait_all_();
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tslot;
    if (threadIdx.x == 0) {
        issue_tile_mma(tmem, sa, sb, dp);
        tc::mma_commit(&bar);
    }
    const bool ok = tc::mbar_wait(&bar, 0, kWaitPolls);
    if (!ok && lane == 0) atomicExch(err, 8u);
    tc::fence_after_sync();
    if (ok) {
        const uint64_t row = i0 + warp * 32 + lane;
        for (uint32_t c0 = 0; c0 < kTile; c0 += 32) {
            float v[32];
            tc::tmem_ld32(tmem + ((warp * 32u) << 16) + c0, v);
            if (row < na)
                for (uint32_t e = 0; e < 32; e++)
                    if (j0 + c0 + e < nb) out[row * nb + j0 + c0 + e] = v[e];
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_free(tmem, 128);
}

// --------------------------------------------------------- filter
// One CTA = 8 warps over a 128-row query tile; warp w reads TMEM lanes
// 32 (w % 4) .. + 31 (its rows) and columns 64 (w / 4) .. + 63 of each tile.
struct FilterParams {
    const __nv_bfloat16* qb;  // query rows, bf16, dp wide
    const float* q32;         // query rows, FP32, stride xs
    const float* qn;          // reference FP32 norms
    const float* qnorm;       // |q| rounded up
    const float* qerr;        // |q - bf16(q)| rounded up
    const uint8_t* qint;      // exact-int rows
    const __nv_bfloat16* xb;
    const float* x32;
    const float* xn;
    const float* xnorm;
    const float* xerr;
    const uint8_t* xint;
    uint64_t n;
    uint32_t xs, d, dp;
    const float* thr_row;     // per query row (top-K bound) or null
    const float* thr_col;     // per base row (rank-k threshold) or null
    int exclude_self;         // skip j == query row (self top-K)
    const uint32_t* rows;     // query rows to process (null: 0 .. nrows-1)
    uint64_t nrows;
    uint64_t split_len;       // base rows per grid.y slice (multiple of 128)
    uint32_t* cnt;            // per query row: hits (atomic; may exceed cap)
    uint32_t cap;
    uint32_t* out_id;         // row * cap + slot
    float* out_key;
    uint32_t* err;
    // leaf mode (init_knn): CTA x = leaf_tiles[x]; rows members[off + 128 rb ..],
    // columns members[off .. off + cnt); the row threshold is its current
    // list's K-th key (+inf while the list holds fewer than list_k); keys are
    // written unchecked, inexact ones flagged by kRecheck in the id
    const LeafTile* leaf_tiles;
    const uint32_t* members;
    const float* list_kd;
    const uint32_t* list_sz;
    uint32_t list_k;
    // bounds over the base rows (columns) of |x| (rounded up), |x - bf16(x)|
    // and the FP32 norm, and whether every base row is exact-integer: they
    // bound eps for a whole row, so most pairs are rejected by one compare
    float bx_norm, bx_err, bx_n;
    int all_exact;
    uint64_t pos_base;  // leaf mode: candidate slot = member position - pos_base (the batch's first)
    // top-K mode: pairs that need the FP32 recheck are written with their
    // approximate key and kRecheck in the id, for recheck_rows_kernel (a
    // 4-thread group per pair instead of one thread here)
    int defer_recheck;
    // the key: 0 = |q|^2 + |x|^2 - 2 <q, x> (l2), 1 = 1 - <q, x> (the ip
    // metric's AKNN distance), 2 = -<q, x> (the ip metric's ground-truth key)
    uint32_t key_mode;
};

constexpr uint32_t kStages = 2;  // base-tile ring; two CTAs fit an SM (shared memory, TMEM)
constexpr uint32_t kFilterThreads = 256;
// Wide form (rows too long to keep the query tile resident, dp > kMaxDp): per
// base tile, the query and base rows pass through a ring of K chunks
// (kWideK elements of 128 rows each, both operands) and the MMAs of the
// chunks accumulate in TMEM.
constexpr uint32_t kWideK = 64;
constexpr uint32_t kWideStages = 4;
constexpr uint32_t kWideMaxDp = 1024;

// The reference's FP32 key |q|^2 + |x|^2 - 2 <q, x> (dataset_gt.cpp:225, 294;
// mode 2, the ip metric: -<q, x>, dataset_gt.cpp:288) with <q, x> in the
// 16-lane AVX-512 order of include/distance.h:89-116, computed by one thread.
__device__ __forceinline__ float ref_key(const float* __restrict__ q, const float* __restrict__ x, uint32_t d,
                                         float qn, float xn, uint32_t mode = 0) {
    const uint32_t d16 = d & ~15u;
    float acc[16];
#pragma unroll
    for (int l = 0; l < 16; l++) acc[l] = 0.f;
    for (uint32_t k0 = 0; k0 < d16; k0 += 16)
#pragma unroll
        for (int l = 0; l < 16; l++) acc[l] = __fmaf_rn(q[k0 + l], x[k0 + l], acc[l]);
    auto fold = [](float (&a)[16]) {
        float t3[8], t6[4];
#pragma unroll
        for (int i = 0; i < 8; i++) t3[i] = __fadd_rn(a[i + 8], a[i]);
#pragma unroll
        for (int i = 0; i < 4; i++) t6[i] = __fadd_rn(t3[i + 4], t3[i]);
        return __fadd_rn(__fadd_rn(t6[0], t6[2]), __fadd_rn(t6[1], t6[3]));
    };
    float ip = fold(acc);
    if (d16 < d) {
        float p[16];
#pragma unroll
        for (int l = 0; l < 16; l++) p[l] = (d16 + l < d) ? __fmul_rn(q[d16 + l], x[d16 + l]) : 0.f;
        ip = __fadd_rn(ip, fold(p));
    }
    if (mode == 2) return -ip;
    return __fsub_rn(__fadd_rn(qn, xn), __fmul_rn(2.0f, ip));
}

template <bool kWide>
__global__ void __launch_bounds__(kFilterThreads, kWide ? 1 : 2) tc_filter_kernel(FilterParams p) {
    extern __shared__ __align__(128) unsigned char sm[];
    // resident form: the query tile, then kStages base tiles; wide form:
    // kWideStages query chunks, then kWideStages base chunks
    const uint32_t tile_bytes = kTile * (kWide ? kWideK : p.dp) * 2;
    unsigned char* sa = sm;
    unsigned char* sb = sm + (size_t)(kWide ? kWideStages : 1) * tile_bytes;
    float* col = reinterpret_cast<float*>(sb + (size_t)(kWide ? kWideStages : kStages) * tile_bytes);  // kStages x 4 x 128
    uint8_t* colint = reinterpret_cast<uint8_t*>(col + kStages * 4 * kTile);    // kStages x 128
    uint64_t* rowid = reinterpret_cast<uint64_t*>(colint + kStages * kTile);    // 128 (aligned: 2*... bytes)
    uint32_t* colid = reinterpret_cast<uint32_t*>(rowid + kTile);                // kStages x 128 (leaf mode)
    __shared__ uint64_t bar[2];
    __shared__ uint64_t cbar[kWideStages];  // wide form: chunk slot free again
    __shared__ uint32_t tslot;
    __shared__ int s_abort;
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t r = (warp & 3u) * 32 + lane;  // this thread's tile row / TMEM lane
    const uint32_t half = warp >> 2;             // column half of each tile

    const bool leaf = p.leaf_tiles != nullptr;
    const LeafTile lt = leaf ? p.leaf_tiles[blockIdx.x] : LeafTile{0, 0, 0};
    const uint32_t* mem = leaf ? p.members + lt.off : nullptr;
    // query rows of this tile
    if (threadIdx.x < kTile) {
        if (leaf) {
            const uint32_t t = lt.rb * kTile + threadIdx.x;
            rowid[threadIdx.x] = t < lt.cnt ? (uint64_t)mem[t] : ~0ull;
        } else {
            const uint64_t t = (uint64_t)blockIdx.x * kTile + threadIdx.x;
            rowid[threadIdx.x] = t < p.nrows ? (p.rows ? p.rows[t] : t) : ~0ull;
        }
    }
    // base columns: positions [js, je) of the base rows, or of the leaf's members
    const uint64_t js = leaf ? 0 : (uint64_t)blockIdx.y * p.split_len;
    const uint64_t je = leaf ? (uint64_t)lt.cnt : min_u64(p.n, js + p.split_len);
    const uint32_t T = js < je ? (uint32_t)((je - js + kTile - 1) / kTile) : 0u;
    if (warp == 0) tc::tmem_alloc(&tslot, 256);
    if (threadIdx.x == 0) {
        tc::mbar_init(&bar[0], 1);
        tc::mbar_init(&bar[1], 1);
        for (uint32_t k = 0; k < kWideStages; k++) tc::mbar_init(&cbar[k], 1);
        tc::fence_mbar_init();
        s_abort = 0;
    }
    __syncthreads();

    // A: the query tile (gathered rows), resident form only
    const uint32_t chunks = kWide ? 0u : p.dp / 8;
    for (uint32_t t = threadIdx.x; t < kTile * chunks; t += blockDim.x) {
        const uint32_t rr = t % kTile, c = t / kTile;
        const uint64_t row = rowid[rr];
        const bool ok = row != ~0ull;
        tc::cp_async16_zfill(sa + (size_t)c * kTile * 16 + rr * 16, p.qb + (ok ? row : 0) * p.dp + 8 * c,
                             ok ? 16u : 0u);
    }
    // base tile t -> stage t % kStages (operand + per-column data)
    auto prefetch = [&](uint32_t t) {
        const uint32_t st = t % kStages;
        const uint64_t j0 = js + (uint64_t)t * kTile;
        unsigned char* dst = sb + (size_t)st * tile_bytes;
        for (uint32_t i = threadIdx.x; i < kTile * chunks; i += blockDim.x) {  // (no operand in the wide form)
            const uint32_t rr = i % kTile, c = i / kTile;
            const uint64_t pos = j0 + rr;
            const bool ok = pos < je;
            const uint64_t row = ok ? (leaf ? (uint64_t)mem[pos] : pos) : 0;
            tc::cp_async16_zfill(dst + (size_t)c * kTile * 16 + rr * 16, p.xb + row * p.dp + 8 * c, ok ? 16u : 0u);
        }
        if (threadIdx.x < kTile) {
            const uint64_t pos = j0 + threadIdx.x;
            const bool ok = pos < je;
            const uint64_t j = ok ? (leaf ? (uint64_t)mem[pos] : pos) : 0;
            if (leaf) colid[st * kTile + threadIdx.x] = (uint32_t)j;
            float* cs = col + (size_t)st * 4 * kTile;
            cs[threadIdx.x] = ok ? p.xn[j] : __int_as_float(0x7f800000);
            cs[kTile + threadIdx.x] = ok ? p.xnorm[j] : 0.f;
            cs[2 * kTile + threadIdx.x] = ok ? p.xerr[j] : 0.f;
            cs[3 * kTile + threadIdx.x] = ok ? (p.thr_col ? p.thr_col[j] : 0.f) : -__int_as_float(0x7f800000);
            colint[st * kTile + threadIdx.x] = ok ? p.xint[j] : 0;
        }
    };
    if (!kWide) {
        if (T > 0) prefetch(0);
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        if (T > 1) prefetch(1);
    }

    // per-row constants of the error bound
    const uint64_t my_row = rowid[r];
    const bool row_ok = my_row != ~0ull;
    const float qn = row_ok ? p.qn[my_row] : 0.f;
    const float qnm = row_ok ? p.qnorm[my_row] : 0.f;
    const float qer = row_ok ? p.qerr[my_row] : 0.f;
    const bool qexact = row_ok && p.qint[my_row] && p.d <= 128;
    float thr_r = (row_ok && p.thr_row) ? p.thr_row[my_row] : 0.f;
    if (leaf && row_ok)
        thr_r = p.list_sz[my_row] >= p.list_k ? p.list_kd[my_row * p.list_k + p.list_k - 1]
                                                : __int_as_float(0x7f800000);
    const float u = 5.9604645e-8f;        // 2^-24
    const float g = 2.0f * p.dp * u;
    // ip keys carry <q, x> once instead of twice: half the product terms; the
    // rounding of 1 - <q, x> (or none for -<q, x>) is below 4 u (1 + |q| |x|)
    const bool l2k = p.key_mode == 0;
    const float kh = l2k ? 1.f : 0.5f;
    const float ca = kh * (2.f * qer + 4.f * g * (qnm + qer) + 4.f * g * qnm + 8.f * u * qnm);
    const float cb = kh * (2.f * qnm + 2.f * qer + 4.f * g * (qnm + qer));
    const float cc = l2k ? 4.f * u : 0.f;
    const float cd = l2k ? 4.f * u * qn : 4.f * u;
    // key~ from the accumulator, in the FP32 steps of the reference's key
    auto approx_key = [&](float xnc, float acc) {
        return l2k ? __fsub_rn(__fadd_rn(qn, xnc), __fmul_rn(2.0f, acc))
                   : (p.key_mode == 1 ? __fsub_rn(1.0f, acc) : -__fadd_rn(acc, 0.0f));  // +0 as the reference's
    };
    const float* qrow = p.q32 + (row_ok ? my_row : 0) * p.xs;
    // eps <= epsmax for every column of this row (eps grows with the column's
    // |x|, |x - bf16(x)| and norm; exact rows against all-exact columns: 0)
    const float epsmax = (qexact && p.all_exact) ? 0.f : fmaf(ca, p.bx_norm, fmaf(cb, p.bx_err, fmaf(cc, p.bx_n, cd)));

    // the filter of tile e's 128 x 128 block (TMEM buffer e & 1, column data
    // in stage e % kStages): each thread its row, each warp half the columns
    auto epilogue = [&](uint32_t e, uint32_t tmem) {
        const uint32_t st = e % kStages;
        const float* cs = col + (size_t)st * 4 * kTile;
        const uint64_t j0 = js + (uint64_t)e * kTile;
        for (uint32_t c0 = half * 64; c0 < half * 64 + 64; c0 += 32) {
            float v[32];
            tc::tmem_ld32(tmem + (((warp & 3u) * 32u) << 16) + (e & 1u) * kTile + c0, v);
            if (!row_ok) continue;
            // columns that survive the row's eps bound, without branches:
            // 4 norms (and thresholds) per shared load
            const bool rowthr = p.thr_row || leaf;
            uint32_t keep = 0;
#pragma unroll
            for (uint32_t k = 0; k < 32; k += 4) {
                const float4 xn4 = *reinterpret_cast<const float4*>(cs + c0 + k);
                const float4 th4 = rowthr ? make_float4(thr_r, thr_r, thr_r, thr_r)
                                          : *reinterpret_cast<const float4*>(cs + 3 * kTile + c0 + k);
                const float xa[4] = {xn4.x, xn4.y, xn4.z, xn4.w}, ta[4] = {th4.x, th4.y, th4.z, th4.w};
#pragma unroll
                for (uint32_t q = 0; q < 4; q++) {
                    const float approx = approx_key(xa[q], v[k + q]);
                    keep |= (approx - epsmax <= ta[q] ? 1u : 0u) << (k + q);
                }
            }
            for (; keep; keep &= keep - 1) {
                const uint32_t k = __ffs(keep) - 1;
                const uint32_t cj = c0 + k;
                const uint64_t j = leaf ? (uint64_t)colid[st * kTile + cj] : j0 + cj;
                const float xn = cs[cj];
                float vk = 0.f;
#pragma unroll
                for (uint32_t q = 0; q < 32; q++)
                    if (q == k) vk = v[q];
                const float approx = approx_key(xn, vk);
                const float thr = rowthr ? thr_r : cs[3 * kTile + cj];
                const bool exact = qexact && colint[st * kTile + cj];
                const float eps =
                    exact ? 0.f : fmaf(ca, cs[kTile + cj], fmaf(cb, cs[2 * kTile + cj], fmaf(cc, xn, cd)));
                if (!(approx - eps <= thr)) continue;
                if (p.exclude_self && j == my_row) continue;
                if (leaf) {
                    // the merge recomputes flagged keys in FP32 and keeps <= its K-th;
                    // slots are indexed by the row's position in the batch of leaves
                    const uint64_t cs0 = lt.off + (uint64_t)lt.rb * kTile + r - p.pos_base;
                    const uint32_t pos = atomicAdd(p.cnt + cs0, 1u);
                    if (pos < p.cap) {
                        p.out_id[cs0 * p.cap + pos] = (uint32_t)j | (exact ? 0u : kRecheck);
                        p.out_key[cs0 * p.cap + pos] = approx;
                    }
                    continue;
                }
                const bool later = p.defer_recheck && !exact;
                const float key = (exact || later) ? approx : ref_key(qrow, p.x32 + j * p.xs, p.d, qn, xn, p.key_mode);
                if (!later && !(key <= thr)) continue;
                const uint32_t pos = atomicAdd(p.cnt + my_row, 1u);
                if (pos < p.cap) {
                    p.out_id[my_row * p.cap + pos] = (uint32_t)j | (later ? kRecheck : 0u);
                    p.out_key[my_row * p.cap + pos] = key;
                }
            }
        }
    };

    if constexpr (!kWide) {
    for (uint32_t t = 0; t <= T; t++) {
        // tile t (prefetched one iteration ahead) and the query tile resident
        // and visible to the tensor cores; TMEM buffer t & 1 free (its last
        // reader, the epilogue of tile t - 2, ran before this barrier)
        asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        if (s_abort) break;  // uniform: read after the barrier
        const uint32_t tmem = tslot;
        if (t < T && threadIdx.x == 0) {
            issue_tile_mma(tmem + (t & 1u) * kTile, sa, sb + (size_t)(t % kStages) * tile_bytes, p.dp);
            tc::mma_commit(&bar[t & 1u]);
        }
        if (t == 0) continue;
        // epilogue of tile e = t - 1 while the tensor cores run tile t
        const uint32_t e = t - 1;
        const bool ok = tc::mbar_wait(&bar[e & 1u], (e >> 1) & 1u, kWaitPolls);
        if (!ok) {
            s_abort = 1;
            atomicExch(p.err, 8u);
        }
        tc::fence_after_sync();
        if (ok) epilogue(e, tmem);
        // stage (t + 1) % 2 held tile e: its MMA finished (waited above); once
        // every warp has left its epilogue the stage is refilled
        if (t + 1 < T) {
            __syncthreads();
            prefetch(t + 1);
        }
        tc::fence_before_sync();
    }
    } else {
        // per base tile t: its nc K chunks through the ring (slot it % kWideStages,
        // free again when the MMAs of chunk it - kWideStages are done), one MMA
        // batch per chunk into TMEM buffer t & 1; then the epilogue of tile t - 1
        // while the tensor cores finish tile t
        const uint32_t nc = p.dp / kWideK;
        uint32_t it = 0;
        bool stop = false;
        for (uint32_t t = 0; t <= T && !stop; t++) {
            const uint32_t tmem = tslot;
            if (t < T) {
                const uint64_t j0 = js + (uint64_t)t * kTile;
                for (uint32_t c = 0; c < nc; c++, it++) {
                    const uint32_t slot = it % kWideStages;
                    if (it >= kWideStages &&
                        !tc::mbar_wait(&cbar[slot], ((it / kWideStages) - 1u) & 1u, kWaitPolls)) {
                        s_abort = 1;
                        atomicExch(p.err, 8u);
                    }
                    unsigned char* da = sa + (size_t)slot * tile_bytes;
                    unsigned char* db = sb + (size_t)slot * tile_bytes;
                    constexpr uint32_t kGroups = kWideK / 8;  // 16-byte groups of a chunk row
                    for (uint32_t i = threadIdx.x; i < kTile * kGroups; i += blockDim.x) {
                        const uint32_t rr = i % kTile, q = i / kTile;
                        const uint64_t row = rowid[rr];
                        const bool oka = row != ~0ull;
                        tc::cp_async16_zfill(da + (size_t)q * kTile * 16 + rr * 16,
                                             p.qb + (oka ? row : 0) * p.dp + c * kWideK + 8 * q, oka ? 16u : 0u);
                        const uint64_t pos = j0 + rr;
                        const bool okb = pos < je;
                        const uint64_t brow = okb ? (leaf ? (uint64_t)mem[pos] : pos) : 0;
                        tc::cp_async16_zfill(db + (size_t)q * kTile * 16 + rr * 16,
                                             p.xb + brow * p.dp + c * kWideK + 8 * q, okb ? 16u : 0u);
                    }
                    if (c == 0) {
                        // column data of tile t: stage t % kStages was last read by
                        // the epilogue of tile t - 2, which every thread has left
                        if (t >= 2) __syncthreads();
                        prefetch(t);
                    }
                    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
                    tc::fence_async_smem();
                    tc::fence_before_sync();
                    __syncthreads();
                    tc::fence_after_sync();
                    if (s_abort) {  // uniform: read after the barrier
                        stop = true;
                        break;
                    }
                    if (threadIdx.x == 0) {
                        issue_tile_mma(tmem + (t & 1u) * kTile, da, db, kWideK, c > 0);
                        tc::mma_commit(&cbar[slot]);
                        if (c + 1 == nc) tc::mma_commit(&bar[t & 1u]);
                    }
                }
                if (stop) break;
            }
            if (t == 0) continue;
            const uint32_t e = t - 1;
            const bool ok = tc::mbar_wait(&bar[e & 1u], (e >> 1) & 1u, kWaitPolls);
            if (!ok) {
                s_abort = 1;
                atomicExch(p.err, 8u);
            }
            tc::fence_after_sync();
            if (ok) epilogue(e, tmem);
            tc::fence_before_sync();
        }
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_free(tslot, 256);
}

// Upper bound of each row's K-th smallest key: the largest reference FP32 key
// to K distinct other rows (the hints, e.g. the AKNN lists).  Warp per row.
__global__ void hint_bound_kernel(const float* __restrict__ x, const float* __restrict__ xn, uint64_t n,
                                  uint32_t xs, uint32_t d, const uint32_t* __restrict__ hints, uint32_t hk,
                                  uint32_t K, float* __restrict__ tau, uint32_t mode) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = w; i < n; i += nw) {
        float mx = -__int_as_float(0x7f800000);
        bool bad = false;
        for (uint32_t k = lane; k < K; k += 32) {
            const uint32_t j = hints[i * hk + k];
            if (j >= n || j == i) {
                bad = true;
                continue;
            }
            mx = fmaxf(mx, ref_key(x + i * xs, x + (uint64_t)j * xs, d, xn[i], xn[j], mode));
        }
        for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
        bad = __any_sync(0xFFFFFFFFu, bad);
        if (lane == 0) tau[i] = bad ? __int_as_float(0x7f800000) : mx;
    }
}

}  // namespace

// Host helpers shared by the tensor-core entry points.
// Maxima of |x|, |x - bf16(x)| and the FP32 norm over n rows, and whether all
// rows are exact-integer (out: 3 float bit patterns as u32, then a flag).
__global__ void row_bounds_kernel(const float* __restrict__ rn, const float* __restrict__ xnorm,
                                  const float* __restrict__ xerr, const uint8_t* __restrict__ xint, uint64_t n,
                                  uint32_t* __restrict__ out) {
    uint32_t a = 0, b = 0, c = 0, e = 1;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        a = max(a, __float_as_uint(fmaxf(xnorm[i], 0.f)));  // non-negative floats order as their bits
        b = max(b, __float_as_uint(fmaxf(xerr[i], 0.f)));
        c = max(c, __float_as_uint(fmaxf(rn[i], 0.f)));
        e &= xint[i] ? 1u : 0u;
    }
    atomicMax(out, a);
    atomicMax(out + 1, b);
    atomicMax(out + 2, c);
    atomicAnd(out + 3, e);
}

int tc_row_bounds(Ctx* c, const float* rn, const float* xnorm, const float* xerr, const uint8_t* xint, uint64_t n,
                  float* bnorm, float* berr, float* bn, int* all_exact) {
    TmpBuf t(c);
    int rc;
    const uint32_t init[4] = {0, 0, 0, 1};
    if ((rc = h2d(c, t, init, 16))) return rc;
    row_bounds_kernel<<<c->sm_count * 4, 256, 0, c->stream>>>(rn, xnorm, xerr, xint, n, t.as<uint32_t>());
    ANQI_CUDA(c, cudaGetLastError());
    uint32_t h[4];
    if ((rc = d2h(c, h, t, 16)) || (rc = sync(c))) return rc;
    std::memcpy(bnorm, &h[0], 4);
    std::memcpy(berr, &h[1], 4);
    std::memcpy(bn, &h[2], 4);
    *all_exact = (int)h[3];
    return ANQI_OK;
}

int tc_prepare_rows(Ctx* c, const float* dx, uint64_t n, uint32_t xs, uint32_t d, uint32_t dp, DevBuf& xb,
                    DevBuf& xnorm, DevBuf& xerr, DevBuf& xint) {
    int rc;
    if ((rc = ensure(c, xb, n * dp * 2)) || (rc = ensure(c, xnorm, n * 4)) || (rc = ensure(c, xerr, n * 4)) ||
        (rc = ensure(c, xint, n)))
        return rc;
    bf16_rows_kernel<<<c->sm_count * 8, 256, 0, c->stream>>>(dx, n, xs, d, dp, xb.as<__nv_bfloat16>(),
                                                             xnorm.as<float>(), xerr.as<float>(), xint.as<uint8_t>());
    ANQI_CUDA(c, cudaGetLastError());
    return ANQI_OK;
}

namespace {

// Rows resident for the tensor path: FP32 copy, reference norms, bf16 copy,
// |x|, |x - bf16(x)|, exact-int flags.
struct TcRows {
    TmpBuf f32, rn, bf, nrm, err, xint;
    explicit TcRows(Ctx* c) : f32(c), rn(c), bf(c), nrm(c), err(c), xint(c) {}
    int load(Ctx* c, const float* host, uint64_t n, uint32_t d, uint32_t xs, uint32_t dp) {
        int rc;
        if ((rc = upload_padded(c, f32, host, n, d, xs)) || (rc = ensure(c, rn, n * 4)) ||
            (rc = compute_norms_device(c, f32.as<float>(), n, d, xs, rn.as<float>())) ||
            (rc = tc_prepare_rows(c, f32.as<float>(), n, xs, d, dp, bf, nrm, err, xint)))
            return rc;
        return ANQI_OK;
    }
};

__global__ void compact_rows_kernel(const uint32_t* __restrict__ cnt, uint32_t cap, const uint64_t* __restrict__ off,
                                    uint64_t nrows, const uint32_t* __restrict__ in_id, const float* __restrict__ in_key,
                                    uint32_t* __restrict__ out_id, float* __restrict__ out_key) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = w; i < nrows; i += nw) {
        const uint32_t m = min(cnt[i], cap);
        for (uint32_t k = lane; k < m; k += 32) {
            out_id[off[i] + k] = in_id[i * cap + k];
            out_key[off[i] + k] = in_key[i * cap + k];
        }
    }
}

// The deferred FP32 recheck of a CSR of (id, key) rows: every entry flagged
// kRecheck gets the reference's FP32 key (ref_key's arithmetic, by a 4-thread
// group in the lane order), the flag cleared.  One warp per row, 8 entries at
// a time.  Keys above the row's bound stay: they sort after the K it keeps.
__global__ void __launch_bounds__(256) recheck_rows_kernel(const uint64_t* __restrict__ off, uint64_t nrows,
                                                           const uint32_t* __restrict__ rows, uint32_t* __restrict__ ids,
                                                           float* __restrict__ keys, const float* __restrict__ x32,
                                                           const float* __restrict__ xn, uint32_t xs, uint32_t d,
                                                           uint32_t mode) {
    const uint32_t lane = threadIdx.x & 31u, gt = lane & 3u, gw = lane >> 2;
    const uint64_t w0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = w0; i < nrows; i += nw) {
        const uint64_t q = rows ? rows[i] : i;
        const uint64_t o0 = off[i], o1 = off[i + 1];
        for (uint64_t e0 = o0; e0 < o1; e0 += 8) {
            const uint64_t e = e0 + gw;
            const bool ok = e < o1;
            const uint32_t raw = ok ? ids[e] : 0u;
            const bool flagged = ok && (raw & kRecheck);
            if (!__any_sync(0xFFFFFFFFu, flagged)) continue;
            const uint32_t j = raw & ~kRecheck;
            const float ip = group_ip(x32 + q * xs, x32 + (uint64_t)(flagged ? j : (uint32_t)q) * xs, d, gt,
                                      0xFFFFFFFFu);
            if (flagged && gt == 0) {
                keys[e] = mode == 2 ? -ip : __fsub_rn(__fadd_rn(xn[q], xn[j]), __fmul_rn(2.0f, ip));
                ids[e] = j;
            }
        }
    }
}

__global__ void take_first_k_kernel(const uint64_t* __restrict__ off, uint64_t nrows, uint32_t K,
                                    const uint32_t* __restrict__ in_id, const float* __restrict__ in_key,
                                    uint32_t* __restrict__ ids, float* __restrict__ keys, uint32_t* __restrict__ err) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nrows * K) return;
    const uint64_t i = t / K, k = t % K;
    if (off[i + 1] - off[i] < K) {
        if (k == 0) atomicExch(err, 5u);
        ids[t] = kEmpty;
        keys[t] = __int_as_float(0x7f800000);
        return;
    }
    ids[t] = in_id[off[i] + k];
    keys[t] = in_key[off[i] + k];
}

size_t filter_smem(uint32_t dp) {
    const size_t operands = dp > kMaxDp ? (size_t)2 * kWideStages * kTile * kWideK * 2 : (size_t)(1 + kStages) * kTile * dp * 2;
    return operands + (size_t)kStages * 4 * kTile * 4 + kStages * kTile + kTile * 8 + (size_t)kStages * kTile * 4;
}

// The padded dimension of the tensor path for d: a multiple of 16 with the
// query tile resident (up to kMaxDp), else a multiple of kWideK for the wide
// form (up to kWideMaxDp); 0 when d is too large.
uint32_t tc_dp(uint32_t d) {
    const uint32_t dp = round_up(d, 16u);
    if (dp <= kMaxDp && filter_smem(dp) <= 227 * 1024) return dp;
    const uint32_t dw = round_up(d, kWideK);
    return dw <= kWideMaxDp ? dw : 0u;
}

// The filter kernel for p.dp (resident or wide form) with its shared memory.
int filter_kernel_for(Ctx* c, uint32_t dp, void (**kern)(FilterParams), size_t* smem) {
    *kern = dp > kMaxDp ? tc_filter_kernel<true> : tc_filter_kernel<false>;
    *smem = filter_smem(dp);
    ANQI_CUDA(c, cudaFuncSetAttribute(*kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*smem));
    return ANQI_OK;
}

int launch_filter(Ctx* c, FilterParams p, uint64_t nrows) {
    if (nrows == 0) return ANQI_OK;
    void (*kern)(FilterParams) = nullptr;
    size_t smem = 0;
    int rc = filter_kernel_for(c, p.dp, &kern, &smem);
    if (rc) return rc;
    const uint64_t gx = (nrows + kTile - 1) / kTile;
    const uint64_t tiles = (p.n + kTile - 1) / kTile;
    uint64_t gy = std::max<uint64_t>(1, ((uint64_t)2 * c->sm_count + gx - 1) / gx);
    gy = std::min<uint64_t>(gy, tiles);
    p.split_len = (tiles + gy - 1) / gy * kTile;
    p.nrows = nrows;
    dim3 grid((unsigned)gx, (unsigned)gy);
    kern<<<grid, kFilterThreads, smem, c->stream>>>(p);
    ANQI_CUDA(c, cudaGetLastError());
    return ANQI_OK;
}

// Runs the filter over all query rows, reruns rows whose hits exceeded the
// capacity with a capacity that fits them, and returns the hits as a CSR
// (off: nq + 1, host and device) sorted by (key, id) within each row.
int filter_to_csr(Ctx* c, FilterParams p, uint64_t nq, uint32_t cap, std::vector<uint64_t>& hoff, TmpBuf& doff,
                  TmpBuf& ids, TmpBuf& keys) {
    TmpBuf cnt(c), oid(c), okey(c);
    int rc;
    if ((rc = ensure(c, cnt, nq * 4)) || (rc = ensure(c, oid, nq * cap * 4)) || (rc = ensure(c, okey, nq * cap * 4)))
        return rc;
    ANQI_CUDA(c, cudaMemsetAsync(cnt.p, 0, nq * 4, c->stream));
    ANQI_CUDA(c, cudaMemsetAsync(c->err.p, 0, 4, c->stream));
    p.cnt = cnt.as<uint32_t>();
    p.cap = cap;
    p.out_id = oid.as<uint32_t>();
    p.out_key = okey.as<float>();
    p.rows = nullptr;
    p.err = c->err.as<uint32_t>();
    if ((rc = launch_filter(c, p, nq))) return rc;
    if ((rc = check_device_error(c, "tensor-core filter"))) return rc;
    std::vector<uint32_t> hc(nq);
    if ((rc = d2h(c, hc.data(), cnt, nq * 4)) || (rc = sync(c))) return rc;
    // rows over capacity: run again with room for all their hits
    std::vector<uint32_t> over;
    uint32_t cap2 = 0;
    for (uint64_t i = 0; i < nq; i++)
        if (hc[i] > cap) {
            over.push_back((uint32_t)i);
            cap2 = std::max(cap2, hc[i]);
        }
    TmpBuf orow(c), ocnt(c), oid2(c), okey2(c);
    if (!over.empty()) {
        const uint64_t no = over.size();
        // rerun outputs are indexed by row id, so they take nq x cap2 entries
        // (ids and keys: 8 bytes per entry) within most of the free device memory
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) free_b = 8ull << 30;
        if (nq * (uint64_t)cap2 * 8 > free_b / 10 * 7)
            return fail(c, ANQI_ERR_CAPACITY, "%zu rows need up to %u candidates each", over.size(), cap2);
        if ((rc = h2d(c, orow, over.data(), no * 4)) || (rc = ensure(c, ocnt, nq * 4)) ||
            (rc = ensure(c, oid2, nq * (uint64_t)cap2 * 4)) || (rc = ensure(c, okey2, nq * (uint64_t)cap2 * 4)))
            return rc;
        ANQI_CUDA(c, cudaMemsetAsync(ocnt.p, 0, nq * 4, c->stream));
        FilterParams q = p;
        q.rows = orow.as<uint32_t>();
        q.cnt = ocnt.as<uint32_t>();
        q.cap = cap2;
        q.out_id = oid2.as<uint32_t>();
        q.out_key = okey2.as<float>();
        if ((rc = launch_filter(c, q, no))) return rc;
        if ((rc = check_device_error(c, "tensor-core filter (capacity rerun)"))) return rc;
    }
    hoff.assign(nq + 1, 0);
    uint64_t maxm = 0;
    for (uint64_t i = 0; i < nq; i++) {
        hoff[i + 1] = hoff[i] + hc[i];
        maxm = std::max<uint64_t>(maxm, hc[i]);
    }
    const uint64_t tot = hoff[nq];
    if ((rc = h2d(c, doff, hoff.data(), (nq + 1) * 8)) || (rc = ensure(c, ids, tot * 4 + 4)) ||
        (rc = ensure(c, keys, tot * 4 + 4)))
        return rc;
    compact_rows_kernel<<<c->sm_count * 8, 256, 0, c->stream>>>(cnt.as<uint32_t>(), cap, doff.as<uint64_t>(), nq,
                                                                oid.as<uint32_t>(), okey.as<float>(),
                                                                ids.as<uint32_t>(), keys.as<float>());
    ANQI_CUDA(c, cudaGetLastError());
    if (!over.empty()) {
        // the rerun rows' full lists replace their truncated ones (row i's
        // hits went to i * cap2; rows not rerun have no hits there)
        compact_rows_kernel<<<c->sm_count * 8, 256, 0, c->stream>>>(ocnt.as<uint32_t>(), cap2, doff.as<uint64_t>(),
                                                                    nq, oid2.as<uint32_t>(), okey2.as<float>(),
                                                                    ids.as<uint32_t>(), keys.as<float>());
        ANQI_CUDA(c, cudaGetLastError());
    }
    return sort_csr_segments(c, doff.as<uint64_t>(), nq, ids.as<uint32_t>(), keys.as<float>(), maxm);
}

}  // namespace

uint32_t tc_padded_dim(uint32_t d) { return tc_dp(d); }

int tc_prep(Ctx* c, const float* d_x, const float* d_norms, uint64_t n, uint32_t xs, uint32_t d, TcPrep& tp) {
    tp.dp = tc_dp(d);
    if (tp.dp == 0) return fail(c, ANQI_ERR_ARGS, "dimension %u too large for the tensor path", d);
    int rc = tc_prepare_rows(c, d_x, n, xs, d, tp.dp, tp.bf, tp.nrm, tp.err, tp.xint);
    if (rc) return rc;
    return tc_row_bounds(c, d_norms, tp.nrm.as<float>(), tp.err.as<float>(), tp.xint.as<uint8_t>(), n, &tp.bnorm,
                         &tp.berr, &tp.bn, &tp.all_exact);
}

void tc_release(Ctx* c, TcPrep& tp) {
    release(c, tp.bf);
    release(c, tp.nrm);
    release(c, tp.err);
    release(c, tp.xint);
}

// ------------------------------------------------------ LocalJoin filter
// Precision form of one LocalJoin round's distances (index.h:1468-1487, in
// the snapshot form of build.cu's join_apply_kernel).  Every pair the round
// pushes is (target, candidate) = (sample a, sample b) of one source u, so
// the Gram matrix of u's samples holds all of them.  A CTA of 4 warps takes 4
// sources: warp w's 32 TMEM lanes (tile rows 32 w .. 32 w + 31) hold the
// samples of source 4 x + w, and one 128 x 128 BF16 tile of the gathered rows
// with themselves on the tensor cores gives each source's pairs in its
// diagonal 32 x 32 block (thread = target row, one tcgen05.ld of the block).
// A pair stays when key~ - eps <= the target's heap top at the start of the
// round (eps as in the filter kernel: bf16 rounding of both rows, FP32
// accumulation, the key's roundings).  A pair above it is rejected by the
// heap push whatever is pushed before it, since a heap's top only falls
// during a round; so pushing only the kept pairs, each with its FP32 key,
// leaves the heaps bit-identical to the FP32 form.
// mask[u * S + a] bit b: candidate b of target a of source u stays.
struct JoinFilterParams {
    const __nv_bfloat16* xb;
    const float* xn;     // reference FP32 norms
    const float* xnorm;  // |x| rounded up
    const float* xerr;   // |x - bf16(x)| rounded up
    uint64_t n;
    uint32_t dp, S, K;
    const uint32_t* samp;
    const uint32_t* scnt;
    const float* hval;   // heaps, top first
    uint32_t* mask;
    uint32_t* err;
};

namespace {

__global__ void __launch_bounds__(128) join_filter_kernel(JoinFilterParams p) {
    extern __shared__ __align__(128) unsigned char sm[];
    __shared__ uint32_t rowid[kTile];
    __shared__ float cn[kTile], cnm[kTile], cer[kTile];
    __shared__ uint64_t bar;
    __shared__ uint32_t tslot;
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u, r = threadIdx.x;
    const uint64_t u = (uint64_t)blockIdx.x * 4 + warp;
    const uint32_t su = u < p.n ? min(p.scnt[u], min(p.S, 32u)) : 0u;
    {
        const bool ok = lane < su;
        const uint32_t id = ok ? p.samp[u * p.S + lane] : kEmpty;
        const bool okid = ok && id < p.n;
        rowid[r] = okid ? id : kEmpty;
        cn[r] = okid ? p.xn[id] : 0.f;
        cnm[r] = okid ? p.xnorm[id] : 0.f;
        cer[r] = okid ? p.xerr[id] : 0.f;
    }
    if (warp == 0) tc::tmem_alloc(&tslot, kTile);
    if (threadIdx.x == 0) {
        tc::mbar_init(&bar, 1);
        tc::fence_mbar_init();
    }
    __syncthreads();
    const uint32_t chunks = p.dp / 8;
    for (uint32_t t = threadIdx.x; t < kTile * chunks; t += blockDim.x) {
        const uint32_t rr = t % kTile, c = t / kTile;
        const uint32_t id = rowid[rr];
        const bool ok = id != kEmpty;
        tc::cp_async16_zfill(sm + (size_t)c * kTile * 16 + rr * 16, p.xb + (uint64_t)(ok ? id : 0u) * p.dp + 8 * c,
                             ok ? 16u : 0u);
    }
    cp_async_wait_all_();
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tslot;
    if (threadIdx.x == 0) {
        issue_tile_mma(tmem, sm, sm, p.dp);  // the tile against itself: A = B
        tc::mma_commit(&bar);
    }
    const bool ok = tc::mbar_wait(&bar, 0, kWaitPolls);
    if (!ok && lane == 0) atomicExch(p.err, 8u);
    tc::fence_after_sync();
    if (ok) {
        float v[32];
        tc::tmem_ld32(tmem + ((warp * 32u) << 16) + warp * 32u, v);
        if (lane < su && rowid[r] != kEmpty) {
            const uint32_t t = rowid[r];
            const float top = p.hval[(uint64_t)t * p.K];
            const float qn = cn[r], qnm = cnm[r], qer = cer[r];
            const float uu = 5.9604645e-8f;  // 2^-24
            const float g = 2.0f * p.dp * uu;
            const float ca = 2.f * qer + 4.f * g * (qnm + qer) + 4.f * g * qnm + 8.f * uu * qnm;
            const float cb = 2.f * qnm + 2.f * qer + 4.f * g * (qnm + qer);
            const float cc = 4.f * uu;
            const float cd = 4.f * uu * qn;
            uint32_t keep = 0;
#pragma unroll
            for (uint32_t b = 0; b < 32; b++) {
                const uint32_t j = warp * 32 + b;
                const float approx = __fsub_rn(__fadd_rn(qn, cn[j]), __fmul_rn(2.0f, v[b]));
                const float eps = fmaf(ca, cnm[j], fmaf(cb, cer[j], fmaf(cc, cn[j], cd)));
                const bool stay = b < su && b != lane && rowid[j] != kEmpty && approx - eps <= top;
                keep |= (stay ? 1u : 0u) << b;
            }
            p.mask[u * p.S + lane] = keep;
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_free(tmem, kTile);
}

}  // namespace

int tc_join_filter(Ctx* c, const TcPrep& tp, const float* d_norms, uint64_t n, const uint32_t* samp,
                   const uint32_t* scnt, uint32_t S, const float* hval, uint32_t K, uint32_t* mask) {
    if (S > 32) return fail(c, ANQI_ERR_ARGS, "tensor-core LocalJoin needs at most 32 samples per row, got %u", S);
    JoinFilterParams p;
    p.xb = tp.bf.as<__nv_bfloat16>();
    p.xn = d_norms;
    p.xnorm = tp.nrm.as<float>();
    p.xerr = tp.err.as<float>();
    p.n = n;
    p.dp = tp.dp;
    p.S = S;
    p.K = K;
    p.samp = samp;
    p.scnt = scnt;
    p.hval = hval;
    p.mask = mask;
    p.err = c->err.as<uint32_t>();
    const size_t smem = (size_t)kTile * tp.dp * 2;
    ANQI_CUDA(c, cudaFuncSetAttribute(join_filter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const uint64_t blocks = (n + 3) / 4;
    if (blocks > 0x7FFFFFFFull) return fail(c, ANQI_ERR_ARGS, "too many rows for the LocalJoin filter");
    join_filter_kernel<<<(unsigned)blocks, 128, smem, c->stream>>>(p);
    ANQI_CUDA(c, cudaGetLastError());
    return ANQI_OK;
}

int tc_leaf_tiles(Ctx* c, const std::vector<LeafRef>& leaves, uint32_t cap, std::vector<LeafTile>& tiles) {
    for (const LeafRef& l : leaves) {
        if (l.cnt > cap + 1) return fail(c, ANQI_ERR_ARGS, "leaf of %u rows exceeds the candidate capacity", l.cnt);
        for (uint32_t rb = 0; rb * kTile < l.cnt; rb++) tiles.push_back({l.off, l.cnt, rb});
    }
    return ANQI_OK;
}

int tc_leaf_filter(Ctx* c, const TcPrep& tp, const float* d_x, const float* d_norms, uint64_t n, uint32_t xs,
                   uint32_t d, const uint32_t* d_members, const LeafTile* d_tiles, size_t ntiles,
                   const float* list_kd, const uint32_t* list_sz, uint32_t K, uint32_t* cnt, uint32_t cap,
                   uint32_t* out_id, float* out_key, uint64_t pos_base, uint32_t key_mode) {
    if (ntiles == 0) return ANQI_OK;
    if (key_mode > 1) return fail(c, ANQI_ERR_ARGS, "leaf tiles take the l2 or ip distance, not mode %u", key_mode);
    FilterParams p{};
    p.qb = p.xb = tp.bf.as<__nv_bfloat16>();
    p.q32 = p.x32 = d_x;
    p.qn = p.xn = d_norms;
    p.qnorm = p.xnorm = tp.nrm.as<float>();
    p.qerr = p.xerr = tp.err.as<float>();
    p.qint = p.xint = tp.xint.as<uint8_t>();
    p.n = n;
    p.xs = xs;
    p.d = d;
    p.dp = tp.dp;
    p.exclude_self = 1;
    p.cnt = cnt;
    p.cap = cap;
    p.out_id = out_id;
    p.out_key = out_key;
    p.err = c->err.as<uint32_t>();
    p.leaf_tiles = d_tiles;
    p.members = d_members;
    p.list_kd = list_kd;
    p.list_sz = list_sz;
    p.list_k = K;
    p.pos_base = pos_base;
    p.key_mode = key_mode;
    p.bx_norm = tp.bnorm;
    p.bx_err = tp.berr;
    p.bx_n = tp.bn;
    p.all_exact = tp.all_exact;
    p.nrows = ntiles * kTile;
    p.split_len = 0;
    void (*kern)(FilterParams) = nullptr;
    size_t smem = 0;
    int rc;
    if ((rc = filter_kernel_for(c, p.dp, &kern, &smem))) return rc;
    kern<<<(unsigned)ntiles, kFilterThreads, smem, c->stream>>>(p);
    ANQI_CUDA(c, cudaGetLastError());
    return ANQI_OK;
}

int tc_leaf_candidates(Ctx* c, const TcPrep& tp, const float* d_x, const float* d_norms, uint64_t n, uint32_t xs,
                       uint32_t d, const uint32_t* d_members, const std::vector<LeafRef>& leaves,
                       const float* list_kd, const uint32_t* list_sz, uint32_t K, uint32_t* cnt, uint32_t cap,
                       uint32_t* out_id, float* out_key, uint64_t pos_base) {
    std::vector<LeafTile> tiles;
    int rc;
    if ((rc = tc_leaf_tiles(c, leaves, cap, tiles))) return rc;
    if (tiles.empty()) return ANQI_OK;
    TmpBuf dt(c);
    if ((rc = h2d(c, dt, tiles.data(), tiles.size() * sizeof(LeafTile)))) return rc;
    if ((rc = tc_leaf_filter(c, tp, d_x, d_norms, n, xs, d, d_members, dt.as<LeafTile>(), tiles.size(), list_kd,
                             list_sz, K, cnt, cap, out_id, out_key, pos_base, 0)))
        return rc;
    return check_device_error(c, "tensor-core init_knn filter");
}

namespace {

FilterParams make_params(const TcRows& Q, const TcRows& X, uint64_t n, uint32_t xs, uint32_t d, uint32_t dp) {
    FilterParams p{};
    p.qb = Q.bf.as<__nv_bfloat16>();
    p.q32 = Q.f32.as<float>();
    p.qn = Q.rn.as<float>();
    p.qnorm = Q.nrm.as<float>();
    p.qerr = Q.err.as<float>();
    p.qint = Q.xint.as<uint8_t>();
    p.xb = X.bf.as<__nv_bfloat16>();
    p.x32 = X.f32.as<float>();
    p.xn = X.rn.as<float>();
    p.xnorm = X.nrm.as<float>();
    p.xerr = X.err.as<float>();
    p.xint = X.xint.as<uint8_t>();
    p.n = n;
    p.xs = xs;
    p.d = d;
    p.dp = dp;
    return p;
}

}  // namespace

}  // namespace anqi

using namespace anqi;

extern "C" {

int anqi_bf16_gram(anqi_ctx* h, const float* a, uint64_t na, const float* b, uint64_t nb, uint32_t d, float* out) {
    if (!h || !a || !b || !out || na == 0 || nb == 0 || d == 0) return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    const uint32_t dp = round_up(d, 16u), xs = round_up(d, 8u);
    if (dp > kMaxDp) return fail(c, ANQI_ERR_ARGS, "dimension %u exceeds the tensor-core tile limit %u", d, kMaxDp);
    TmpBuf da(c), db(c), ab(c), bb(c), an(c), ae(c), ai(c), bn(c), be(c), bi(c), dout(c);
    int rc;
    if ((rc = upload_padded(c, da, a, na, d, xs)) || (rc = upload_padded(c, db, b, nb, d, xs)) ||
        (rc = tc_prepare_rows(c, da.as<float>(), na, xs, d, dp, ab, an, ae, ai)) ||
        (rc = tc_prepare_rows(c, db.as<float>(), nb, xs, d, dp, bb, bn, be, bi)) ||
        (rc = ensure(c, dout, na * nb * 4)))
        return rc;
    ANQI_CUDA(c, cudaMemsetAsync(c->err.p, 0, 4, c->stream));
    const size_t smem = (size_t)2 * kTile * dp * 2;
    ANQI_CUDA(c, cudaFuncSetAttribute(gram_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 grid((unsigned)((na + kTile - 1) / kTile), (unsigned)((nb + kTile - 1) / kTile));
    gram_kernel<<<grid, 128, smem, c->stream>>>(ab.as<__nv_bfloat16>(), na, bb.as<__nv_bfloat16>(), nb, dp,
                                                dout.as<float>(), c->err.as<uint32_t>());
    ANQI_CUDA(c, cudaGetLastError());
    if ((rc = check_device_error(c, "bf16 gram"))) return rc;
    if ((rc = d2h(c, out, dout, na * nb * 4))) return rc;
    return sync(c);
}

int anqi_rknn_ground_truth_tc(anqi_ctx* h, const float* base, uint64_t n, const float* query, uint64_t nq,
                              uint32_t d, const float* rk2, uint32_t* off, uint32_t* ids, float* keys, uint64_t cap,
                              uint64_t* total) {
    return anqi_rknn_ground_truth_tc_metric(h, base, n, query, nq, d, rk2, ANQI_METRIC_L2, off, ids, keys, cap,
                                            total);
}

int anqi_rknn_ground_truth_tc_metric(anqi_ctx* h, const float* base, uint64_t n, const float* query, uint64_t nq,
                                     uint32_t d, const float* rk2, uint32_t metric, uint32_t* off, uint32_t* ids,
                                     float* keys, uint64_t cap, uint64_t* total) {
    if (!h || !base || !query || !rk2 || !off || n == 0 || nq == 0 || d == 0 || metric > ANQI_METRIC_IP)
        return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    const uint32_t dp = tc_dp(d), xs = round_up(d, 8u);
    if (dp == 0) return fail(c, ANQI_ERR_ARGS, "dimension %u too large for the tensor path", d);
    TcRows X(c), Q(c);
    TmpBuf dr(c), doff(c), did(c), dkey(c);
    int rc;
    if ((rc = X.load(c, base, n, d, xs, dp)) || (rc = Q.load(c, query, nq, d, xs, dp)) || (rc = h2d(c, dr, rk2, n * 4)))
        return rc;
    FilterParams p = make_params(Q, X, n, xs, d, dp);
    if ((rc = tc_row_bounds(c, X.rn.as<float>(), X.nrm.as<float>(), X.err.as<float>(), X.xint.as<uint8_t>(), n,
                            &p.bx_norm, &p.bx_err, &p.bx_n, &p.all_exact)))
        return rc;
    p.thr_col = dr.as<float>();
    p.key_mode = metric == ANQI_METRIC_IP ? 2u : 0u;
    std::vector<uint64_t> hoff;
    if ((rc = filter_to_csr(c, p, nq, 256, hoff, doff, did, dkey))) return rc;
    const uint64_t tot = hoff[nq];
    if (total) *total = tot;
    if (tot > cap || tot > 0xFFFFFFFFull)
        return fail(c, ANQI_ERR_CAPACITY, "reverse-kNN output needs %llu entries", (unsigned long long)tot);
    for (uint64_t i = 0; i <= nq; i++) off[i] = (uint32_t)hoff[i];
    if (tot) {
        if (ids && (rc = d2h(c, ids, did, tot * 4))) return rc;
        if (keys && (rc = d2h(c, keys, dkey, tot * 4))) return rc;
    }
    return sync(c);
}

int anqi_exact_topk_tc(anqi_ctx* h, const float* base, uint64_t n, uint32_t d, uint32_t K, const uint32_t* hints,
                       uint32_t hint_k, uint32_t* ids, float* keys) {
    return anqi_exact_topk_tc_metric(h, base, n, d, K, hints, hint_k, ANQI_METRIC_L2, ids, keys);
}

int anqi_exact_topk_tc_metric(anqi_ctx* h, const float* base, uint64_t n, uint32_t d, uint32_t K,
                              const uint32_t* hints, uint32_t hint_k, uint32_t metric, uint32_t* ids, float* keys) {
    if (!h || !base || !ids || !keys || d == 0 || K == 0 || K > 256 || metric > ANQI_METRIC_IP) return ANQI_ERR_ARGS;
    const uint32_t mode = metric == ANQI_METRIC_IP ? 2u : 0u;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    if (K >= n) return fail(c, ANQI_ERR_ARGS, "require K < base vector count");
    const uint32_t dp = tc_dp(d), xs = round_up(d, 8u);
    if (dp == 0) return fail(c, ANQI_ERR_ARGS, "dimension %u too large for the tensor path", d);
    // hints: the caller's (e.g. AKNN lists) or an AKNN build here
    std::vector<uint32_t> own;
    if (!hints) {
        anqi_aknn_params ap{};
        ap.k = std::max<uint32_t>(K, 100);
        ap.leaf = 500;
        ap.trees = 64;
        ap.ef = 600;
        ap.ef_alpha = 8;
        ap.seed = 10;
        ap.nn_sample = 20;
        ap.precision = 1;
        ap.metric = metric;
        if (ap.k >= n) ap.k = (uint32_t)n - 1;
        own.resize(n * ap.k);
        std::vector<float> od(n * ap.k);
        int rc0 = anqi_aknn_build(h, base, n, d, &ap, own.data(), od.data(), nullptr);
        if (rc0) return rc0;
        hints = own.data();
        hint_k = ap.k;
    }
    if (hint_k < K) return fail(c, ANQI_ERR_ARGS, "need at least K = %u hints per row, got %u", K, hint_k);
    TcRows X(c);
    TmpBuf dh(c), tau(c), doff(c), did(c), dkey(c), ko(c), kk(c);
    int rc;
    if ((rc = X.load(c, base, n, d, xs, dp)) || (rc = h2d(c, dh, hints, n * hint_k * 4)) || (rc = ensure(c, tau, n * 4)))
        return rc;
    hint_bound_kernel<<<c->sm_count * 8, 256, 0, c->stream>>>(X.f32.as<float>(), X.rn.as<float>(), n, xs, d,
                                                              dh.as<uint32_t>(), hint_k, K, tau.as<float>(), mode);
    ANQI_CUDA(c, cudaGetLastError());
    FilterParams p = make_params(X, X, n, xs, d, dp);
    if ((rc = tc_row_bounds(c, X.rn.as<float>(), X.nrm.as<float>(), X.err.as<float>(), X.xint.as<uint8_t>(), n,
                            &p.bx_norm, &p.bx_err, &p.bx_n, &p.all_exact)))
        return rc;
    p.thr_row = tau.as<float>();
    p.exclude_self = 1;
    p.defer_recheck = 1;
    p.key_mode = mode;
    std::vector<uint64_t> hoff;
    if ((rc = filter_to_csr(c, p, n, K + 156, hoff, doff, did, dkey))) return rc;
    // the deferred FP32 rechecks, then each row again in (key, id) order
    recheck_rows_kernel<<<c->sm_count * 8, 256, 0, c->stream>>>(doff.as<uint64_t>(), n, nullptr, did.as<uint32_t>(),
                                                                dkey.as<float>(), X.f32.as<float>(), X.rn.as<float>(),
                                                                xs, d, mode);
    ANQI_CUDA(c, cudaGetLastError());
    {
        uint64_t maxm = 0;
        for (uint64_t i = 0; i < n; i++) maxm = std::max<uint64_t>(maxm, hoff[i + 1] - hoff[i]);
        if ((rc = sort_csr_segments(c, doff.as<uint64_t>(), n, did.as<uint32_t>(), dkey.as<float>(), maxm))) return rc;
    }
    if ((rc = ensure(c, ko, n * K * 4)) || (rc = ensure(c, kk, n * K * 4))) return rc;
    ANQI_CUDA(c, cudaMemsetAsync(c->err.p, 0, 4, c->stream));
    const uint64_t tk = n * K;
    take_first_k_kernel<<<(unsigned)((tk + 255) / 256), 256, 0, c->stream>>>(
        doff.as<uint64_t>(), n, K, did.as<uint32_t>(), dkey.as<float>(), ko.as<uint32_t>(), kk.as<float>(),
        c->err.as<uint32_t>());
    ANQI_CUDA(c, cudaGetLastError());
    if ((rc = check_device_error(c, "exact top-K (tensor path)"))) return rc;
    if ((rc = d2h(c, ids, ko, n * K * 4)) || (rc = d2h(c, keys, kk, n * K * 4))) return rc;
    return sync(c);
}

}  // extern "C"
