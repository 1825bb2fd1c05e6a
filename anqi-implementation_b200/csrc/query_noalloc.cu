// Allocation-free reverse-kNN query: the search + postfilter of
// rknn_search_kernel (query.cu) for callers that cannot allocate device
// memory themselves and cannot let a library allocate it either -- for
// example code running inside a host framework whose device memory all
// comes from its own pool (so a cudaMalloc would fragment or overrun it),
// callers that must not synchronize the device the way cudaMalloc/cudaFree
// can, or a process whose memory budget was fixed before it started.  Such a
// caller owns every input and output buffer; this entry point allocates
// nothing and creates no context, stream or event.
//
// Its working memory (per-query visited bitmaps, visit logs, candidate
// lists, a work counter and an error word) lives in one file-scope device
// array of kNoAllocBytes (16 MiB).  Because it is a static __device__
// variable, every GPU on which this library is loaded reserves those 16 MiB
// for as long as the process lives.  The array is shared by all calls on a
// device and keeps whatever the last call left in it: each call zeroes the
// part it uses before its search kernel runs, and two calls whose work
// overlaps on the GPU (different streams, or different host threads) race on
// it -- serialize them.  The first call on each device looks up the array's
// device address (cudaGetSymbolAddress, with that device current); make that
// first call before any stream capture begins.  Every call also ends by
// reading the error word back and synchronizing the caller's stream, so no
// call can be made while that stream is being captured.
//
// Concurrency: each query in flight holds one slot of the array (a visited
// bitmap of n/8 bytes plus 40 KB of log and candidate list).  A block runs up
// to four warps, one query each, and fewer when fewer slots fit, down to one
// slot: n up to about 134 million objects.  At n = 1M a slot is 166 KB, so
// about 100 queries run at once (25 four-warp blocks on 148 SMs): this entry
// point trades throughput for owning no memory.
#include <algorithm>
#include <cfloat>
#include <mutex>

#include "common.cuh"
#include "internal.h"
#include "util.cuh"

namespace anqi {
namespace {

constexpr size_t kNoAllocBytes = (size_t)ANQI_NOALLOC_SCRATCH_BYTES;
constexpr uint32_t kNoAllocWords = (uint32_t)(kNoAllocBytes / 4);
constexpr uint32_t kHeaderWords = 64;  // [0] work counter, [1] error word
constexpr uint32_t kLogCap = 2048;
constexpr uint32_t kCandCap = 8192;
constexpr uint32_t kMaxL = 1024;
constexpr uint32_t kWarps = 4;  // most warps per block (fewer when fewer slots fit)

static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocWords];

struct NoAllocParams {
    anqi_device_index ix;
    const float* queries;
    const float* thr;
    uint32_t nq, L, max_pred;
    uint32_t* pred_count;
    uint32_t* pred_ids;
    uint32_t* n_dist;
    uint32_t* scratch;  // device address of g_noalloc_scratch
    uint32_t words;     // bitmap words per slot
    uint32_t slot_words;
};

__device__ __forceinline__ uint32_t na_expand(const NoAllocParams& p, uint32_t node, uint32_t* bits, uint32_t* vlog,
                                              uint32_t& nlog, uint32_t* ni, uint32_t lane, uint32_t* err) {
    const uint32_t* lk = p.ix.links + (size_t)node * p.ix.degree;
    const uint32_t dg = min(p.ix.deg[node], p.ix.degree);
    uint32_t id0 = kEmpty, id1 = kEmpty;
    bool f0 = false, f1 = false;
    if (lane < dg) {
        id0 = lk[lane];
        if (id0 < p.ix.n) f0 = visit_first(bits, id0);
        else set_error(err, kDevBadId);
    }
    if (lane + 32 < dg) {
        id1 = lk[lane + 32];
        if (id1 < p.ix.n) f1 = visit_first(bits, id1);
        else set_error(err, kDevBadId);
    }
    const unsigned b0 = __ballot_sync(kAll, f0), b1 = __ballot_sync(kAll, f1);
    const uint32_t c0 = __popc(b0), lt = lane_lt_mask();
    const uint32_t p0 = __popc(b0 & lt), p1 = c0 + __popc(b1 & lt);
    if (f0) {
        ni[p0] = id0;
        if (nlog + p0 < kLogCap) vlog[nlog + p0] = id0;
    }
    if (f1) {
        ni[p1] = id1;
        if (nlog + p1 < kLogCap) vlog[nlog + p1] = id1;
    }
    const uint32_t m = c0 + __popc(b1);
    nlog += m;
    __syncwarp();
    return m;
}

__device__ __forceinline__ void na_distances(const NoAllocParams& p, const float* qhat, const uint32_t* ni, float* nd,
                                             uint32_t m, uint32_t gw, uint32_t gt) {
    const uint32_t dim = p.ix.d + 2;
    for (uint32_t r0 = 0; r0 < m; r0 += 8) {
        const uint32_t idx = r0 + gw;
        const bool ok = idx < m;
        const uint32_t id = ni[ok ? idx : r0];
        const float dd = group_l2sqr(p.ix.lifted + (size_t)id * p.ix.lifted_stride, qhat, dim, gt, kAll);
        if (ok && gt == 0) nd[idx] = dd;
    }
    __syncwarp();
}

__device__ __forceinline__ void na_in_range(const NoAllocParams& p, double R2, const float* nd, const uint32_t* ni,
                                            uint32_t m, uint32_t* cl, uint32_t& ncand, bool& overflow, uint32_t lane) {
    const bool in0 = lane < m && (double)nd[lane] <= R2;
    const bool in1 = lane + 32 < m && (double)nd[lane + 32] <= R2;
    const unsigned b0 = __ballot_sync(kAll, in0), b1 = __ballot_sync(kAll, in1);
    const uint32_t c0 = __popc(b0), lt = lane_lt_mask();
    const uint32_t q0 = ncand + __popc(b0 & lt), q1 = ncand + c0 + __popc(b1 & lt);
    if (in0) {
        if (q0 < kCandCap) cl[q0] = ni[lane];
        else overflow = true;
    }
    if (in1) {
        if (q1 < kCandCap) cl[q1] = ni[lane + 32];
        else overflow = true;
    }
    ncand = min(ncand + c0 + __popc(b1), kCandCap);
    overflow = __any_sync(kAll, overflow);
    __syncwarp();
}

extern __shared__ __align__(16) unsigned char na_smem[];

// Same search as rknn_search_kernel: lift, RP-tree entry, greedy beam merged
// batch-wise, bounded flood, then key = IP(o,o) + IP(q,q) - 2 IP(o,q) against
// thr[o]; IP(o,o) is computed per candidate (as the reference does) instead of
// coming from a precomputed norm array.  Results: pred_ids[q * max_pred + i].
__global__ void __launch_bounds__(32 * kWarps) noalloc_search_kernel(NoAllocParams p) {
    const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5, gt = lane & 3u, gw = lane >> 2;
    const uint32_t slot = blockIdx.x * (blockDim.x >> 5) + wib;
    const uint32_t ls = p.ix.lifted_stride, bs = p.ix.base_stride, dim = p.ix.d + 2;
    const size_t per_warp = (size_t)(4 * p.L + 128 + ls + bs) * 4;
    float* qhat = reinterpret_cast<float*>(na_smem + wib * per_warp);
    float* qraw = qhat + ls;
    float* bdA = qraw + bs;
    uint32_t* biA = reinterpret_cast<uint32_t*>(bdA + p.L);
    float* bdB = reinterpret_cast<float*>(biA + p.L);
    uint32_t* biB = reinterpret_cast<uint32_t*>(bdB + p.L);
    float* nd = reinterpret_cast<float*>(biB + p.L);
    uint32_t* ni = reinterpret_cast<uint32_t*>(nd + 64);
    uint32_t* work = p.scratch;
    uint32_t* err = p.scratch + 1;
    uint32_t* mine = p.scratch + kHeaderWords + (size_t)slot * p.slot_words;
    uint32_t* bits = mine;
    uint32_t* vlog = bits + p.words;
    uint32_t* cl = vlog + kLogCap;
    VisitSlot vs{bits, vlog, kLogCap, p.words};
    const double R2_l2 = p.ix.mstar2 + 1.0;
    const bool is_ip = p.ix.metric == ANQI_METRIC_IP;
    for (;;) {
        uint32_t qi = 0;
        if (lane == 0) qi = atomicAdd(work, 1u);
        qi = __shfl_sync(kAll, qi, 0);
        if (qi >= p.nq) break;
        const float* q = p.queries + (size_t)qi * bs;
        for (uint32_t j = lane; j < bs; j += 32) qraw[j] = j < p.ix.d ? q[j] : 0.0f;
        // the ip metric's radius is per query: |s q|^2 (double, index order) + 1 + M*^2
        double R2 = R2_l2;
        if (is_ip) {
            double qn2s = 0.0;
            for (uint32_t j = 0; j < p.ix.d; j++) {
                const double t = __dmul_rn((double)q[j], p.ix.scale);
                qn2s = __dadd_rn(qn2s, __dmul_rn(t, t));
            }
            R2 = __dadd_rn(__dadd_rn(qn2s, 1.0), p.ix.mstar2);
        }
        for (uint32_t j = lane; j < ls; j += 32) {
            float v = 0.0f;
            if (j < p.ix.d) v = __double2float_rn(__dmul_rn((double)q[j], p.ix.scale));
            else if (j == p.ix.d) v = 1.0f;
            qhat[j] = v;
        }
        __syncwarp();
        // descent; a child index outside the tree is reported and the search
        // starts from object 0
        uint32_t v = p.ix.tree_nodes - 1;
        bool bad_tree = false;
        for (uint32_t depth = 0; p.ix.tree_left[v] != kEmpty && depth < 4096; depth++) {
            const float ip = group_ip(p.ix.tree_hyperplane + (size_t)v * ls, qhat, dim, gt, kAll);
            const float margin = __fsub_rn(ip, p.ix.tree_offset[v]);
            const uint32_t c = (margin > kSplitEps) ? p.ix.tree_right[v] : p.ix.tree_left[v];
            if (c >= p.ix.tree_nodes) {
                bad_tree = true;
                break;
            }
            v = c;
        }
        if (bad_tree && lane == 0) set_error(err, kDevBadId);
        uint32_t ep = bad_tree ? 0u : p.ix.tree_leaf_first[v];
        if (ep == kEmpty || ep >= p.ix.n) ep = 0;
        const float dep = group_l2sqr(p.ix.lifted + (size_t)ep * ls, qhat, dim, gt, kAll);
        if (lane == 0) {
            visit_first(bits, ep);
            vlog[0] = ep;
            bdA[0] = dep;
            biA[0] = ep;
        }
        uint32_t nlog = 1, ncand = 0;
        bool overflow = false;
        if ((double)dep <= R2) {
            if (lane == 0) cl[0] = ep;
            ncand = 1;
        }
        __syncwarp();
        float* bd = bdA;
        uint32_t* bi = biA;
        float* od = bdB;
        uint32_t* oi = biB;
        uint32_t size = 1, cur = 0;
        while (cur < size && !overflow) {
            const uint32_t node = bi[cur] & kIdMask;
            __syncwarp();
            if (lane == 0) bi[cur] = node | kExpanded;
            __syncwarp();
            uint32_t nxt = size;
            for (uint32_t s0 = cur + 1; s0 < size; s0 += 32) {
                const uint32_t idx = s0 + lane;
                const unsigned b = __ballot_sync(kAll, idx < size && !(bi[idx] & kExpanded));
                if (b) {
                    nxt = s0 + __ffs(b) - 1;
                    break;
                }
            }
            const uint32_t m = na_expand(p, node, bits, vlog, nlog, ni, lane, err);
            if (m == 0) {
                cur = nxt;
                continue;
            }
            na_distances(p, qhat, ni, nd, m, gw, gt);
            na_in_range(p, R2, nd, ni, m, cl, ncand, overflow, lane);
            warp_sort_batch64(nd, ni, m);
            const uint32_t ns = warp_merge(bd, bi, size, nd, ni, m, p.L, od, oi, false);
            uint32_t cb = 0xFFFFFFFFu;
            if (nxt < size) cb = nxt + lower_rank(nd, ni, m, bd[nxt], bi[nxt]);
            const uint32_t cn = lower_rank(bd, bi, size, nd[0], ni[0]);
            __syncwarp();
            float* td = bd;
            bd = od;
            od = td;
            uint32_t* ti = bi;
            bi = oi;
            oi = ti;
            size = ns;
            cur = min(min(cb, cn), ns);
        }
        uint32_t head = 0;
        while (head < ncand && !overflow) {
            const uint32_t node = cl[head++];
            const uint32_t m = na_expand(p, node, bits, vlog, nlog, ni, lane, err);
            if (m == 0) continue;
            na_distances(p, qhat, ni, nd, m, gw, gt);
            na_in_range(p, R2, nd, ni, m, cl, ncand, overflow, lane);
        }
        if (overflow && lane == 0) set_error(err, kDevCandOverflow);
        const float qn = group_ip(qraw, qraw, p.ix.d, gt, kAll);
        uint32_t npred = 0;
        for (uint32_t r0 = 0; r0 < ncand; r0 += 8) {
            const uint32_t idx = r0 + gw;
            const bool ok = idx < ncand;
            const uint32_t o = cl[ok ? idx : r0];
            const float* orow = p.ix.base + (size_t)o * bs;
            const float dot = group_ip(orow, qraw, p.ix.d, gt, kAll);
            const float on = group_ip(orow, orow, p.ix.d, gt, kAll);
            const float key = is_ip ? -dot : __fsub_rn(__fadd_rn(on, qn), __fmul_rn(2.0f, dot));
            const bool pass = ok && (double)key <= (double)p.thr[o];
            const unsigned b = __ballot_sync(kAll, pass && gt == 0);
            if (pass && gt == 0) {
                const uint32_t w = npred + __popc(b & lane_lt_mask());
                if (w < p.max_pred) p.pred_ids[(size_t)qi * p.max_pred + w] = o;
            }
            npred += __popc(b);
        }
        if (lane == 0) {
            p.pred_count[qi] = npred;
            if (p.n_dist) p.n_dist[qi] = nlog;
            if (npred > p.max_pred) set_error(err, kDevOutOverflow);
        }
        visit_clear(vs, nlog);
    }
}

__global__ void noalloc_clear_kernel(uint32_t* scratch, uint64_t words) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < words; t += (uint64_t)gridDim.x * blockDim.x)
        scratch[t] = 0u;
}

std::mutex g_setup_mu;
uint32_t* g_scratch_addr[256] = {};
int g_sm_count[256] = {};

}  // namespace
}  // namespace anqi

using namespace anqi;

extern "C" int anqi_rknn_query_noalloc(const anqi_device_index* ix, const float* queries, uint32_t nq,
                                       const float* thresholds, uint32_t L, uint32_t max_pred, uint32_t* pred_count,
                                       uint32_t* pred_ids, uint32_t* n_dist, void* stream) {
    if (!ix || !queries || !thresholds || !pred_count || (!pred_ids && max_pred) || nq == 0 || L == 0)
        return ANQI_ERR_ARGS;
    if (L > kMaxL || ix->metric > ANQI_METRIC_IP || ix->n == 0 || ix->n >= 0x7FFFFFFFull || ix->d == 0 || ix->degree == 0 || ix->degree > 64 ||
        ix->tree_nodes == 0 || !ix->base || !ix->lifted || !ix->deg || !ix->links || !ix->tree_left ||
        !ix->tree_right || !ix->tree_offset || !ix->tree_hyperplane || !ix->tree_leaf_first)
        return ANQI_ERR_ARGS;
    // rows are read as float4: strides multiple of 4 floats, rows 16-byte aligned
    if (ix->base_stride < ix->d || ix->lifted_stride < ix->d + 2 || (ix->base_stride & 3u) ||
        (ix->lifted_stride & 3u) || ((uintptr_t)ix->base & 15u) || ((uintptr_t)ix->lifted & 15u) ||
        ((uintptr_t)ix->tree_hyperplane & 15u) || ((uintptr_t)queries & 15u))
        return ANQI_ERR_ARGS;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) return ANQI_ERR_DEVICE;
    uint32_t* scratch = nullptr;
    int sms = 0;
    {
        std::lock_guard<std::mutex> lock(g_setup_mu);
        if (!g_scratch_addr[dev]) {
            uint32_t* ptr = nullptr;
            if (cudaGetSymbolAddress((void**)&ptr, g_noalloc_scratch) != cudaSuccess || !ptr) return ANQI_ERR_DEVICE;
            int s = 0;
            if (cudaDeviceGetAttribute(&s, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return ANQI_ERR_DEVICE;
            g_sm_count[dev] = s;
            g_scratch_addr[dev] = ptr;
        }
        scratch = g_scratch_addr[dev];
        sms = g_sm_count[dev];
    }
    const uint32_t words = (uint32_t)((ix->n + 31) / 32);
    const uint64_t slot_words = (uint64_t)words + kLogCap + kCandCap;
    const uint64_t fit = (kNoAllocWords - kHeaderWords) / slot_words;
    if (fit == 0) return ANQI_ERR_CAPACITY;  // n too large for the fixed scratch (above about 134M objects)
    // one query slot per warp: blocks of up to kWarps warps, fewer when fewer slots fit
    const uint32_t wpb = (uint32_t)std::min<uint64_t>(kWarps, fit);
    const size_t smem = (size_t)(4 * L + 128 + ix->lifted_stride + ix->base_stride) * 4 * wpb;
    if (smem > 227 * 1024) return ANQI_ERR_ARGS;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaFuncSetAttribute(noalloc_search_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        return ANQI_ERR_DEVICE;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, noalloc_search_kernel, 32 * wpb, smem) !=
            cudaSuccess ||
        per_sm < 1)
        return ANQI_ERR_DEVICE;
    uint64_t blocks = std::min<uint64_t>((uint64_t)per_sm * sms, fit / wpb);
    blocks = std::min<uint64_t>(blocks, (nq + wpb - 1) / wpb);
    if (blocks == 0) blocks = 1;
    if (blocks * wpb > fit) return ANQI_ERR_CAPACITY;
    // zero the header and every slot this call uses (the array keeps the last call's contents)
    const uint64_t used = kHeaderWords + blocks * wpb * slot_words;
    noalloc_clear_kernel<<<sms * 4, 256, 0, st>>>(scratch, used);
    NoAllocParams p;
    p.ix = *ix;
    p.queries = queries;
    p.thr = thresholds;
    p.nq = nq;
    p.L = L;
    p.max_pred = max_pred;
    p.pred_count = pred_count;
    p.pred_ids = pred_ids;
    p.n_dist = n_dist;
    p.scratch = scratch;
    p.words = words;
    p.slot_words = (uint32_t)slot_words;
    noalloc_search_kernel<<<(unsigned)blocks, 32 * wpb, smem, st>>>(p);
    if (cudaGetLastError() != cudaSuccess) return ANQI_ERR_DEVICE;
    uint32_t err = 0;
    if (cudaMemcpyAsync(&err, scratch + 1, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return ANQI_ERR_DEVICE;
    switch (err) {
        case kDevOk: return ANQI_OK;
        case kDevCandOverflow:
        case kDevOutOverflow: return ANQI_ERR_CAPACITY;
        case kDevBadId: return ANQI_ERR_FORMAT;
        default: return ANQI_ERR_DEVICE;
    }
}
