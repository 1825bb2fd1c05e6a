// Index construction: AKNN source (init_knn + gather) and the lifted G48 graph
// (warm start, LocalJoin, gather + alpha-RNG prune, commit_edges).
//
// Reference: include/index.h:1071-1295 (build_index), 1300-1367
// (build_approx_knn), 1372-1461 (init_knn), 1468-1487 (nndescent_refine),
// 1491-1525 (gather_candidates), 225-281 + 772-829 (sort_unique_candidates,
// rng_extend, prune_pool_to_ids), 907-930 (commit_edges); include/heap.h
// (push_nolock / check_push / push_reverse).
//
// Per-row work is one warp; distances are exact FP32 in the AVX lane order
// (common.cuh), so a stage given the same inputs produces the reference's
// outputs bit for bit:
//  * gather: the beam (queue cap ef) is merged batch-wise like the query beam;
//    the pool is either kept whole (graph: the prune scans it in (dist, id)
//    order) or reduced to its best K+1 (AKNN: the answer is the K best ids
//    other than the row).
//  * init_knn: every row keeps the K smallest unique leaf-mates by (dist, id)
//    in a sorted list; one launch per tree so each row has one writer.
//  * LocalJoin: "snapshot" form -- every row samples the first <= S live slots
//    of its heap at round start; each target heap then receives, in ascending
//    source order, the other sampled ids of each source that sampled it, and
//    pushes them with the reference's max-heap semantics.  The reference's
//    in-place form mutates heaps while other rows sample them, so it is racy
//    across threads; its outputs are matched statistically.
#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cstdlib>

#include "beam.cuh"
#include "internal.h"
#include "util.cuh"

namespace anqi {

using Clock = std::chrono::steady_clock;
static double ms_since(Clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
}

// ------------------------------------------------------------ gather

// kModeVamana: one pass of the global Vamana refine (index.h:856-875,
// 1262-1285): the beam runs over the current graph from the row's entry,
// without a pool cap, then the row's g0 list joins the pool, which is pruned
// as in select mode.
enum GatherMode : int { kModeAknn = 0, kModeSelect = 1, kModeCommit = 2, kModeVamana = 3 };

// Pair keys: L2 through the norms (index.h:172-176); the ip metric's distance
// 1 - <a, b>, one sequential sum per pair and so one lane per pair
// (distance.h:170-174); the ip ground truth's key -<a, b> in the lane order
// (dataset_gt.cpp:224).
enum KeyMode : uint32_t { kKeyL2 = 0, kKeyIpDist = 1, kKeyNegIp = 2 };

struct GatherParams {
    const float* x;
    const float* norms;
    uint64_t n;
    uint32_t stride, dim;
    // forward lists: n x K ids (kEmpty = empty slot) and their stored distances
    const uint32_t* g_ids;
    const float* g_vals;
    uint32_t K;
    const uint64_t* rev_off;
    const uint32_t* rev_ids;
    uint32_t ef, cap;
    int mode;
    uint32_t out_k;
    uint32_t* out_ids;
    float* out_d;
    uint32_t M;
    float alpha;
    uint32_t* O;       // select output / commit input (n x M)
    uint32_t* O_deg;
    uint32_t* links;   // commit output
    uint32_t* deg;
    // per-slot scratch
    uint32_t* vis_bits;
    uint32_t vis_words;
    uint32_t* vis_log;
    uint32_t log_cap;
    float* pool_d;
    uint32_t* pool_i;
    uint32_t pool_cap;  // power of two
    uint32_t sort_words;  // 2 * kSortSmem in select / commit mode, 0 for AKNN
    uint32_t hash_cap, hash_shift;  // shared-memory visited table per warp (power of two, 0 = none)
    uint32_t* gtab;                 // per-slot L2-resident visited tables (all kEmpty between rows)
    uint32_t gcap, gshift;          // entries per slot (power of two, 0 = none)
    uint32_t ip;    // AKNN mode only: keys are the ip metric's 1 - <a, b>
    uint32_t cols;  // AKNN mode, d = 128: rows stored in chunk column order (group_ip_cols)
    // Vamana mode: the current graph (links n x cur_M, degrees) and each row's entry
    const uint32_t* cur_links;
    const uint32_t* cur_deg;
    uint32_t cur_M;
    const uint32_t* entry;
    uint32_t* next_row;
    const uint32_t* row_order;  // work item -> row (rows of one RP-tree leaf together), or null for identity
    // AKNN mode with rows renumbered for locality (gather_kernel<.., .., true>):
    // row number -> original id.  Lists, rows and norms are given in the new
    // numbering; (dist, id) ties and the output use the original ids.
    const uint32_t* perm;
    // edge-policy prunes: the rows [row_base, row_base + row_count) of the work
    // list (row_count 0: all), each writing its pool (pool_cap entries apart)
    // and its size to the dump buffers instead of pruning it
    uint64_t row_base;
    uint32_t row_count;
    // Vamana mode: also append the row's current links (the batched style,
    // append_current_edges, index.h:759-765)
    uint32_t cur_append;
    float* dump_d;
    uint32_t* dump_i;
    uint32_t* dump_n;
    unsigned long long* pool_total;
    uint32_t* err;
};

constexpr uint32_t kSortSmem = 1024;  // pool entries sorted in shared memory per warp

// Distances of batch ids to row i: (n_i + n_j) - 2 ip(x_i, x_j).
template <bool kIp>
__device__ __forceinline__ void batch_d2(const GatherParams& p, uint64_t i, const uint32_t* ni, float* nd, uint32_t m,
                                         uint32_t gw, uint32_t gt) {
    const float* xi = p.x + i * p.stride;
    if constexpr (kIp) {
        for (uint32_t idx = threadIdx.x & 31u; idx < m; idx += 32)
            nd[idx] = ip_dist_seq(xi, p.x + (uint64_t)ni[idx] * p.stride, p.dim);
        __syncwarp();
        return;
    }
    const float ni_norm = p.norms[i];
    for (uint32_t r0 = 0; r0 < m; r0 += 8) {
        const uint32_t idx = r0 + gw;
        const bool ok = idx < m;
        const uint32_t j = ni[ok ? idx : r0];
        const float ip = p.cols ? group_ip_cols<128>(xi, p.x + (uint64_t)j * p.stride, gt, kAll)
                                : group_ip(xi, p.x + (uint64_t)j * p.stride, p.dim, gt, kAll);
        if (ok && gt == 0) nd[idx] = norm_d2(ni_norm, p.norms[j], ip);
    }
    __syncwarp();
}

// alpha-RNG prune of the sorted candidates (sd/si, m entries, duplicates adjacent)
// of row i into sel (<= M).  index.h:267-281.
__device__ uint32_t rng_prune(const GatherParams& p, uint64_t i, const float* sd, const uint32_t* si, uint32_t m,
                              uint32_t* sel, uint32_t gw, uint32_t gt) {
    uint32_t nsel = 0;
    uint32_t prev = kEmpty;
    for (uint32_t q = 0; q < m && nsel < p.M; q++) {
        const uint32_t cid = si[q];
        const float dc = sd[q];
        if (cid == prev) continue;  // duplicate id (same distance) after sort-unique
        prev = cid;
        if (cid == (uint32_t)i || cid >= p.n) continue;
        bool occluded = false;
        const float nc = p.norms[cid];
        const float* xc = p.x + (uint64_t)cid * p.stride;
        for (uint32_t s0 = 0; s0 < nsel && !occluded; s0 += 8) {
            const uint32_t j = s0 + gw;
            const bool ok = j < nsel;
            const uint32_t sid = sel[ok ? j : s0];
            const float ip = group_ip(p.x + (uint64_t)sid * p.stride, xc, p.dim, gt, kAll);
            const float dsc = norm_d2(p.norms[sid], nc, ip);
            occluded = __any_sync(kAll, ok && __fmul_rn(p.alpha, dsc) < dc);
        }
        if (!occluded) {
            if ((threadIdx.x & 31u) == 0) sel[nsel] = cid;
            __syncwarp();
            nsel++;
        }
    }
    __syncwarp();
    return nsel;
}

// Sort m pool entries by (dist, id): in shared memory when small, else in the
// slot's global scratch (pool_cap is a power of two).
__device__ void sort_pool(float* d, uint32_t* id, uint32_t m, float* sm_d, uint32_t* sm_i, uint32_t cap,
                          const float** out_d, const uint32_t** out_i) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t np2 = next_pow2(max(m, 2u));
    const float inf = __int_as_float(0x7f800000);
    if (np2 <= kSortSmem) {
        for (uint32_t t = lane; t < np2; t += 32) {
            sm_d[t] = t < m ? d[t] : inf;
            sm_i[t] = t < m ? id[t] : kEmpty;
        }
        __syncwarp();
        warp_sort_pairs(sm_d, sm_i, np2);
        *out_d = sm_d;
        *out_i = sm_i;
    } else {
        for (uint32_t t = m + lane; t < np2 && t < cap; t += 32) {
            d[t] = inf;
            id[t] = kEmpty;
        }
        __syncwarp();
        warp_sort_pairs(d, id, min(np2, cap));
        *out_d = d;
        *out_i = id;
    }
}

extern __shared__ __align__(16) unsigned char g_build_smem[];

// Per-warp shared words before the visited table (a multiple of 4 words: its
// 16-byte buckets) and in total (a multiple of 4 words, so every warp's region
// keeps that alignment).
__host__ __device__ __forceinline__ size_t gather_smem_pre(uint32_t ef, uint32_t topk_cap, uint32_t sort_words) {
    return (2 * (size_t)ef + 2 * (size_t)topk_cap + (topk_cap ? 128 : 0) + 128 + 64 + sort_words + 3) & ~(size_t)3;
}

__host__ __device__ __forceinline__ size_t gather_smem_words(uint32_t ef, uint32_t topk_cap, uint32_t sort_words,
                                                             uint32_t hash_cap, uint32_t win_words = 0) {
    return gather_smem_pre(ef, topk_cap, sort_words) + hash_cap + 256 + win_words;
}

// Visits one chunk of up to 64 list ids (slots lane and lane + 32): ids seen
// for the first time go to ni (with their seed distances v0/v1 in nd when
// `vals`) in slot order, and the visits that went to the visited tables are
// logged.  kWin: ids in [wbase, wbase + kWinBits) are visited in the warp's
// window bitmap `win` instead (not logged).  Returns the count of first visits.
template <bool kWin = false>
__device__ __forceinline__ uint32_t gather_visit(const GatherParams& p, Visited& vis, uint32_t& nlog, uint32_t id0,
                                                 uint32_t id1, float v0, float v1, bool vals, uint32_t* ni, float* nd,
                                                 uint32_t lane, uint32_t* win = nullptr, uint32_t wbase = 0) {
    vis_room(vis, nlog, 64, lane, p.err);
    uint32_t r0 = 0, r1 = 0;
    bool f0 = false, f1 = false, g0 = true, g1 = true;  // g: a table visit (logged)
    if constexpr (kWin) {
        if (id0 < p.n) f0 = visit_id(vis, win, wbase, id0, r0, g0, p.err);
        if (id1 < p.n) f1 = visit_id(vis, win, wbase, id1, r1, g1, p.err);
    } else {
        f0 = id0 < p.n && vis_first(vis, id0, r0, p.err);
        f1 = id1 < p.n && vis_first(vis, id1, r1, p.err);
    }
    const unsigned b0 = __ballot_sync(kAll, f0), b1 = __ballot_sync(kAll, f1);
    const uint32_t cnt0 = __popc(b0), lt = lane_lt_mask();
    const uint32_t q0 = __popc(b0 & lt), q1 = cnt0 + __popc(b1 & lt);
    const unsigned h0 = kWin ? __ballot_sync(kAll, f0 && g0) : b0, h1 = kWin ? __ballot_sync(kAll, f1 && g1) : b1;
    const uint32_t l0 = __popc(h0 & lt), l1 = __popc(h0) + __popc(h1 & lt);
    const bool logs = vis.level != 0;
    if (f0) {
        ni[q0] = id0;
        if (vals) nd[q0] = v0;
        if (logs && g0 && nlog + l0 < p.log_cap) vis.vlog[nlog + l0] = r0;
    }
    if (f1) {
        ni[q1] = id1;
        if (vals) nd[q1] = v1;
        if (logs && g1 && nlog + l1 < p.log_cap) vis.vlog[nlog + l1] = r1;
    }
    nlog += __popc(h0) + __popc(h1);
    __syncwarp();
    return cnt0 + __popc(b1);
}

// A row's pool (np entries) to dump entry t of the chunk, for the policy prune.
__device__ __forceinline__ void dump_pool(const GatherParams& p, uint32_t t, const float* pd, const uint32_t* pi,
                                          uint32_t np, uint32_t lane) {
    float* dd = p.dump_d + (uint64_t)t * p.pool_cap;
    uint32_t* di = p.dump_i + (uint64_t)t * p.pool_cap;
    for (uint32_t e = lane; e < np; e += 32) {
        dd[e] = pd[e];
        di[e] = pi[e];
    }
    if (lane == 0) p.dump_n[t] = np;
    __syncwarp();
}

// kIp: the AKNN mode in the ip metric; kVam: the Vamana mode; kRen: the AKNN
// mode over rows renumbered for locality (p.perm), whose visits near the row
// go to a per-warp window bitmap (separate instances, so each mode keeps its
// registers and occupancy)
template <bool kIp, bool kVam = false, bool kRen = false, bool kDump = false, bool kRows = kDump>
__global__ void __launch_bounds__(128, kVam ? 5 : 7) gather_kernel(GatherParams p) {
    const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5, gt = lane & 3u, gw = lane >> 2;
    const uint32_t slot = blockIdx.x * (blockDim.x >> 5) + wib;
    const uint32_t topk_cap = (p.mode == kModeAknn && p.ef < p.out_k + 1) ? p.out_k + 1 : 0;
    const size_t per_warp = gather_smem_words(p.ef, topk_cap, p.sort_words, p.hash_cap, kRen ? kWinWords : 0) * 4;
    unsigned char* my = g_build_smem + wib * per_warp;
    float* bd = reinterpret_cast<float*>(my);  // the beam (queue cap ef), sorted, expanded flag in the id's top bit
    uint32_t* bi = reinterpret_cast<uint32_t*>(bd + p.ef);
    float* td = reinterpret_cast<float*>(bi + p.ef);  // best out_k + 1 of the pool when ef is smaller
    uint32_t* ti = reinterpret_cast<uint32_t*>(td + topk_cap);
    float* nd = reinterpret_cast<float*>(ti + topk_cap);
    uint32_t* ni = reinterpret_cast<uint32_t*>(nd + 64);
    float* nd2 = reinterpret_cast<float*>(ni + 64);  // a copy of the batch for the top-K list
    uint32_t* ni2 = reinterpret_cast<uint32_t*>(nd2 + (topk_cap ? 64 : 0));
    uint32_t* sel = ni2 + (topk_cap ? 64 : 0);
    float* sm_d = reinterpret_cast<float*>(sel + 64);
    uint32_t* sm_i = reinterpret_cast<uint32_t*>(sm_d + p.sort_words / 2);
    uint32_t* tab = reinterpret_cast<uint32_t*>(my) + gather_smem_pre(p.ef, topk_cap, p.sort_words);
    uint32_t* lst = tab + p.hash_cap;  // 256 list ids of the expansion being visited
    uint32_t* win = lst + 256;         // kRen: the window bitmap (kWinWords)
    // (dist, id) order of the beam and the top-K list: through the original ids when renumbered
    const auto ord = [&]() {
        if constexpr (kRen) return PermOrder{p.perm};
        else return IdOrder{};
    }();
    uint32_t* bits = p.vis_bits + (size_t)slot * p.vis_words;
    uint32_t* vlog = p.vis_log + (size_t)slot * p.log_cap;
    float* pd = p.pool_d + (size_t)slot * p.pool_cap;
    uint32_t* pi = p.pool_i + (size_t)slot * p.pool_cap;
    VisitSlot vs{bits, vlog, p.log_cap, p.vis_words};
    for (uint32_t t = lane; t < p.hash_cap; t += 32) tab[t] = kEmpty;
    __syncwarp();

    for (;;) {
        uint32_t row = 0;
        if (lane == 0) row = atomicAdd(p.next_row, 1u);
        row = __shfl_sync(kAll, row, 0);
        if (row >= (kRows ? (uint64_t)p.row_count : p.n)) break;
        const uint64_t i = kRows ? (p.row_order ? p.row_order[p.row_base + row] : p.row_base + row)
                                 : (p.row_order ? p.row_order[row] : row);
        if (i >= p.n) {
            if (lane == 0) set_error(p.err, kDevBadId);
            continue;
        }

        if (p.mode == kModeCommit) {
            // cand = O_i + R_i with fresh distances (index.h:921-929)
            const uint32_t od = p.O_deg[i];
            const uint64_t r0 = p.rev_off[i], r1 = p.rev_off[i + 1];
            const uint32_t tot = od + (uint32_t)(r1 - r0);
            uint32_t np = 0;
            for (uint32_t c0 = 0; c0 < tot; c0 += 64) {
                const uint32_t m = min(64u, tot - c0);
                for (uint32_t t = lane; t < m; t += 32) {
                    const uint32_t pos = c0 + t;
                    ni[t] = pos < od ? p.O[i * p.M + pos] : p.rev_ids[r0 + (pos - od)];
                }
                __syncwarp();
                batch_d2<kIp>(p, i, ni, nd, m, gw, gt);
                for (uint32_t t = lane; t < m; t += 32) {
                    if (np + t < p.pool_cap) {
                        pd[np + t] = nd[t];
                        pi[np + t] = ni[t];
                    }
                }
                np += m;
                __syncwarp();
            }
            if (np > p.pool_cap) {
                if (lane == 0) set_error(p.err, kDevPoolOverflow);
                np = p.pool_cap;
            }
            if constexpr (kDump) {
                dump_pool(p, row, pd, pi, np, lane);
                continue;
            }
            const float* sd;
            const uint32_t* si;
            sort_pool(pd, pi, np, sm_d, sm_i, p.pool_cap, &sd, &si);
            const uint32_t nsel = rng_prune(p, i, sd, si, np, sel, gw, gt);
            for (uint32_t t = lane; t < p.M; t += 32) p.links[i * p.M + t] = t < nsel ? sel[t] : kEmpty;
            if (lane == 0) p.deg[i] = nsel;
            __syncwarp();
            continue;
        }

        // ---- gather_candidates, index.h:1491-1525
        Visited vis{tab,  p.hash_cap, p.hash_shift, p.gtab ? p.gtab + (size_t)slot * p.gcap : nullptr,
                    p.gcap, p.gshift, bits, vlog, p.log_cap, p.hash_cap ? 0u : (p.gcap ? 1u : 2u)};
        uint32_t size = 0, tsize = 0, nlog = 0;
        uint32_t lo = 0;  // beam entries before lo are expanded
        uint64_t npool = 0;
        // kRen: the window of row numbers around the row
        uint32_t wbase = 0;
        if constexpr (kRen) {
            wbase = i > kWinBits / 2 ? (uint32_t)i - kWinBits / 2 : 0u;
            if (p.n <= kWinBits) wbase = 0;
            else if ((uint64_t)wbase > p.n - kWinBits) wbase = (uint32_t)(p.n - kWinBits);
            for (uint32_t t = lane; t < kWinWords; t += 32) win[t] = 0u;
            __syncwarp();
        }
        // one visited batch: pool (select mode), beam and top-K list
        auto take = [&](uint32_t m) {
            if (p.mode == kModeSelect || kVam) {
                for (uint32_t t = lane; t < m; t += 32)
                    if (npool + t < p.pool_cap) {
                        pd[npool + t] = nd[t];
                        pi[npool + t] = ni[t];
                    }
            }
            npool += m;
            if (topk_cap) {
                for (uint32_t t = lane; t < m; t += 32) {
                    nd2[t] = nd[t];
                    ni2[t] = ni[t];
                }
                __syncwarp();
                beam_insert(td, ti, tsize, topk_cap, nd2, ni2, m, lane, ord);
            }
            lo = min(lo, beam_insert(bd, bi, size, p.ef, nd, ni, m, lane, ord));
        };
        // seeds: the row's entry (Vamana), or the row's own list with its stored distances
        if constexpr (kVam) {
            const uint32_t ep = p.entry[i] < p.n ? p.entry[i] : 0u;
            const uint32_t m = gather_visit(p, vis, nlog, lane == 0 ? ep : kEmpty, kEmpty, 0.f, 0.f, false, ni, nd, lane);
            if (m) {
                batch_d2<kIp>(p, i, ni, nd, m, gw, gt);
                take(m);
            }
        }
        for (uint32_t c0 = 0; !kVam && c0 < p.K; c0 += 64) {
            const uint32_t m0 = min(64u, p.K - c0);
            uint32_t id0 = kEmpty, id1 = kEmpty;
            float v0 = 0.f, v1 = 0.f;
            if (lane < m0) {
                id0 = p.g_ids[i * p.K + c0 + lane];
                v0 = p.g_vals[i * p.K + c0 + lane];
            }
            if (lane + 32 < m0) {
                id1 = p.g_ids[i * p.K + c0 + lane + 32];
                v1 = p.g_vals[i * p.K + c0 + lane + 32];
            }
            const uint32_t m = gather_visit<kRen>(p, vis, nlog, id0, id1, v0, v1, true, ni, nd, lane, win, wbase);
            if (m) take(m);
        }
        // expansions: the closest unexpanded entry, its forward then reverse list
        for (;;) {
            uint32_t cur = size;
            for (uint32_t s0 = lo; s0 < size; s0 += 32) {
                const uint32_t idx = s0 + lane;
                const bool un = idx < size && !(bi[idx] & kExpanded);
                const unsigned b = __ballot_sync(kAll, un);
                if (b) {
                    cur = s0 + __ffs(b) - 1;
                    break;
                }
            }
            if (cur >= size) break;
            const uint32_t node = bi[cur] & kIdMask;
            __syncwarp();
            if (lane == 0) bi[cur] = node | kExpanded;
            __syncwarp();
            lo = cur + 1;
            constexpr bool vam = kVam;
            const uint64_t r0 = vam ? 0 : p.rev_off[node], r1 = vam ? 0 : p.rev_off[node + 1];
            const uint32_t tot = vam ? min(p.cur_deg[node], p.cur_M) : p.K + (uint32_t)(r1 - r0);
            // list slots in chunks of 64 (slot c0 + lane, c0 + lane + 32); the
            // ids of four chunks are loaded together, one memory round trip
            for (uint32_t c0 = 0; c0 < tot; c0 += 256) {
                uint32_t ids[8];
#pragma unroll
                for (uint32_t u = 0; u < 8; u++) {
                    const uint32_t pa = c0 + lane + 32 * u;
                    ids[u] = pa >= tot ? kEmpty
                             : vam      ? p.cur_links[(uint64_t)node * p.cur_M + pa]
                             : (pa < p.K ? p.g_ids[(uint64_t)node * p.K + pa] : p.rev_ids[r0 + (pa - p.K)]);
                }
#pragma unroll
                for (uint32_t u = 0; u < 8; u++) lst[32 * u + lane] = ids[u];
                // Visited prefilter: one read-only probe per id, four in flight
                // at a time; an id found there is visited (late in a row almost
                // every id is), the rest take the exact path below.  Within one
                // expansion the order in which chunks are inserted does not
                // change the beam or the pool after sorting.
                uint32_t maybe = 0;  // bit u: ids[u] may be a first visit
#pragma unroll
                for (uint32_t h = 0; h < 8; h += 4) {
                    uint4 q[4];
#pragma unroll
                    for (uint32_t k = 0; k < 4; k++) {
                        const uint32_t id = ids[h + k], w = id - wbase;
                        if (kRen && w < kWinBits) q[k] = make_uint4(win[w >> 5], 0, 0, 0);
                        else q[k] = id < p.n ? probe_visited(vis, id) : make_uint4(0, 0, 0, 0);
                    }
#pragma unroll
                    for (uint32_t k = 0; k < 4; k++) {
                        const uint32_t id = ids[h + k], w = id - wbase;
                        const bool found = (kRen && w < kWinBits) ? ((q[k].x >> (w & 31u)) & 1u) != 0u
                                                                 : probe_found(vis, q[k], id);
                        if (id < p.n && !found) maybe |= 1u << (h + k);
                    }
                }
                __syncwarp();
                for (uint32_t u = 0; u < 8 && c0 + 32 * u < tot; u += 2) {
                    const bool a0 = (maybe >> u) & 1u, a1 = (maybe >> (u + 1)) & 1u;
                    if (!__any_sync(kAll, a0 || a1)) continue;
                    const uint32_t m = gather_visit<kRen>(p, vis, nlog, a0 ? lst[32 * u + lane] : kEmpty,
                                                          a1 ? lst[32 * u + 32 + lane] : kEmpty, 0.f, 0.f, false, ni,
                                                          nd, lane, win, wbase);
                    if (m == 0) continue;
                    batch_d2<kIp>(p, i, ni, nd, m, gw, gt);
                    take(m);
                }
                __syncwarp();
            }
            if (npool >= p.cap) break;
        }
        if constexpr (kVam) {
            // append_aknn_edges (index.h:767-770): the row's g0 list, fresh distances
            for (uint32_t c0 = 0; c0 < p.K; c0 += 32) {
                const uint32_t t = c0 + lane;
                const uint32_t j = t < p.K ? p.g_ids[i * p.K + t] : kEmpty;
                const bool ok = j < p.n && j != (uint32_t)i;
                const unsigned b = __ballot_sync(kAll, ok);
                if (ok) ni[__popc(b & lane_lt_mask())] = j;
                __syncwarp();
                const uint32_t m = __popc(b);
                if (m == 0) continue;
                batch_d2<kIp>(p, i, ni, nd, m, gw, gt);
                if (lane < m && npool + lane < p.pool_cap) {
                    pd[npool + lane] = nd[lane];
                    pi[npool + lane] = ni[lane];
                }
                npool += m;
                __syncwarp();
            }
            // append_current_edges (index.h:759-765): the row's links at the batch's start
            const uint32_t cdeg = p.cur_append ? min(p.cur_deg[i], p.cur_M) : 0u;
            for (uint32_t c0 = 0; c0 < cdeg; c0 += 32) {
                const uint32_t t = c0 + lane;
                const uint32_t j = t < cdeg ? p.cur_links[i * p.cur_M + t] : kEmpty;
                const bool ok = j < p.n && j != (uint32_t)i;
                const unsigned b = __ballot_sync(kAll, ok);
                if (ok) ni[__popc(b & lane_lt_mask())] = j;
                __syncwarp();
                const uint32_t m = __popc(b);
                if (m == 0) continue;
                batch_d2<kIp>(p, i, ni, nd, m, gw, gt);
                if (lane < m && npool + lane < p.pool_cap) {
                    pd[npool + lane] = nd[lane];
                    pi[npool + lane] = ni[lane];
                }
                npool += m;
                __syncwarp();
            }
        }
        if (lane == 0) atomicAdd(p.pool_total, (unsigned long long)npool);

        if (p.mode == kModeAknn) {
            // index.h:1355-1361: sorted pool, first K ids != i
            const float* ld = topk_cap ? td : bd;
            const uint32_t* li = topk_cap ? ti : bi;
            const uint32_t ls = topk_cap ? tsize : size;
            // position of i (if present) among the first out_k + 1 entries
            uint32_t self_pos = kEmpty;
            for (uint32_t t = lane; t < min(ls, p.out_k + 1); t += 32)
                if ((li[t] & kIdMask) == (uint32_t)i) self_pos = t;
            for (int o = 16; o > 0; o >>= 1) self_pos = min(self_pos, __shfl_xor_sync(kAll, self_pos, o));
            // kRen: the row's original id and its neighbours' original ids
            const uint64_t orow = kRen ? (uint64_t)p.perm[i] : i;
            for (uint32_t t = lane; t < p.out_k; t += 32) {
                const uint32_t src = (self_pos != kEmpty && t >= self_pos) ? t + 1 : t;
                const bool ok = src < ls;
                const uint32_t id = ok ? (li[src] & kIdMask) : kEmpty;
                p.out_ids[orow * p.out_k + t] = (kRen && ok) ? p.perm[id] : id;
                p.out_d[orow * p.out_k + t] = ok ? ld[src] : FLT_MAX;
            }
        } else {
            // prune_pool_to_ids: sort_unique_candidates + rng_extend (index.h:772-829)
            uint32_t np = (uint32_t)(npool < (uint64_t)p.pool_cap ? npool : (uint64_t)p.pool_cap);
            if (npool > p.pool_cap && lane == 0) set_error(p.err, kDevPoolOverflow);
            if constexpr (kDump) {
                dump_pool(p, row, pd, pi, np, lane);
            } else {
                const float* sd;
                const uint32_t* si;
                sort_pool(pd, pi, np, sm_d, sm_i, p.pool_cap, &sd, &si);
                const uint32_t nsel = rng_prune(p, i, sd, si, np, sel, gw, gt);
                for (uint32_t t = lane; t < p.M; t += 32) p.O[i * p.M + t] = t < nsel ? sel[t] : kEmpty;
                if (lane == 0) p.O_deg[i] = nsel;
            }
        }
        __syncwarp();
        vis_release(vis, vs, nlog, lane);
        for (uint32_t t = lane; t < p.hash_cap; t += 32) tab[t] = kEmpty;
        __syncwarp();
    }
}

// ------------------------------------------------------- Vamana entries

// The entry of each row for the Vamana refine (rptrees.h:108-123): the RP-tree
// descent of the row's own vector, |margin| <= 1e-6 to the left (the
// reference draws a random side there), and the first point of the leaf
// reached, 0 for an empty leaf or a child outside the tree.  One 4-lane group
// per row, the reference's lane order.
__global__ void __launch_bounds__(128) tree_entry_kernel(const float* __restrict__ x, uint64_t n, uint32_t stride,
                                                         uint32_t dim, const uint32_t* __restrict__ left,
                                                         const uint32_t* __restrict__ right,
                                                         const float* __restrict__ offset,
                                                         const float* __restrict__ hyper,
                                                         const uint32_t* __restrict__ leaf_first, uint32_t n_nodes,
                                                         uint32_t* __restrict__ entry) {
    const uint32_t lane = threadIdx.x & 31u, gt = lane & 3u, gw = lane >> 2;
    const uint64_t w = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t r0 = w * 8; r0 < n; r0 += nw * 8) {
        const uint64_t i = r0 + gw;
        const bool ok = i < n;
        uint32_t v = 0;
        bool done = !ok, bad = false;
        for (uint32_t depth = 0; depth < 4096; depth++) {
            if (!done && left[v] == kEmpty) done = true;
            if (__all_sync(kAll, done)) break;
            const float ip = group_ip(hyper + (size_t)(done ? 0u : v) * stride, x + (ok ? i : 0) * stride, dim, gt,
                                      kAll);
            if (!done) {
                const float m = __fsub_rn(ip, offset[v]);
                const uint32_t nx = m > kSplitEps ? right[v] : left[v];
                if (nx >= n_nodes) {
                    bad = done = true;
                } else {
                    v = nx;
                }
            }
        }
        if (ok && gt == 0) {
            const uint32_t ep = bad ? 0u : leaf_first[v];
            entry[i] = ep < n ? ep : 0u;
        }
    }
}

// ------------------------------------------------------- warm start

// index.h:1210-1217: heap (cap K) of each row from its first `width` warm ids.
// Rows [row0, row0 + rows) of n; cand holds their candidates, row by row.
__global__ void warm_start_kernel(const float* __restrict__ x, const float* __restrict__ norms, uint64_t n,
                                  uint64_t row0, uint64_t rows, uint32_t stride, uint32_t dim,
                                  const uint32_t* __restrict__ cand, uint32_t cstride, uint32_t width, uint32_t K,
                                  uint32_t* __restrict__ hid, float* __restrict__ hval) {
    extern __shared__ __align__(16) unsigned char sm[];
    const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5, gt = lane & 3u, gw = lane >> 2;
    const size_t per_warp = (size_t)(2 * width + 2 * K) * 4;
    uint32_t* cid = reinterpret_cast<uint32_t*>(sm + wib * per_warp);
    float* cd = reinterpret_cast<float*>(cid + width);
    uint32_t* hi = reinterpret_cast<uint32_t*>(cd + width);
    float* hv = reinterpret_cast<float*>(hi + K);
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t loc = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; loc < rows; loc += nw) {
        const uint64_t i = row0 + loc;
        for (uint32_t t = lane; t < width; t += 32) cid[t] = cand[loc * cstride + t];
        for (uint32_t t = lane; t < K; t += 32) {
            hi[t] = kEmpty;
            hv[t] = FLT_MAX;
        }
        __syncwarp();
        const float* xi = x + i * stride;
        for (uint32_t r0 = 0; r0 < width; r0 += 8) {
            const uint32_t idx = r0 + gw;
            const uint32_t j = idx < width ? cid[idx] : kEmpty;
            const bool ok = j < n && j != (uint32_t)i;
            const uint32_t jj = ok ? j : (uint32_t)i;
            const float ip = group_ip(xi, x + (uint64_t)jj * stride, dim, gt, kAll);
            if (idx < width && gt == 0) cd[idx] = norm_d2(norms[i], norms[jj], ip);
        }
        __syncwarp();
        if (lane == 0) {
            for (uint32_t t = 0; t < width; t++) {
                const uint32_t j = cid[t];
                if (j != (uint32_t)i && j < n) heap_push(hi, hv, K, j, cd[t]);
            }
        }
        __syncwarp();
        for (uint32_t t = lane; t < K; t += 32) {
            hid[i * K + t] = hi[t];
            hval[i * K + t] = hv[t];
        }
        __syncwarp();
    }
}

// ------------------------------------------------------------ LocalJoin

__global__ void join_sample_kernel(const uint32_t* __restrict__ hid, uint64_t n, uint32_t K, uint32_t S,
                                   uint32_t* __restrict__ samp, uint32_t* __restrict__ scnt,
                                   uint32_t* __restrict__ incnt) {
    for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < n; u += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t c = 0;
        for (uint32_t s = 0; s < K && c < S; s++) {
            const uint32_t v = hid[u * K + s];
            if (v != kEmpty && v < n) {
                samp[u * S + c++] = v;
                atomicAdd(incnt + v, 1u);
            }
        }
        scnt[u] = c;
    }
}

__global__ void join_fill_kernel(const uint32_t* __restrict__ samp, const uint32_t* __restrict__ scnt, uint64_t n,
                                 uint32_t S, const uint64_t* __restrict__ off, uint32_t* __restrict__ fill,
                                 uint64_t* __restrict__ inc) {
    for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < n; u += (uint64_t)gridDim.x * blockDim.x) {
        for (uint32_t a = 0; a < scnt[u]; a++) {
            const uint32_t x = samp[u * S + a];
            const uint32_t pos = atomicAdd(fill + x, 1u);
            inc[off[x] + pos] = (u << 8) | a;
        }
    }
}

__global__ void __launch_bounds__(128) join_apply_kernel(const float* __restrict__ x, const float* __restrict__ norms,
                                                         uint64_t n, uint32_t stride, uint32_t dim,
                                                         const uint32_t* __restrict__ samp,
                                                         const uint32_t* __restrict__ scnt, uint32_t S,
                                                         const uint64_t* __restrict__ off, uint64_t* __restrict__ inc,
                                                         uint32_t* __restrict__ hid, float* __restrict__ hval, uint32_t K,
                                                         uint64_t* __restrict__ sort_scratch, uint32_t scratch_cap,
                                                         unsigned long long* __restrict__ upd, uint32_t* err,
                                                         const uint32_t* __restrict__ mask) {
    extern __shared__ __align__(16) unsigned char sm[];
    constexpr uint32_t kIncSmem = 512;
    const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5, gt = lane & 3u, gw = lane >> 2;
    const uint32_t slot = blockIdx.x * (blockDim.x >> 5) + wib;
    constexpr uint32_t kBatch = 128;
    const size_t per_warp = (size_t)(2 * kIncSmem + 2 * K + 2 * kBatch) * 4;
    uint64_t* sinc = reinterpret_cast<uint64_t*>(sm + wib * per_warp);
    uint32_t* hi = reinterpret_cast<uint32_t*>(sinc + kIncSmem);
    float* hv = reinterpret_cast<float*>(hi + K);
    uint32_t* bi = reinterpret_cast<uint32_t*>(hv + K);
    float* bd = reinterpret_cast<float*>(bi + kBatch);
    uint64_t* gscr = sort_scratch + (size_t)slot * scratch_cap;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    unsigned long long local_upd = 0;
    for (uint64_t t = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; t < n; t += nw) {
        const uint64_t o0 = off[t];
        const uint32_t s = (uint32_t)(off[t + 1] - o0);
        if (s == 0) continue;
        const uint32_t np2 = next_pow2(max(s, 2u));
        uint64_t* buf;
        if (np2 <= kIncSmem) buf = sinc;
        else if (np2 <= scratch_cap) buf = gscr;
        else {
            if (lane == 0) set_error(err, kDevSortOverflow);
            continue;
        }
        for (uint32_t k = lane; k < np2; k += 32) buf[k] = k < s ? inc[o0 + k] : ~0ull;
        __syncwarp();
        warp_sort_u64(buf, np2);
        for (uint32_t k = lane; k < K; k += 32) {
            hi[k] = hid[t * K + k];
            hv[k] = hval[t * K + k];
        }
        __syncwarp();
        const float* xt = x + t * stride;
        const float nt = norms[t];
        uint32_t m = 0;
        auto flush = [&]() {
            for (uint32_t r0 = 0; r0 < m; r0 += 8) {
                const uint32_t idx = r0 + gw;
                const bool ok = idx < m;
                const uint32_t w = bi[ok ? idx : r0];
                const float ip = group_ip(xt, x + (uint64_t)w * stride, dim, gt, kAll);
                if (ok && gt == 0) bd[idx] = norm_d2(nt, norms[w], ip);
            }
            __syncwarp();
            if (lane == 0)
                for (uint32_t q = 0; q < m; q++) local_upd += heap_push(hi, hv, K, bi[q], bd[q]);
            __syncwarp();
            m = 0;
        };
        for (uint32_t e = 0; e < s; e++) {
            const uint64_t key = buf[e];
            const uint64_t u = key >> 8;
            const uint32_t a = (uint32_t)(key & 0xFF);
            const uint32_t cu = scnt[u];
            // candidates: the other sampled ids of u, in sample order
            if (m + cu > kBatch + 1) flush();
            if (mask) {
                // precision form (S <= 32): only the candidates the tensor-core
                // filter kept; the others would be rejected by the push
                const uint32_t mk = mask[u * S + a] & (cu >= 32 ? kAll : ((1u << cu) - 1u));
                if ((mk >> lane) & 1u) bi[m + __popc(mk & lane_lt_mask())] = samp[u * S + lane];
                __syncwarp();
                m += __popc(mk);
                continue;
            }
            for (uint32_t b = lane; b < cu; b += 32) {
                if (b == a) continue;
                const uint32_t pos = m + (b < a ? b : b - 1);
                bi[pos] = samp[u * S + b];
            }
            __syncwarp();
            m += cu - 1;
        }
        flush();
        for (uint32_t k = lane; k < K; k += 32) {
            hid[t * K + k] = hi[k];
            hval[t * K + k] = hv[k];
        }
        __syncwarp();
    }
    if (lane == 0 && local_upd) atomicAdd(upd, local_upd);
}

// ------------------------------------------------------------ reverse CSR

__global__ void count_targets_kernel(const uint32_t* __restrict__ ids, uint64_t n, uint32_t K, uint32_t* __restrict__ cnt) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < n * K; t += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t v = ids[t];
        if (v < n) atomicAdd(cnt + v, 1u);
    }
}

__global__ void fill_reverse_kernel(const uint32_t* __restrict__ ids, uint64_t n, uint32_t K,
                                    const uint64_t* __restrict__ off, uint32_t* __restrict__ fill,
                                    uint32_t* __restrict__ rev) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < n * K; t += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t v = ids[t];
        if (v < n) rev[off[v] + atomicAdd(fill + v, 1u)] = (uint32_t)(t / K);
    }
}

// ------------------------------------------------------------ locality numbering
// The AKNN gather's visited tests and row reads stay local when rows that
// visit one another carry nearby numbers.  Rows are numbered component by
// component of the list graph (min-label propagation over the lists, both
// directions), in tree 0's leaf order inside a component.  The numbering
// changes no result: the gather breaks (dist, id) ties and writes its output
// through the original ids.

__device__ __forceinline__ uint32_t ld_cg_u32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.global.cg.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// One propagation round, a warp per row: the smallest label of the row and its
// list goes to all of them; *changed is set when any label fell.
__global__ void label_prop_kernel(const uint32_t* __restrict__ ids, uint64_t n, uint32_t K, uint32_t* lab,
                                  uint32_t* changed) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
        uint32_t m = ld_cg_u32(lab + i);
        for (uint32_t j = lane; j < K; j += 32) {
            const uint32_t v = ids[i * K + j];
            if (v < n) m = min(m, ld_cg_u32(lab + v));
        }
        for (int o = 16; o > 0; o >>= 1) m = min(m, __shfl_xor_sync(kAll, m, o));
        bool fell = false;
        if (lane == 0 && atomicMin(lab + i, m) > m) fell = true;
        for (uint32_t j = lane; j < K; j += 32) {
            const uint32_t v = ids[i * K + j];
            if (v < n && ld_cg_u32(lab + v) > m && atomicMin(lab + v, m) > m) fell = true;
        }
        if (__any_sync(kAll, fell) && lane == 0) atomicOr(changed, 1u);
    }
}

// lab[i] = lab[lab[i]]: every label is the number of a row of the same
// component, so one jump follows a chain of propagated labels.
__global__ void label_jump_kernel(uint32_t* lab, uint64_t n) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t l = ld_cg_u32(lab + i);
        const uint32_t l2 = ld_cg_u32(lab + l);
        if (l2 < l) atomicMin(lab + i, l2);
    }
}

__global__ void label_init_kernel(uint32_t* lab, uint64_t n) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        lab[i] = (uint32_t)i;
}

__global__ void inverse_perm_kernel(const uint32_t* __restrict__ perm, uint64_t n, uint32_t* __restrict__ inv) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        inv[perm[i]] = (uint32_t)i;
}

// Lists in the new numbering: row k is original row perm[k], its ids mapped by
// inv (empty slots stay empty), its values as they are.
__global__ void renumber_lists_kernel(const uint32_t* __restrict__ ids, const float* __restrict__ vals,
                                      const uint32_t* __restrict__ perm, const uint32_t* __restrict__ inv, uint64_t n,
                                      uint32_t K, uint32_t* __restrict__ ids2, float* __restrict__ vals2) {
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n * K; t += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t k = t / K;
        const uint64_t src = (uint64_t)perm[k] * K + (t - k * K);
        const uint32_t v = ids[src];
        ids2[t] = v < n ? inv[v] : kEmpty;
        vals2[t] = vals[src];
    }
}

// ------------------------------------------------------------ init_knn

constexpr uint32_t kLeafRows = 16;

// CTA (leaf, row block): K smallest unique leaf-mates by (dist, id) merged into
// each row's sorted list (kd/ki, n x K, size ksz).
__global__ void __launch_bounds__(256) leaf_topk_kernel(const float* __restrict__ x, const float* __restrict__ norms,
                                                        uint64_t n, uint32_t stride, uint32_t dim,
                                                        const uint32_t* __restrict__ ids,
                                                        const LeafRef* __restrict__ leaves, uint32_t K,
                                                        uint32_t tile_rows, float* __restrict__ kd,
                                                        uint32_t* __restrict__ ki, uint32_t* __restrict__ ksz,
                                                        uint32_t mode) {
    extern __shared__ __align__(16) unsigned char sm[];
    const LeafRef lf = leaves[blockIdx.x];
    const uint32_t rb = blockIdx.y * kLeafRows;
    if (rb >= lf.cnt) return;
    const uint32_t rows = min(kLeafRows, lf.cnt - rb);
    const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5, gt = lane & 3u, gw = lane >> 2;
    const uint32_t nwarp = blockDim.x >> 5;
    float* rv = reinterpret_cast<float*>(sm);                        // kLeafRows x stride
    float* tv = rv + (size_t)kLeafRows * stride;                     // tile_rows x stride
    float* ld = tv + (size_t)tile_rows * stride;                     // 2 x kLeafRows x K
    uint32_t* li = reinterpret_cast<uint32_t*>(ld + 2 * kLeafRows * K);
    float* bd = reinterpret_cast<float*>(li + 2 * kLeafRows * K);    // nwarp x 64
    uint32_t* bi = reinterpret_cast<uint32_t*>(bd + nwarp * 64);
    uint32_t* tid = bi + nwarp * 64;                                 // tile ids
    uint32_t* rsz = tid + tile_rows;                                 // row sizes
    uint32_t* rbuf = rsz + kLeafRows;                                // which half holds the list
    const uint32_t* mem = ids + lf.off;
    for (uint32_t t = threadIdx.x; t < rows * stride; t += blockDim.x) {
        const uint32_t r = t / stride, j = t % stride;
        rv[t] = x[(uint64_t)mem[rb + r] * stride + j];
    }
    for (uint32_t t = threadIdx.x; t < rows * K; t += blockDim.x) {
        const uint32_t r = t / K, k = t % K;
        const uint64_t row = mem[rb + r];
        ld[r * K + k] = kd[row * K + k];
        li[r * K + k] = ki[row * K + k];
    }
    for (uint32_t r = threadIdx.x; r < rows; r += blockDim.x) {
        rsz[r] = ksz[mem[rb + r]];
        rbuf[r] = 0;
    }
    __syncthreads();
    float* wd = bd + wib * 64;
    uint32_t* wi = bi + wib * 64;
    for (uint32_t c0 = 0; c0 < lf.cnt; c0 += tile_rows) {
        const uint32_t tr = min(tile_rows, lf.cnt - c0);
        for (uint32_t t = threadIdx.x; t < tr * (stride / 4); t += blockDim.x) {
            const uint32_t r = t / (stride / 4), q = t % (stride / 4);
            reinterpret_cast<float4*>(tv)[t] = reinterpret_cast<const float4*>(x + (uint64_t)mem[c0 + r] * stride)[q];
        }
        for (uint32_t t = threadIdx.x; t < tr; t += blockDim.x) tid[t] = mem[c0 + t];
        __syncthreads();
        for (uint32_t r = wib; r < rows; r += nwarp) {
            const uint32_t rid = mem[rb + r];
            const float nr = norms[rid];
            float* cur_d = ld + (rbuf[r] * kLeafRows + r) * K;
            uint32_t* cur_i = li + (rbuf[r] * kLeafRows + r) * K;
            float* alt_d = ld + ((1 - rbuf[r]) * kLeafRows + r) * K;
            uint32_t* alt_i = li + ((1 - rbuf[r]) * kLeafRows + r) * K;
            uint32_t size = rsz[r];
            for (uint32_t b0 = 0; b0 < tr; b0 += 64) {
                const uint32_t bm = min(64u, tr - b0);
                // distances for the batch
                if (mode == kKeyIpDist) {
                    for (uint32_t idx = lane; idx < bm; idx += 32) {
                        const uint32_t q = b0 + idx;
                        wd[idx] = ip_dist_seq(rv + (size_t)r * stride, tv + (size_t)q * stride, dim);
                        wi[idx] = tid[q];
                    }
                } else {
                    for (uint32_t r0 = 0; r0 < bm; r0 += 8) {
                        const uint32_t idx = r0 + gw;
                        const bool ok = idx < bm;
                        const uint32_t q = b0 + (ok ? idx : r0);
                        const float ip = group_ip(rv + (size_t)r * stride, tv + (size_t)q * stride, dim, gt, kAll);
                        if (ok && gt == 0) {
                            wd[idx] = mode == kKeyNegIp ? -ip : norm_d2(nr, norms[tid[q]], ip);
                            wi[idx] = tid[q];
                        }
                    }
                }
                __syncwarp();
                // filter: not self, better than the current K-th
                uint32_t kept = 0;
                for (uint32_t s0 = 0; s0 < bm; s0 += 32) {
                    const uint32_t s = s0 + lane;
                    bool keep = false;
                    float dv = 0;
                    uint32_t iv = 0;
                    if (s < bm) {
                        dv = wd[s];
                        iv = wi[s];
                        keep = iv != rid && (size < K || nb_less(dv, iv, cur_d[K - 1], cur_i[K - 1]));
                    }
                    const unsigned b = __ballot_sync(kAll, keep);
                    __syncwarp();
                    if (keep) {
                        const uint32_t w = kept + __popc(b & lane_lt_mask());
                        wd[w] = dv;
                        wi[w] = iv;
                    }
                    kept += __popc(b);
                    __syncwarp();
                }
                if (kept == 0) continue;
                warp_sort_batch64(wd, wi, kept);
                size = warp_merge(cur_d, cur_i, size, wd, wi, kept, K, alt_d, alt_i, true);
                float* t1 = cur_d; cur_d = alt_d; alt_d = t1;
                uint32_t* t2 = cur_i; cur_i = alt_i; alt_i = t2;
                if (lane == 0) rbuf[r] ^= 1u;
                __syncwarp();
            }
            if (lane == 0) rsz[r] = size;
            __syncwarp();
        }
        __syncthreads();
    }
    for (uint32_t t = threadIdx.x; t < rows * K; t += blockDim.x) {
        const uint32_t r = t / K, k = t % K;
        const uint64_t row = mem[rb + r];
        const uint32_t h = rbuf[r];
        kd[row * K + k] = ld[(h * kLeafRows + r) * K + k];
        ki[row * K + k] = li[(h * kLeafRows + r) * K + k];
    }
    for (uint32_t r = threadIdx.x; r < rows; r += blockDim.x) ksz[mem[rb + r]] = rsz[r];
}

// Merges one tree's tensor-core init_knn candidates (tc_leaf_candidates) into
// every row's list: flagged keys are recomputed in FP32 in the leaf_topk_kernel
// arithmetic (mode kKeyL2: the AVX lane order; kKeyIpDist: 1 - <a, b> summed
// in sequence), candidates that cannot enter are dropped,
// the rest sorted and merged with duplicates of list entries removed.  The
// list stays the K smallest unique (key, id) of all candidates seen, whatever
// their order.  Resets cnt.  One warp per row.
__global__ void __launch_bounds__(128) leaf_merge_kernel(const float* __restrict__ x, const float* __restrict__ norms,
                                                         uint64_t n, uint32_t stride, uint32_t dim,
                                                         const uint32_t* __restrict__ members, uint64_t pos_base,
                                                         uint64_t nslots, uint32_t* __restrict__ cnt, uint32_t cap,
                                                         const uint32_t* __restrict__ cid,
                                                         const float* __restrict__ ckey, uint32_t K,
                                                         float* __restrict__ kd, uint32_t* __restrict__ ki,
                                                         uint32_t* __restrict__ ksz, uint32_t* __restrict__ err,
                                                         uint32_t mode) {
    const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5, gt = lane & 3u, gw = lane >> 2;
    float* ld = reinterpret_cast<float*>(g_build_smem) + (size_t)wib * (4 * K + 128);
    uint32_t* li = reinterpret_cast<uint32_t*>(ld + 2 * K);
    float* wd = reinterpret_cast<float*>(li + 2 * K);
    uint32_t* wi = reinterpret_cast<uint32_t*>(wd + 64);
    const uint64_t w0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t sl = w0; sl < nslots; sl += nw) {
        uint32_t m = cnt[sl];
        if (m == 0) continue;
        const uint64_t row = members[pos_base + sl];
        if (m > cap) {
            if (lane == 0) set_error(err, kDevPoolOverflow);
            m = cap;
        }
        uint32_t size = ksz[row];
        for (uint32_t t = lane; t < size; t += 32) {
            ld[t] = kd[row * K + t];
            li[t] = ki[row * K + t];
        }
        uint32_t h = 0;  // which half holds the list
        __syncwarp();
        const float nr = norms[row];
        const float* xi = x + row * stride;
        for (uint32_t c0 = 0; c0 < m; c0 += 64) {
            const uint32_t bm = min(64u, m - c0);
            bool flag = false;
            for (uint32_t t = lane; t < bm; t += 32) {
                const uint32_t id = cid[sl * cap + c0 + t];
                wi[t] = id & ~kRecheck;
                wd[t] = ckey[sl * cap + c0 + t];
                flag |= (id & kRecheck) != 0;
            }
            __syncwarp();
            if (__any_sync(kAll, flag) && mode == kKeyIpDist) {
                // the ip distance in the sequential order of leaf_topk_kernel
                for (uint32_t t = lane; t < bm; t += 32)
                    if (cid[sl * cap + c0 + t] & kRecheck) wd[t] = ip_dist_seq(xi, x + (uint64_t)wi[t] * stride, dim);
                __syncwarp();
            } else if (__any_sync(kAll, flag)) {
                for (uint32_t r0 = 0; r0 < bm; r0 += 8) {
                    const uint32_t idx = r0 + gw;
                    const bool ok = idx < bm;
                    const uint32_t j = wi[ok ? idx : r0];
                    const bool re = ok && (cid[sl * cap + c0 + idx] & kRecheck);
                    if (__any_sync(kAll, re)) {
                        const float ip = group_ip(xi, x + (uint64_t)j * stride, dim, gt, kAll);
                        if (re && gt == 0) wd[idx] = norm_d2(nr, norms[j], ip);
                    }
                }
                __syncwarp();
            }
            float* cd = ld + h * K;
            uint32_t* ci = li + h * K;
            uint32_t kept = 0;
            for (uint32_t s0 = 0; s0 < bm; s0 += 32) {
                const uint32_t s1 = s0 + lane;
                bool keep = false;
                float dv = 0;
                uint32_t iv = 0;
                if (s1 < bm) {
                    dv = wd[s1];
                    iv = wi[s1];
                    keep = iv != (uint32_t)row && iv < n && (size < K || nb_less(dv, iv, cd[K - 1], ci[K - 1]));
                }
                const unsigned b = __ballot_sync(kAll, keep);
                __syncwarp();
                if (keep) {
                    const uint32_t w = kept + __popc(b & lane_lt_mask());
                    wd[w] = dv;
                    wi[w] = iv;
                }
                kept += __popc(b);
                __syncwarp();
            }
            if (kept == 0) continue;
            warp_sort_batch64(wd, wi, kept);
            size = warp_merge(cd, ci, size, wd, wi, kept, K, ld + (1 - h) * K, li + (1 - h) * K, true);
            h ^= 1u;
        }
        for (uint32_t t = lane; t < size; t += 32) {
            kd[row * K + t] = ld[h * K + t];
            ki[row * K + t] = li[h * K + t];
        }
        if (lane == 0) {
            ksz[row] = size;
            cnt[sl] = 0;
        }
        __syncwarp();
    }
}

__global__ void init_lists_kernel(float* kd, uint32_t* ki, uint32_t* ksz, uint64_t n, uint32_t K) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < n * K; t += (uint64_t)gridDim.x * blockDim.x) {
        kd[t] = FLT_MAX;
        ki[t] = kEmpty;
        if (t < n) ksz[t] = 0;
    }
}

// index.h:1452-1460: rows with fewer than K entries get random ids (this
// project's counter hash instead of mt19937; the id may be the row itself).
__global__ void random_fill_kernel(const float* __restrict__ x, const float* __restrict__ norms, uint64_t n,
                                   uint32_t stride, uint32_t dim, uint64_t seed, uint32_t K, float* kd, uint32_t* ki,
                                   uint32_t* ksz, uint32_t ip) {
    const uint32_t lane = threadIdx.x & 31u, gt = lane & 3u;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
        uint32_t size = ksz[i];
        if (size >= K) continue;
        const uint32_t miss = K - size;
        float* d = kd + i * K;
        uint32_t* id = ki + i * K;
        for (uint32_t t = 0; t < miss; t++) {
            const uint32_t r = (uint32_t)(hash64(hash64(seed + 0x51ED270Bull) ^ (i << 20) ^ t) % n);
            // every lane forms the same key (the ip metric's is one sequential sum)
            const float v = ip ? ip_dist_seq(x + i * stride, x + (uint64_t)r * stride, dim)
                               : norm_d2(norms[i], norms[r], group_ip(x + i * stride, x + (uint64_t)r * stride, dim,
                                                                     gt, kAll));
            bool dup = false;
            for (uint32_t s = lane; s < size; s += 32) dup |= id[s] == r;
            dup = __any_sync(kAll, dup);
            if (!dup && (size < K || nb_less(v, r, d[K - 1], id[K - 1]))) {
                if (lane == 0) {
                    uint32_t pos = size < K ? size : K - 1;
                    while (pos > 0 && nb_less(v, r, d[pos - 1], id[pos - 1])) {
                        d[pos] = d[pos - 1];
                        id[pos] = id[pos - 1];
                        pos--;
                    }
                    d[pos] = v;
                    id[pos] = r;
                }
                if (size < K) size++;
            }
            __syncwarp();
        }
        if (lane == 0) ksz[i] = size;
    }
}

// sorted ascending list -> descending array, a valid max-heap (parents >= children)
__global__ void list_to_heap_kernel(const float* kd, const uint32_t* ki, const uint32_t* ksz, uint64_t n, uint32_t K,
                                    float* hv, uint32_t* hi) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < n * K; t += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i = t / K;
        const uint32_t k = (uint32_t)(t % K), s = ksz[i];
        // heap slot k holds the (K-1-k)-th smallest; empty slots first (FLT_MAX)
        const uint32_t src = K - 1 - k;
        hv[t] = src < s ? kd[i * K + src] : FLT_MAX;
        hi[t] = src < s ? ki[i * K + src] : kEmpty;
    }
}

// ------------------------------------------------------------ host side

struct Dev {
    Ctx* c;
    explicit Dev(Ctx* ctx) : c(ctx) {}
};

static int upload_rows(Ctx* c, DevBuf& dx, DevBuf& dn, const float* x, uint64_t n, uint32_t dim, uint32_t stride) {
    int rc = upload_padded(c, dx, x, n, dim, stride);
    if (rc) return rc;
    if ((rc = ensure(c, dn, n * 4))) return rc;
    return compute_norms_device(c, dx.as<float>(), n, dim, stride, dn.as<float>());
}

static int build_reverse(Ctx* c, const uint32_t* d_ids, uint64_t n, uint32_t K, DevBuf& off, DevBuf& rev) {
    TmpBuf cnt(c), fill(c);
    int rc;
    if ((rc = ensure(c, cnt, n * 4)) || (rc = ensure(c, fill, n * 4)) || (rc = ensure(c, off, (n + 1) * 8))) return rc;
    ANQI_CUDA(c, cudaMemsetAsync(cnt.p, 0, n * 4, c->stream));
    ANQI_CUDA(c, cudaMemsetAsync(fill.p, 0, n * 4, c->stream));
    const int blocks = c->sm_count * 8;
    count_targets_kernel<<<blocks, 256, 0, c->stream>>>(d_ids, n, K, cnt.as<uint32_t>());
    ANQI_CUDA(c, cudaGetLastError());
    if ((rc = device_scan(c, cnt.as<uint32_t>(), off.as<uint64_t>(), n))) return rc;
    uint64_t total = 0;
    ANQI_CUDA(c, cudaMemcpy(&total, off.as<uint64_t>() + n, 8, cudaMemcpyDeviceToHost));
    if ((rc = ensure(c, rev, total * 4 + 4))) return rc;
    fill_reverse_kernel<<<blocks, 256, 0, c->stream>>>(d_ids, n, K, off.as<uint64_t>(), fill.as<uint32_t>(),
                                                      rev.as<uint32_t>());
    ANQI_CUDA(c, cudaGetLastError());
    return sync(c);
}

// The locality numbering of the gather (label propagation on the device, a
// counting sort by label in tree-0 order on the host): perm (new -> original)
// and inv (original -> new).  order: tree 0's permutation.
static int locality_order(Ctx* c, const uint32_t* d_ids, uint64_t n, uint32_t K, const uint32_t* d_order, DevBuf& perm,
                          DevBuf& inv) {
    TmpBuf lab(c), flag(c);
    int rc;
    if ((rc = ensure(c, lab, n * 4)) || (rc = ensure(c, flag, 4)) || (rc = ensure(c, perm, n * 4)) ||
        (rc = ensure(c, inv, n * 4)))
        return rc;
    const int blocks = c->sm_count * 8;
    label_init_kernel<<<blocks, 256, 0, c->stream>>>(lab.as<uint32_t>(), n);
    ANQI_CUDA(c, cudaGetLastError());
    // rounds until no label falls (bounded; a cut-off round count only
    // weakens the locality, never a result)
    for (int round = 0; round < 64; round++) {
        ANQI_CUDA(c, cudaMemsetAsync(flag.p, 0, 4, c->stream));
        label_prop_kernel<<<blocks, 256, 0, c->stream>>>(d_ids, n, K, lab.as<uint32_t>(), flag.as<uint32_t>());
        label_jump_kernel<<<blocks, 256, 0, c->stream>>>(lab.as<uint32_t>(), n);
        ANQI_CUDA(c, cudaGetLastError());
        uint32_t changed = 0;
        if ((rc = d2h(c, &changed, flag, 4)) || (rc = sync(c))) return rc;
        if (!changed) break;
    }
    std::vector<uint32_t> hl(n), ho(n), start(n + 1, 0), out(n);
    ANQI_CUDA(c, cudaMemcpyAsync(ho.data(), d_order, n * 4, cudaMemcpyDeviceToHost, c->stream));
    if ((rc = d2h(c, hl.data(), lab, n * 4)) || (rc = sync(c))) return rc;
    for (uint64_t i = 0; i < n; i++) {
        if (hl[i] >= n) return fail(c, ANQI_ERR_DEVICE, "locality numbering: label out of range");
        start[hl[i] + 1]++;
    }
    for (uint64_t l = 0; l < n; l++) start[l + 1] += start[l];
    for (uint64_t k = 0; k < n; k++) {
        const uint32_t o = ho[k];
        if (o >= n) return fail(c, ANQI_ERR_DEVICE, "locality numbering: bad tree order");
        out[start[hl[o]]++] = o;
    }
    if ((rc = h2d(c, perm, out.data(), n * 4))) return rc;
    inverse_perm_kernel<<<blocks, 256, 0, c->stream>>>(perm.as<uint32_t>(), n, inv.as<uint32_t>());
    ANQI_CUDA(c, cudaGetLastError());
    return ANQI_OK;
}

static uint64_t max_reverse(Ctx* c, const DevBuf& off, uint64_t n) {
    std::vector<uint64_t> h(n + 1);
    cudaMemcpy(h.data(), off.p, (n + 1) * 8, cudaMemcpyDeviceToHost);
    uint64_t m = 0;
    for (uint64_t i = 0; i < n; i++) m = std::max(m, h[i + 1] - h[i]);
    return m;
}

// Runs gather_kernel over all rows.
static int run_gather(Ctx* c, GatherParams p, uint64_t max_rev, uint64_t* pool_total, double* kernel_ms = nullptr) {
    const int warps_per_block = 4;
    const uint32_t topk_cap = (p.mode == kModeAknn && p.ef < p.out_k + 1) ? p.out_k + 1 : 0;
    p.sort_words = p.mode == kModeAknn ? 0 : 2 * kSortSmem;
    // the log covers a row's first visits up to the pool cap plus one expansion
    // (a row past it clears its whole bitmap instead)
    const uint32_t log_cap = (uint32_t)std::min<uint64_t>(
        p.n, std::max<uint64_t>(8192, std::min<uint64_t>(32768, (uint64_t)p.cap + p.K + max_rev + 64)));
    // visited set: an L2-resident table per slot (bucketed probing: a lookup
    // is one 16-byte L2 load), then the bitmap; measured at 1M x 128 this beats
    // any shared-memory table in front of it, which costs occupancy
    // (ANQI_B200_GATHER_HASH="S,G" sets the shared and L2 table sizes)
    uint32_t hash_cap = 0, gcap = p.mode == kModeCommit ? 0 : 4096;
    if (const char* e = std::getenv("ANQI_B200_GATHER_HASH")) {
        char* end = nullptr;
        hash_cap = (uint32_t)std::strtoul(e, &end, 10);
        gcap = (end && *end == ',') ? (uint32_t)std::strtoul(end + 1, nullptr, 10) : 0;
    }
    if (hash_cap & (hash_cap - 1)) hash_cap = 0;
    if ((gcap & (gcap - 1)) || (uint64_t)gcap / 8 * 5 > log_cap) gcap = 0;  // the log must cover level 1
    p.hash_cap = hash_cap;
    p.hash_shift = hash_cap ? 32u - (uint32_t)__builtin_ctz(hash_cap) : 0u;
    p.gcap = gcap;
    p.gshift = gcap ? 32u - (uint32_t)__builtin_ctz(gcap) : 0u;
    const bool ren = p.mode == kModeAknn && p.perm && !p.ip;
    if (p.perm && !ren) return fail(c, ANQI_ERR_ARGS, "renumbered rows are an AKNN-mode (l2) option");
    const size_t per_warp = gather_smem_words(p.ef, topk_cap, p.sort_words, hash_cap, ren ? kWinWords : 0) * 4;
    const size_t smem = per_warp * warps_per_block;
    if (smem > 227 * 1024) return fail(c, ANQI_ERR_ARGS, "explore range %u too large", p.ef);
    const bool policy = c->edge.active && (p.mode == kModeSelect || p.mode == kModeCommit || p.mode == kModeVamana);
    if (policy && p.ip) return fail(c, ANQI_ERR_ARGS, "edge policies are an l2 graph option");
    // a subset of the work list: rows [row_base, row_base + row_count) of it
    const bool sub = p.row_count != 0;
    if (sub && (p.ip || ren)) return fail(c, ANQI_ERR_ARGS, "row subsets are a select / commit / Vamana option");
    const uint64_t rb0 = sub ? p.row_base : 0, rc0 = sub ? p.row_count : p.n;
    auto* kern = p.mode == kModeVamana ? (policy ? gather_kernel<false, true, false, true>
                                                 : (sub ? gather_kernel<false, true, false, false, true>
                                                        : gather_kernel<false, true>))
                 : p.ip                  ? gather_kernel<true>
                 : ren                   ? gather_kernel<false, false, true>
                 : policy                ? gather_kernel<false, false, false, true>
                 : sub                   ? gather_kernel<false, false, false, false, true>
                                         : gather_kernel<false>;
    ANQI_CUDA(c, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    ANQI_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * warps_per_block, smem));
    if (per_sm < 1) return fail(c, ANQI_ERR_DEVICE, "gather kernel does not fit on an SM");
    uint32_t blocks = std::min<uint64_t>((uint64_t)per_sm * c->sm_count, (rc0 + warps_per_block - 1) / warps_per_block);
    const uint32_t slots = blocks * warps_per_block;
    const uint32_t words = (uint32_t)((p.n + 31) / 32);
    uint64_t need = (uint64_t)p.cap + p.K + max_rev + 64;
    if (p.mode == kModeCommit) need = p.M + max_rev + 64;
    if (p.mode == kModeVamana)  // every visit of an uncapped beam, g0, the current links
        need = (uint64_t)p.ef * 128 + p.K + (p.cur_append ? p.cur_M : 0) + 64;
    const uint32_t pool_cap = p.mode == kModeAknn ? 1u : (uint32_t)std::min<uint64_t>(1ull << 30, 1ull << (64 - __builtin_clzll(need)));
    // per-slot scratch, kept by the context between builds (the first build
    // maps it; later ones reuse it)
    DevBuf& bits = c->g_bits;
    DevBuf& vlog = c->g_vlog;
    DevBuf& pd = c->g_pd;
    DevBuf& pi = c->g_pi;
    DevBuf& gtab = c->g_gtab;
    int rc;
    if ((rc = ensure(c, bits, (size_t)slots * words * 4)) || (rc = ensure(c, vlog, (size_t)slots * log_cap * 4)) ||
        (rc = ensure(c, pd, (size_t)slots * pool_cap * 4)) || (rc = ensure(c, pi, (size_t)slots * pool_cap * 4)) ||
        (gcap && (rc = ensure(c, gtab, (size_t)slots * gcap * 4))))
        return rc;
    ANQI_CUDA(c, cudaMemsetAsync(bits.p, 0, (size_t)slots * words * 4, c->stream));
    if (gcap) ANQI_CUDA(c, cudaMemsetAsync(gtab.p, 0xFF, (size_t)slots * gcap * 4, c->stream));
    p.gtab = gcap ? gtab.as<uint32_t>() : nullptr;
    ANQI_CUDA(c, cudaMemsetAsync(c->counters.p, 0, 64, c->stream));
    p.vis_bits = bits.as<uint32_t>();
    p.vis_words = words;
    p.vis_log = vlog.as<uint32_t>();
    p.log_cap = log_cap;
    p.pool_d = pd.as<float>();
    p.pool_i = pi.as<uint32_t>();
    p.pool_cap = pool_cap;
    p.next_row = c->counters.as<uint32_t>();
    p.pool_total = reinterpret_cast<unsigned long long*>(c->counters.as<uint32_t>() + 2);
    p.err = c->err.as<uint32_t>();
    // the L2 tables persist in L2 for this launch (the query tables' window is
    // set again by the next search)
    if (gcap) {
        set_l2_window(c, gtab.p, (size_t)slots * gcap * 4);
        c->l2_window = false;
    }
    ANQI_CUDA(c, cudaEventRecord(c->ev0, c->stream));
    if (!policy) {
        kern<<<blocks, 32 * warps_per_block, smem, c->stream>>>(p);
        ANQI_CUDA(c, cudaGetLastError());
    } else {
        // pools dumped a chunk of rows at a time (about 1 GB), each chunk
        // pruned under the edge policy into O (select, Vamana) or the links (commit)
        uint64_t chunk = std::max<uint64_t>(1, std::min<uint64_t>(p.n, (1ull << 30) / (pool_cap * 8ull)));
        if (const char* e = std::getenv("ANQI_B200_POLICY_CHUNK_ROWS")) chunk = std::max<uint64_t>(1, std::strtoull(e, nullptr, 10));
        if ((rc = ensure(c, c->pol_dump_d, chunk * pool_cap * 4)) || (rc = ensure(c, c->pol_dump_i, chunk * pool_cap * 4)) ||
            (rc = ensure(c, c->pol_dump_n, chunk * 4)))
            return rc;
        p.dump_d = c->pol_dump_d.as<float>();
        p.dump_i = c->pol_dump_i.as<uint32_t>();
        p.dump_n = c->pol_dump_n.as<uint32_t>();
        uint32_t* out = p.mode == kModeCommit ? p.links : p.O;
        uint32_t* out_deg = p.mode == kModeCommit ? p.deg : p.O_deg;
        for (uint64_t r0 = rb0; r0 < rb0 + rc0; r0 += chunk) {
            p.row_base = r0;
            p.row_count = (uint32_t)std::min<uint64_t>(chunk, rb0 + rc0 - r0);
            ANQI_CUDA(c, cudaMemsetAsync(p.next_row, 0, 4, c->stream));
            kern<<<blocks, 32 * warps_per_block, smem, c->stream>>>(p);
            ANQI_CUDA(c, cudaGetLastError());
            if ((rc = run_policy_prune(c, p.x, p.norms, p.n, p.stride, p.dim, p.M, p.alpha, p.dump_d, p.dump_i,
                                       p.dump_n, pool_cap, p.row_order, r0, p.row_count, out, out_deg)))
                return rc;
        }
    }
    ANQI_CUDA(c, cudaEventRecord(c->ev1, c->stream));
    rc = check_device_error(c, "gather");  // synchronizes
    if (gcap) clear_l2_window(c);
    if (rc) return rc;
    if (kernel_ms) {
        float ms = 0;
        ANQI_CUDA(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
        *kernel_ms += ms;
    }
    if (pool_total) ANQI_CUDA(c, cudaMemcpy(pool_total, p.pool_total, 8, cudaMemcpyDeviceToHost));
    return ANQI_OK;
}

static GatherParams base_params(const DevBuf& dx, const DevBuf& dn, uint64_t n, uint32_t stride, uint32_t dim) {
    GatherParams p{};
    p.x = dx.as<float>();
    p.norms = dn.as<float>();
    p.n = n;
    p.stride = stride;
    p.dim = dim;
    return p;
}

// LocalJoin rounds on device heaps; returns rounds done and update counts.
// precision 1: the round's distances filtered on BF16 tensor-core tiles first
// (tc_join_filter), only the kept pairs recomputed in FP32 and pushed; the
// heaps equal the FP32 form's.  Needs S <= 32; falls back to FP32 otherwise.
static int run_localjoin(Ctx* c, const DevBuf& dx, const DevBuf& dn, uint64_t n, uint32_t stride, uint32_t dim,
                         DevBuf& hid, DevBuf& hval, uint32_t K, uint32_t S, uint32_t max_rounds,
                         std::vector<uint64_t>& updates, uint32_t precision = 0) {
    if (S > 120) S = 120;  // index.h:1470
    TmpBuf samp(c), scnt(c), incnt(c), off(c), fill(c), inc(c), scratch(c), upd(c), mask(c);
    int rc;
    if ((rc = ensure(c, samp, n * S * 4)) || (rc = ensure(c, scnt, n * 4)) || (rc = ensure(c, incnt, n * 4)) ||
        (rc = ensure(c, off, (n + 1) * 8)) || (rc = ensure(c, fill, n * 4)) || (rc = ensure(c, upd, 8)))
        return rc;
    const bool tensor = precision == 1 && S <= 32 && dim <= 256;
    TcPrep tp;
    if (tensor && ((rc = tc_prep(c, dx.as<float>(), dn.as<float>(), n, stride, dim, tp)) ||
                   (rc = ensure(c, mask, n * S * 4)))) {
        tc_release(c, tp);
        return rc;
    }
    struct Release {
        Ctx* c;
        TcPrep& tp;
        ~Release() { tc_release(c, tp); }
    } release_tp{c, tp};
    const int blocks = c->sm_count * 8;
    for (uint32_t it = 0; it < max_rounds; it++) {
        ANQI_CUDA(c, cudaMemsetAsync(incnt.p, 0, n * 4, c->stream));
        ANQI_CUDA(c, cudaMemsetAsync(fill.p, 0, n * 4, c->stream));
        ANQI_CUDA(c, cudaMemsetAsync(upd.p, 0, 8, c->stream));
        join_sample_kernel<<<blocks, 256, 0, c->stream>>>(hid.as<uint32_t>(), n, K, S, samp.as<uint32_t>(),
                                                         scnt.as<uint32_t>(), incnt.as<uint32_t>());
        ANQI_CUDA(c, cudaGetLastError());
        if (tensor && (rc = tc_join_filter(c, tp, dn.as<float>(), n, samp.as<uint32_t>(), scnt.as<uint32_t>(), S,
                                           hval.as<float>(), K, mask.as<uint32_t>())))
            return rc;
        if ((rc = device_scan(c, incnt.as<uint32_t>(), off.as<uint64_t>(), n))) return rc;
        std::vector<uint64_t> hoff(n + 1);
        ANQI_CUDA(c, cudaMemcpy(hoff.data(), off.p, (n + 1) * 8, cudaMemcpyDeviceToHost));
        uint64_t maxin = 0;
        for (uint64_t i = 0; i < n; i++) maxin = std::max(maxin, hoff[i + 1] - hoff[i]);
        if ((rc = ensure(c, inc, hoff[n] * 8 + 8))) return rc;
        join_fill_kernel<<<blocks, 256, 0, c->stream>>>(samp.as<uint32_t>(), scnt.as<uint32_t>(), n, S,
                                                       off.as<uint64_t>(), fill.as<uint32_t>(), inc.as<uint64_t>());
        ANQI_CUDA(c, cudaGetLastError());
        const int wpb = 4;
        const size_t smem = (size_t)(2 * 512 + 2 * K + 2 * 128) * 4 * wpb;
        ANQI_CUDA(c, cudaFuncSetAttribute(join_apply_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int per_sm = 0;
        ANQI_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, join_apply_kernel, 32 * wpb, smem));
        const uint32_t jb = std::max(1, per_sm) * c->sm_count;
        const uint32_t scratch_cap = maxin > 512 ? (uint32_t)(1ull << (64 - __builtin_clzll(maxin - 1))) : 1;
        if ((rc = ensure(c, scratch, (size_t)jb * wpb * scratch_cap * 8))) return rc;
        join_apply_kernel<<<jb, 32 * wpb, smem, c->stream>>>(dx.as<float>(), dn.as<float>(), n, stride, dim,
                                                             samp.as<uint32_t>(), scnt.as<uint32_t>(), S,
                                                             off.as<uint64_t>(), inc.as<uint64_t>(), hid.as<uint32_t>(),
                                                             hval.as<float>(), K, scratch.as<uint64_t>(), scratch_cap,
                                                             upd.as<unsigned long long>(), c->err.as<uint32_t>(),
                                                             tensor ? mask.as<uint32_t>() : nullptr);
        ANQI_CUDA(c, cudaGetLastError());
        if ((rc = check_device_error(c, "localjoin"))) return rc;
        uint64_t u = 0;
        ANQI_CUDA(c, cudaMemcpy(&u, upd.p, 8, cudaMemcpyDeviceToHost));
        updates.push_back(u);
        if (u < n / 200) break;  // index.h:1485
    }
    return ANQI_OK;
}

static int run_warm_start(Ctx* c, const DevBuf& dx, const DevBuf& dn, uint64_t n, uint32_t stride, uint32_t dim,
                          const uint32_t* d_cand, uint32_t cstride, uint32_t width, uint32_t K, DevBuf& hid,
                          DevBuf& hval, uint64_t row0 = 0, uint64_t rows = ~0ull) {
    int rc;
    if (rows == ~0ull) rows = n;
    if ((rc = ensure(c, hid, n * K * 4)) || (rc = ensure(c, hval, n * K * 4))) return rc;
    const int wpb = 4;
    const size_t smem = (size_t)(2 * width + 2 * K) * 4 * wpb;
    ANQI_CUDA(c, cudaFuncSetAttribute(warm_start_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    warm_start_kernel<<<c->sm_count * 8, 32 * wpb, smem, c->stream>>>(dx.as<float>(), dn.as<float>(), n, row0, rows,
                                                                      stride, dim, d_cand, cstride, width, K,
                                                                      hid.as<uint32_t>(), hval.as<float>());
    ANQI_CUDA(c, cudaGetLastError());
    return sync(c);
}

static int run_commit(Ctx* c, const DevBuf& dx, const DevBuf& dn, uint64_t n, uint32_t stride, uint32_t dim,
                      DevBuf& O, DevBuf& Odeg, uint32_t M, float alpha, DevBuf& links_buf, DevBuf& deg_buf,
                      const uint32_t* row_order, double* kernel_ms);

static int run_select_commit(Ctx* c, const DevBuf& dx, const DevBuf& dn, uint64_t n, uint32_t stride, uint32_t dim,
                             const DevBuf& hid, const DevBuf& hval, uint32_t K, uint32_t M, uint32_t ef, uint32_t cap,
                             float alpha, DevBuf& O, DevBuf& Odeg, DevBuf* links, DevBuf* deg, uint64_t* pool_total,
                             const uint32_t* row_order = nullptr, double* kernel_ms = nullptr) {
    TmpBuf roff(c), rev(c);
    int rc = build_reverse(c, hid.as<uint32_t>(), n, K, roff, rev);
    if (rc) return rc;
    const uint64_t mr = max_reverse(c, roff, n);
    if ((rc = ensure(c, O, n * M * 4)) || (rc = ensure(c, Odeg, n * 4))) return rc;
    GatherParams p = base_params(dx, dn, n, stride, dim);
    p.g_ids = hid.as<uint32_t>();
    p.g_vals = hval.as<float>();
    p.K = K;
    p.rev_off = roff.as<uint64_t>();
    p.rev_ids = rev.as<uint32_t>();
    p.ef = ef;
    p.cap = cap;
    p.mode = kModeSelect;
    p.M = M;
    p.alpha = alpha;
    p.O = O.as<uint32_t>();
    p.O_deg = Odeg.as<uint32_t>();
    p.row_order = row_order;
    if ((rc = run_gather(c, p, mr, pool_total, kernel_ms))) return rc;
    if (!links) return ANQI_OK;
    return run_commit(c, dx, dn, n, stride, dim, O, Odeg, M, alpha, *links, *deg, row_order, kernel_ms);
}

// commit_edges (index.h:907-930): reverse lists of O, then per row O_i + R_i
// pruned to the final adjacency.
static int run_commit(Ctx* c, const DevBuf& dx, const DevBuf& dn, uint64_t n, uint32_t stride, uint32_t dim,
                      DevBuf& O, DevBuf& Odeg, uint32_t M, float alpha, DevBuf& links_buf, DevBuf& deg_buf,
                      const uint32_t* row_order, double* kernel_ms) {
    int rc;
    DevBuf* links = &links_buf;
    DevBuf* deg = &deg_buf;
    TmpBuf roff2(c), rev2(c);
    if ((rc = build_reverse(c, O.as<uint32_t>(), n, M, roff2, rev2))) return rc;
    const uint64_t mr2 = max_reverse(c, roff2, n);
    if ((rc = ensure(c, *links, n * M * 4)) || (rc = ensure(c, *deg, n * 4))) return rc;
    GatherParams q = base_params(dx, dn, n, stride, dim);
    q.mode = kModeCommit;
    q.K = 1;
    q.ef = 4;
    q.M = M;
    q.alpha = alpha;
    q.O = O.as<uint32_t>();
    q.O_deg = Odeg.as<uint32_t>();
    q.rev_off = roff2.as<uint64_t>();
    q.rev_ids = rev2.as<uint32_t>();
    q.links = links->as<uint32_t>();
    q.deg = deg->as<uint32_t>();
    q.row_order = row_order;
    return run_gather(c, q, mr2, nullptr, kernel_ms);
}

// One pass of the global Vamana refine over the current graph (dl, dd: n x M,
// degrees), rows' entries given: the Vamana-mode gather (beam of width Lb
// over the graph + the row's g0 list, pruned) -> O, then commit_edges -> dl, dd.
static int run_vamana_pass(Ctx* c, const DevBuf& dx, const DevBuf& dn, uint64_t n, uint32_t stride, uint32_t dim,
                           const DevBuf& hid, uint32_t K, const uint32_t* d_entry, uint32_t Lb, uint32_t M,
                           float alpha, DevBuf& dl, DevBuf& dd, DevBuf& O, DevBuf& Odeg, const uint32_t* row_order,
                           uint64_t* pool_total, double* kernel_ms, bool commit = true) {
    int rc;
    if ((rc = ensure(c, O, n * M * 4)) || (rc = ensure(c, Odeg, n * 4))) return rc;
    GatherParams p = base_params(dx, dn, n, stride, dim);
    p.g_ids = hid.as<uint32_t>();
    p.K = K;
    p.ef = Lb;
    p.cap = 0xFFFFFFFFu;
    p.mode = kModeVamana;
    p.M = M;
    p.alpha = alpha;
    p.O = O.as<uint32_t>();
    p.O_deg = Odeg.as<uint32_t>();
    p.cur_links = dl.as<uint32_t>();
    p.cur_deg = dd.as<uint32_t>();
    p.cur_M = M;
    p.entry = d_entry;
    p.row_order = row_order;
    if ((rc = run_gather(c, p, 0, pool_total, kernel_ms))) return rc;
    if (!commit) return ANQI_OK;
    return run_commit(c, dx, dn, n, stride, dim, O, Odeg, M, alpha, dl, dd, row_order, kernel_ms);
}

// Entries of every row from the context's entry tree (the last graph build's).
// ------------------------------------------------- the batched Vamana style
// index.h:936-1065.  The insertion order is the reference's: std::mt19937_64
// seeded from one value (the 64-bit Mersenne Twister of Matsumoto and
// Nishimura) and std::shuffle as GCC's library performs it on 32-bit ids --
// Fisher-Yates from the front, two positions per bounded draw
// (Brackett-Rozinsky and Lemire's batched ranged integers), each bounded draw
// by Lemire's multiply-and-reject -- restated here.
struct Mt64 {
    uint64_t mt[312];
    uint32_t idx = 312;
    explicit Mt64(uint64_t seed) {
        mt[0] = seed;
        for (uint32_t i = 1; i < 312; i++) mt[i] = 6364136223846793005ull * (mt[i - 1] ^ (mt[i - 1] >> 62)) + i;
    }
    uint64_t next() {
        if (idx >= 312) {
            for (uint32_t i = 0; i < 312; i++) {
                const uint64_t y = (mt[i] & 0xFFFFFFFF80000000ull) | (mt[(i + 1) % 312] & 0x7FFFFFFFull);
                mt[i] = mt[(i + 156) % 312] ^ (y >> 1) ^ ((y & 1ull) ? 0xB5026F5AA96619E9ull : 0ull);
            }
            idx = 0;
        }
        uint64_t x = mt[idx++];
        x ^= (x >> 29) & 0x5555555555555555ull;
        x ^= (x << 17) & 0x71D67FFFEDA60000ull;
        x ^= (x << 37) & 0xFFF7EEE000000000ull;
        return x ^ (x >> 43);
    }
    uint64_t below(uint64_t range) {  // uniform in [0, range)
        unsigned __int128 prod = (unsigned __int128)next() * range;
        uint64_t low = (uint64_t)prod;
        if (low < range) {
            const uint64_t threshold = (0ull - range) % range;
            while (low < threshold) {
                prod = (unsigned __int128)next() * range;
                low = (uint64_t)prod;
            }
        }
        return (uint64_t)(prod >> 64);
    }
};

static void shuffle_ids(std::vector<uint32_t>& a, Mt64& g) {
    const uint64_t n = a.size();
    if (n < 2) return;
    uint64_t i = 1;
    if (n % 2 == 0) std::swap(a[i++], a[g.below(2)]);
    while (i < n) {
        const uint64_t b1 = i + 2, x = g.below((i + 1) * b1);
        std::swap(a[i++], a[x / b1]);
        std::swap(a[i++], a[x % b1]);
    }
}

// The batch's rows take their new links (write_ids for every batch row).
__global__ void batch_write_kernel(const uint32_t* __restrict__ order, uint64_t floor_, uint32_t bsz,
                                   const uint32_t* __restrict__ O, const uint32_t* __restrict__ Od, uint32_t M,
                                   uint32_t* __restrict__ links, uint32_t* __restrict__ deg) {
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < (uint64_t)bsz * M;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t node = order[floor_ + t / M];
        const uint32_t j = (uint32_t)(t % M);
        links[node * M + j] = O[node * M + j];
        if (j == 0) deg[node] = Od[node];
    }
}

// Reverse edges of the batch: counts per target, the targets touched (listed
// once each, in any order), the largest count; then the sources per target.
__global__ void batch_count_kernel(const uint32_t* __restrict__ order, uint64_t floor_, uint32_t bsz,
                                   const uint32_t* __restrict__ O, const uint32_t* __restrict__ Od, uint32_t M,
                                   uint64_t n, uint32_t* __restrict__ cnt, uint32_t* __restrict__ touched,
                                   uint32_t* __restrict__ nt_max) {
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < (uint64_t)bsz * M;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t node = order[floor_ + t / M];
        const uint32_t j = (uint32_t)(t % M);
        if (j >= Od[node]) continue;
        const uint32_t dst = O[node * M + j];
        if (dst >= n) continue;
        const uint32_t old = atomicAdd(cnt + dst, 1u);
        if (old == 0) touched[atomicAdd(nt_max, 1u)] = dst;
        atomicMax(nt_max + 1, old + 1);
    }
}

__global__ void batch_fill_kernel(const uint32_t* __restrict__ order, uint64_t floor_, uint32_t bsz,
                                  const uint32_t* __restrict__ O, const uint32_t* __restrict__ Od, uint32_t M,
                                  uint64_t n, const uint64_t* __restrict__ off, uint32_t* __restrict__ fill,
                                  uint32_t* __restrict__ rev) {
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < (uint64_t)bsz * M;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t node = order[floor_ + t / M];
        const uint32_t j = (uint32_t)(t % M);
        if (j >= Od[node]) continue;
        const uint32_t dst = O[node * M + j];
        if (dst >= n) continue;
        rev[off[dst] + atomicAdd(fill + dst, 1u)] = (uint32_t)node;
    }
}

__global__ void fill_u32_kernel(uint32_t* a, uint64_t n, uint32_t v) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        a[i] = v;
}

// vamana_batch_refine on the device graph (dl, dd: n x M, degrees), g0 = the
// build's heaps (n x K).
static int run_vamana_batch(Ctx* c, const DevBuf& dx, const DevBuf& dn, uint64_t n, uint32_t stride, uint32_t dim,
                            const DevBuf& hid, uint32_t K, const anqi_graph_params& gp, DevBuf& dl, DevBuf& dd,
                            uint64_t* pool_total) {
    const int passes = (int)gp.vamana_passes;
    const uint32_t M = gp.degree, Lb = gp.vamana_L ? gp.vamana_L : 128;
    if (n == 0 || passes <= 0) return ANQI_OK;
    double frac = gp.vamana_batch_frac;
    if (frac <= 0.0) frac = 0.02;
    const double mb = frac * (double)n;
    uint64_t max_batch = std::min<uint64_t>((uint64_t)std::max(1.0, mb), gp.vamana_max_batch);
    if (max_batch == 0) max_batch = n;
    double base = gp.vamana_batch_base;
    if (base <= 1.0) base = 2.0;
    // the batches of a pass: [floor, ceiling) of the order
    std::vector<std::pair<uint64_t, uint64_t>> batches;
    uint64_t largest = 1;
    for (uint64_t count = 0, inc = 0; count < n;) {
        uint64_t floor_ = count, ceiling;
        const double p0 = std::pow(base, (double)inc);
        if (p0 <= (double)max_batch) {
            floor_ = (uint64_t)p0 - 1;
            ceiling = std::min<uint64_t>((uint64_t)std::pow(base, (double)(inc + 1)) - 1, n);
        } else {
            ceiling = std::min<uint64_t>(count + max_batch, n);
        }
        count = ceiling;
        inc++;
        if (ceiling <= floor_ || floor_ >= n) continue;
        batches.push_back({floor_, ceiling});
        largest = std::max(largest, ceiling - floor_);
    }
    if (largest * M > 0xFFFFFFFFull) return fail(c, ANQI_ERR_ARGS, "Vamana batch of %llu rows too large",
                                                (unsigned long long)largest);
    TmpBuf dord(c), dent(c), dO(c), dOd(c), cnt(c), fill(c), roff(c), rev(c), touched(c), ntm(c);
    int rc;
    const uint64_t tcap = std::min<uint64_t>(n, largest * M);
    if ((rc = ensure(c, dord, n * 4)) || (rc = ensure(c, dent, n * 4)) || (rc = ensure(c, dO, n * M * 4ull)) ||
        (rc = ensure(c, dOd, n * 4)) || (rc = ensure(c, cnt, n * 4)) || (rc = ensure(c, fill, n * 4)) ||
        (rc = ensure(c, roff, (n + 1) * 8)) || (rc = ensure(c, rev, largest * M * 4ull + 4)) ||
        (rc = ensure(c, touched, tcap * 4 + 4)) || (rc = ensure(c, ntm, 8)))
        return rc;
    const int blocks = c->sm_count * 8;
    fill_u32_kernel<<<blocks, 256, 0, c->stream>>>(dent.as<uint32_t>(), n, gp.vamana_entry < n ? gp.vamana_entry : 0u);
    ANQI_CUDA(c, cudaMemsetAsync(cnt.p, 0, n * 4, c->stream));
    ANQI_CUDA(c, cudaMemsetAsync(fill.p, 0, n * 4, c->stream));
    std::vector<uint32_t> order(n);
    for (uint64_t i = 0; i < n; i++) order[i] = (uint32_t)i;
    for (int pass = 0; pass < passes; pass++) {
        const float alpha = (gp.vamana_early_alpha_one && pass + 1 < passes) ? gp.vamana_early_alpha : gp.alpha;
        Mt64 g(gp.seed + 0x9e3779b97f4a7c15ull * (uint64_t)(pass + 1));
        shuffle_ids(order, g);
        if ((rc = h2d(c, dord, order.data(), n * 4))) return rc;
        for (const auto& bt : batches) {
            const uint64_t floor_ = bt.first;
            const uint32_t bsz = (uint32_t)(bt.second - bt.first);
            // the batch's rows: beam from the entry + g0 + current links, pruned -> O
            GatherParams p = base_params(dx, dn, n, stride, dim);
            p.g_ids = hid.as<uint32_t>();
            p.K = K;
            p.ef = Lb;
            p.cap = 0xFFFFFFFFu;
            p.mode = kModeVamana;
            p.M = M;
            p.alpha = alpha;
            p.O = dO.as<uint32_t>();
            p.O_deg = dOd.as<uint32_t>();
            p.cur_links = dl.as<uint32_t>();
            p.cur_deg = dd.as<uint32_t>();
            p.cur_M = M;
            p.cur_append = 1;
            p.entry = dent.as<uint32_t>();
            p.row_order = dord.as<uint32_t>();
            p.row_base = floor_;
            p.row_count = bsz;
            if ((rc = run_gather(c, p, 0, pool_total))) return rc;
            batch_write_kernel<<<blocks, 256, 0, c->stream>>>(dord.as<uint32_t>(), floor_, bsz, dO.as<uint32_t>(),
                                                            dOd.as<uint32_t>(), M, dl.as<uint32_t>(),
                                                            dd.as<uint32_t>());
            // every row the batch now links to: its links + those batch rows, pruned in place
            ANQI_CUDA(c, cudaMemsetAsync(ntm.p, 0, 8, c->stream));
            batch_count_kernel<<<blocks, 256, 0, c->stream>>>(dord.as<uint32_t>(), floor_, bsz, dO.as<uint32_t>(),
                                                            dOd.as<uint32_t>(), M, n, cnt.as<uint32_t>(),
                                                            touched.as<uint32_t>(), ntm.as<uint32_t>());
            ANQI_CUDA(c, cudaGetLastError());
            if ((rc = device_scan(c, cnt.as<uint32_t>(), roff.as<uint64_t>(), n))) return rc;
            batch_fill_kernel<<<blocks, 256, 0, c->stream>>>(dord.as<uint32_t>(), floor_, bsz, dO.as<uint32_t>(),
                                                           dOd.as<uint32_t>(), M, n, roff.as<uint64_t>(),
                                                           fill.as<uint32_t>(), rev.as<uint32_t>());
            ANQI_CUDA(c, cudaGetLastError());
            uint32_t nt[2] = {0, 0};
            if ((rc = d2h(c, nt, ntm, 8)) || (rc = sync(c))) return rc;
            if (nt[0] > 0) {
                GatherParams q = base_params(dx, dn, n, stride, dim);
                q.mode = kModeCommit;
                q.K = 1;
                q.ef = 4;
                q.M = M;
                q.alpha = alpha;
                q.O = dl.as<uint32_t>();
                q.O_deg = dd.as<uint32_t>();
                q.rev_off = roff.as<uint64_t>();
                q.rev_ids = rev.as<uint32_t>();
                q.links = dl.as<uint32_t>();
                q.deg = dd.as<uint32_t>();
                q.row_order = touched.as<uint32_t>();
                q.row_base = 0;
                q.row_count = nt[0];
                if ((rc = run_gather(c, q, nt[1], nullptr))) return rc;
            }
            // counts and fill cursors back to zero for the next batch
            fill_u32_kernel<<<blocks, 256, 0, c->stream>>>(cnt.as<uint32_t>(), n, 0u);
            fill_u32_kernel<<<blocks, 256, 0, c->stream>>>(fill.as<uint32_t>(), n, 0u);
            ANQI_CUDA(c, cudaGetLastError());
        }
    }
    return sync(c);
}

static int vamana_entries(Ctx* c, const DevBuf& dx, uint64_t n, uint32_t stride, uint32_t dim, DevBuf& ent) {
    const uint32_t nn = c->t_nodes;
    if (nn == 0 || c->t_dim != dim) return fail(c, ANQI_ERR_ARGS, "no entry tree for the Vamana refine");
    std::vector<uint32_t> lf(nn, kEmpty);
    for (uint32_t v = 0; v < nn; v++)
        if (c->t_left[v] == kEmpty && c->t_leaf_cnt[v] > 0) lf[v] = c->t_perm[c->t_leaf_off[v]];
    TmpBuf tl(c), tr(c), to(c), th(c), tf(c);
    int rc;
    if ((rc = h2d(c, tl, c->t_left.data(), nn * 4)) || (rc = h2d(c, tr, c->t_right.data(), nn * 4)) ||
        (rc = h2d(c, to, c->t_offset.data(), nn * 4)) || (rc = upload_padded(c, th, c->t_hyper.data(), nn, dim, stride)) ||
        (rc = h2d(c, tf, lf.data(), nn * 4)) || (rc = ensure(c, ent, n * 4)))
        return rc;
    tree_entry_kernel<<<c->sm_count * 8, 128, 0, c->stream>>>(dx.as<float>(), n, stride, dim, tl.as<uint32_t>(),
                                                              tr.as<uint32_t>(), to.as<float>(), th.as<float>(),
                                                              tf.as<uint32_t>(), nn, ent.as<uint32_t>());
    ANQI_CUDA(c, cudaGetLastError());
    return sync(c);
}

// init_knn over leaves; lists kd/ki/ksz already initialised.
static int run_leaf_topk(Ctx* c, const DevBuf& dx, const DevBuf& dn, uint64_t n, uint32_t stride, uint32_t dim,
                         const uint32_t* d_ids, const std::vector<LeafRef>& leaves, uint32_t K, DevBuf& kd, DevBuf& ki,
                         DevBuf& ksz, uint32_t mode = kKeyL2) {
    if (leaves.empty()) return ANQI_OK;
    uint32_t maxcnt = 0;
    for (const LeafRef& l : leaves) maxcnt = std::max(maxcnt, l.cnt);
    uint32_t tile_rows = std::min<uint32_t>(64, std::max<uint32_t>(8, (48 * 1024) / (stride * 4)) / 8 * 8);
    const uint32_t nwarp = 8;
    const size_t smem = ((size_t)kLeafRows * stride + (size_t)tile_rows * stride + 4 * (size_t)kLeafRows * K +
                         2 * nwarp * 64 + tile_rows + 2 * kLeafRows) * 4;
    if (smem > 227 * 1024) return fail(c, ANQI_ERR_ARGS, "init_knn tile does not fit (dim %u, K %u)", dim, K);
    if (mode > kKeyNegIp) return fail(c, ANQI_ERR_ARGS, "unknown key mode %u", mode);
    ANQI_CUDA(c, cudaFuncSetAttribute(leaf_topk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    TmpBuf dl(c);
    int rc = h2d(c, dl, leaves.data(), leaves.size() * sizeof(LeafRef));
    if (rc) return rc;
    dim3 grid((unsigned)leaves.size(), (maxcnt + kLeafRows - 1) / kLeafRows);
    leaf_topk_kernel<<<grid, 32 * nwarp, smem, c->stream>>>(dx.as<float>(), dn.as<float>(), n, stride, dim, d_ids,
                                                            dl.as<LeafRef>(), K, tile_rows, kd.as<float>(),
                                                            ki.as<uint32_t>(), ksz.as<uint32_t>(), mode);
    ANQI_CUDA(c, cudaGetLastError());
    return sync(c);
}

static int init_lists(Ctx* c, DevBuf& kd, DevBuf& ki, DevBuf& ksz, uint64_t n, uint32_t K) {
    int rc;
    if ((rc = ensure(c, kd, n * K * 4)) || (rc = ensure(c, ki, n * K * 4)) || (rc = ensure(c, ksz, n * 4))) return rc;
    init_lists_kernel<<<c->sm_count * 8, 256, 0, c->stream>>>(kd.as<float>(), ki.as<uint32_t>(), ksz.as<uint32_t>(), n, K);
    ANQI_CUDA(c, cudaGetLastError());
    return ANQI_OK;
}

}  // namespace anqi

using namespace anqi;

extern "C" {

int anqi_graph_warm_start(anqi_ctx* h, const float* x, uint64_t n, uint32_t dim, const uint32_t* cand, uint32_t stride,
                          uint32_t width, uint32_t K, uint32_t* ids, float* vals) {
    if (!h || !x || !cand || !ids || !vals || n == 0 || dim == 0 || K == 0 || width > stride || width > 4096)
        return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    const uint32_t xs = round_up(dim, 8);
    TmpBuf dx(c), dn(c), dc(c), hid(c), hv(c);
    int rc;
    if ((rc = upload_rows(c, dx, dn, x, n, dim, xs)) || (rc = h2d(c, dc, cand, n * stride * 4ull)) ||
        (rc = run_warm_start(c, dx, dn, n, xs, dim, dc.as<uint32_t>(), stride, width, K, hid, hv)) ||
        (rc = d2h(c, ids, hid, n * K * 4)) || (rc = d2h(c, vals, hv, n * K * 4)))
        return rc;
    return sync(c);
}

int anqi_graph_localjoin(anqi_ctx* h, const float* x, uint64_t n, uint32_t dim, uint32_t K, uint32_t sample,
                         uint32_t max_rounds, uint32_t* ids, float* vals, uint64_t* updates, uint32_t* rounds_done) {
    return anqi_graph_localjoin_precision(h, x, n, dim, K, sample, max_rounds, 0, ids, vals, updates, rounds_done,
                                          nullptr);
}

int anqi_graph_localjoin_precision(anqi_ctx* h, const float* x, uint64_t n, uint32_t dim, uint32_t K, uint32_t sample,
                                   uint32_t max_rounds, uint32_t precision, uint32_t* ids, float* vals,
                                   uint64_t* updates, uint32_t* rounds_done, float* join_ms) {
    if (!h || !x || !ids || !vals || n == 0 || dim == 0 || K == 0 || precision > 1) return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    const uint32_t xs = round_up(dim, 8);
    TmpBuf dx(c), dn(c), hid(c), hv(c);
    int rc;
    if ((rc = upload_rows(c, dx, dn, x, n, dim, xs)) || (rc = h2d(c, hid, ids, n * K * 4)) ||
        (rc = h2d(c, hv, vals, n * K * 4)))
        return rc;
    std::vector<uint64_t> up;
    ANQI_CUDA(c, cudaEventRecord(c->ev2, c->stream));
    if ((rc = run_localjoin(c, dx, dn, n, xs, dim, hid, hv, K, sample, max_rounds, up, precision))) return rc;
    ANQI_CUDA(c, cudaEventRecord(c->ev3, c->stream));
    if (join_ms) {
        ANQI_CUDA(c, cudaEventSynchronize(c->ev3));
        ANQI_CUDA(c, cudaEventElapsedTime(join_ms, c->ev2, c->ev3));
    }
    if (updates)
        for (size_t i = 0; i < up.size(); i++) updates[i] = up[i];
    if (rounds_done) *rounds_done = (uint32_t)up.size();
    if ((rc = d2h(c, ids, hid, n * K * 4)) || (rc = d2h(c, vals, hv, n * K * 4))) return rc;
    return sync(c);
}

// Clears the context's edge policy when the entry point that set it returns.
struct PolicyScope {
    Ctx* c;
    ~PolicyScope() { clear_edge_policy(c); }
};

int anqi_graph_select(anqi_ctx* h, const float* x, uint64_t n, uint32_t dim, const uint32_t* g_ids,
                      const float* g_vals, uint32_t K, uint32_t M, uint32_t ef, uint32_t cap, float alpha, uint32_t* O,
                      uint32_t* O_deg) {
    return anqi_graph_select_policy(h, x, n, dim, g_ids, g_vals, K, M, ef, cap, alpha, nullptr, O, O_deg);
}

int anqi_graph_select_policy(anqi_ctx* h, const float* x, uint64_t n, uint32_t dim, const uint32_t* g_ids,
                             const float* g_vals, uint32_t K, uint32_t M, uint32_t ef, uint32_t cap, float alpha,
                             const anqi_edge_policy* edge, uint32_t* O, uint32_t* O_deg) {
    if (!h || !x || !g_ids || !g_vals || !O || !O_deg || n == 0 || M == 0 || M > 64 || ef == 0) return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    const uint32_t xs = round_up(dim, 8);
    TmpBuf dx(c), dn(c), hid(c), hv(c), dO(c), dOd(c);
    PolicyScope scope{c};
    int rc;
    if ((rc = set_edge_policy(c, edge, n))) return rc;
    if ((rc = upload_rows(c, dx, dn, x, n, dim, xs)) || (rc = h2d(c, hid, g_ids, n * K * 4)) ||
        (rc = h2d(c, hv, g_vals, n * K * 4)) ||
        (rc = run_select_commit(c, dx, dn, n, xs, dim, hid, hv, K, M, ef, cap, alpha, dO, dOd, nullptr, nullptr,
                                nullptr)) ||
        (rc = d2h(c, O, dO, n * M * 4)) || (rc = d2h(c, O_deg, dOd, n * 4)))
        return rc;
    return sync(c);
}

int anqi_graph_commit(anqi_ctx* h, const float* x, uint64_t n, uint32_t dim, const uint32_t* O, const uint32_t* O_deg,
                      uint32_t M, float alpha, uint32_t* links, uint32_t* deg) {
    return anqi_graph_commit_policy(h, x, n, dim, O, O_deg, M, alpha, nullptr, links, deg);
}

int anqi_graph_commit_policy(anqi_ctx* h, const float* x, uint64_t n, uint32_t dim, const uint32_t* O,
                             const uint32_t* O_deg, uint32_t M, float alpha, const anqi_edge_policy* edge,
                             uint32_t* links, uint32_t* deg) {
    if (!h || !x || !O || !O_deg || !links || !deg || n == 0 || M == 0 || M > 64) return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    const uint32_t xs = round_up(dim, 8);
    TmpBuf dx(c), dn(c), dO(c), dOd(c), roff(c), rev(c), dl(c), dd(c);
    PolicyScope scope{c};
    int rc;
    if ((rc = set_edge_policy(c, edge, n))) return rc;
    if ((rc = upload_rows(c, dx, dn, x, n, dim, xs)) || (rc = h2d(c, dO, O, n * M * 4)) ||
        (rc = h2d(c, dOd, O_deg, n * 4)) || (rc = build_reverse(c, dO.as<uint32_t>(), n, M, roff, rev)) ||
        (rc = ensure(c, dl, n * M * 4)) || (rc = ensure(c, dd, n * 4)))
        return rc;
    GatherParams q = base_params(dx, dn, n, xs, dim);
    q.mode = kModeCommit;
    q.K = 1;
    q.ef = 4;
    q.M = M;
    q.alpha = alpha;
    q.O = dO.as<uint32_t>();
    q.O_deg = dOd.as<uint32_t>();
    q.rev_off = roff.as<uint64_t>();
    q.rev_ids = rev.as<uint32_t>();
    q.links = dl.as<uint32_t>();
    q.deg = dd.as<uint32_t>();
    if ((rc = run_gather(c, q, max_reverse(c, roff, n), nullptr))) return rc;
    if ((rc = d2h(c, links, dl, n * M * 4)) || (rc = d2h(c, deg, dd, n * 4))) return rc;
    return sync(c);
}

int anqi_graph_vamana_batch_refine(anqi_ctx* h, const float* x, uint64_t n, uint32_t dim, uint32_t* links,
                                   uint32_t* deg, const uint32_t* g0, uint32_t K, const anqi_graph_params* gp) {
    if (!h || !x || !links || !deg || !g0 || !gp || n == 0 || dim == 0 || K == 0 || gp->degree == 0 ||
        gp->degree > 64 || (gp->vamana_L ? gp->vamana_L : 128) > 1024)
        return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    const uint32_t xs = round_up(dim, 8), M = gp->degree;
    TmpBuf dx(c), dn(c), dl(c), dd(c), dg(c);
    PolicyScope scope{c};
    int rc;
    if ((rc = set_edge_policy(c, gp->edge, n)) || (rc = upload_rows(c, dx, dn, x, n, dim, xs)) ||
        (rc = h2d(c, dl, links, n * M * 4ull)) || (rc = h2d(c, dd, deg, n * 4)) || (rc = h2d(c, dg, g0, n * K * 4ull)))
        return rc;
    if ((rc = run_vamana_batch(c, dx, dn, n, xs, dim, dg, K, *gp, dl, dd, nullptr))) return rc;
    if ((rc = d2h(c, links, dl, n * M * 4ull)) || (rc = d2h(c, deg, dd, n * 4))) return rc;
    return sync(c);
}

int anqi_graph_vamana_select(anqi_ctx* h, const float* x, uint64_t n, uint32_t dim, const uint32_t* links,
                             const uint32_t* deg, uint32_t M, const uint32_t* g0, uint32_t K, const uint32_t* entry,
                             uint32_t Lb, float alpha, uint32_t* O, uint32_t* O_deg) {
    if (!h || !x || !links || !deg || !g0 || !entry || !O || !O_deg || n == 0 || dim == 0 || M == 0 || M > 64 ||
        K == 0 || Lb == 0 || Lb > 1024)
        return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    for (uint64_t i = 0; i < n; i++) {
        if (deg[i] > M || entry[i] >= n) return fail(c, ANQI_ERR_FORMAT, "invalid graph row or entry %llu", (unsigned long long)i);
        for (uint32_t j = 0; j < deg[i]; j++)
            if (links[i * M + j] >= n) return fail(c, ANQI_ERR_FORMAT, "invalid neighbor id in graph row %llu", (unsigned long long)i);
    }
    const uint32_t xs = round_up(dim, 8);
    TmpBuf dx(c), dn(c), dl(c), dd(c), dg(c), de(c), dO(c), dOd(c);
    int rc;
    if ((rc = upload_rows(c, dx, dn, x, n, dim, xs)) || (rc = h2d(c, dl, links, n * M * 4ull)) ||
        (rc = h2d(c, dd, deg, n * 4)) || (rc = h2d(c, dg, g0, n * K * 4ull)) || (rc = h2d(c, de, entry, n * 4)))
        return rc;
    uint64_t pool_total = 0;
    if ((rc = run_vamana_pass(c, dx, dn, n, xs, dim, dg, K, de.as<uint32_t>(), Lb, M, alpha, dl, dd, dO, dOd, nullptr,
                              &pool_total, nullptr, false)))
        return rc;
    if ((rc = d2h(c, O, dO, n * M * 4ull)) || (rc = d2h(c, O_deg, dOd, n * 4))) return rc;
    return sync(c);
}

static void graph_build_reset(Ctx* c) {
    GraphBuild& g = c->gb;
    for (DevBuf* b : {&g.dx, &g.dn, &g.hid, &g.hv, &g.order}) release(c, *b);
    g.seen.clear();
    g.seen.shrink_to_fit();
    g.active = false;
    g.rows_done = 0;
    g.has_edge = false;
    g.edge_resid.clear();
    g.edge_resid.shrink_to_fit();
    g.edge_mu.clear();
    g.edge_mu.shrink_to_fit();
}

int anqi_graph_build_begin(anqi_ctx* h, const float* x, uint64_t n, uint32_t dim, const anqi_graph_params* gp) {
    if (!h || !x || !gp || n < 2 || dim == 0 || gp->degree == 0 || gp->degree > 64 || gp->nn_k == 0 ||
        gp->nn_k > 256 || gp->warm_width == 0 || gp->leaf == 0)
        return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    graph_build_reset(c);
    GraphBuild& g = c->gb;
    g.n = n;
    g.dim = dim;
    g.xs = round_up(dim, 8);
    g.gp = *gp;
    g.gp.edge = nullptr;
    g.has_edge = gp->edge && gp->edge->flags != 0;
    if (g.has_edge) {
        // the policy and its tables, kept for the prunes of _finish
        const anqi_edge_policy& e = *gp->edge;
        if (e.nks > 8 || ((e.flags & (ANQI_EDGE_COVER | ANQI_EDGE_BALL | ANQI_EDGE_AUTO)) && (!e.resid || !e.nk)) ||
            ((e.flags & ANQI_EDGE_LSG) && !e.mu))
            return fail(c, ANQI_ERR_ARGS, "invalid edge policy");
        g.edge = e;
        g.edge_resid.assign(e.resid ? e.resid : nullptr, e.resid ? e.resid + n * (uint64_t)e.nk : nullptr);
        g.edge_mu.assign(e.mu ? e.mu : nullptr, e.mu ? e.mu + n : nullptr);
        g.edge.resid = g.edge_resid.empty() ? nullptr : g.edge_resid.data();
        g.edge.mu = g.edge_mu.empty() ? nullptr : g.edge_mu.data();
    }
    int rc;
    if ((rc = upload_rows(c, g.dx, g.dn, x, n, dim, g.xs))) return rc;
    // entry tree: make_forest with one tree (index.h:1111-1120)
    const auto t = Clock::now();
    ForestOut f;
    const uint32_t cap_nodes = (uint32_t)std::min<uint64_t>(4 * n + 8, 0xFFFFFFF0ull);
    rc = build_forest(c, g.dx.as<float>(), n, dim, g.xs, 1, gp->leaf, gp->max_depth ? gp->max_depth : 100, gp->seed,
                      cap_nodes, f);
    if (rc) {
        release(c, f.perm);
        release(c, f.hyper);
        graph_build_reset(c);
        return rc;
    }
    c->t_nodes = f.n_nodes[0];
    c->t_left.assign(f.left.begin(), f.left.begin() + c->t_nodes);
    c->t_right.assign(f.right.begin(), f.right.begin() + c->t_nodes);
    c->t_offset.assign(f.offset.begin(), f.offset.begin() + c->t_nodes);
    c->t_leaf_off.assign(f.leaf_off.begin(), f.leaf_off.begin() + c->t_nodes);
    c->t_leaf_cnt.assign(f.leaf_cnt.begin(), f.leaf_cnt.begin() + c->t_nodes);
    c->t_hyper.resize((size_t)c->t_nodes * dim);
    c->t_perm.resize(n);
    c->t_dim = dim;
    cudaMemcpy2D(c->t_hyper.data(), dim * 4, f.hyper.p, g.xs * 4, dim * 4, c->t_nodes, cudaMemcpyDeviceToHost);
    cudaMemcpy(c->t_perm.data(), f.perm.p, n * 4, cudaMemcpyDeviceToHost);
    for (uint32_t v = 0; v < c->t_nodes; v++)
        if (c->t_left[v] == kEmpty) std::memset(c->t_hyper.data() + (size_t)v * dim, 0, dim * 4);
    // the entry tree's leaf order groups nearby rows: the gathers run them together
    rc = ensure(c, g.order, n * 4);
    if (!rc && cudaMemcpyAsync(g.order.p, f.perm.p, n * 4, cudaMemcpyDeviceToDevice, c->stream) != cudaSuccess)
        rc = fail(c, ANQI_ERR_DEVICE, "row order copy failed");
    release(c, f.perm);
    release(c, f.hyper);
    if (!rc && ((rc = ensure(c, g.hid, n * gp->nn_k * 4ull)) || (rc = ensure(c, g.hv, n * gp->nn_k * 4ull))))
        ;
    if (rc) {
        graph_build_reset(c);
        return rc;
    }
    g.forest_ms = ms_since(t);
    g.warm_ms = 0;
    g.seen.assign(n, 0);
    g.active = true;
    return ANQI_OK;
}

int anqi_graph_build_warm_rows(anqi_ctx* h, uint64_t row0, uint64_t rows, const uint32_t* ids, uint32_t stride) {
    if (!h || !ids || rows == 0) return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    GraphBuild& g = c->gb;
    if (!g.active) return fail(c, ANQI_ERR_ARGS, "no graph build in progress (anqi_graph_build_begin)");
    if (row0 >= g.n || rows > g.n - row0 || stride < g.gp.warm_width)
        return fail(c, ANQI_ERR_ARGS, "warm-start rows [%llu, +%llu) or stride %u outside the build",
                    (unsigned long long)row0, (unsigned long long)rows, stride);
    for (uint64_t r = row0; r < row0 + rows; r++)
        if (g.seen[r]) return fail(c, ANQI_ERR_ARGS, "warm-start row %llu delivered twice", (unsigned long long)r);
    cudaSetDevice(c->device);
    const auto t = Clock::now();
    TmpBuf dw(c);
    int rc;
    if ((rc = h2d(c, dw, ids, rows * stride * 4ull)) ||
        (rc = run_warm_start(c, g.dx, g.dn, g.n, g.xs, g.dim, dw.as<uint32_t>(), stride, g.gp.warm_width, g.gp.nn_k,
                             g.hid, g.hv, row0, rows)))
        return rc;
    std::fill(g.seen.begin() + row0, g.seen.begin() + row0 + rows, 1);
    g.rows_done += rows;
    g.warm_ms += ms_since(t);
    return ANQI_OK;
}

int anqi_graph_build_finish(anqi_ctx* h, uint32_t* deg, uint32_t* links, anqi_build_stats* st) {
    if (!h || !deg || !links) return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    GraphBuild& g = c->gb;
    if (!g.active) return fail(c, ANQI_ERR_ARGS, "no graph build in progress (anqi_graph_build_begin)");
    if (g.rows_done != g.n) {
        const uint64_t done = g.rows_done, n = g.n;
        graph_build_reset(c);
        return fail(c, ANQI_ERR_ARGS, "warm start covers %llu of %llu rows", (unsigned long long)done,
                    (unsigned long long)n);
    }
    cudaSetDevice(c->device);
    const auto t0 = Clock::now();
    const anqi_graph_params& gp = g.gp;
    const uint64_t n = g.n;
    TmpBuf dO(c), dOd(c), dl(c), dd(c);
    auto t = Clock::now();
    std::vector<uint64_t> up;
    int rc = run_localjoin(c, g.dx, g.dn, n, g.xs, g.dim, g.hid, g.hv, gp.nn_k, gp.join_sample ? gp.join_sample : 20,
                           gp.join_iters, up, gp.precision);
    const double join_ms = ms_since(t);
    t = Clock::now();
    uint64_t pool_total = 0;
    double gather_kernel_ms = 0;
    const uint32_t cap = std::max<uint32_t>(gp.degree, gp.ef_alpha * gp.explore);
    const char* ord_env = std::getenv("ANQI_B200_ORDER");
    PolicyScope scope{c};
    if (!rc && g.has_edge) rc = set_edge_policy(c, &g.edge, n);
    if (!rc)
        rc = run_select_commit(c, g.dx, g.dn, n, g.xs, g.dim, g.hid, g.hv, gp.nn_k, gp.degree, gp.explore, cap,
                               gp.alpha, dO, dOd, &dl, &dd, &pool_total,
                               ord_env && ord_env[0] == '0' ? nullptr : g.order.as<uint32_t>(), &gather_kernel_ms);
    // optional global Vamana refine (index.h:1262-1285): every row's entry
    // from the entry tree, then `vamana_passes` passes over the graph
    if (!rc && gp.vamana_passes > 0 && gp.vamana_batch)
        rc = run_vamana_batch(c, g.dx, g.dn, n, g.xs, g.dim, g.hid, gp.nn_k, gp, dl, dd, &pool_total);
    else if (!rc && gp.vamana_passes > 0) {
        TmpBuf ent(c);
        rc = vamana_entries(c, g.dx, n, g.xs, g.dim, ent);
        for (uint32_t pass = 0; pass < gp.vamana_passes && !rc; pass++)
            rc = run_vamana_pass(c, g.dx, g.dn, n, g.xs, g.dim, g.hid, gp.nn_k, ent.as<uint32_t>(),
                                 gp.vamana_L ? gp.vamana_L : 128, gp.degree, gp.alpha, dl, dd, dO, dOd,
                                 ord_env && ord_env[0] == '0' ? nullptr : g.order.as<uint32_t>(), &pool_total,
                                 nullptr);
    }
    const double gather_ms = ms_since(t);
    if (!rc && !(rc = d2h(c, links, dl, n * gp.degree * 4ull)) && !(rc = d2h(c, deg, dd, n * 4))) rc = sync(c);
    if (!rc && st) {
        st->forest_ms = g.forest_ms;
        st->init_ms = g.warm_ms;
        st->join_ms = join_ms;
        st->reverse_ms = 0;
        st->gather_ms = gather_ms;
        st->gather_kernel_ms = gather_kernel_ms;
        st->total_ms = g.forest_ms + g.warm_ms + ms_since(t0);
        uint64_t tot = 0;
        for (uint64_t u : up) tot += u;
        st->join_updates = tot;
        st->pool_total = pool_total;
    }
    graph_build_reset(c);
    return rc;
}

int anqi_graph_build(anqi_ctx* h, const float* x, uint64_t n, uint32_t dim, const uint32_t* warm_ids,
                     uint32_t warm_stride, const anqi_graph_params* gp, uint32_t* deg, uint32_t* links,
                     anqi_build_stats* st) {
    if (!h || !x || !warm_ids || !gp || !deg || !links || n < 2 || dim == 0 || gp->degree == 0 || gp->degree > 64 ||
        gp->nn_k == 0 || gp->nn_k > 256 || gp->warm_width > warm_stride || gp->leaf == 0)
        return ANQI_ERR_ARGS;
    int rc;
    if ((rc = anqi_graph_build_begin(h, x, n, dim, gp))) return rc;
    if ((rc = anqi_graph_build_warm_rows(h, 0, n, warm_ids, warm_stride))) {
        graph_build_reset(&h->c);
        return rc;
    }
    return anqi_graph_build_finish(h, deg, links, st);
}

int anqi_graph_tree_size(anqi_ctx* h, uint32_t* n_nodes, uint64_t* n_points) {
    if (!h || !n_nodes || !n_points) return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    if (c->t_nodes == 0) return fail(c, ANQI_ERR_ARGS, "no graph built in this context");
    *n_nodes = c->t_nodes;
    *n_points = c->t_perm.size();
    return ANQI_OK;
}

int anqi_graph_tree_copy(anqi_ctx* h, uint32_t* left, uint32_t* right, float* offset, float* hyperplane,
                         uint32_t* leaf_off, uint32_t* leaf_cnt, uint32_t* perm) {
    if (!h || !left || !right || !offset || !hyperplane || !leaf_off || !leaf_cnt || !perm) return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    if (c->t_nodes == 0) return fail(c, ANQI_ERR_ARGS, "no graph built in this context");
    std::memcpy(left, c->t_left.data(), c->t_nodes * 4);
    std::memcpy(right, c->t_right.data(), c->t_nodes * 4);
    std::memcpy(offset, c->t_offset.data(), c->t_nodes * 4);
    std::memcpy(hyperplane, c->t_hyper.data(), c->t_hyper.size() * 4);
    std::memcpy(leaf_off, c->t_leaf_off.data(), c->t_nodes * 4);
    std::memcpy(leaf_cnt, c->t_leaf_cnt.data(), c->t_nodes * 4);
    std::memcpy(perm, c->t_perm.data(), c->t_perm.size() * 4);
    return ANQI_OK;
}

int anqi_aknn_init(anqi_ctx* h, const float* x, uint64_t n, uint32_t dim, const uint64_t* leaf_off,
                   const uint32_t* leaf_ids, uint64_t n_leaves, uint32_t K, uint32_t* ids, float* dists) {
    return anqi_aknn_init_metric(h, x, n, dim, leaf_off, leaf_ids, n_leaves, K, ANQI_METRIC_L2, ids, dists);
}

int anqi_aknn_init_metric(anqi_ctx* h, const float* x, uint64_t n, uint32_t dim, const uint64_t* leaf_off,
                          const uint32_t* leaf_ids, uint64_t n_leaves, uint32_t K, uint32_t metric, uint32_t* ids,
                          float* dists) {
    if (!h || !x || !leaf_off || !leaf_ids || !ids || !dists || n == 0 || dim == 0 || K == 0 || K > 256 ||
        metric > ANQI_METRIC_IP)
        return ANQI_ERR_ARGS;
    const uint32_t mode = metric == ANQI_METRIC_IP ? kKeyIpDist : kKeyL2;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    const uint32_t xs = round_up(dim, 8);
    TmpBuf dx(c), dn(c), dids(c), kd(c), ki(c), ksz(c);
    int rc;
    const uint64_t tot = leaf_off[n_leaves];
    if ((rc = upload_rows(c, dx, dn, x, n, dim, xs)) || (rc = h2d(c, dids, leaf_ids, tot * 4 + 4)) ||
        (rc = init_lists(c, kd, ki, ksz, n, K)))
        return rc;
    // leaves are applied in batches in which every row appears at most once
    std::vector<uint8_t> seen(n, 0);
    std::vector<LeafRef> batch;
    std::vector<uint64_t> batch_rows;
    for (uint64_t l = 0; l <= n_leaves; l++) {
        bool conflict = false;
        if (l < n_leaves)
            for (uint64_t a = leaf_off[l]; a < leaf_off[l + 1] && !conflict; a++) conflict = seen[leaf_ids[a]];
        if (l == n_leaves || conflict) {
            if ((rc = run_leaf_topk(c, dx, dn, n, xs, dim, dids.as<uint32_t>(), batch, K, kd, ki, ksz, mode))) return rc;
            for (uint64_t r : batch_rows) seen[r] = 0;
            batch.clear();
            batch_rows.clear();
            if (l == n_leaves) break;
        }
        batch.push_back({leaf_off[l], (uint32_t)(leaf_off[l + 1] - leaf_off[l]), 0});
        for (uint64_t a = leaf_off[l]; a < leaf_off[l + 1]; a++) {
            seen[leaf_ids[a]] = 1;
            batch_rows.push_back(leaf_ids[a]);
        }
    }
    if ((rc = d2h(c, ids, ki, n * K * 4)) || (rc = d2h(c, dists, kd, n * K * 4))) return rc;
    return sync(c);
}

int anqi_aknn_gather(anqi_ctx* h, const float* x, uint64_t n, uint32_t dim, const uint32_t* g_ids, const float* g_vals,
                     uint32_t K, uint32_t ef, uint32_t cap, uint32_t out_k, uint32_t* ids, float* dists) {
    return anqi_aknn_gather_metric(h, x, n, dim, g_ids, g_vals, K, ef, cap, out_k, ANQI_METRIC_L2, ids, dists);
}

int anqi_aknn_gather_metric(anqi_ctx* h, const float* x, uint64_t n, uint32_t dim, const uint32_t* g_ids,
                            const float* g_vals, uint32_t K, uint32_t ef, uint32_t cap, uint32_t out_k, uint32_t metric,
                            uint32_t* ids, float* dists) {
    if (!h || !x || !g_ids || !g_vals || !ids || !dists || n == 0 || K == 0 || ef == 0 || out_k == 0 || out_k > 1024 ||
        metric > ANQI_METRIC_IP)
        return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    const uint32_t xs = round_up(dim, 8);
    TmpBuf dx(c), dn(c), hid(c), hv(c), roff(c), rev(c), oi(c), od(c);
    int rc;
    if ((rc = upload_rows(c, dx, dn, x, n, dim, xs)) || (rc = h2d(c, hid, g_ids, n * K * 4)) ||
        (rc = h2d(c, hv, g_vals, n * K * 4)) || (rc = build_reverse(c, hid.as<uint32_t>(), n, K, roff, rev)) ||
        (rc = ensure(c, oi, n * out_k * 4)) || (rc = ensure(c, od, n * out_k * 4)))
        return rc;
    GatherParams p = base_params(dx, dn, n, xs, dim);
    p.g_ids = hid.as<uint32_t>();
    p.g_vals = hv.as<float>();
    p.K = K;
    p.rev_off = roff.as<uint64_t>();
    p.rev_ids = rev.as<uint32_t>();
    p.ef = ef;
    p.cap = cap;
    p.mode = kModeAknn;
    p.ip = metric == ANQI_METRIC_IP;
    p.out_k = out_k;
    p.out_ids = oi.as<uint32_t>();
    p.out_d = od.as<float>();
    if ((rc = run_gather(c, p, max_reverse(c, roff, n), nullptr))) return rc;
    if ((rc = d2h(c, ids, oi, n * out_k * 4)) || (rc = d2h(c, dists, od, n * out_k * 4))) return rc;
    return sync(c);
}

int anqi_aknn_build(anqi_ctx* h, const float* base, uint64_t n, uint32_t d, const anqi_aknn_params* ap, uint32_t* ids,
                    float* dists, anqi_build_stats* st) {
    if (!h || !base || !ap || !ids || !dists || n == 0 || d == 0 || ap->k == 0 || ap->k > 256 || ap->trees == 0 ||
        ap->leaf == 0 || ap->ef == 0 || ap->metric > ANQI_METRIC_IP)
        return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    if (n <= ap->k) return fail(c, ANQI_ERR_FORMAT, "n must exceed K");
    const bool ip = ap->metric == ANQI_METRIC_IP;
    if (ip && ap->nn_iters > 0) return fail(c, ANQI_ERR_ARGS, "LocalJoin rounds are implemented for metric l2 only");
    const auto t0 = Clock::now();
    const uint32_t xs = round_up(d, 8);
    const uint32_t K = ap->k;
    TmpBuf dx(c), dn(c), kd(c), ki(c), ksz(c), roff(c), rev(c), oi(c), od(c), hv(c), hi(c);
    int rc;
    if ((rc = upload_rows(c, dx, dn, base, n, d, xs)) || (rc = init_lists(c, kd, ki, ksz, n, K))) return rc;
    auto t = Clock::now();
    ForestOut f;
    const uint32_t cap_nodes = (uint32_t)std::min<uint64_t>(16 * n / ap->leaf + 1024, 4 * n + 8);
    rc = build_forest(c, dx.as<float>(), n, d, xs, ap->trees, ap->leaf, 100, ap->seed, cap_nodes, f, ip);
    const double forest_ms = ms_since(t);
    t = Clock::now();
    if (!rc) {
        // init_knn, one tree at a time (index.h:1433-1449)
        std::vector<std::vector<LeafRef>> tree_leaves(ap->trees);
        uint32_t maxcnt = 0;
        for (uint32_t tr = 0; tr < ap->trees; tr++)
            for (uint32_t v = 0; v < f.n_nodes[tr]; v++) {
                const size_t g = (size_t)tr * cap_nodes + v;
                if (f.left[g] == kEmpty && f.leaf_cnt[g] > 1) {
                    tree_leaves[tr].push_back({(uint64_t)tr * n + f.leaf_off[g], f.leaf_cnt[g], 0});
                    maxcnt = std::max(maxcnt, f.leaf_cnt[g]);
                }
            }
        // the tensor-core tiles: query tile resident up to 256 (padded)
        // dimensions, K-chunked up to 1024
        if (ap->precision == 1 && tc_padded_dim(d) != 0) {
            // BF16 tensor-core leaf tiles: candidates per tree, then the merge
            TcPrep tp;
            // candidate buffers (n x cap entries; GBs at 1M) are kept by the
            // context: allocating them anew for every build cost up to seconds
            DevBuf& ccnt = c->init_cnt;
            DevBuf& cid = c->init_cid;
            DevBuf& ckey = c->init_key;
            const uint32_t cap = round_up(std::max(maxcnt, 2u), 32u);
            // candidate slots for batches of leaves covering up to brows rows (~1 GB)
            uint64_t want = (512ull << 20) / (cap * 4ull);
            if (const char* e = std::getenv("ANQI_B200_INIT_BATCH_ROWS")) want = std::strtoull(e, nullptr, 10);
            const uint64_t brows = std::min<uint64_t>(n, std::max<uint64_t>(maxcnt, want));
            if (!(rc = tc_prep(c, dx.as<float>(), dn.as<float>(), n, xs, d, tp)) && !(rc = ensure(c, ccnt, brows * 4)) &&
                !(rc = ensure(c, cid, brows * (size_t)cap * 4)) && !(rc = ensure(c, ckey, brows * (size_t)cap * 4))) {
                auto cu = [&](cudaError_t e, const char* what) { return e == cudaSuccess ? ANQI_OK : cuda_check(c, e, what); };
                rc = cu(cudaMemsetAsync(ccnt.p, 0, brows * 4, c->stream), "cudaMemsetAsync");
                const int wpb = 4;
                const size_t msmem = (size_t)(4 * K + 128) * 4 * wpb;
                if (!rc && msmem > 48 * 1024)
                    rc = cu(cudaFuncSetAttribute(leaf_merge_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)msmem),
                            "cudaFuncSetAttribute");
                // every tree's batches planned on the host first, their tiles
                // uploaded once: the filter and merge launches then follow
                // each other on the stream without a host round trip
                struct BatchPlan {
                    uint64_t base, nslots;
                    size_t t0, nt;
                };
                std::vector<LeafTile> tiles;
                std::vector<BatchPlan> plan;
                for (uint32_t tr = 0; tr < ap->trees && !rc; tr++) {
                    // leaves in permutation order, in batches of contiguous positions
                    std::vector<LeafRef>& lv = tree_leaves[tr];
                    std::sort(lv.begin(), lv.end(), [](const LeafRef& a, const LeafRef& b) { return a.off < b.off; });
                    for (size_t l0 = 0; l0 < lv.size() && !rc;) {
                        const uint64_t base = lv[l0].off;
                        size_t l1 = l0;
                        while (l1 < lv.size() && lv[l1].off + lv[l1].cnt - base <= brows) l1++;
                        const std::vector<LeafRef> batch(lv.begin() + l0, lv.begin() + l1);
                        const size_t t0 = tiles.size();
                        rc = tc_leaf_tiles(c, batch, cap, tiles);
                        plan.push_back({base, lv[l1 - 1].off + lv[l1 - 1].cnt - base, t0, tiles.size() - t0});
                        l0 = l1;
                    }
                }
                TmpBuf dtiles(c);
                if (!rc) rc = h2d(c, dtiles, tiles.data(), std::max<size_t>(1, tiles.size()) * sizeof(LeafTile));
                for (size_t b = 0; b < plan.size() && !rc; b++) {
                    const BatchPlan& bp = plan[b];
                    rc = tc_leaf_filter(c, tp, dx.as<float>(), dn.as<float>(), n, xs, d, f.perm.as<uint32_t>(),
                                        dtiles.as<LeafTile>() + bp.t0, bp.nt, kd.as<float>(), ksz.as<uint32_t>(), K,
                                        ccnt.as<uint32_t>(), cap, cid.as<uint32_t>(), ckey.as<float>(), bp.base,
                                        ip ? kKeyIpDist : kKeyL2);
                    if (rc) break;
                    leaf_merge_kernel<<<c->sm_count * 8, 32 * wpb, msmem, c->stream>>>(
                        dx.as<float>(), dn.as<float>(), n, xs, d, f.perm.as<uint32_t>(), bp.base, bp.nslots,
                        ccnt.as<uint32_t>(), cap, cid.as<uint32_t>(), ckey.as<float>(), K, kd.as<float>(),
                        ki.as<uint32_t>(), ksz.as<uint32_t>(), c->err.as<uint32_t>(), ip ? kKeyIpDist : kKeyL2);
                    rc = cu(cudaGetLastError(), "leaf_merge_kernel");
                }
                if (!rc) rc = check_device_error(c, "tensor-core init_knn");
            }
            tc_release(c, tp);
        } else {
            for (uint32_t tr = 0; tr < ap->trees && !rc; tr++)
                rc = run_leaf_topk(c, dx, dn, n, xs, d, f.perm.as<uint32_t>(), tree_leaves[tr], K, kd, ki, ksz,
                                   ip ? kKeyIpDist : kKeyL2);
        }
    }
    // tree 0's leaf order groups the rows of one leaf: the gather runs them together
    TmpBuf order(c);
    if (!rc && !(rc = ensure(c, order, n * 4)))
        rc = cudaMemcpyAsync(order.p, f.perm.p, n * 4, cudaMemcpyDeviceToDevice, c->stream) == cudaSuccess
                 ? ANQI_OK
                 : fail(c, ANQI_ERR_DEVICE, "row order copy failed");
    release(c, f.perm);
    release(c, f.hyper);
    if (rc) return rc;
    random_fill_kernel<<<c->sm_count * 8, 128, 0, c->stream>>>(dx.as<float>(), dn.as<float>(), n, xs, d, ap->seed, K,
                                                               kd.as<float>(), ki.as<uint32_t>(), ksz.as<uint32_t>(), ip);
    ANQI_CUDA(c, cudaGetLastError());
    if ((rc = sync(c))) return rc;
    const double init_ms = ms_since(t);
    t = Clock::now();
    std::vector<uint64_t> up;
    if (ap->nn_iters > 0) {
        // optional LocalJoin on the AKNN heaps (index.h:1314-1333)
        if ((rc = ensure(c, hv, n * K * 4)) || (rc = ensure(c, hi, n * K * 4))) return rc;
        list_to_heap_kernel<<<c->sm_count * 8, 256, 0, c->stream>>>(kd.as<float>(), ki.as<uint32_t>(),
                                                                    ksz.as<uint32_t>(), n, K, hv.as<float>(),
                                                                    hi.as<uint32_t>());
        ANQI_CUDA(c, cudaGetLastError());
        if ((rc = run_localjoin(c, dx, dn, n, xs, d, hi, hv, K, ap->nn_sample ? ap->nn_sample : 20, ap->nn_iters, up)))
            return rc;
    }
    const double join_ms = ms_since(t);
    t = Clock::now();
    const DevBuf& gid = ap->nn_iters > 0 ? static_cast<const DevBuf&>(hi) : static_cast<const DevBuf&>(ki);
    const DevBuf& gval = ap->nn_iters > 0 ? static_cast<const DevBuf&>(hv) : static_cast<const DevBuf&>(kd);
    GatherParams p = base_params(dx, dn, n, xs, d);
    // l2: the gather runs over rows renumbered for locality (lists, rows and
    // norms permuted; ANQI_B200_GATHER_RENUMBER=0 keeps the original numbering)
    const char* ren_env = std::getenv("ANQI_B200_GATHER_RENUMBER");
    const bool ren = !ip && !(ren_env && ren_env[0] == '0');
    TmpBuf dxc(c), rperm(c), rinv(c), rids(c), rvals(c), rnorm(c);
    if (ren) {
        if ((rc = locality_order(c, gid.as<uint32_t>(), n, K, order.as<uint32_t>(), rperm, rinv)) ||
            (rc = ensure(c, rids, n * K * 4)) || (rc = ensure(c, rvals, n * K * 4)) || (rc = ensure(c, rnorm, n * 4)) ||
            (rc = ensure(c, dxc, n * xs * 4ull)))
            return rc;
        const int blocks = c->sm_count * 8;
        renumber_lists_kernel<<<blocks, 256, 0, c->stream>>>(gid.as<uint32_t>(), gval.as<float>(), rperm.as<uint32_t>(),
                                                            rinv.as<uint32_t>(), n, K, rids.as<uint32_t>(),
                                                            rvals.as<float>());
        // d = 128: rows in chunk column order (two shuffles per distance
        // instead of the lane tree's nine; the same bits)
        permute_rows_kernel<<<blocks, 256, 0, c->stream>>>(dx.as<float>(), dxc.as<float>(), rperm.as<uint32_t>(), n, xs,
                                                           d == 128 ? 128u : 0u);
        permute_vals_kernel<<<blocks, 256, 0, c->stream>>>(dn.as<float>(), rnorm.as<float>(), rperm.as<uint32_t>(), n);
        ANQI_CUDA(c, cudaGetLastError());
        if ((rc = build_reverse(c, rids.as<uint32_t>(), n, K, roff, rev))) return rc;
        p.x = dxc.as<float>();
        p.norms = rnorm.as<float>();
        p.cols = d == 128 ? 1 : 0;
        p.g_ids = rids.as<uint32_t>();
        p.g_vals = rvals.as<float>();
        p.perm = rperm.as<uint32_t>();
    } else {
        if ((rc = build_reverse(c, gid.as<uint32_t>(), n, K, roff, rev))) return rc;
        // d = 128: the gather reads its rows in chunk column order
        if (d == 128 && !ip) {
            if ((rc = ensure(c, dxc, n * xs * 4ull))) return rc;
            if ((rc = chunk_cols(c, dx.as<float>(), dxc.as<float>(), n, xs, 128))) return rc;
            p.x = dxc.as<float>();
            p.cols = 1;
        }
        p.g_ids = gid.as<uint32_t>();
        p.g_vals = gval.as<float>();
    }
    const double reverse_ms = ms_since(t);
    t = Clock::now();
    if ((rc = ensure(c, oi, n * K * 4)) || (rc = ensure(c, od, n * K * 4))) return rc;
    p.K = K;
    p.rev_off = roff.as<uint64_t>();
    p.rev_ids = rev.as<uint32_t>();
    p.ef = ap->ef;
    p.cap = std::max<uint32_t>(K, (ap->ef_alpha ? ap->ef_alpha : 8) * ap->ef);
    p.mode = kModeAknn;
    p.ip = ip;
    p.out_k = K;
    p.out_ids = oi.as<uint32_t>();
    p.out_d = od.as<float>();
    // rows of one RP-tree leaf run together (the renumbered rows are in that order already)
    p.row_order = ren || (std::getenv("ANQI_B200_ORDER") && std::getenv("ANQI_B200_ORDER")[0] == '0')
                      ? nullptr
                      : order.as<uint32_t>();
    uint64_t pool_total = 0;
    double gather_kernel_ms = 0;
    if ((rc = run_gather(c, p, max_reverse(c, roff, n), &pool_total, &gather_kernel_ms))) return rc;
    const double gather_ms = ms_since(t);
    if ((rc = d2h(c, ids, oi, n * K * 4)) || (rc = d2h(c, dists, od, n * K * 4)) || (rc = sync(c))) return rc;
    if (st) {
        st->forest_ms = forest_ms;
        st->init_ms = init_ms;
        st->join_ms = join_ms;
        st->reverse_ms = reverse_ms;
        st->gather_ms = gather_ms;
        st->gather_kernel_ms = gather_kernel_ms;
        st->total_ms = ms_since(t0);
        uint64_t tot = 0;
        for (uint64_t u : up) tot += u;
        st->join_updates = tot;
        st->pool_total = pool_total;
    }
    return ANQI_OK;
}

// tools/dataset_gt.cpp:206-248: the whole base is one candidate set, every row
// keeps its K smallest (key, id) over all other rows.
__global__ void iota_kernel(uint32_t* a, uint64_t n) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < n; t += (uint64_t)gridDim.x * blockDim.x)
        a[t] = (uint32_t)t;
}

int anqi_exact_topk(anqi_ctx* h, const float* base, uint64_t n, uint32_t d, uint32_t K, uint32_t* ids, float* keys) {
    return anqi_exact_topk_metric(h, base, n, d, K, ANQI_METRIC_L2, ids, keys);
}

int anqi_exact_topk_metric(anqi_ctx* h, const float* base, uint64_t n, uint32_t d, uint32_t K, uint32_t metric,
                           uint32_t* ids, float* keys) {
    if (!h || !base || !ids || !keys || d == 0 || K == 0 || K > 256 || metric > ANQI_METRIC_IP) return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    if (K >= n) return fail(c, ANQI_ERR_ARGS, "require K < base vector count");
    const uint32_t xs = round_up(d, 8);
    TmpBuf dx(c), dn(c), dids(c), kd(c), ki(c), ksz(c);
    int rc;
    if ((rc = upload_rows(c, dx, dn, base, n, d, xs)) || (rc = ensure(c, dids, n * 4)) ||
        (rc = init_lists(c, kd, ki, ksz, n, K)))
        return rc;
    iota_kernel<<<c->sm_count * 8, 256, 0, c->stream>>>(dids.as<uint32_t>(), n);
    ANQI_CUDA(c, cudaGetLastError());
    std::vector<LeafRef> all{{0, (uint32_t)n, 0}};
    if ((rc = run_leaf_topk(c, dx, dn, n, xs, d, dids.as<uint32_t>(), all, K, kd, ki, ksz,
                            metric == ANQI_METRIC_IP ? kKeyNegIp : kKeyL2)))
        return rc;
    if ((rc = d2h(c, ids, ki, n * K * 4)) || (rc = d2h(c, keys, kd, n * K * 4))) return rc;
    return sync(c);
}

}  // extern "C"
