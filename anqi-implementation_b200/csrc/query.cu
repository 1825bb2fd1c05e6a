// Reverse-kNN query path: query lift, RP-tree entry, greedy beam + bounded
// flood over the lifted G48 graph, FP32 postfilter against the LRQ thresholds.
//
// Reference: src/rknn_query.cpp:2714-2765 (per-query work of the timed loop),
// include/index.h:1535-1640 (range_search), include/neighbor.h:43-141 (the
// ordered beam queue), include/rptrees.h:108-124 (entry descent).
//
// Design.  One warp owns one query at a time and pulls queries from a global
// counter (persistent grid), in RP-tree leaf order.  The beam is one sorted
// (dist, id) array in shared memory; an expansion's fresh neighbours are
// filtered, sorted and inserted in place as a batch, which leaves exactly the
// top-L set and first-unexpanded cursor that the reference's one-at-a-time
// binary insertion leaves, because the queue order is a total order on
// (dist, id) and no id is inserted twice.  The flood's visited set is a
// closure, so its result does not depend on visit order either.  Distances are
// computed by 4-thread groups in the AVX-512 lane order (common.cuh), so every
// comparison against R2 and every beam decision matches the reference's FP32
// arithmetic bit for bit.  Objects are renumbered in breadth-first graph order
// at index load; the visited set is a per-warp window bitmap around the entry
// object in shared memory, backed by visited tables and a per-warp bitmap
// over all objects (beam.cuh).  Fresh lifted rows arrive by TMA bulk copies.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdlib>

#include "beam.cuh"
#include "internal.h"
#include "tc.cuh"

namespace anqi {

struct SearchParams {
    const float* lifted;
    const float* base;
    const float* onorm;
    const uint32_t* links;
    const uint32_t* deg;
    const uint32_t* tleft;
    const uint32_t* tright;
    const float* toffset;
    const float* thyper;
    const uint32_t* tleaf;
    uint64_t n;
    uint32_t dim, d, lstride, bstride, degree, troot;
    uint32_t stage_rows;  // rows per staging round: 8, 4 or 2 (long rows)
    double scale, R2, mstar2;
    float R2f;  // the largest float <= R2 (float distances compare the same against either)
    uint32_t ip;  // the ip metric: per-query R2 (qR2f) and postfilter key -<o, q>
    float* qR2f;  // ip: per query, the largest float <= |s q|^2 + 1 + M*^2 (rknn_entry_kernel)
    const float* thr;  // slot-major thresholds
    const float* queries;
    const uint32_t* entry;  // entry object per query (rknn_entry_kernel)
    const uint32_t* perm;   // object id -> original id (objects are renumbered for locality)
    const uint32_t* order;  // work item -> query (leaf-ordered), or null for identity
    const uint32_t* qL;
    const uint8_t* qslot;
    uint32_t L_all, slot_all, nq, L_max;
    uint32_t* vis_bits;
    uint32_t vis_words;
    uint32_t* vis_log;
    uint32_t log_cap;
    uint32_t* cand_scratch;
    uint32_t cand_cap;
    uint32_t* work;
    unsigned long long* fill;  // [0] predicted ids, [1] candidate ids
    uint32_t* pred_buf;
    uint64_t pred_cap;
    uint32_t* cand_buf;
    uint64_t cand_out_cap;
    int keep_cand;
    uint32_t* npred;
    uint32_t* ncand;
    uint32_t* ndist;
    uint32_t* nexp;
    uint32_t* nflood;
    unsigned long long* pred_at;
    unsigned long long* cand_at;
    uint32_t* err;
    uint32_t hash_cap;    // shared-memory visited table entries per warp (power of two, 0 = none)
    uint32_t hash_shift;  // 32 - log2(hash_cap)
    uint32_t* gtab;       // per-slot global visited tables (gcap entries each, all ANQI_EMPTY between queries)
    uint32_t gcap;        // entries per slot (power of two, 0 = none)
    uint32_t gshift;      // 32 - log2(gcap)
    uint32_t drop_row_copies;  // test fault: issue no row copies, so the bounded row waits run out
    uint32_t post_rows;        // candidate tile: base rows per postfilter round (<= stage_rows)
};

constexpr unsigned kFull = 0xFFFFFFFFu;

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Rows per staging round fixed at compile time for the d = 128 instance (8
// rows, 4-thread groups); 0 = from the launch parameters.
template <uint32_t kDim>
constexpr uint32_t kSearchRows = kDim == 130 ? 8u : 0u;

// The d = 128 instance also has its row stride fixed, and reads the lifted
// rows and the lifted query in chunk column order (common.cuh), which
// anqi_index_load gives the lifted rows for that dimension.
constexpr uint32_t kColsDim = 130;
template <uint32_t kDim>
constexpr uint32_t kSearchLStride = kDim ? (kDim + 7) / 8 * 8 : 0u;
template <uint32_t kDim>
__device__ __forceinline__ uint32_t search_lstride(const SearchParams& p) {
    return kSearchLStride<kDim> ? kSearchLStride<kDim> : p.lstride;
}

// Bulk (TMA) copy of one row into shared memory, completing on the warp's
// mbarrier; and the arrive that sets the bytes a phase waits for.  The
// staging buffer is written by the generic proxy only through cp.async (the
// entry row and the postfilter's base rows); the kernel orders those writes
// before later bulk copies with one proxy fence per query, after the entry
// row.  Reads of staged rows are complete (their values consumed) before the
// warp issues the next copies into them.
__device__ __forceinline__ void bulk_row(float* dst, const float* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
                 ::"r"(tc::smem_u32(dst)), "l"(src), "r"(bytes), "r"(tc::smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void bar_expect(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(tc::smem_u32(bar)), "r"(bytes)
                 : "memory");
}

constexpr uint32_t kRowWaitPolls = 1u << 22;

// Objects are numbered in breadth-first order of the graph (anqi_index_load),
// so a query's visits fall mostly near its entry object: the window bitmap of
// beam.cuh covers the kWinBits ids around the entry.

template <uint32_t kDim>
__device__ __forceinline__ uint32_t expand_links(const SearchParams& p, uint32_t l0, uint32_t l1, uint32_t dg,
                                                 Visited& vis, uint32_t& nlog, uint32_t* ni, uint32_t lane,
                                                 float* stage, uint64_t* bar, uint32_t* win, uint32_t wbase) {
    const uint32_t srows = kSearchRows<kDim> ? kSearchRows<kDim> : p.stage_rows;
    bool f0 = false, f1 = false, bad = false, g0 = false, g1 = false;
    uint32_t r0 = 0, r1 = 0;
    if (lane < dg) {
        if (l0 < p.n) f0 = visit_id(vis, win, wbase, l0, r0, g0, p.err);
        else bad = true;
    }
    if (lane + 32 < dg) {
        if (l1 < p.n) f1 = visit_id(vis, win, wbase, l1, r1, g1, p.err);
        else bad = true;
    }
    if (bad) set_error(p.err, kDevBadId);
    const unsigned b0 = __ballot_sync(kFull, f0), b1 = __ballot_sync(kFull, f1);
    const uint32_t c0 = __popc(b0), lt = lanemask_lt();
    const uint32_t p0 = __popc(b0 & lt), p1 = c0 + __popc(b1 & lt);
    const uint32_t m = c0 + __popc(b1);
    const uint32_t ls = search_lstride<kDim>(p), rb = ls * 4;
    if (m) {
        if (lane == 0) bar_expect(bar, min(m, srows) * rb);
        if (!p.drop_row_copies) {
            if (f0 && p0 < srows) bulk_row(stage + (size_t)p0 * ls, p.lifted + (size_t)l0 * ls, rb, bar);
            if (f1 && p1 < srows) bulk_row(stage + (size_t)p1 * ls, p.lifted + (size_t)l1 * ls, rb, bar);
        }
    }
    if (f0) ni[p0] = l0;
    if (f1) ni[p1] = l1;
    // table visits are counted (the level's load) and, above level 0, logged
    // for the clean-up; window visits are neither
    if (__any_sync(kFull, (f0 && g0) || (f1 && g1))) {
        const unsigned h0 = __ballot_sync(kFull, f0 && g0), h1 = __ballot_sync(kFull, f1 && g1);
        const uint32_t q0 = nlog + __popc(h0 & lt), q1 = nlog + __popc(h0) + __popc(h1 & lt);
        const bool logs = vis.level != 0;
        if (logs && f0 && g0 && q0 < p.log_cap) vis.vlog[q0] = r0;
        if (logs && f1 && g1 && q1 < p.log_cap) vis.vlog[q1] = r1;
        nlog += __popc(h0) + __popc(h1);
    }
    __syncwarp();
    return m;
}

// Issues the loads of node's degree and link slots lane and lane + 32.  No
// instruction here uses the loaded values, so the warp does not wait for them
// until it expands the node (usually one expansion later).  Slots at or past
// the degree are never used; the links array has 64 padding entries, so the
// loads past the last row stay in bounds, and degrees were checked against the
// slot count at index load.
__device__ __forceinline__ void load_links(const SearchParams& p, uint32_t node, uint32_t lane, uint32_t& l0,
                                           uint32_t& l1, uint32_t& dg) {
    const uint32_t* lk = p.links + (size_t)node * p.degree;
    dg = p.deg[node];
    l0 = lk[lane];
    l1 = lk[lane + 32];
}

// Distance of staged row `row` to the lifted query by a group of G threads
// (thread gt of the group): the reference's lane order for G = 4, 8, 16.
template <int G>
__device__ __forceinline__ float row_l2sqr(const float* row, const float* qhat, uint32_t dim, uint32_t gt) {
    if constexpr (G == 4) return group_l2sqr(row, qhat, dim, gt, kFull);
    else return group_l2sqr_w<G>(row, qhat, dim, gt, kFull);
}

// Distances of the m fresh neighbours to the lifted query.  Rows arrive by
// bulk copy, stage_rows per round (the first round was requested by
// expand_links); each round is one phase of bar (parity ph).  Rows are
// reduced by groups of 32 / stage_rows threads (4, 8 or 16: long rows are
// staged 4 or 2 at a time).  Returns false when a wait ran out (the error
// word is set).
template <uint32_t kDim>
__device__ __forceinline__ bool fresh_distances(const SearchParams& p, const float* qhat, const uint32_t* ni,
                                                float* nd, uint32_t m, float* stage, uint64_t* bar, uint32_t& ph,
                                                uint32_t lane) {
    const uint32_t dim = kDim ? kDim : p.dim;
    const uint32_t srows = kSearchRows<kDim> ? kSearchRows<kDim> : p.stage_rows;
    const uint32_t ls = search_lstride<kDim>(p), rb = ls * 4;
    for (uint32_t r0 = 0; r0 < m; r0 += srows) {
        const uint32_t nr = min(m - r0, srows);
        if (r0 > 0) {
            if (lane == 0) bar_expect(bar, nr * rb);
            if (lane < nr) bulk_row(stage + (size_t)lane * ls, p.lifted + (size_t)ni[r0 + lane] * ls, rb, bar);
        }
        if (!tc::mbar_wait(bar, ph, kRowWaitPolls)) {
            set_error(p.err, kDevWaitTimeout);
            return false;
        }
        ph ^= 1u;
        if (srows == 2) {
            const uint32_t gw = lane >> 4, gt = lane & 15u;
            const float da = row_l2sqr<16>(stage + (size_t)gw * ls, qhat, dim, gt);
            if (gt == 0 && gw < nr) nd[r0 + gw] = da;
        } else if (srows == 4) {
            const uint32_t gw = lane >> 3, gt = lane & 7u;
            const float da = row_l2sqr<8>(stage + (size_t)gw * ls, qhat, dim, gt);
            if (gt == 0 && gw < nr) nd[r0 + gw] = da;
        } else {
            const uint32_t gw = lane >> 2, gt = lane & 3u;
            const bool oka = gw < nr;
            const float* row = oka ? stage + (size_t)gw * ls : stage;
            float da;
            if constexpr (kDim == kColsDim) da = group_l2sqr_cols<kColsDim>(row, qhat, gt, kFull);
            else da = row_l2sqr<4>(row, qhat, dim, gt);
            if (gt == 0 && oka) nd[r0 + gw] = da;
        }
        __syncwarp();
    }
    return true;
}

// Appends fresh neighbours within R2 to the candidate / flood list (visit
// order).  For a float x, (double)x <= R2 exactly when x <= R2f, the largest
// float not above R2.
__device__ __forceinline__ void append_in_range(const SearchParams& p, float r2f, const float* nd, const uint32_t* ni,
                                                uint32_t m, uint32_t* cl, uint32_t& ncand, bool& overflow,
                                                uint32_t lane) {
    const bool in0 = lane < m && nd[lane] <= r2f;
    const bool in1 = lane + 32 < m && nd[lane + 32] <= r2f;
    const unsigned b0 = __ballot_sync(kFull, in0), b1 = __ballot_sync(kFull, in1);
    const uint32_t c0 = __popc(b0), lt = lanemask_lt();
    const uint32_t pos0 = ncand + __popc(b0 & lt), pos1 = ncand + c0 + __popc(b1 & lt);
    if (in0) {
        if (pos0 < p.cand_cap) cl[pos0] = ni[lane];
        else overflow = true;
    }
    if (in1) {
        if (pos1 < p.cand_cap) cl[pos1] = ni[lane + 32];
        else overflow = true;
    }
    ncand += c0 + __popc(b1);
    if (ncand > p.cand_cap) ncand = p.cand_cap;
    overflow = __any_sync(kFull, overflow);
    __syncwarp();
}

extern __shared__ __align__(16) unsigned char g_smem[];

// Rows per staging round: 8 rows of up to 1 KB, else 4 of up to 2 KB, else 2.
__device__ __host__ __forceinline__ uint32_t stage_rows_for(uint32_t lstride, uint32_t bstride) {
    const uint32_t w = lstride > bstride ? lstride : bstride;
    return w <= 256 ? 8u : (w <= 512 ? 4u : 2u);
}

__device__ __host__ __forceinline__ size_t search_smem_words(uint32_t L_max, uint32_t lstride, uint32_t bstride,
                                                             uint32_t hash_cap) {
    return (size_t)2 * L_max + 128 + lstride + kWinWords +
           stage_rows_for(lstride, bstride) * (size_t)(lstride > bstride ? lstride : bstride) + hash_cap + 8;
}

// kWpb warps per block (one query each): 2, 4 or 8, the block shape the
// autotuner picks; 32 warps per SM at 64 registers in every shape.
template <uint32_t kDim, uint32_t kWpb>
__global__ void __launch_bounds__(32 * kWpb, 32 / kWpb) rknn_search_kernel(SearchParams p) {
    const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5, gt = lane & 3u, gw = lane >> 2;
    const uint32_t slot = blockIdx.x * (blockDim.x >> 5) + wib;
    const uint32_t ls = search_lstride<kDim>(p);
    const size_t per_warp = search_smem_words(p.L_max, ls, p.bstride, p.hash_cap) * 4;
    unsigned char* my = g_smem + wib * per_warp;
    float* qhat = reinterpret_cast<float*>(my);
    uint32_t* win = reinterpret_cast<uint32_t*>(qhat + ls);  // window bitmap, kWinWords
    float* bd = reinterpret_cast<float*>(win + kWinWords);  // the beam: sorted (dist, id), expanded flag in the id's top bit
    uint32_t* bi = reinterpret_cast<uint32_t*>(bd + p.L_max);
    float* nd = reinterpret_cast<float*>(bi + p.L_max);
    uint32_t* ni = reinterpret_cast<uint32_t*>(nd + 64);
    float* stage = reinterpret_cast<float*>(ni + 64);  // stage_rows staged rows of max(lstride, bstride)
    const uint32_t srows = kSearchRows<kDim> ? kSearchRows<kDim> : p.stage_rows;
    uint32_t* tab = reinterpret_cast<uint32_t*>(stage + srows * (size_t)max(ls, p.bstride));
    uint64_t* bar = reinterpret_cast<uint64_t*>(tab + p.hash_cap);  // row-copy mbarrier of this warp
    uint32_t ph = 0;
    if (lane == 0) {
        tc::mbar_init(bar, 1);
        tc::fence_mbar_init();
    }
    __syncwarp();
    uint32_t* bits = p.vis_bits + (size_t)slot * p.vis_words;
    uint32_t* vlog = p.vis_log + (size_t)slot * p.log_cap;
    uint32_t* cl = p.cand_scratch + (size_t)slot * p.cand_cap;
    VisitSlot vs{bits, vlog, p.log_cap, p.vis_words};
    for (uint32_t t = lane; t < p.hash_cap; t += 32) tab[t] = kEmpty;
    for (uint32_t t = lane; t < kWinWords; t += 32) win[t] = 0u;
    __syncwarp();
    const PermOrder ord{p.perm};

    for (;;) {
        uint32_t w = 0;
        if (lane == 0) w = atomicAdd(p.work, 1u);
        w = __shfl_sync(kFull, w, 0);
        if (w >= p.nq) break;
        const uint32_t qi = p.order ? p.order[w] : w;
        const uint32_t L = min(p.qL ? p.qL[qi] : p.L_all, p.L_max);
        const uint32_t tslot = p.qslot ? p.qslot[qi] : p.slot_all;
        const float* q = p.queries + (size_t)qi * p.bstride;
        const float r2f = p.ip ? p.qR2f[qi] : p.R2f;
        // query lift, rknn_query.cpp:2724-2729 (in the rows' column order)
        for (uint32_t j = lane; j < ls; j += 32) {
            float v = 0.0f;
            if (j < p.d) v = __double2float_rn(__dmul_rn((double)q[j], p.scale));
            else if (j == p.d) v = 1.0f;
            qhat[kDim == kColsDim ? chunk_col_pos(j, kColsDim / 16 * 16) : j] = v;
        }
        __syncwarp();
        uint32_t ep = p.entry[qi];
        if (ep >= p.n) ep = 0;
        // the window of ids around the entry object
        uint32_t wbase = ep > kWinBits / 2 ? ep - kWinBits / 2 : 0u;
        if (p.n <= kWinBits) wbase = 0;
        else if ((uint64_t)wbase > p.n - kWinBits) wbase = (uint32_t)(p.n - kWinBits);

        Visited vis{tab,  p.hash_cap, p.hash_shift, p.gtab ? p.gtab + (size_t)slot * p.gcap : nullptr,
                    p.gcap, p.gshift, bits, vlog, p.log_cap, p.hash_cap ? 0u : (p.gcap ? 1u : 2u)};
        stage_row_async(stage, p.lifted + (size_t)ep * ls, ls, lane, 32);
        cp_async_wait_all();
        // generic-proxy writes to the staging buffer (this row, the last
        // query's base rows) before the bulk copies of this query
        tc::fence_async_smem();
        __syncwarp();
        float dep;
        if constexpr (kDim == kColsDim) dep = group_l2sqr_cols<kColsDim>(stage, qhat, gt, kFull);
        else dep = group_l2sqr(stage, qhat, p.dim, gt, kFull);
        __syncwarp();
        if (lane == 0) {
            win[(ep - wbase) >> 5] |= 1u << ((ep - wbase) & 31u);  // the entry lies in the window
            bd[0] = dep;
            bi[0] = ep;
        }
        uint32_t nlog = 0, nvis = 1, ncand = 0, nexp = 0, nfl = 0;
        bool overflow = false;
        if (dep <= r2f) {
            if (lane == 0) cl[0] = ep;
            ncand = 1;
        }
        __syncwarp();
        uint32_t size = 1, cur = 0;
        // links of the next node to expand, loaded while the current merge runs
        uint32_t pre_node = kEmpty, pl0 = kEmpty, pl1 = kEmpty, pdg = 0;

        // ---- greedy beam (index.h:1613-1624), then the bounded flood
        // (index.h:1626-1638), as one loop so the expansion code exists once
        // in the kernel (instruction fetch)
        bool flood = false;
        uint32_t head = 0;
        for (;;) {
            uint32_t node, nxt = 0;
            if (!flood) {
                if (cur >= size || overflow) {
                    flood = true;
                    if (ncand > 0 && !overflow) {
                        pre_node = cl[0];
                        load_links(p, pre_node, lane, pl0, pl1, pdg);
                    }
                    continue;
                }
                node = bi[cur] & kIdMask;
                __syncwarp();
                if (lane == 0) bi[cur] = node | kExpanded;
                __syncwarp();
                nexp++;
                // entries before cur are all expanded; nxt = the next unexpanded one
                nxt = size;
                for (uint32_t s0 = cur + 1; s0 < size; s0 += 32) {
                    const uint32_t idx = s0 + lane;
                    const bool un = idx < size && !(bi[idx] & kExpanded);
                    const unsigned b = __ballot_sync(kFull, un);
                    if (b) {
                        nxt = s0 + __ffs(b) - 1;
                        break;
                    }
                }
            } else {
                if (head >= ncand || overflow) break;
                node = cl[head++];
                nfl++;
            }
            uint32_t l0, l1, dg;
            if (node == pre_node) {
                l0 = pl0;
                l1 = pl1;
                dg = pdg;
            } else {
                load_links(p, node, lane, l0, l1, dg);
            }
            // links of the likely next node, an expansion ahead of their use:
            // the old beam's next unexpanded entry (unless a fresh neighbour
            // ranks before it), or the flood's next candidate
            if (!flood && nxt < size) {
                pre_node = bi[nxt] & kIdMask;
                load_links(p, pre_node, lane, pl0, pl1, pdg);
            } else if (flood && head < ncand) {
                pre_node = cl[head];
                load_links(p, pre_node, lane, pl0, pl1, pdg);
            }
            vis_room(vis, nlog, p.degree, lane, p.err);
            const uint32_t m = expand_links<kDim>(p, l0, l1, dg, vis, nlog, ni, lane, stage, bar, win, wbase);
            nvis += m;
            uint32_t mk = 0;
            if (m != 0) {
                if (!fresh_distances<kDim>(p, qhat, ni, nd, m, stage, bar, ph, lane)) return;
                append_in_range(p, r2f, nd, ni, m, cl, ncand, overflow, lane);
                if (!flood) {
                    const bool full = size >= L;
                    mk = sort_fresh_kept<PermOrder, true>(nd, ni, m, full, full ? bd[L - 1] : 0.f,
                                                          full ? bi[L - 1] : 0u, lane, ord);
                }
            }
            if (flood) continue;
            if (mk == 0) {
                // no fresh entry enters the beam: only the cursor moves (to
                // nxt, whose links are on their way)
                cur = nxt;
                continue;
            }
            // Batch insert of the mk kept entries (sorted) into the sorted
            // beam.  Fresh entry r lands at r + (beam entries before it);
            // beam entry j at j + (fresh entries before it); only entries from
            // cn (the rank of the best fresh one) on move.
            uint32_t r0 = 0, r1 = 0;
            if (lane < mk) r0 = lower_rank(bd, bi, size, nd[lane], ni[lane], ord);
            if (lane + 32 < mk) r1 = lower_rank(bd, bi, size, nd[lane + 32], ni[lane + 32], ord);
            const uint32_t cn = __shfl_sync(kFull, r0, 0);
            const uint32_t ns = min(L, size + mk);
            // first unexpanded entry of the merged beam: the old beam's next
            // one if it ranks before every fresh entry, else the best fresh one
            const bool old_next = nxt < cn;
            const uint32_t nc = old_next ? nxt : cn;
            if (!old_next) {
                pre_node = ni[0];
                load_links(p, pre_node, lane, pl0, pl1, pdg);
            }
            __syncwarp();
            // move beam entries [cn, size) right, highest first, so no entry is
            // overwritten before it is read
            for (uint32_t hi = size; hi > cn; hi = hi > cn + 32 ? hi - 32 : cn) {
                const uint32_t j = hi - 1 - lane;
                const bool mv = lane < hi - cn;
                float dv = 0.f;
                uint32_t iv = 0, pos = ns;
                if (mv) {
                    dv = bd[j];
                    iv = bi[j];
                    pos = j + lower_rank(nd, ni, mk, dv, iv, ord);
                }
                __syncwarp();
                if (pos < ns) {
                    bd[pos] = dv;
                    bi[pos] = iv;
                }
                __syncwarp();
            }
            if (lane < mk && lane + r0 < ns) {
                bd[lane + r0] = nd[lane];
                bi[lane + r0] = ni[lane];
            }
            if (lane + 32 < mk && lane + 32 + r1 < ns) {
                bd[lane + 32 + r1] = nd[lane + 32];
                bi[lane + 32 + r1] = ni[lane + 32];
            }
            __syncwarp();
            size = ns;
            cur = nc;
        }

        if (overflow && lane == 0) set_error(p.err, kDevCandOverflow);

        // ---- candidates out (optional), then the postfilter
        unsigned long long cat = 0;
        if (p.keep_cand) {
            if (lane == 0) {
                cat = atomicAdd(&p.fill[1], (unsigned long long)ncand);
                if (cat + ncand > p.cand_out_cap) set_error(p.err, kDevOutOverflow);
            }
            cat = __shfl_sync(kFull, cat, 0);
            if (cat + ncand <= p.cand_out_cap)
                for (uint32_t i = lane; i < ncand; i += 32) p.cand_buf[cat + i] = p.perm[cl[i]];
            __syncwarp();
        }
        // rknn_query.cpp:2555-2561: key = IP(o,o) + IP(q,q) - 2 IP(o,q) <= (double) thr[o];
        // the ip metric's key is -IP(o,q)
        const float qn = group_ip(q, q, p.d, gt, kFull);
        const float* thr = p.thr + (size_t)tslot * p.n;
        uint32_t npred = 0;
        // base rows in rounds of prow (the candidate tile), G = 32 / prow threads per row
        const uint32_t prow = min(p.post_rows, srows);
        const uint32_t G = prow == 8 ? 4u : (prow == 4 ? 8u : 16u);
        const uint32_t pg = prow == 8 ? lane >> 2 : (prow == 4 ? lane >> 3 : lane >> 4), pt = lane & (G - 1);
        float* brow = stage + (size_t)pg * max(ls, p.bstride);
        for (uint32_t r0 = 0; r0 < ncand; r0 += prow) {
            const uint32_t idx = r0 + pg;
            const bool ok = idx < ncand;
            const uint32_t o = cl[ok ? idx : r0];
            if (ok) stage_row_async(brow, p.base + (size_t)o * p.bstride, p.bstride, pt, G);
            cp_async_wait_all();
            __syncwarp();
            const float* rr = ok ? brow : stage;
            const float ip = G == 4 ? group_ip(rr, q, p.d, pt, kFull)
                                    : (G == 8 ? group_ip_w<8>(rr, q, p.d, pt, kFull)
                                              : group_ip_w<16>(rr, q, p.d, pt, kFull));
            const float key = p.ip ? -ip : __fsub_rn(__fadd_rn(p.onorm[o], qn), __fmul_rn(2.0f, ip));
            const bool pass = ok && key <= thr[o];  // (double) of both sides in the reference: same order
            const unsigned b = __ballot_sync(kFull, pass && pt == 0);
            __syncwarp();
            if (pass && pt == 0) cl[npred + __popc(b & lanemask_lt())] = o;
            npred += __popc(b);
            __syncwarp();
        }
        unsigned long long at = 0;
        if (lane == 0) {
            at = atomicAdd(&p.fill[0], (unsigned long long)npred);
            if (at + npred > p.pred_cap) set_error(p.err, kDevOutOverflow);
            p.npred[qi] = npred;
            p.ncand[qi] = ncand;
            p.ndist[qi] = nvis;
            p.nexp[qi] = nexp;
            p.nflood[qi] = nfl;
            p.pred_at[qi] = at;
            p.cand_at[qi] = cat;
        }
        at = __shfl_sync(kFull, at, 0);
        if (at + npred <= p.pred_cap)
            for (uint32_t i = lane; i < npred; i += 32) p.pred_buf[at + i] = p.perm[cl[i]];
        vis_release(vis, vs, nlog, lane);
        for (uint32_t t = lane; t < p.hash_cap; t += 32) tab[t] = kEmpty;
        for (uint32_t t = lane; t < kWinWords; t += 32) win[t] = 0u;
        __syncwarp();
    }
}

// Query lift and RP-tree entry (rknn_query.cpp:2724-2729, rptrees.h:108-124;
// |margin| <= EPS goes left): every 4-lane group of a warp descends for its
// own query (qpw queries per warp, 8 unless the rows are long), staging each
// hyperplane with cp.async and reducing in the reference's lane order.
// Writes the entry object and the leaf node reached; the leaf orders the
// search's work list.
__global__ void __launch_bounds__(128) rknn_entry_kernel(SearchParams p, uint32_t* __restrict__ enode,
                                                         uint32_t* __restrict__ entry, uint32_t qpw) {
    const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5, gt = lane & 3u, gw = lane >> 2;
    float* qhat = reinterpret_cast<float*>(g_smem) + ((size_t)wib * qpw + (gw < qpw ? gw : 0)) * 2 * p.lstride;
    float* stage = qhat + p.lstride;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t q0 = (blockIdx.x * (blockDim.x >> 5) + wib) * qpw; q0 < p.nq; q0 += warps * qpw) {
        const uint32_t qi = q0 + gw;
        const bool ok = gw < qpw && qi < p.nq;
        if (ok) {
            const float* q = p.queries + (size_t)qi * p.bstride;
            for (uint32_t j = gt; j < p.lstride; j += 4) {
                float v = 0.0f;
                if (j < p.d) v = __double2float_rn(__dmul_rn((double)q[j], p.scale));
                else if (j == p.d) v = 1.0f;
                qhat[j] = v;
            }
        }
        __syncwarp();
        uint32_t v = p.troot;
        bool done = !ok;
        for (uint32_t depth = 0; depth < 4096; depth++) {
            if (!done && p.tleft[v] == kEmpty) done = true;
            if (__all_sync(kFull, done)) break;
            if (!done) stage_row_async(stage, p.thyper + (size_t)v * p.lstride, p.lstride, gt, 4);
            cp_async_wait_all();
            __syncwarp();
            const float ip = group_ip(done ? qhat : stage, qhat, p.dim, gt, kFull);
            __syncwarp();
            if (!done) {
                const float margin = __fsub_rn(ip, p.toffset[v]);
                v = (margin < -kSplitEps) ? p.tleft[v] : (margin > kSplitEps ? p.tright[v] : p.tleft[v]);
            }
        }
        if (ok && gt == 0) {
            uint32_t ep = p.tleaf[v];
            if (ep == kEmpty || ep >= p.n) ep = 0;
            entry[qi] = ep;
            enode[qi] = v;
            if (p.ip) {
                // rknn_query.cpp:2724-2729: qn2s sums (q_j s)^2 in index order in
                // double (multiply, then add); R2 = qn2s + 1 + M*^2
                const float* q = p.queries + (size_t)qi * p.bstride;
                double qn2s = 0.0;
                for (uint32_t j = 0; j < p.d; j++) {
                    const double t = __dmul_rn((double)q[j], p.scale);
                    qn2s = __dadd_rn(qn2s, __dmul_rn(t, t));
                }
                p.qR2f[qi] = __double2float_rd(__dadd_rn(__dadd_rn(qn2s, 1.0), p.mstar2));
            }
        }
        __syncwarp();
    }
}

// Counting sort of the queries by entry leaf: queries that start in the same
// leaf run at about the same time and share the rows they fetch in L2.  The
// order inside a leaf is arbitrary; it changes scheduling, not results.
__global__ void leaf_count_kernel(const uint32_t* __restrict__ enode, uint32_t nq, uint32_t* __restrict__ cnt) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += gridDim.x * blockDim.x)
        atomicAdd(cnt + enode[q], 1u);
}

__global__ void leaf_scatter_kernel(const uint32_t* __restrict__ enode, uint32_t nq, uint32_t* __restrict__ cursor,
                                    uint32_t* __restrict__ order) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += gridDim.x * blockDim.x)
        order[atomicAdd(cursor + enode[q], 1u)] = q;
}

// Exclusive scan of counts (nq) into off (nq + 1), one block of 1024 threads:
// tiles of 4,096 counts, 4 consecutive per thread, warp-shuffle scans.
__global__ void __launch_bounds__(1024) scan_counts_kernel(const uint32_t* __restrict__ cnt, uint32_t nq,
                                                           uint32_t* __restrict__ off) {
    __shared__ uint32_t wsum[32];
    const uint32_t t = threadIdx.x, lane = t & 31u, w = t >> 5;
    uint32_t carry = 0;
    for (uint32_t base = 0; base < nq; base += 4096) {
        uint32_t v[4], loc[4], s0 = 0;
#pragma unroll
        for (uint32_t k = 0; k < 4; k++) {
            const uint32_t idx = base + 4 * t + k;
            v[k] = idx < nq ? cnt[idx] : 0u;
            loc[k] = s0;
            s0 += v[k];
        }
        uint32_t x = s0;  // inclusive scan over the warp
#pragma unroll
        for (uint32_t o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[w] = x;
        __syncthreads();
        if (w == 0) {
            uint32_t z = wsum[lane];
#pragma unroll
            for (uint32_t o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, z, o);
                if (lane >= o) z += y;
            }
            wsum[lane] = z;
        }
        __syncthreads();
        const uint32_t pre = carry + (w ? wsum[w - 1] : 0u) + x - s0;
#pragma unroll
        for (uint32_t k = 0; k < 4; k++) {
            const uint32_t idx = base + 4 * t + k;
            if (idx < nq) off[idx] = pre + loc[k];
        }
        carry += wsum[31];
        __syncthreads();
    }
    if (t == 0) off[nq] = carry;
}

__global__ void gather_csr_kernel(const uint32_t* __restrict__ src, const unsigned long long* __restrict__ at,
                                  const uint32_t* __restrict__ off, uint32_t nq, uint32_t* __restrict__ dst) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t q = w; q < nq; q += nw) {
        const uint32_t c = off[q + 1] - off[q];
        const unsigned long long s = at[q];
        for (uint32_t i = lane; i < c; i += 32) dst[off[q] + i] = src[s + i];
    }
}

// Per query recall / precision / candidate recall (rknn_query.cpp:2784-2799);
// gt ids are sorted ascending per query for binary search.
__global__ void evaluate_kernel(const uint32_t* __restrict__ pred_off, const uint32_t* __restrict__ pred,
                                const uint32_t* __restrict__ cand_off, const uint32_t* __restrict__ cand,
                                const uint32_t* __restrict__ gt_off, const uint32_t* __restrict__ gt_sorted,
                                uint32_t nq, double* __restrict__ out /* nq x 3, NaN for empty truth */) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t q = w; q < nq; q += nw) {
        const uint32_t* g = gt_sorted + gt_off[q];
        const uint32_t ng = gt_off[q + 1] - gt_off[q];
        auto member = [&](uint32_t id) {
            uint32_t lo = 0, hi = ng;
            while (lo < hi) {
                uint32_t mid = (lo + hi) >> 1;
                if (g[mid] < id) lo = mid + 1;
                else hi = mid;
            }
            return lo < ng && g[lo] == id;
        };
        uint32_t hit = 0, chit = 0;
        const uint32_t np = pred_off[q + 1] - pred_off[q];
        for (uint32_t i = lane; i < np; i += 32) hit += member(pred[pred_off[q] + i]);
        uint32_t nc = 0;
        if (cand) {
            nc = cand_off[q + 1] - cand_off[q];
            for (uint32_t i = lane; i < nc; i += 32) chit += member(cand[cand_off[q] + i]);
        }
        for (int o = 16; o > 0; o >>= 1) {
            hit += __shfl_xor_sync(kFull, hit, o);
            chit += __shfl_xor_sync(kFull, chit, o);
        }
        if (lane == 0) {
            double nan = __longlong_as_double(0x7ff8000000000000ull);
            if (ng == 0) {
                out[3 * (size_t)q] = nan;
                out[3 * (size_t)q + 1] = nan;
                out[3 * (size_t)q + 2] = nan;
            } else {
                out[3 * (size_t)q] = (double)hit / ng;
                out[3 * (size_t)q + 1] = np == 0 ? 1.0 : (double)hit / np;
                out[3 * (size_t)q + 2] = (double)chit / ng;
            }
        }
    }
}

// Sums of the per-query metrics over queries with non-empty truth, in a fixed
// order (thread t owns a contiguous range; thread 0 adds the partials in t
// order), so the result does not depend on scheduling.  out: recall,
// precision, F1, candidate recall, |C|, |P|, graph distances, count.
__global__ void eval_sums_kernel(const double* __restrict__ rows, const uint32_t* __restrict__ npred,
                                 const uint32_t* __restrict__ ncand, const uint32_t* __restrict__ ndist,
                                 uint32_t nq, double* __restrict__ out) {
    __shared__ double part[256][8];
    const uint32_t t = threadIdx.x, T = blockDim.x;
    const uint32_t chunk = (nq + T - 1) / T;
    const uint32_t b = min(nq, t * chunk), e = min(nq, b + chunk);
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (uint32_t q = b; q < e; q++) {
        const double r = rows[3 * (size_t)q], p = rows[3 * (size_t)q + 1];
        if (r != r) continue;
        acc[0] += r;
        acc[1] += p;
        acc[2] += (r + p > 0.0) ? 2.0 * r * p / (r + p) : 0.0;
        acc[3] += rows[3 * (size_t)q + 2];
        acc[4] += (double)ncand[q];
        acc[5] += (double)npred[q];
        acc[6] += (double)ndist[q];
        acc[7] += 1.0;
    }
    for (int j = 0; j < 8; j++) part[t][j] = acc[j];
    __syncthreads();
    if (t == 0) {
        double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (uint32_t i = 0; i < T; i++)
            for (int j = 0; j < 8; j++) s[j] += part[i][j];
        for (int j = 0; j < 8; j++) out[j] = s[j];
    }
}

// dst[i] = src[perm[i]] for rows of `stride` floats (warp per row).
// With cols_full > 0, each row's first cols_full elements are stored in chunk
// column order (common.cuh).
__global__ void permute_rows_kernel(const float* __restrict__ src, float* __restrict__ dst,
                                    const uint32_t* __restrict__ perm, uint64_t n, uint32_t stride,
                                    uint32_t cols_full) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t w0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = w0; i < n; i += nw) {
        const float* s = src + (uint64_t)perm[i] * stride;
        if (cols_full) {
            for (uint32_t t = lane; t < stride; t += 32) dst[i * stride + t] = s[chunk_col_pos(t, cols_full)];
            continue;
        }
        const float4* s4 = reinterpret_cast<const float4*>(s);
        float4* d4 = reinterpret_cast<float4*>(dst + i * stride);
        for (uint32_t t = lane; t < stride / 4; t += 32) d4[t] = s4[t];
    }
}

// dst[i] = src[perm[i]] for one value per object.
__global__ void permute_vals_kernel(const float* __restrict__ src, float* __restrict__ dst,
                                    const uint32_t* __restrict__ perm, uint64_t n) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        dst[i] = src[perm[i]];
}

static int slot_for_k(Ctx* c, uint32_t k) {
    for (int s = 0; s < Ctx::kThrSlots; s++)
        if (c->thr_k[s] == k) return s;
    return -1;
}

static int claim_slot(Ctx* c, uint32_t k) {
    int s = slot_for_k(c, k);
    if (s >= 0) return s;
    for (s = 0; s < Ctx::kThrSlots; s++)
        if (c->thr_k[s] == 0) return s;
    return 0;  // evict slot 0
}

static int ensure_thr_table(Ctx* c, uint64_t n) {
    if (c->thr_n != n) {
        for (int s = 0; s < Ctx::kThrSlots; s++) c->thr_k[s] = 0;
        c->thr_n = n;
    }
    return ensure(c, c->thr_table, (size_t)Ctx::kThrSlots * n * 4);
}

static size_t search_smem_per_warp(const Ctx* c, uint32_t L_max, uint32_t hash_cap) {
    return search_smem_words(L_max, c->ix.lstride, c->ix.bstride, hash_cap) * 4;
}

using SearchKernel = void (*)(SearchParams);

// The search kernel for lifted dimension dim (130, d = 128, has its distance
// loops unrolled at compile time) and block shape wpb.
template <uint32_t kDim>
static SearchKernel search_kernel_wpb(uint32_t wpb) {
    return wpb == 2 ? rknn_search_kernel<kDim, 2> : (wpb == 8 ? rknn_search_kernel<kDim, 8> : rknn_search_kernel<kDim, 4>);
}
static SearchKernel search_kernel_for(uint32_t dim, uint32_t wpb) {
    return dim == kColsDim ? search_kernel_wpb<kColsDim>(wpb) : search_kernel_wpb<0>(wpb);
}

// One launch configuration of the search: the visited-set sizes, the block
// shape (warps per block) and the postfilter's candidate tile (base rows per
// round).  The autotuner times the candidates per batch shape.
struct SearchCfg {
    uint32_t hash_cap = 0;  // shared-memory table entries per warp
    uint32_t gcap = 0;      // global (L2-resident) table entries per warp
    uint32_t wpb = 4;       // warps per block
    uint32_t post_rows = 8; // candidate tile
    uint32_t blocks = 0;
    size_t smem = 0;
    uint64_t code() const { return hash_cap | (uint64_t)gcap << 24 | (uint64_t)wpb << 48 | (uint64_t)post_rows << 56; }
};

static int search_cfg(Ctx* c, uint32_t hash_cap, uint32_t gcap, uint32_t wpb, uint32_t post_rows, SearchCfg& cfg) {
    const Batch& b = c->batch;
    cfg.hash_cap = hash_cap;
    cfg.gcap = gcap;
    cfg.wpb = wpb;
    cfg.post_rows = std::min(post_rows, stage_rows_for(c->ix.lstride, c->ix.bstride));
    cfg.smem = search_smem_per_warp(c, b.L_max, hash_cap) * wpb;
    if (cfg.smem > 227 * 1024) return ANQI_ERR_ARGS;
    auto kern = search_kernel_for(c->ix.dim, wpb);
    ANQI_CUDA(c, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cfg.smem));
    int per_sm = 0;
    ANQI_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * wpb, cfg.smem));
    if (per_sm < 1) return ANQI_ERR_ARGS;
    cfg.blocks = std::min<uint32_t>((uint32_t)per_sm * c->sm_count, (b.nq + wpb - 1) / wpb);
    return ANQI_OK;
}

}  // namespace anqi

using namespace anqi;

extern "C" {

int anqi_index_load(anqi_ctx* h, const anqi_index_desc* x) {
    if (!h || !x || !x->base || !x->lifted || !x->deg || !x->links || !x->tree_left || !x->tree_right ||
        !x->tree_offset || !x->tree_hyperplane || !x->tree_leaf_first || x->n == 0 || x->d == 0 ||
        x->degree == 0 || x->tree_nodes == 0)
        return h ? fail(&h->c, ANQI_ERR_ARGS, "anqi_index_load: missing or empty argument") : ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    if (x->degree > 64) return fail(c, ANQI_ERR_ARGS, "graph degree %u > 64 is not supported", x->degree);
    if (x->n >= 0x7FFFFFFFull) return fail(c, ANQI_ERR_ARGS, "n must be < 2^31");
    if (x->metric > ANQI_METRIC_IP) return fail(c, ANQI_ERR_ARGS, "unknown metric %u", x->metric);
    // index.h:1840-1861 validation: degrees and neighbour ids in range
    for (uint64_t i = 0; i < x->n; i++) {
        if (x->deg[i] > x->degree) return fail(c, ANQI_ERR_FORMAT, "invalid adjacency data: deg[%llu]", (unsigned long long)i);
        const uint32_t* lk = x->links + i * x->degree;
        for (uint32_t j = 0; j < x->deg[i]; j++)
            if (lk[j] >= x->n) return fail(c, ANQI_ERR_FORMAT, "invalid neighbor id in graph row %llu", (unsigned long long)i);
    }
    for (uint32_t v = 0; v < x->tree_nodes; v++) {
        const bool leaf = x->tree_left[v] == ANQI_EMPTY;
        if (!leaf && (x->tree_left[v] >= x->tree_nodes || x->tree_right[v] >= x->tree_nodes))
            return fail(c, ANQI_ERR_FORMAT, "invalid RP tree node %u", v);
    }
    QueryIndex& ix = c->ix;
    ix.loaded = false;
    ix.n = x->n;
    ix.d = x->d;
    ix.dim = x->d + 2;
    ix.degree = x->degree;
    ix.bstride = round_up(x->d, 8);
    ix.lstride = round_up(x->d + 2, 8);
    ix.tree_nodes = x->tree_nodes;
    ix.troot = x->tree_nodes - 1;
    ix.metric = x->metric;
    ix.scale = x->scale;
    ix.mstar2 = x->mstar2;
    int rc;
    // Renumber the objects in breadth-first order of the graph (from object 0,
    // then from the smallest object not reached): a search's visits then fall
    // on nearby numbers, which the search kernel's window bitmap exploits.
    // ANQI_B200_RENUMBER=0 keeps the given order.
    const uint64_t n = x->n;
    std::vector<uint32_t> perm;
    perm.reserve(n);
    const char* ren = std::getenv("ANQI_B200_RENUMBER");
    if (ren && ren[0] == '0') {
        for (uint64_t i = 0; i < n; i++) perm.push_back((uint32_t)i);
    } else {
        std::vector<uint8_t> seen(n, 0);
        uint64_t head = 0;
        for (uint64_t s0 = 0; s0 < n; s0++) {
            if (seen[s0]) continue;
            seen[s0] = 1;
            perm.push_back((uint32_t)s0);
            while (head < perm.size()) {
                const uint32_t u = perm[head++];
                const uint32_t* lk = x->links + (uint64_t)u * x->degree;
                for (uint32_t j = 0; j < x->deg[u]; j++)
                    if (!seen[lk[j]]) {
                        seen[lk[j]] = 1;
                        perm.push_back(lk[j]);
                    }
            }
        }
    }
    // 64 padding entries: the search loads link slots 0..63 of a row whatever its degree
    std::vector<uint32_t> rank(n), deg_r(n), links_r(n * (size_t)x->degree + 64, kEmpty), leaf_r(x->tree_leaf_first,
                                                                                         x->tree_leaf_first + x->tree_nodes);
    for (uint64_t i = 0; i < n; i++) rank[perm[i]] = (uint32_t)i;
    for (uint64_t i = 0; i < n; i++) {
        const uint32_t o = perm[i];
        deg_r[i] = x->deg[o];
        const uint32_t* lk = x->links + (uint64_t)o * x->degree;
        for (uint32_t j = 0; j < x->deg[o]; j++) links_r[i * x->degree + j] = rank[lk[j]];
    }
    for (uint32_t& e : leaf_r)
        if (e < n) e = rank[e];
    {
        TmpBuf tb(c), tl(c);
        if ((rc = upload_padded(c, tb, x->base, n, x->d, ix.bstride)) ||
            (rc = upload_padded(c, tl, x->lifted, n, ix.dim, ix.lstride)) || (rc = h2d(c, ix.perm, perm.data(), n * 4)) ||
            (rc = ensure(c, ix.base, n * (size_t)ix.bstride * 4)) || (rc = ensure(c, ix.lifted, n * (size_t)ix.lstride * 4)))
            return rc;
        const uint32_t blocks = c->sm_count * 8;
        permute_rows_kernel<<<blocks, 256, 0, c->stream>>>(tb.as<float>(), ix.base.as<float>(), ix.perm.as<uint32_t>(),
                                                           n, ix.bstride, 0u);
        // the d = 128 search instance reads its lifted rows in chunk column order
        permute_rows_kernel<<<blocks, 256, 0, c->stream>>>(tl.as<float>(), ix.lifted.as<float>(),
                                                           ix.perm.as<uint32_t>(), n, ix.lstride,
                                                           ix.dim == kColsDim ? kColsDim / 16 * 16 : 0u);
        ANQI_CUDA(c, cudaGetLastError());
        if ((rc = sync(c))) return rc;
    }
    if ((rc = ensure(c, ix.onorm, n * 4)) || (rc = h2d(c, ix.deg, deg_r.data(), n * 4)) ||
        (rc = h2d(c, ix.links, links_r.data(), links_r.size() * 4)) ||
        (rc = h2d(c, ix.tleft, x->tree_left, x->tree_nodes * 4)) ||
        (rc = h2d(c, ix.tright, x->tree_right, x->tree_nodes * 4)) ||
        (rc = h2d(c, ix.toffset, x->tree_offset, x->tree_nodes * 4)) ||
        (rc = upload_padded(c, ix.thyper, x->tree_hyperplane, x->tree_nodes, ix.dim, ix.lstride)) ||
        (rc = h2d(c, ix.tleaf, leaf_r.data(), x->tree_nodes * 4)))
        return rc;
    if ((rc = compute_norms_device(c, ix.base.as<float>(), x->n, x->d, ix.bstride, ix.onorm.as<float>()))) return rc;
    if ((rc = sync(c))) return rc;
    for (int s = 0; s < Ctx::kThrSlots; s++) c->thr_k[s] = 0;
    ix.loaded = true;
    return ANQI_OK;
}

int anqi_set_thresholds(anqi_ctx* h, uint32_t k, const float* thr) {
    if (!h || !thr || k == 0) return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    if (!c->ix.loaded) return fail(c, ANQI_ERR_ARGS, "anqi_set_thresholds: no index loaded");
    int rc = ensure_thr_table(c, c->ix.n);
    if (rc) return rc;
    const int s = claim_slot(c, k);
    // stored by object number (objects are renumbered)
    TmpBuf t(c);
    if ((rc = h2d(c, t, thr, c->ix.n * 4))) return rc;
    permute_vals_kernel<<<c->sm_count * 8, 256, 0, c->stream>>>(t.as<float>(), c->thr_table.as<float>() + (size_t)s * c->ix.n,
                                                               c->ix.perm.as<uint32_t>(), c->ix.n);
    ANQI_CUDA(c, cudaGetLastError());
    if ((rc = sync(c))) return rc;
    c->thr_k[s] = k;
    return ANQI_OK;
}

int anqi_verifier_materialize(anqi_ctx* h, uint32_t k, double radius_scale) {
    if (!h || k == 0) return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    if (!c->vf.loaded) return fail(c, ANQI_ERR_ARGS, "anqi_verifier_materialize: no verifier loaded");
    if (k > c->vf.nk) return fail(c, ANQI_ERR_ARGS, "LRQ verifier is not ready for k=%u", k);
    if (!c->ix.loaded || c->ix.n != c->vf.n)
        return fail(c, ANQI_ERR_ARGS, "anqi_verifier_materialize: verifier and index sizes differ");
    int rc = ensure_thr_table(c, c->ix.n);
    if (rc) return rc;
    const int s = claim_slot(c, k);
    c->thr_k[s] = 0;
    TmpBuf t(c);
    if ((rc = ensure(c, t, c->ix.n * 4)) || (rc = lrq_materialize_device(c, c->vf, k, radius_scale, t.as<float>())))
        return rc;
    permute_vals_kernel<<<c->sm_count * 8, 256, 0, c->stream>>>(t.as<float>(), c->thr_table.as<float>() + (size_t)s * c->ix.n,
                                                               c->ix.perm.as<uint32_t>(), c->ix.n);
    ANQI_CUDA(c, cudaGetLastError());
    if ((rc = sync(c))) return rc;
    c->thr_k[s] = k;
    return ANQI_OK;
}

}  // extern "C"

// The upload; with sync_after false the copies may still be in flight from
// the caller's buffers on return (anqi_rknn_query, which synchronizes before
// it returns).
static int query_upload(anqi_ctx* h, const float* queries, uint32_t nq, const uint32_t* k_per_query, uint32_t k_all,
                        const uint32_t* L_per_query, uint32_t L_all, bool sync_after) {
    if (!h || !queries || nq == 0) return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    if (!c->ix.loaded) return fail(c, ANQI_ERR_ARGS, "anqi_query_upload: no index loaded");
    Batch& b = c->batch;
    b.nq = nq;
    b.have_results = false;
    c->gt_nq = 0;  // a resident ground truth belongs to the previous batch
    std::vector<uint8_t> slots;
    uint32_t slot_all = 0;
    if (k_per_query) {
        slots.resize(nq);
        uint32_t last_k = 0;
        int last_s = -1;  // slot of last_k (batches hold runs of equal k)
        for (uint32_t i = 0; i < nq; i++) {
            if (last_s < 0 || k_per_query[i] != last_k) {
                last_k = k_per_query[i];
                last_s = slot_for_k(c, last_k);
                if (last_s < 0) return fail(c, ANQI_ERR_ARGS, "no thresholds materialized for k=%u", last_k);
            }
            slots[i] = (uint8_t)last_s;
        }
    } else {
        int s = slot_for_k(c, k_all);
        if (s < 0) return fail(c, ANQI_ERR_ARGS, "no thresholds materialized for k=%u", k_all);
        slot_all = (uint32_t)s;
    }
    uint32_t L_max = L_all;
    bool L_zero = false;
    if (L_per_query) {
        L_max = 0;
        for (uint32_t i = 0; i < nq; i++) {
            L_max = std::max(L_max, L_per_query[i]);
            L_zero |= L_per_query[i] == 0;
        }
    }
    if (L_max == 0 || L_max > 4096) return fail(c, ANQI_ERR_ARGS, "beam width must be in [1, 4096]");
    if (L_zero) return fail(c, ANQI_ERR_ARGS, "beam width must be positive");
    b.L_max = round_up(L_max, 4);
    b.has_k = k_per_query != nullptr;
    b.has_L = L_per_query != nullptr;
    b.k_all = slot_all;
    b.L_all = L_all;
    int rc;
    if ((rc = upload_padded(c, b.q, queries, nq, c->ix.d, c->ix.bstride))) return rc;
    if (b.has_k && (rc = h2d(c, b.qslot, slots.data(), nq))) return rc;
    if (b.has_L && (rc = h2d(c, b.qL, L_per_query, nq * 4ull))) return rc;
    const size_t q4 = (size_t)nq * 4, q8 = (size_t)nq * 8;
    if ((rc = ensure(c, b.npred, q4)) || (rc = ensure(c, b.ncand, q4)) || (rc = ensure(c, b.ndist, q4)) ||
        (rc = ensure(c, b.nexp, q4)) || (rc = ensure(c, b.nflood, q4)) || (rc = ensure(c, b.pred_at, q8)) ||
        (rc = ensure(c, b.cand_at, q8)) || (rc = ensure(c, b.pred_off, q4 + 4)) ||
        (rc = ensure(c, b.cand_off, q4 + 4)))
        return rc;
    return sync_after ? sync(c) : ANQI_OK;
}

extern "C" int anqi_query_upload(anqi_ctx* h, const float* queries, uint32_t nq, const uint32_t* k_per_query,
                                 uint32_t k_all, const uint32_t* L_per_query, uint32_t L_all) {
    return query_upload(h, queries, nq, k_per_query, k_all, L_per_query, L_all, true);
}

extern "C" {

// Entry objects of the batch (lift + RP-tree descent) and, unless
// ANQI_B200_ORDER=0, the work list ordered by entry leaf.
static int prepare_entries(Ctx* c, bool* ordered) {
    Batch& b = c->batch;
    const QueryIndex& ix = c->ix;
    int rc;
    const uint32_t nq = b.nq;
    if ((rc = ensure(c, b.entry, nq * 4ull)) || (rc = ensure(c, b.enode, nq * 4ull)) ||
        (rc = ensure(c, b.order, nq * 4ull)) || (rc = ensure(c, b.leaf_cnt, 2 * (ix.tree_nodes + 1ull) * 4)) ||
        (ix.metric == ANQI_METRIC_IP && (rc = ensure(c, b.qr2, nq * 4ull))))
        return rc;
    SearchParams p{};
    p.queries = b.q.as<float>();
    p.nq = nq;
    p.n = ix.n;
    p.d = ix.d;
    p.dim = ix.dim;
    p.bstride = ix.bstride;
    p.lstride = ix.lstride;
    p.scale = ix.scale;
    p.tleft = ix.tleft.as<uint32_t>();
    p.tright = ix.tright.as<uint32_t>();
    p.toffset = ix.toffset.as<float>();
    p.thyper = ix.thyper.as<float>();
    p.tleaf = ix.tleaf.as<uint32_t>();
    p.troot = ix.troot;
    p.ip = ix.metric == ANQI_METRIC_IP;
    p.mstar2 = ix.mstar2;
    p.qR2f = p.ip ? b.qr2.as<float>() : nullptr;
    // 8 queries per warp (one per 4-lane group) while their rows fit 48 KB per block
    const uint32_t qpw = 4ull * 8 * 2 * ix.lstride * 4 <= 48 * 1024 ? 8u : 1u;
    const size_t smem = 4ull * qpw * 2 * ix.lstride * 4;
    if (smem > 48 * 1024)
        ANQI_CUDA(c, cudaFuncSetAttribute(rknn_entry_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const uint32_t blocks = std::min<uint32_t>(c->sm_count * 8, (nq + 4 * qpw - 1) / (4 * qpw));
    rknn_entry_kernel<<<blocks, 128, smem, c->stream>>>(p, b.enode.as<uint32_t>(), b.entry.as<uint32_t>(), qpw);
    const char* env = std::getenv("ANQI_B200_ORDER");
    *ordered = !(env && env[0] == '0');
    if (*ordered) {
        uint32_t* cnt = b.leaf_cnt.as<uint32_t>();
        uint32_t* cursor = cnt + ix.tree_nodes + 1;
        const uint32_t tb = std::min<uint32_t>(c->sm_count * 4, (nq + 255) / 256);
        ANQI_CUDA(c, cudaMemsetAsync(cnt, 0, ix.tree_nodes * 4ull, c->stream));
        leaf_count_kernel<<<tb, 256, 0, c->stream>>>(b.enode.as<uint32_t>(), nq, cnt);
        scan_counts_kernel<<<1, 1024, 0, c->stream>>>(cnt, ix.tree_nodes, cursor);
        leaf_scatter_kernel<<<tb, 256, 0, c->stream>>>(b.enode.as<uint32_t>(), nq, cursor, b.order.as<uint32_t>());
    }
    ANQI_CUDA(c, cudaGetLastError());
    return ANQI_OK;
}

// Enqueues one search launch with configuration cfg (counters cleared, CUDA
// events around the kernel) on the context's stream; no host synchronization,
// so it can be captured into a graph.
static int enqueue_search(Ctx* c, const SearchCfg& cfg, int keep_candidates, bool capturing = false) {
    Batch& b = c->batch;
    const QueryIndex& ix = c->ix;
    int rc;
    if ((rc = ensure(c, b.pred_buf, b.pred_cap * 4))) return rc;
    if (keep_candidates && (rc = ensure(c, b.cand_buf, b.cand_cap * 4))) return rc;
    ANQI_CUDA(c, cudaMemsetAsync(c->counters.p, 0, 64, c->stream));
    SearchParams p{};
    p.lifted = ix.lifted.as<float>();
    p.base = ix.base.as<float>();
    p.onorm = ix.onorm.as<float>();
    p.links = ix.links.as<uint32_t>();
    p.deg = ix.deg.as<uint32_t>();
    p.tleft = ix.tleft.as<uint32_t>();
    p.tright = ix.tright.as<uint32_t>();
    p.toffset = ix.toffset.as<float>();
    p.thyper = ix.thyper.as<float>();
    p.tleaf = ix.tleaf.as<uint32_t>();
    p.n = ix.n;
    p.dim = ix.dim;
    p.d = ix.d;
    p.lstride = ix.lstride;
    p.bstride = ix.bstride;
    p.degree = ix.degree;
    p.troot = ix.troot;
    p.stage_rows = stage_rows_for(ix.lstride, ix.bstride);
    p.scale = ix.scale;
    p.R2 = ix.mstar2 + 1.0;  // rknn_query.cpp:2729, eps = 0
    p.R2f = (float)p.R2;
    if ((double)p.R2f > p.R2) p.R2f = std::nextafter(p.R2f, -INFINITY);
    p.mstar2 = ix.mstar2;
    p.ip = ix.metric == ANQI_METRIC_IP;
    p.qR2f = p.ip ? b.qr2.as<float>() : nullptr;
    p.thr = c->thr_table.as<float>();
    p.queries = b.q.as<float>();
    p.entry = b.entry.as<uint32_t>();
    p.perm = ix.perm.as<uint32_t>();
    p.order = b.ordered ? b.order.as<uint32_t>() : nullptr;
    p.qL = b.has_L ? b.qL.as<uint32_t>() : nullptr;
    p.qslot = b.has_k ? b.qslot.as<uint8_t>() : nullptr;
    p.L_all = b.L_all;
    p.slot_all = b.k_all;
    p.nq = b.nq;
    p.L_max = b.L_max;
    p.vis_bits = c->vis_bits.as<uint32_t>();
    p.vis_words = c->vis_words;
    p.vis_log = c->vis_log.as<uint32_t>();
    p.log_cap = c->log_cap;
    p.cand_scratch = c->cand_scratch.as<uint32_t>();
    p.cand_cap = c->cand_cap;
    p.work = c->counters.as<uint32_t>();
    p.fill = reinterpret_cast<unsigned long long*>(c->counters.as<uint32_t>() + 4);
    p.pred_buf = b.pred_buf.as<uint32_t>();
    p.pred_cap = b.pred_cap;
    p.cand_buf = keep_candidates ? b.cand_buf.as<uint32_t>() : nullptr;
    p.cand_out_cap = keep_candidates ? b.cand_cap : 0;
    p.keep_cand = keep_candidates;
    p.npred = b.npred.as<uint32_t>();
    p.ncand = b.ncand.as<uint32_t>();
    p.ndist = b.ndist.as<uint32_t>();
    p.nexp = b.nexp.as<uint32_t>();
    p.nflood = b.nflood.as<uint32_t>();
    p.pred_at = b.pred_at.as<unsigned long long>();
    p.cand_at = b.cand_at.as<unsigned long long>();
    p.err = c->err.as<uint32_t>();
    p.hash_cap = cfg.hash_cap;
    p.hash_shift = cfg.hash_cap ? 32u - (uint32_t)__builtin_ctz(cfg.hash_cap) : 0u;
    p.gcap = cfg.gcap;
    p.gshift = cfg.gcap ? 32u - (uint32_t)__builtin_ctz(cfg.gcap) : 0u;
    p.gtab = cfg.gcap ? c->vis_gtab.as<uint32_t>() : nullptr;
    p.drop_row_copies = (c->inject & ANQI_FAULT_DROP_ROW_COPIES) ? 1u : 0u;
    p.post_rows = cfg.post_rows;
    auto kern = search_kernel_for(ix.dim, cfg.wpb);
    ANQI_CUDA(c, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cfg.smem));
    // in a captured graph the events become event-record nodes (so the replay
    // is timed like a plain launch)
    const unsigned ef = capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
    ANQI_CUDA(c, cudaEventRecordWithFlags(c->ev0, c->stream, ef));
    kern<<<cfg.blocks, 32 * cfg.wpb, cfg.smem, c->stream>>>(p);
    ANQI_CUDA(c, cudaGetLastError());
    ANQI_CUDA(c, cudaEventRecordWithFlags(c->ev1, c->stream, ef));
    return ANQI_OK;
}

// Reads back the output fill and the error word of the last search (one
// synchronization); ms = the search kernel's device time.  Returns
// ANQI_ERR_CAPACITY (and the needed fill) when an output buffer was too small.
static int check_search(Ctx* c, float* ms, unsigned long long* fill) {
    int rc;
    ANQI_CUDA(c, cudaMemcpyAsync(fill, c->counters.as<uint32_t>() + 4, 16, cudaMemcpyDeviceToHost, c->stream));
    uint32_t err = 0;
    ANQI_CUDA(c, cudaMemcpyAsync(&err, c->err.p, 4, cudaMemcpyDeviceToHost, c->stream));
    if ((rc = sync(c))) return rc;
    if (err == kDevOutOverflow) {
        ANQI_CUDA(c, cudaMemsetAsync(c->err.p, 0, 4, c->stream));
        return ANQI_ERR_CAPACITY;
    }
    if ((rc = check_device_error(c, "rknn search"))) return rc;
    ANQI_CUDA(c, cudaEventElapsedTime(ms, c->ev0, c->ev1));
    return ANQI_OK;
}

static int launch_search(Ctx* c, const SearchCfg& cfg, int keep_candidates, float* ms, unsigned long long* fill) {
    int rc = enqueue_search(c, cfg, keep_candidates);
    return rc ? rc : check_search(c, ms, fill);
}

// Enqueues the CSR offsets and the compaction of the last search's output.
static int enqueue_compaction(Ctx* c, int keep_candidates) {
    Batch& b = c->batch;
    scan_counts_kernel<<<1, 1024, 0, c->stream>>>(b.npred.as<uint32_t>(), b.nq, b.pred_off.as<uint32_t>());
    gather_csr_kernel<<<c->sm_count * 4, 256, 0, c->stream>>>(b.pred_buf.as<uint32_t>(),
                                                              b.pred_at.as<unsigned long long>(),
                                                              b.pred_off.as<uint32_t>(), b.nq,
                                                              b.pred_csr.as<uint32_t>());
    if (keep_candidates) {
        scan_counts_kernel<<<1, 1024, 0, c->stream>>>(b.ncand.as<uint32_t>(), b.nq, b.cand_off.as<uint32_t>());
        gather_csr_kernel<<<c->sm_count * 4, 256, 0, c->stream>>>(b.cand_buf.as<uint32_t>(),
                                                                  b.cand_at.as<unsigned long long>(),
                                                                  b.cand_off.as<uint32_t>(), b.nq,
                                                                  b.cand_csr.as<uint32_t>());
    }
    ANQI_CUDA(c, cudaGetLastError());
    return ANQI_OK;
}

}  // extern "C"

// The run; with sync_after false it returns once the last kernel is enqueued
// (the search itself is always waited for: its output sizes are checked).
static int query_run(anqi_ctx* h, int keep_candidates, anqi_query_stats* st, bool sync_after) {
    if (!h) return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    Batch& b = c->batch;
    if (!c->ix.loaded || b.nq == 0) return fail(c, ANQI_ERR_ARGS, "anqi_query_run: no index or batch");
    const QueryIndex& ix = c->ix;
    int rc;
    // candidate visited-set configurations (shared-memory entries, L2 table
    // entries); ANQI_B200_HASH="S" or "S,G" forces one of them
    const char* forced = std::getenv("ANQI_B200_HASH");
    uint32_t f_hc = 0, f_gc = 0;
    if (forced) {
        char* end = nullptr;
        f_hc = (uint32_t)std::strtoul(forced, &end, 10);
        if (end && *end == ',') f_gc = (uint32_t)std::strtoul(end + 1, nullptr, 10);
    }
    static const uint32_t kCandidates[][2] = {{0, 0},       {1024, 0},    {2048, 0},   {4096, 0}, {0, 2048},
                                                  {0, 4096},    {512, 4096},  {1024, 4096}};
    // block shapes (warps per block) and candidate tiles; ANQI_B200_SHAPE="W"
    // or "W,T" forces one
    const char* fshape = std::getenv("ANQI_B200_SHAPE");
    uint32_t f_w = 0, f_t = 0;
    if (fshape) {
        char* end = nullptr;
        f_w = (uint32_t)std::strtoul(fshape, &end, 10);
        if (end && *end == ',') f_t = (uint32_t)std::strtoul(end + 1, nullptr, 10);
    }
    static const uint32_t kShapes[][2] = {{4, 8}, {2, 8}, {8, 8}, {4, 4}, {2, 4}, {8, 4}};
    // cfgs: every (visited set, shape) candidate; the first shape is the default
    std::vector<SearchCfg> cfgs;
    for (const auto& shape : kShapes) {
        if (fshape && (shape[0] != f_w || (f_t && shape[1] != f_t))) continue;
        for (const auto& cand : kCandidates) {
            if (forced && (cand[0] != f_hc || cand[1] != f_gc)) continue;
            if (!forced && cand[0] == 4096) continue;  // measured slower everywhere (occupancy); kept forcible
            if (cand[1] && (uint64_t)cand[1] / 8 * 5 > std::min<uint64_t>(ix.n, 16384)) continue;  // log must cover it
            SearchCfg g;
            if (search_cfg(c, cand[0], cand[1], shape[0], shape[1], g) == ANQI_OK) cfgs.push_back(g);
        }
    }
    if (cfgs.empty()) return fail(c, ANQI_ERR_ARGS, "beam width %u needs too much shared memory", b.L_max);
    uint32_t slots = 0, gslots = 0, gcap_max = 0;
    for (const SearchCfg& g : cfgs) {
        slots = std::max(slots, g.blocks * g.wpb);
        if (g.gcap) gslots = std::max(gslots, g.blocks * g.wpb);
        gcap_max = std::max(gcap_max, g.gcap);
    }
    // per-slot L2-resident tables, ANQI_EMPTY between queries
    if (gcap_max && (c->gtab_slots < gslots || c->gtab_cap < gcap_max)) {
        const size_t bytes = (size_t)gslots * gcap_max * 4;
        if ((rc = ensure(c, c->vis_gtab, bytes))) return rc;
        ANQI_CUDA(c, cudaMemsetAsync(c->vis_gtab.p, 0xFF, bytes, c->stream));
        c->gtab_slots = gslots;
        c->gtab_cap = gcap_max;
        c->l2_window = false;  // the tables moved: the window is set again below
    }
    // the visited tables stay in L2 while the search streams rows past them
    if (gcap_max && !c->l2_window) {
        set_l2_window(c, c->vis_gtab.p, (size_t)c->gtab_slots * c->gtab_cap * 4);
        c->l2_window = true;
    }
    // per-slot scratch (bitmap, log, candidate list) for the largest configuration
    const uint32_t words = (uint32_t)((ix.n + 31) / 32);
    const uint32_t log_cap = (uint32_t)std::min<uint64_t>(ix.n, 16384);
    const uint32_t cand_cap = (uint32_t)std::min<uint64_t>(ix.n, 65536);
    if (c->vis_slots < slots || c->vis_words != words || c->log_cap != log_cap || c->cand_cap != cand_cap) {
        if ((rc = ensure(c, c->vis_bits, (size_t)slots * words * 4)) ||
            (rc = ensure(c, c->vis_log, (size_t)slots * log_cap * 4)) ||
            (rc = ensure(c, c->cand_scratch, (size_t)slots * cand_cap * 4)))
            return rc;
        ANQI_CUDA(c, cudaMemsetAsync(c->vis_bits.p, 0, (size_t)slots * words * 4, c->stream));
        c->vis_slots = slots;
        c->vis_words = words;
        c->log_cap = log_cap;
        c->cand_cap = cand_cap;
    }
    if ((rc = prepare_entries(c, &b.ordered))) return rc;
    if (b.pred_cap == 0) b.pred_cap = std::max<uint64_t>(1024, (uint64_t)b.nq * 128);
    if (keep_candidates && b.cand_cap == 0) b.cand_cap = std::max<uint64_t>(1024, (uint64_t)b.nq * 256);
    // autotune once per (n, L_max, nq): time every configuration, keep the fastest
    const uint64_t key = ix.n * 1000003ull ^ ((uint64_t)b.L_max << 40) ^ ((uint64_t)b.nq << 20);
    SearchCfg best = cfgs[0];
    auto it = c->tuned.find(key);
    if (it != c->tuned.end()) {
        for (const SearchCfg& g : cfgs)
            if (g.code() == it->second) best = g;
    } else if (cfgs.size() > 1) {
        // coordinate descent: the visited sets at the first shape, then every
        // shape with the fastest visited set
        float best_ms = 1e30f;
        auto time_cfg = [&](const SearchCfg& g) -> int {
            float ms = 0;
            unsigned long long fill[2];
            int r = launch_search(c, g, 0, &ms, fill);
            if (r == ANQI_ERR_CAPACITY) {
                b.pred_cap = std::max<uint64_t>(b.pred_cap, fill[0] + 1024);
                r = launch_search(c, g, 0, &ms, fill);
            }
            if (r) return r;
            if (ms < best_ms) {
                best_ms = ms;
                best = g;
            }
            return ANQI_OK;
        };
        for (const SearchCfg& g : cfgs)
            if (g.wpb == cfgs[0].wpb && g.post_rows == cfgs[0].post_rows && (rc = time_cfg(g))) return rc;
        const SearchCfg vis = best;
        for (const SearchCfg& g : cfgs)
            if (g.hash_cap == vis.hash_cap && g.gcap == vis.gcap &&
                (g.wpb != cfgs[0].wpb || g.post_rows != cfgs[0].post_rows) && (rc = time_cfg(g)))
                return rc;
        c->tuned[key] = best.code();
    }
    for (int attempt = 0; attempt < 3; attempt++) {
        float ms = 0;
        unsigned long long fill[2] = {0, 0};
        rc = launch_search(c, best, keep_candidates, &ms, fill);
        if (rc == ANQI_ERR_CAPACITY) {
            b.pred_cap = std::max<uint64_t>(b.pred_cap, fill[0] + 1024);
            if (keep_candidates) b.cand_cap = std::max<uint64_t>(b.cand_cap, fill[1] + 1024);
            continue;
        }
        if (rc) return rc;
        // CSR offsets + compaction (the CSR buffers hold the whole output
        // capacity, so a replayed graph never outgrows them)
        if ((rc = ensure(c, b.pred_csr, std::max<uint64_t>(b.pred_cap, 1) * 4))) return rc;
        if (keep_candidates && (rc = ensure(c, b.cand_csr, std::max<uint64_t>(b.cand_cap, 1) * 4))) return rc;
        if ((rc = enqueue_compaction(c, keep_candidates))) return rc;
        c->last_cfg_hash = best.hash_cap;
        c->last_cfg_gcap = best.gcap;
        c->last_cfg_blocks = best.blocks;
        c->last_cfg_smem = best.smem;
        c->last_cfg_wpb = best.wpb;
        c->last_cfg_post = best.post_rows;
        b.have_results = true;
        b.have_cands = keep_candidates != 0;
        if (st) {
            st->search_ms = ms;
            st->visited_table = best.hash_cap;
            st->visited_l2_table = best.gcap;
            st->warps_per_block = best.wpb;
            st->candidate_tile = best.post_rows;
        }
        return sync_after ? sync(c) : ANQI_OK;
    }
    return fail(c, ANQI_ERR_CAPACITY, "rknn search: output capacity could not be satisfied");
}

extern "C" int anqi_query_run(anqi_ctx* h, int keep_candidates, anqi_query_stats* st) {
    return query_run(h, keep_candidates, st, true);
}

extern "C" {

// Everything a captured query graph depends on: batch shape and mode, search
// configuration, output capacities and every device buffer it touches.
static std::vector<uint64_t> query_graph_key(Ctx* c, int keep_candidates) {
    const Batch& b = c->batch;
    const QueryIndex& ix = c->ix;
    auto u = [](const void* q) { return (uint64_t)(uintptr_t)q; };
    return {b.nq, b.L_max, (uint64_t)b.has_k, (uint64_t)b.has_L, b.k_all, b.L_all, (uint64_t)keep_candidates,
            (uint64_t)b.ordered, c->last_cfg_hash, c->last_cfg_gcap, c->last_cfg_blocks, c->last_cfg_smem,
            c->last_cfg_wpb, c->last_cfg_post,
            b.pred_cap, b.cand_cap, u(b.q.p), u(b.qslot.p), u(b.qL.p), u(b.pred_buf.p), u(b.cand_buf.p),
            u(b.pred_csr.p), u(b.cand_csr.p), u(b.pred_off.p), u(b.cand_off.p), u(b.entry.p), u(b.enode.p),
            u(b.order.p), u(b.leaf_cnt.p), u(b.npred.p), u(b.ncand.p), u(b.ndist.p), u(b.nexp.p), u(b.nflood.p),
            u(b.pred_at.p), u(b.cand_at.p), u(c->vis_bits.p), u(c->vis_log.p), u(c->cand_scratch.p),
            u(c->vis_gtab.p), u(c->thr_table.p), u(c->counters.p), u(c->err.p), u(ix.lifted.p), u(ix.base.p),
            u(ix.links.p), u(ix.thyper.p), ix.n, c->vis_words, c->log_cap, c->cand_cap};
}

static void drop_query_graph(Ctx* c) {
    if (c->qgraph) cudaGraphExecDestroy(c->qgraph);
    c->qgraph = nullptr;
    c->qgraph_key.clear();
}

int anqi_query_counters(anqi_ctx* h, anqi_query_stats* st) {
    if (!h || !st) return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    Batch& b = c->batch;
    if (!b.have_results) return fail(c, ANQI_ERR_ARGS, "anqi_query_counters: no results");
    std::vector<uint32_t> v(b.nq);
    uint64_t sums[5] = {0, 0, 0, 0, 0};
    DevBuf* arr[5] = {&b.ndist, &b.nexp, &b.ncand, &b.npred, &b.nflood};
    for (int a = 0; a < 5; a++) {
        ANQI_CUDA(c, cudaMemcpyAsync(v.data(), arr[a]->p, b.nq * 4ull, cudaMemcpyDeviceToHost, c->stream));
        int rc = sync(c);
        if (rc) return rc;
        for (uint32_t x : v) sums[a] += x;
    }
    st->n_dist = sums[0];
    st->n_expand = sums[1];
    st->n_cand = sums[2];
    st->n_pred = sums[3];
    st->n_flood = sums[4];
    return ANQI_OK;
}

int anqi_query_run_graph(anqi_ctx* h, int keep_candidates, anqi_query_stats* st) {
    if (!h) return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    Batch& b = c->batch;
    if (!c->ix.loaded || b.nq == 0) return fail(c, ANQI_ERR_ARGS, "anqi_query_run_graph: no index or batch");
    int rc;
    if (c->qgraph && c->qgraph_key == query_graph_key(c, keep_candidates)) {
        ANQI_CUDA(c, cudaGraphLaunch(c->qgraph, c->stream));
        float ms = 0;
        unsigned long long fill[2] = {0, 0};
        rc = check_search(c, &ms, fill);
        if (rc == ANQI_OK) {
            b.have_results = true;
            b.have_cands = keep_candidates != 0;
            if (st) {
                st->search_ms = ms;
                st->visited_table = c->last_cfg_hash;
                st->visited_l2_table = c->last_cfg_gcap;
                st->warps_per_block = c->last_cfg_wpb;
                st->candidate_tile = c->last_cfg_post;
            }
            return ANQI_OK;
        }
        if (rc != ANQI_ERR_CAPACITY) return rc;
        drop_query_graph(c);  // outgrew the captured capacity: run the sized path, capture again
    }
    // the plain path sizes buffers, autotunes and produces this batch's results
    if ((rc = anqi_query_run(h, keep_candidates, st))) return rc;
    drop_query_graph(c);
    SearchCfg cfg;
    cfg.hash_cap = c->last_cfg_hash;
    cfg.gcap = c->last_cfg_gcap;
    cfg.blocks = c->last_cfg_blocks;
    cfg.smem = c->last_cfg_smem;
    cfg.wpb = c->last_cfg_wpb;
    cfg.post_rows = c->last_cfg_post;
    bool ordered = false;
    cudaGraph_t g = nullptr;
    ANQI_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    rc = prepare_entries(c, &ordered);
    if (!rc) rc = enqueue_search(c, cfg, keep_candidates, true);
    if (!rc) rc = enqueue_compaction(c, keep_candidates);
    const cudaError_t ce = cudaStreamEndCapture(c->stream, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (ce != cudaSuccess) return cuda_check(c, ce, "cudaStreamEndCapture");
    const cudaError_t ie = cudaGraphInstantiate(&c->qgraph, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) {
        c->qgraph = nullptr;
        return cuda_check(c, ie, "cudaGraphInstantiate");
    }
    c->qgraph_key = query_graph_key(c, keep_candidates);
    return ANQI_OK;
}

int anqi_query_download(anqi_ctx* h, uint32_t* pred_off, uint32_t* pred_ids, uint64_t pred_cap, uint32_t* cand_off,
                        uint32_t* cand_ids, uint64_t cand_cap, uint32_t* n_dist) {
    if (!h || !pred_off) return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    Batch& b = c->batch;
    if (!b.have_results) return fail(c, ANQI_ERR_ARGS, "anqi_query_download: no results");
    ANQI_CUDA(c, cudaMemcpyAsync(pred_off, b.pred_off.p, (b.nq + 1ull) * 4, cudaMemcpyDeviceToHost, c->stream));
    int rc = sync(c);
    if (rc) return rc;
    if (pred_ids && pred_off[b.nq] > pred_cap)
        return fail(c, ANQI_ERR_CAPACITY, "pred_ids needs %u entries", pred_off[b.nq]);
    if (pred_ids && pred_off[b.nq])
        ANQI_CUDA(c, cudaMemcpyAsync(pred_ids, b.pred_csr.p, pred_off[b.nq] * 4ull, cudaMemcpyDeviceToHost, c->stream));
    if (cand_off) {
        if (!b.have_cands) return fail(c, ANQI_ERR_ARGS, "candidates were not kept");
        ANQI_CUDA(c, cudaMemcpyAsync(cand_off, b.cand_off.p, (b.nq + 1ull) * 4, cudaMemcpyDeviceToHost, c->stream));
        if ((rc = sync(c))) return rc;
        if (cand_ids && cand_off[b.nq] > cand_cap)
            return fail(c, ANQI_ERR_CAPACITY, "cand_ids needs %u entries", cand_off[b.nq]);
        if (cand_ids && cand_off[b.nq])
            ANQI_CUDA(c, cudaMemcpyAsync(cand_ids, b.cand_csr.p, cand_off[b.nq] * 4ull, cudaMemcpyDeviceToHost,
                                         c->stream));
    }
    if (n_dist) ANQI_CUDA(c, cudaMemcpyAsync(n_dist, b.ndist.p, b.nq * 4ull, cudaMemcpyDeviceToHost, c->stream));
    return sync(c);
}

int anqi_rknn_query(anqi_ctx* h, const float* queries, uint32_t nq, const uint32_t* k_per_query, uint32_t k_all,
                    const uint32_t* L_per_query, uint32_t L_all, uint32_t* pred_off, uint32_t* pred_ids,
                    uint64_t pred_cap, uint32_t* cand_off, uint32_t* cand_ids, uint64_t cand_cap, uint32_t* n_dist,
                    anqi_query_stats* st) {
    if (!h) return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    ANQI_CUDA(c, cudaEventRecord(c->ev2, c->stream));
    // no host round trip between the upload, the run and the first copy back;
    // on an error the stream is drained before the caller's buffers are
    // handed back
    int rc = query_upload(h, queries, nq, k_per_query, k_all, L_per_query, L_all, false);
    if (!rc) rc = query_run(h, cand_off != nullptr, st, false);
    if (rc) {
        cudaStreamSynchronize(c->stream);
        return rc;
    }
    rc = anqi_query_download(h, pred_off, pred_ids, pred_cap, cand_off, cand_ids, cand_cap, n_dist);
    if (rc) return rc;
    ANQI_CUDA(c, cudaEventRecord(c->ev3, c->stream));
    if ((rc = sync(c))) return rc;
    if (st) {
        float ms = 0;
        ANQI_CUDA(c, cudaEventElapsedTime(&ms, c->ev2, c->ev3));
        st->total_ms = ms;
        st->h2d_bytes = (uint64_t)nq * c->ix.d * 4 + (k_per_query ? nq * 4ull : 0) + (L_per_query ? nq * 4ull : 0);
        st->d2h_bytes = (nq + 1ull) * 4 + (uint64_t)pred_off[nq] * 4 + (n_dist ? nq * 4ull : 0) +
                        (cand_off ? (nq + 1ull) * 4 + (uint64_t)cand_off[nq] * 4 : 0);
    }
    return ANQI_OK;
}

int anqi_query_evaluate(anqi_ctx* h, const uint32_t* gt_off, const uint32_t* gt_ids, uint64_t gt_total,
                        double* recall_sum, double* precision_sum, double* cand_recall_sum, uint32_t* nonempty) {
    if (!h || !gt_off) return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    Batch& b = c->batch;
    if (!b.have_results) return fail(c, ANQI_ERR_ARGS, "anqi_query_evaluate: no results");
    if (gt_off[b.nq] != gt_total) return fail(c, ANQI_ERR_ARGS, "ground-truth offsets disagree with gt_total");
    std::vector<uint32_t> sorted(gt_ids, gt_ids + gt_total);
    for (uint32_t q = 0; q < b.nq; q++) std::sort(sorted.begin() + gt_off[q], sorted.begin() + gt_off[q + 1]);
    TmpBuf doff(c), dids(c), dout(c);
    int rc;
    if ((rc = h2d(c, doff, gt_off, (b.nq + 1ull) * 4)) || (rc = h2d(c, dids, sorted.data(), gt_total * 4 + 4)) ||
        (rc = ensure(c, dout, b.nq * 24ull)))
        return rc;
    evaluate_kernel<<<c->sm_count * 4, 256, 0, c->stream>>>(
        b.pred_off.as<uint32_t>(), b.pred_csr.as<uint32_t>(), b.have_cands ? b.cand_off.as<uint32_t>() : nullptr,
        b.have_cands ? b.cand_csr.as<uint32_t>() : nullptr, doff.as<uint32_t>(), dids.as<uint32_t>(), b.nq,
        dout.as<double>());
    ANQI_CUDA(c, cudaGetLastError());
    std::vector<double> out(b.nq * 3ull);
    ANQI_CUDA(c, cudaMemcpyAsync(out.data(), dout.p, b.nq * 24ull, cudaMemcpyDeviceToHost, c->stream));
    if ((rc = sync(c))) return rc;
    double r = 0, p = 0, cr = 0;
    uint32_t ne = 0;
    for (uint32_t q = 0; q < b.nq; q++) {
        if (out[3ull * q] != out[3ull * q]) continue;
        r += out[3ull * q];
        p += out[3ull * q + 1];
        cr += out[3ull * q + 2];
        ne++;
    }
    if (recall_sum) *recall_sum = r;
    if (precision_sum) *precision_sum = p;
    if (cand_recall_sum) *cand_recall_sum = cr;
    if (nonempty) *nonempty = ne;
    return ANQI_OK;
}

int anqi_gt_load(anqi_ctx* h, const uint32_t* gt_off, const uint32_t* gt_ids, uint64_t gt_total) {
    if (!h || !gt_off || (gt_total && !gt_ids)) return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    Batch& b = c->batch;
    if (b.nq == 0) return fail(c, ANQI_ERR_ARGS, "anqi_gt_load: upload the query batch first");
    if (gt_off[0] != 0 || gt_off[b.nq] != gt_total) return fail(c, ANQI_ERR_FORMAT, "ground-truth offsets disagree");
    std::vector<uint32_t> sorted(gt_ids, gt_ids + gt_total);
    for (uint32_t q = 0; q < b.nq; q++) {
        if (gt_off[q + 1] < gt_off[q]) return fail(c, ANQI_ERR_FORMAT, "ground-truth offsets not ascending");
        std::sort(sorted.begin() + gt_off[q], sorted.begin() + gt_off[q + 1]);
    }
    int rc;
    if ((rc = h2d(c, c->gt_off, gt_off, (b.nq + 1ull) * 4)) || (rc = h2d(c, c->gt_ids, sorted.data(), gt_total * 4 + 4)) ||
        (rc = ensure(c, c->eval_rows, b.nq * 24ull)) || (rc = ensure(c, c->eval_sums, 64)))
        return rc;
    c->gt_nq = b.nq;
    return sync(c);
}

int anqi_query_evaluate_sums(anqi_ctx* h, anqi_eval_sums* out) {
    if (!h || !out) return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    Batch& b = c->batch;
    if (!b.have_results) return fail(c, ANQI_ERR_ARGS, "anqi_query_evaluate_sums: no results");
    if (c->gt_nq != b.nq || !c->gt_off.p) return fail(c, ANQI_ERR_ARGS, "anqi_query_evaluate_sums: no ground truth for this batch");
    evaluate_kernel<<<c->sm_count * 4, 256, 0, c->stream>>>(
        b.pred_off.as<uint32_t>(), b.pred_csr.as<uint32_t>(), b.have_cands ? b.cand_off.as<uint32_t>() : nullptr,
        b.have_cands ? b.cand_csr.as<uint32_t>() : nullptr, c->gt_off.as<uint32_t>(), c->gt_ids.as<uint32_t>(), b.nq,
        c->eval_rows.as<double>());
    eval_sums_kernel<<<1, 256, 0, c->stream>>>(c->eval_rows.as<double>(), b.npred.as<uint32_t>(),
                                               b.ncand.as<uint32_t>(), b.ndist.as<uint32_t>(), b.nq,
                                               c->eval_sums.as<double>());
    ANQI_CUDA(c, cudaGetLastError());
    double s[8];
    ANQI_CUDA(c, cudaMemcpyAsync(s, c->eval_sums.p, 64, cudaMemcpyDeviceToHost, c->stream));
    int rc;
    if ((rc = sync(c))) return rc;
    out->recall = s[0];
    out->precision = s[1];
    out->f1 = s[2];
    out->cand_recall = s[3];
    out->cand = s[4];
    out->pred = s[5];
    out->graph_dist = s[6];
    out->nonempty = (uint32_t)s[7];
    return ANQI_OK;
}

}  // extern "C"
