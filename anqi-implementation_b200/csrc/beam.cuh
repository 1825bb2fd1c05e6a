// Per-warp search state shared by the query and index-construction kernels:
// the three-level visited set and the in-place batch insert into a sorted
// (dist, id) beam.
#pragma once

#include "common.cuh"
#include "util.cuh"

namespace anqi {

// The visited set of one query, in up to three levels:
//   0  an open-addressing table in the warp's shared memory (atomicCAS,
//      linear probing, kept at or below 5/8 load);
//   1  a per-slot open-addressing table in global memory, small enough that
//      all slots' tables stay resident in L2 (same rules);
//   2  the per-slot bitmap over all n ids.
// Before an expansion could push the current level past its load limit, its
// ids move one level up.  The log records, per first visit, what the clean-up
// at the end of the query needs: nothing at level 0, the table position at
// level 1, the id at level 2.
struct Visited {
    uint32_t* tab;
    uint32_t cap, shift;
    uint32_t* gtab;
    uint32_t gcap, gshift;
    uint32_t* bits;
    uint32_t* vlog;
    uint32_t log_cap;
    uint32_t level;
};

// 16-byte bucket loads (shared: the warp's own table; global: bypassing L1,
// since the table is updated by atomics at L2) and the shared-memory CAS.
__device__ __forceinline__ uint4 ld_bucket_shared(const uint32_t* p) {
    uint4 v;
    asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];\n"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "r"((uint32_t)__cvta_generic_to_shared(p))
                 : "memory");
    return v;
}

__device__ __forceinline__ uint4 ld_bucket_global(const uint32_t* p) {
    uint4 v;
    asm volatile("ld.global.cg.v4.u32 {%0, %1, %2, %3}, [%4];\n"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p)
                 : "memory");
    return v;
}

__device__ __forceinline__ uint32_t cas_shared(uint32_t* p, uint32_t cmp, uint32_t val) {
    uint32_t old;
    asm volatile("atom.shared.cas.b32 %0, [%1], %2, %3;\n"
                 : "=r"(old)
                 : "r"((uint32_t)__cvta_generic_to_shared(p)), "r"(cmp), "r"(val)
                 : "memory");
    return old;
}

// Inserts id into an open-addressing table of 4-slot buckets (bucketed linear
// probing); returns true on first insertion and the slot used in pos.  A
// bucket's occupied slots are always a prefix and no entry is removed while
// the table is in use, so a bucket with a free slot ends the search: a lookup
// is one 16-byte load in the common case, and only an insertion takes an
// atomic.  A failed CAS (another lane of the warp took the slot) reads the
// bucket again.  cap is a power of two >= 8; iterations are bounded.
template <bool kShared>
__device__ __forceinline__ bool table_insert(uint32_t* t, uint32_t cap, uint32_t shift, uint32_t id, uint32_t& pos,
                                             uint32_t* err) {
    const uint32_t nb = cap >> 2;
    uint32_t b = (id * 0x9E3779B1u) >> (shift + 2);
    for (uint32_t it = 0; it < 2 * nb + 64; it++) {
        const uint4 v = kShared ? ld_bucket_shared(t + 4 * b) : ld_bucket_global(t + 4 * b);
        if (v.x == id || v.y == id || v.z == id || v.w == id) return false;
        const uint32_t e = v.x == kEmpty ? 0u : v.y == kEmpty ? 1u : v.z == kEmpty ? 2u : v.w == kEmpty ? 3u : 4u;
        if (e == 4u) {
            b = (b + 1) & (nb - 1);
            continue;
        }
        const uint32_t slot = 4 * b + e;
        const uint32_t old = kShared ? cas_shared(t + slot, kEmpty, id) : atomicCAS(t + slot, kEmpty, id);
        if (old == kEmpty) {
            pos = slot;
            return true;
        }
        if (old == id) return false;
    }
    set_error(err, kDevWaitTimeout);  // unreachable at or below 5/8 load
    return false;
}

__device__ __forceinline__ bool vis_first(Visited& v, uint32_t id, uint32_t& pos, uint32_t* err) {
    if (v.level == 0) return table_insert<true>(v.tab, v.cap, v.shift, id, pos, err);
    if (v.level == 1) return table_insert<false>(v.gtab, v.gcap, v.gshift, id, pos, err);
    pos = id;
    return visit_first(v.bits, id);
}

// Read-only probe of the visited set for id: the id's first bucket (levels 0
// and 1) or its bitmap word (level 2, in .x).  probe_found tells whether the
// probe alone shows id visited; nothing leaves the set while it is in use, so
// "found" is final, and "not found" needs vis_first.  Probes of many ids can
// be in flight at once.
__device__ __forceinline__ uint4 probe_visited(const Visited& v, uint32_t id) {
    if (v.level == 2) {
        uint32_t w;
        asm volatile("ld.global.cg.u32 %0, [%1];\n" : "=r"(w) : "l"(v.bits + (id >> 5)) : "memory");
        return make_uint4(w, 0, 0, 0);
    }
    const bool sh = v.level == 0;
    const uint32_t b = (id * 0x9E3779B1u) >> ((sh ? v.shift : v.gshift) + 2);
    return sh ? ld_bucket_shared(v.tab + 4 * b) : ld_bucket_global(v.gtab + 4 * b);
}

__device__ __forceinline__ bool probe_found(const Visited& v, const uint4& q, uint32_t id) {
    if (v.level == 2) return (q.x >> (id & 31u)) & 1u;
    return q.x == id || q.y == id || q.z == id || q.w == id;
}

// Level 0 -> 1 (gtab present) or 0 -> 2 (warp-collective); nlog entries move.
static __device__ void vis_up_from_shared(Visited& v, uint32_t lane, uint32_t* err) {
    const uint32_t to = v.gcap ? 1u : 2u;
    uint32_t pos0 = 0;
    for (uint32_t t0 = 0; t0 < v.cap; t0 += 32) {
        const uint32_t id = v.tab[t0 + lane];
        const bool has = id != kEmpty;
        uint32_t rec = id;
        if (has) {
            if (to == 1) table_insert<false>(v.gtab, v.gcap, v.gshift, id, rec, err);
            else atomicOr(v.bits + (id >> 5), 1u << (id & 31u));
        }
        const unsigned b = __ballot_sync(kAll, has);
        if (has) {
            const uint32_t at = pos0 + __popc(b & lane_lt_mask());
            if (at < v.log_cap) v.vlog[at] = rec;
        }
        pos0 += __popc(b);
    }
    __syncwarp();
    v.level = to;
}

// Level 1 -> 2 (warp-collective): positions in the log become ids.
static __device__ void vis_up_from_global(Visited& v, uint32_t nlog, uint32_t lane) {
    const uint32_t m = min(nlog, v.log_cap);
    for (uint32_t i = lane; i < m; i += 32) {
        const uint32_t pos = v.vlog[i];
        const uint32_t id = v.gtab[pos];
        v.gtab[pos] = kEmpty;
        atomicOr(v.bits + (id >> 5), 1u << (id & 31u));
        v.vlog[i] = id;
    }
    __syncwarp();
    v.level = 2;
}

// Makes room for `more` first visits: moves up while the level's limit would be passed.
__device__ __forceinline__ void vis_room(Visited& v, uint32_t nlog, uint32_t more, uint32_t lane, uint32_t* err) {
    if (v.level == 0 && nlog + more > v.cap / 8 * 5) vis_up_from_shared(v, lane, err);
    if (v.level == 1 && nlog + more > v.gcap / 8 * 5) vis_up_from_global(v, nlog, lane);
}

// End of query: leaves level 1 / 2 storage clean (the shared table is reset by the caller).
__device__ __forceinline__ void vis_release(Visited& v, const VisitSlot& vs, uint32_t nlog, uint32_t lane) {
    if (v.level == 1) {
        for (uint32_t i = lane; i < nlog; i += 32) v.gtab[v.vlog[i]] = kEmpty;
        __syncwarp();
    } else if (v.level == 2) {
        visit_clear(vs, nlog);
    }
}

// Window bitmap: when objects are numbered for locality (graph or RP-tree
// order), one search's visits fall mostly within a few thousand ids of where
// it starts.  A per-warp bitmap in shared memory covers kWinBits ids from
// wbase; visits outside it go to the visited tables.
constexpr uint32_t kWinBits = 4096;
constexpr uint32_t kWinWords = kWinBits / 32;

// Visits the links of node (slots l0 = link[lane], l1 = link[lane + 32], dg =
// degree): collects the ids seen for the first time into ni[0..m) in link-slot
// order and logs the table visits (levels 1 and 2).  The lifted rows of the first
// stage_rows of them are requested at once, one bulk copy per row into
// stage[slot], completing on bar.  Returns m.
// A first visit of id in the window bitmap (win covers [wbase, wbase +
// kWinBits)) or else in the visited tables; `logged` tells which.
__device__ __forceinline__ bool visit_id(Visited& vis, uint32_t* win, uint32_t wbase, uint32_t id, uint32_t& rec,
                                         bool& logged, uint32_t* err) {
    const uint32_t w = id - wbase;
    if (w < kWinBits) {
        logged = false;
        const uint32_t bit = 1u << (w & 31u);
        return (atomicOr(win + (w >> 5), bit) & bit) == 0u;
    }
    logged = true;
    return vis_first(vis, id, rec, err);
}

// Of the m (<= 64) fresh (dist, id) entries in nd/ni, keeps those that can
// enter the beam -- all of them while the beam is not full, else those ranking
// before its last entry (td, tid), since any other would land at rank >= L --
// and sorts them ascending into nd/ni[0..m').  Returns m'.  Small batches (the
// common case after the first expansions) are ranked by counting over the kept
// entries only; larger ones use the register bitonic network, after which the
// kept entries are a prefix.
template <class Ord = IdOrder, bool kCompact = false>
__device__ __forceinline__ uint32_t sort_fresh_kept(float* nd, uint32_t* ni, uint32_t m, bool full, float td,
                                                    uint32_t tid, uint32_t lane, Ord ord = Ord()) {
    if (m <= 32) {
        const float dv = lane < m ? nd[lane] : 0.f;
        const uint32_t iv = lane < m ? ni[lane] : kEmpty;
        const bool keep = lane < m && (!full || ord(dv, iv, td, tid));
        const unsigned km = __ballot_sync(kAll, keep);
        // rank by distance alone, counting equal distances; only kept lanes
        // use their rank
        uint32_t rank = 0, ties = 0;
        for (unsigned r = km; r; r &= r - 1) {
            const int s = __ffs(r) - 1;
            const float ds = __shfl_sync(kAll, dv, s);
            rank += ds < dv ? 1u : 0u;
            ties += (ds == dv && s != (int)lane) ? 1u : 0u;
        }
        if (__any_sync(kAll, keep && ties != 0)) {
            // two kept entries at one distance: rank by the full order
            rank = 0;
            for (unsigned r = km; r; r &= r - 1) {
                const int s = __ffs(r) - 1;
                const float ds = __shfl_sync(kAll, dv, s);
                const uint32_t is = __shfl_sync(kAll, iv, s);
                rank += (keep && ord(ds, is, dv, iv)) ? 1u : 0u;
            }
        }
        __syncwarp();
        if (keep) {
            nd[rank] = dv;
            ni[rank] = iv;
        }
        __syncwarp();
        return __popc(km);
    }
    const float inf = __int_as_float(0x7f800000);
    float d0 = lane < m ? nd[lane] : inf;
    uint32_t i0 = lane < m ? ni[lane] : kEmpty;
    float d1 = lane + 32 < m ? nd[lane + 32] : inf;
    uint32_t i1 = lane + 32 < m ? ni[lane + 32] : kEmpty;
    warp_sort64<Ord, kCompact>(d0, i0, d1, i1, ord);
    __syncwarp();
    nd[lane] = d0;
    ni[lane] = i0;
    nd[lane + 32] = d1;
    ni[lane + 32] = i1;
    const bool k0 = lane < m && (!full || ord(d0, i0, td, tid));
    const bool k1 = lane + 32 < m && (!full || ord(d1, i1, td, tid));
    const uint32_t kept = __popc(__ballot_sync(kAll, k0)) + __popc(__ballot_sync(kAll, k1));
    __syncwarp();
    return kept;
}

// Inserts the m (<= 64) fresh entries of nd/ni (any order; their ids are not
// in the beam) into the sorted beam bd/bi of `size` entries and capacity cap,
// in place: the beam becomes the cap best of the union in (dist, id) order,
// which is what inserting them one at a time by binary search
// (neighbor.h:61-111) leaves.  Fresh entry r lands at r + (beam entries before
// it), beam entry j at j + (fresh entries before it); entries before cn, the
// rank of the best kept fresh entry, do not move.  Returns cn (size when no
// fresh entry enters).  Warp-collective; nd/ni are reordered.
template <class Ord = IdOrder>
__device__ __forceinline__ uint32_t beam_insert(float* bd, uint32_t* bi, uint32_t& size, uint32_t cap, float* nd,
                                                uint32_t* ni, uint32_t m, uint32_t lane, Ord ord = Ord()) {
    if (m == 0) return size;
    const bool full = size >= cap;
    const uint32_t mk = sort_fresh_kept(nd, ni, m, full, full ? bd[cap - 1] : 0.f, full ? bi[cap - 1] : 0u, lane, ord);
    if (mk == 0) return size;
    uint32_t r0 = 0, r1 = 0;
    if (lane < mk) r0 = lower_rank(bd, bi, size, nd[lane], ni[lane], ord);
    if (lane + 32 < mk) r1 = lower_rank(bd, bi, size, nd[lane + 32], ni[lane + 32], ord);
    const uint32_t cn = __shfl_sync(kAll, r0, 0);
    const uint32_t ns = min(cap, size + mk);
    __syncwarp();
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
    return cn;
}

}  // namespace anqi
