// Edge policies of the G48 prune on the device (prune_pool_to_ids under
// ANQI_EDGE_POLICY, include/index.h:283-829).
//
// The select, commit and Vamana gathers write each row's candidate pool to a
// chunk buffer instead of pruning it (GatherParams::dump_*); this kernel then
// prunes every pool of the chunk under the policy, one warp per row:
// sort_unique_candidates, then the policy's passes (rng_extend, the ball and
// LSG orders with their occlusion tests, residual-cover edges, the
// verification-constrained bubble optimizer), each a warp-cooperative loop
// over the sorted candidates with the selection in shared memory.
//
// Arithmetic as in the reference: pair distances FP32 through the norms in the
// AVX lane order; the ball, LSG and residual keys in double, one rounding per
// operation (no fused multiply-add; the reference's keys match that form on its
// own outputs).  LSG's pow: alpha 1 is exact; other exponents use the device's
// double pow, within 2 ulp of the correctly rounded power, so two LSG keys
// closer than that may order differently from the reference's glibc pow.
#include <cfloat>

#include "common.cuh"
#include "internal.h"
#include "util.cuh"

namespace anqi {

namespace {

constexpr uint32_t kPolCover = 1, kPolBall = 2, kPolPure = 4, kPolLsg = 8, kPolAuto = 16, kPolAutoFull = 32;
constexpr uint32_t kPolWarps = 4;  // warps per block
__device__ __forceinline__ double inf_d() { return __longlong_as_double(0x7FF0000000000000ll); }

struct PolicyParams {
    const float* x;
    const float* norms;
    uint64_t n;
    uint32_t stride, dim, M;
    float alpha;
    DevPolicyView pol;
    // the chunk's pools: entry t at pool_d / pool_i [t * pool_cap ..], pool_n[t] entries
    const float* pool_d;
    const uint32_t* pool_i;
    const uint32_t* pool_n;
    uint32_t pool_cap;
    const uint32_t* rows;  // row of entry t: rows[row_base + t], or row_base + t
    uint64_t row_base;
    uint32_t nrows;
    uint32_t* out;      // n x M (kEmpty padded)
    uint32_t* out_deg;  // n
    // per-warp scratch (global), sizes from PolicyScratch
    unsigned char* scratch;
    size_t warp_bytes;
    uint32_t cap;              // power of two >= pool_cap
    uint32_t umax, tmax, wmax;  // bubble optimizer bounds
    uint32_t* next;
    uint32_t* err;
};

struct WarpScratch {
    uint64_t* key;   // cap: (id, d) sort
    uint64_t* cand;  // cap: (d, id) sorted unique candidates
    double* ka;      // cap: order A (ball / residual scores)
    uint32_t* ia;
    float* da;
    double* kb;  // cap: order B (LSG)
    uint32_t* ib;
    float* db;
    // bubble optimizer
    uint32_t* univ;  // umax
    float* ud;       // umax: raw distance to the base
    double* power;   // umax
    uint64_t* ver;   // umax x wmax
    uint64_t* rt;    // umax x wmax
    uint64_t* tkey;  // tmax: targets (d, id)
    int* vc;         // tmax
    int* rc;         // tmax
    uint64_t* req;   // wmax
    uint64_t* zr;    // wmax: route count 0
    uint64_t* ov;    // wmax: verify count 1
    uint64_t* orr;   // wmax: route count 1
    uint32_t* selu;  // 64: the selection as universe indices
};

__host__ __device__ inline size_t align16(size_t b) { return (b + 15) & ~(size_t)15; }

__host__ __device__ inline size_t warp_scratch_bytes(uint32_t cap, uint32_t umax, uint32_t tmax, uint32_t wmax) {
    size_t b = 0;
    b += align16((size_t)cap * 8) * 2;                                          // key, cand
    b += (align16((size_t)cap * 8) + align16((size_t)cap * 4) * 2) * 2;         // orders A, B
    b += align16((size_t)umax * 4) * 2 + align16((size_t)umax * 8);             // univ, ud, power
    b += align16((size_t)umax * wmax * 8) * 2;                                  // ver, rt
    b += align16((size_t)tmax * 8) + align16((size_t)tmax * 4) * 2;             // tkey, vc, rc
    b += align16((size_t)wmax * 8) * 4 + align16(64 * 4);                       // masks, selu
    return b;
}

__device__ WarpScratch carve(const PolicyParams& p, uint32_t warp) {
    unsigned char* b = p.scratch + (size_t)warp * p.warp_bytes;
    WarpScratch s;
    auto take = [&](size_t bytes) {
        unsigned char* r = b;
        b += align16(bytes);
        return r;
    };
    s.key = reinterpret_cast<uint64_t*>(take((size_t)p.cap * 8));
    s.cand = reinterpret_cast<uint64_t*>(take((size_t)p.cap * 8));
    s.ka = reinterpret_cast<double*>(take((size_t)p.cap * 8));
    s.ia = reinterpret_cast<uint32_t*>(take((size_t)p.cap * 4));
    s.da = reinterpret_cast<float*>(take((size_t)p.cap * 4));
    s.kb = reinterpret_cast<double*>(take((size_t)p.cap * 8));
    s.ib = reinterpret_cast<uint32_t*>(take((size_t)p.cap * 4));
    s.db = reinterpret_cast<float*>(take((size_t)p.cap * 4));
    s.univ = reinterpret_cast<uint32_t*>(take((size_t)p.umax * 4));
    s.ud = reinterpret_cast<float*>(take((size_t)p.umax * 4));
    s.power = reinterpret_cast<double*>(take((size_t)p.umax * 8));
    s.ver = reinterpret_cast<uint64_t*>(take((size_t)p.umax * p.wmax * 8));
    s.rt = reinterpret_cast<uint64_t*>(take((size_t)p.umax * p.wmax * 8));
    s.tkey = reinterpret_cast<uint64_t*>(take((size_t)p.tmax * 8));
    s.vc = reinterpret_cast<int*>(take((size_t)p.tmax * 4));
    s.rc = reinterpret_cast<int*>(take((size_t)p.tmax * 4));
    s.req = reinterpret_cast<uint64_t*>(take((size_t)p.wmax * 8));
    s.zr = reinterpret_cast<uint64_t*>(take((size_t)p.wmax * 8));
    s.ov = reinterpret_cast<uint64_t*>(take((size_t)p.wmax * 8));
    s.orr = reinterpret_cast<uint64_t*>(take((size_t)p.wmax * 8));
    s.selu = reinterpret_cast<uint32_t*>(take(64 * 4));
    return s;
}

// float <-> unsigned keys with the same order
__device__ __forceinline__ uint32_t fkey(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u >> 31) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float fval(uint32_t k) {
    return __uint_as_float((k >> 31) ? (k & 0x7FFFFFFFu) : ~k);
}

// Bitonic sort of n_pow2 (key, id, d) triples ascending by (key, id) (warp).
__device__ void warp_sort_dkey(double* k, uint32_t* id, float* d, uint32_t n_pow2) {
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t s = 2; s <= n_pow2; s <<= 1) {
        for (uint32_t j = s >> 1; j > 0; j >>= 1) {
            for (uint32_t i = lane; i < n_pow2; i += 32) {
                const uint32_t q = i ^ j;
                if (q > i) {
                    const bool up = (i & s) == 0;
                    const double ki = k[i], kq = k[q];
                    const uint32_t ii = id[i], iq = id[q];
                    const bool gt = ki > kq || (ki == kq && ii > iq);
                    if (gt == up) {
                        k[i] = kq;
                        k[q] = ki;
                        id[i] = iq;
                        id[q] = ii;
                        const float t = d[i];
                        d[i] = d[q];
                        d[q] = t;
                    }
                }
            }
            __syncwarp();
        }
    }
}

struct RowCtx {
    const PolicyParams* p;
    WarpScratch s;
    uint32_t* sel;  // shared, 64
    float* seld;    // shared, 64: the raw distance of each selected id to the base
    uint32_t nsel;
    uint32_t nc;    // unique candidates in s.cand
    uint64_t base;
    uint32_t lane, gw, gt;
};

__device__ __forceinline__ float pair_d2(const PolicyParams& p, uint32_t a, uint32_t b, uint32_t gt) {
    const float ip = group_ip(p.x + (uint64_t)a * p.stride, p.x + (uint64_t)b * p.stride, p.dim, gt, kAll);
    return norm_d2(p.norms[a], p.norms[b], ip);
}

__device__ __forceinline__ bool in_sel(const RowCtx& r, uint32_t id) {
    const bool h = (r.lane < r.nsel && r.sel[r.lane] == id) || (r.lane + 32 < r.nsel && r.sel[r.lane + 32] == id);
    return __any_sync(kAll, h);
}

__device__ __forceinline__ void push_sel(RowCtx& r, uint32_t id, float d) {
    if (r.lane == 0) {
        r.sel[r.nsel] = id;
        r.seld[r.nsel] = d;
    }
    __syncwarp();
    r.nsel++;
}

// edge_radj / edge_sort_radj (index.h:292-303)
__device__ __forceinline__ double radj(const DevPolicyView& q, uint32_t id, uint32_t k) {
    return __dmul_rn(q.scale2, (double)q.resid[(uint64_t)id * q.nk + (k - 1)]);
}
__device__ double sort_radj(const DevPolicyView& q, uint32_t id) {
    if (!(q.flags & kPolBall) || q.nks == 0) return 0.0;
    double best = -inf_d();
    for (uint32_t t = 0; t < q.nks; t++) {
        const double v = radj(q, id, q.ks[t]);
        best = best < v ? v : best;
    }
    return isfinite(best) ? best : 0.0;
}

// ball_occludes_distance (index.h:478-495): all (or any) k occlude
__device__ bool ball_occludes(const PolicyParams& p, uint64_t base, uint32_t sid, float dbase_cid, float dsc) {
    const DevPolicyView& q = p.pol;
    if (!(q.flags & kPolBall) || q.nks == 0) return false;
    bool any = false, all = true;
    for (uint32_t t = 0; t < q.nks; t++) {
        const uint32_t k = q.ks[t];
        const double lhs = __dsub_rn(__dmul_rn((double)p.alpha, (double)dsc), __dmul_rn(q.lambda, radj(q, sid, k)));
        const double rhs = __dsub_rn((double)dbase_cid, __dmul_rn(q.lambda, radj(q, (uint32_t)base, k)));
        const bool occ = lhs < rhs;
        any = any || occ;
        all = all && occ;
    }
    return q.occ_all ? all : any;
}

// lsg_distance2 (index.h:719-725)
__device__ double lsg_d2(const DevPolicyView& q, uint32_t a, uint32_t b, double raw) {
    if (!(q.flags & kPolLsg) || q.lsg_alpha == 0.0) return raw;
    const double mp = __dmul_rn((double)q.mu[a], (double)q.mu[b]);
    const double denom = q.lsg_alpha == 1.0 ? mp : pow(mp, q.lsg_alpha);
    if (!isfinite(denom) || denom <= 0.0) return raw;
    return __ddiv_rn(raw, denom);
}

// rng_extend (index.h:264-278) over the (d, id) candidates
__device__ void rng_extend(RowCtx& r, uint32_t cap) {
    const PolicyParams& p = *r.p;
    for (uint32_t q = 0; q < r.nc && r.nsel < cap; q++) {
        const uint64_t key = r.s.cand[q];
        const uint32_t cid = (uint32_t)key;
        const float dc = fval((uint32_t)(key >> 32));
        if (in_sel(r, cid)) continue;
        bool occluded = false;
        for (uint32_t s0 = 0; s0 < r.nsel && !occluded; s0 += 8) {
            const uint32_t j = s0 + r.gw;
            const bool ok = j < r.nsel;
            const float dsc = pair_d2(p, r.sel[ok ? j : s0], cid, r.gt);
            occluded = __any_sync(kAll, ok && __fmul_rn(p.alpha, dsc) < dc);
        }
        if (!occluded) push_sel(r, cid, dc);
    }
}

// ball_sort_candidates (index.h:501-510) into order A
__device__ void ball_order(RowCtx& r) {
    const PolicyParams& p = *r.p;
    const uint32_t np2 = next_pow2(max(r.nc, 2u));
    for (uint32_t t = r.lane; t < np2; t += 32) {
        if (t < r.nc) {
            const uint64_t key = r.s.cand[t];
            const uint32_t id = (uint32_t)key;
            const float d = fval((uint32_t)(key >> 32));
            r.s.ka[t] = (p.pol.flags & kPolBall) ? __dsub_rn((double)d, __dmul_rn(p.pol.lambda, sort_radj(p.pol, id)))
                                                 : (double)d;
            r.s.ia[t] = id;
            r.s.da[t] = d;
        } else {
            r.s.ka[t] = inf_d();
            r.s.ia[t] = kEmpty;
            r.s.da[t] = FLT_MAX;
        }
    }
    __syncwarp();
    if (p.pol.flags & kPolBall) warp_sort_dkey(r.s.ka, r.s.ia, r.s.da, np2);
}

// rng_extend_ball (index.h:512-527) over order A
__device__ void rng_extend_ball(RowCtx& r, uint32_t cap) {
    const PolicyParams& p = *r.p;
    for (uint32_t q = 0; q < r.nc && r.nsel < cap; q++) {
        const uint32_t cid = r.s.ia[q];
        const float d2c = r.s.da[q];
        if (in_sel(r, cid)) continue;
        bool occluded = false;
        for (uint32_t s0 = 0; s0 < r.nsel && !occluded; s0 += 8) {
            const uint32_t j = s0 + r.gw;
            const bool ok = j < r.nsel;
            const uint32_t sid = r.sel[ok ? j : s0];
            const float dsc = pair_d2(p, sid, cid, r.gt);
            occluded = __any_sync(kAll, ok && ball_occludes(p, r.base, sid, d2c, dsc));
        }
        if (!occluded) push_sel(r, cid, d2c);
    }
}

// lsg_sort_candidates (index.h:727-737) into order B
__device__ void lsg_order(RowCtx& r) {
    const PolicyParams& p = *r.p;
    const uint32_t np2 = next_pow2(max(r.nc, 2u));
    for (uint32_t t = r.lane; t < np2; t += 32) {
        if (t < r.nc) {
            const uint64_t key = r.s.cand[t];
            const uint32_t id = (uint32_t)key;
            const float d = fval((uint32_t)(key >> 32));
            r.s.kb[t] = lsg_d2(p.pol, (uint32_t)r.base, id, (double)d);
            r.s.ib[t] = id;
            r.s.db[t] = d;
        } else {
            r.s.kb[t] = inf_d();
            r.s.ib[t] = kEmpty;
            r.s.db[t] = FLT_MAX;
        }
    }
    __syncwarp();
    warp_sort_dkey(r.s.kb, r.s.ib, r.s.db, np2);
}

// rng_extend_lsg (index.h:739-754) over order B
__device__ void rng_extend_lsg(RowCtx& r, uint32_t cap) {
    const PolicyParams& p = *r.p;
    for (uint32_t q = 0; q < r.nc && r.nsel < cap; q++) {
        const uint32_t cid = r.s.ib[q];
        const double key = r.s.kb[q];
        if (in_sel(r, cid)) continue;
        bool occluded = false;
        for (uint32_t s0 = 0; s0 < r.nsel && !occluded; s0 += 8) {
            const uint32_t j = s0 + r.gw;
            const bool ok = j < r.nsel;
            const uint32_t sid = r.sel[ok ? j : s0];
            const float dsc = pair_d2(p, sid, cid, r.gt);
            const double l = lsg_d2(p.pol, sid, cid, (double)dsc);
            occluded = __any_sync(kAll, ok && __dmul_rn((double)p.alpha, l) < key);
        }
        if (!occluded) push_sel(r, cid, r.s.db[q]);
    }
}

// add_residual_cover_edges (index.h:441-476): per k, the unselected
// candidates of positive residual by (d - lambda scale^2 risk, id), up to
// per_k of them
__device__ void residual_cover(RowCtx& r) {
    const PolicyParams& p = *r.p;
    const DevPolicyView& q = p.pol;
    if (!(q.flags & kPolCover) || r.nsel >= p.M) return;
    const uint32_t total = min(q.budget, p.M - r.nsel);
    if (total == 0 || q.nks == 0) return;
    const uint32_t per_k = max(1u, (total + q.nks - 1) / q.nks);
    uint32_t added_total = 0;
    for (uint32_t t = 0; t < q.nks; t++) {
        if (added_total >= total || r.nsel >= p.M) break;
        const uint32_t k = q.ks[t];
        // eligible candidates, compacted into order A
        uint32_t m = 0;
        for (uint32_t c0 = 0; c0 < r.nc; c0 += 32) {
            const uint32_t c = c0 + r.lane;
            bool ok = false;
            double score = 0.0;
            uint32_t cid = kEmpty;
            float d = 0.f;
            if (c < r.nc) {
                const uint64_t key = r.s.cand[c];
                cid = (uint32_t)key;
                d = fval((uint32_t)(key >> 32));
                const double residual = (double)q.resid[(uint64_t)cid * q.nk + (k - 1)];
                const double risk = residual > 0.0 ? residual : 0.0;
                ok = risk > 0.0 && cid != (uint32_t)r.base;
                score = __dsub_rn((double)d, __dmul_rn(__dmul_rn(q.lambda, q.scale2), risk));
            }
            // selected at the start of this k's list
            bool sel = false;
            for (uint32_t s = 0; s < r.nsel; s++) sel = sel || r.sel[s] == cid;
            ok = ok && !sel;
            const unsigned b = __ballot_sync(kAll, ok);
            if (ok) {
                const uint32_t w = m + __popc(b & lane_lt_mask());
                r.s.ka[w] = score;
                r.s.ia[w] = cid;
                r.s.da[w] = d;
            }
            m += __popc(b);
        }
        __syncwarp();
        const uint32_t m2 = next_pow2(max(m, 2u));
        for (uint32_t w = m + r.lane; w < m2; w += 32) {
            r.s.ka[w] = inf_d();
            r.s.ia[w] = kEmpty;
            r.s.da[w] = FLT_MAX;
        }
        __syncwarp();
        warp_sort_dkey(r.s.ka, r.s.ia, r.s.da, m2);
        uint32_t added_k = 0;
        for (uint32_t w = 0; w < m; w++) {
            if (r.nsel >= p.M || added_total >= total || added_k >= per_k) break;
            push_sel(r, r.s.ia[w], r.s.da[w]);
            added_k++;
            added_total++;
        }
    }
}

// optimize_verification_constrained_bubble (index.h:531-717)
__device__ void bubble(RowCtx& r) {
    const PolicyParams& p = *r.p;
    const DevPolicyView& q = p.pol;
    if (!(q.flags & kPolAuto) || r.nsel == 0 || r.nc == 0) return;
    WarpScratch& s = r.s;
    const uint32_t lane = r.lane;
    ball_order(r);
    // the universe: the selection, then up to `limit` ball-ordered alternatives
    for (uint32_t u = lane; u < r.nsel; u += 32) {
        s.univ[u] = r.sel[u];
        s.ud[u] = r.seld[u];
    }
    uint32_t nu = r.nsel;
    const uint32_t limit = (q.flags & kPolAutoFull) ? r.nc : q.auto_cand;
    uint32_t alternatives = 0;
    for (uint32_t c0 = 0; c0 < r.nc && alternatives < limit; c0 += 32) {
        const uint32_t c = c0 + lane;
        bool fresh = false;
        if (c < r.nc) {
            fresh = true;
            for (uint32_t t = 0; t < r.nsel; t++) fresh = fresh && r.sel[t] != s.ia[c];
        }
        const unsigned b = __ballot_sync(kAll, fresh);
        const uint32_t rank = __popc(b & lane_lt_mask());
        if (fresh && alternatives + rank < limit) {
            s.univ[nu + rank] = s.ia[c];
            s.ud[nu + rank] = s.da[c];
        }
        const uint32_t took = min((uint32_t)__popc(b), limit - alternatives);
        nu += took;
        alternatives += took;
    }
    __syncwarp();
    if (alternatives == 0) return;
    // targets, sorted by (d, id)
    uint32_t T;
    if (q.flags & kPolAutoFull) {
        T = r.nc;
        for (uint32_t t = lane; t < T; t += 32) s.tkey[t] = s.cand[t];
    } else {
        T = nu;
        const uint32_t t2 = next_pow2(max(T, 2u));
        for (uint32_t t = lane; t < t2; t += 32)
            s.tkey[t] = t < T ? ((uint64_t)fkey(s.ud[t]) << 32) | s.univ[t] : ~0ull;
        __syncwarp();
        warp_sort_u64(s.tkey, t2);
    }
    __syncwarp();
    const uint32_t W = (T + 63) / 64;
    for (uint32_t u = lane; u < nu; u += 32)
        s.power[u] = __dsub_rn((double)s.ud[u], __dmul_rn(q.lambda, sort_radj(q, s.univ[u])));
    __syncwarp();
    // signatures: the verify and route bits of every (member, target) pair,
    // one 64-target word at a time, eight pairs per round (one per 4-lane group)
    const uint32_t rounds = (T + 7) / 8;
    for (uint32_t u = 0; u < nu; u++) {
        const uint32_t id = s.univ[u];
        uint64_t vw = 0, rw = 0;
        for (uint32_t rd = 0; rd < rounds; rd++) {
            const uint32_t ti = rd * 8 + r.gw;
            const bool ok = ti < T;
            const uint64_t tk = s.tkey[ok ? ti : 0];
            const uint32_t tid = (uint32_t)tk;
            const float td = fval((uint32_t)(tk >> 32));
            const float dsc = pair_d2(p, id, tid, r.gt);
            const float dd = id == tid ? 0.0f : dsc;
            const bool vb = ok && (id == tid || __fmul_rn(p.alpha, dd) < td);
            const bool rb = ok && ball_occludes(p, r.base, id, td, dd);
            const unsigned bv = __ballot_sync(kAll, vb && r.gt == 0), br = __ballot_sync(kAll, rb && r.gt == 0);
            uint32_t v8 = 0, r8 = 0;
            for (uint32_t g = 0; g < 8; g++) {
                v8 |= ((bv >> (4 * g)) & 1u) << g;
                r8 |= ((br >> (4 * g)) & 1u) << g;
            }
            vw |= (uint64_t)v8 << ((rd & 7u) * 8);
            rw |= (uint64_t)r8 << ((rd & 7u) * 8);
            if ((rd & 7u) == 7u || rd + 1 == rounds) {
                if (lane == 0) {
                    s.ver[(uint64_t)u * W + (rd >> 3)] = vw;
                    s.rt[(uint64_t)u * W + (rd >> 3)] = rw;
                }
                vw = 0;
                rw = 0;
            }
        }
    }
    __syncwarp();
    // the selection (universe indices 0 .. nsel-1) and its counts
    const uint32_t nsel = r.nsel;
    for (uint32_t t = lane; t < nsel; t += 32) s.selu[t] = t;
    for (uint32_t ti = lane; ti < T; ti += 32) {
        int v = 0, c = 0;
        for (uint32_t t = 0; t < nsel; t++) {
            v += (int)((s.ver[(uint64_t)t * W + (ti >> 6)] >> (ti & 63u)) & 1u);
            c += (int)((s.rt[(uint64_t)t * W + (ti >> 6)] >> (ti & 63u)) & 1u);
        }
        s.vc[ti] = v;
        s.rc[ti] = c;
    }
    __syncwarp();
    for (uint32_t w = lane; w < W; w += 32) {
        uint64_t m = 0;
        for (uint32_t b = 0; b < 64 && w * 64 + b < T; b++)
            if (s.vc[w * 64 + b] > 0) m |= 1ull << b;
        s.req[w] = m;
    }
    __syncwarp();
    const uint32_t max_swaps = min(q.auto_swaps, alternatives);
    for (uint32_t swaps = 0; swaps < max_swaps; swaps++) {
        for (uint32_t w = lane; w < W; w += 32) {
            uint64_t z = 0, o1 = 0, r1 = 0;
            for (uint32_t b = 0; b < 64 && w * 64 + b < T; b++) {
                const uint32_t ti = w * 64 + b;
                if (s.rc[ti] == 0) z |= 1ull << b;
                if (s.vc[ti] == 1) o1 |= 1ull << b;
                if (s.rc[ti] == 1) r1 |= 1ull << b;
            }
            s.zr[w] = z;
            s.ov[w] = o1;
            s.orr[w] = r1;
        }
        __syncwarp();
        // best (q, slot): highest route gain, then highest power gain, first in (q, slot) order
        long best_gain = LONG_MIN;
        double best_pg = -inf_d();
        uint64_t best_e = ~0ull;
        const uint64_t np = (uint64_t)nu * nsel;
        for (uint64_t e = lane; e < np; e += 32) {
            const uint32_t qq = (uint32_t)(e / nsel), slot = (uint32_t)(e - (uint64_t)qq * nsel);
            bool is_selected = false;
            for (uint32_t t = 0; t < nsel; t++) is_selected = is_selected || s.selu[t] == qq;
            if (is_selected) continue;
            const uint32_t old = s.selu[slot];
            long newly = 0, lost = 0;
            bool feasible = true;
            for (uint32_t w = 0; w < W; w++) {
                const uint64_t qv = s.ver[(uint64_t)qq * W + w], qr = s.rt[(uint64_t)qq * W + w];
                const uint64_t ovv = s.ver[(uint64_t)old * W + w], orw = s.rt[(uint64_t)old * W + w];
                newly += __popcll(qr & s.zr[w]);
                if (s.req[w] & ovv & s.ov[w] & ~qv) feasible = false;
                lost += __popcll(orw & s.orr[w] & ~qr);
            }
            if (!feasible) continue;
            const long gain = newly - lost;
            const double pg = __dsub_rn(s.power[old], s.power[qq]);
            if (gain > best_gain || (gain == best_gain && pg > best_pg)) {
                best_gain = gain;
                best_pg = pg;
                best_e = e;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const long og = __shfl_xor_sync(kAll, best_gain, o);
            const double op = __shfl_xor_sync(kAll, best_pg, o);
            const uint64_t oe = __shfl_xor_sync(kAll, best_e, o);
            const bool better = og > best_gain || (og == best_gain && (op > best_pg || (op == best_pg && oe < best_e)));
            if (better) {
                best_gain = og;
                best_pg = op;
                best_e = oe;
            }
        }
        if (best_e == ~0ull || best_gain < 0 || (best_gain == 0 && best_pg <= 1e-12)) break;
        const uint32_t bq = (uint32_t)(best_e / nsel), bslot = (uint32_t)(best_e - (uint64_t)bq * nsel);
        const uint32_t old = s.selu[bslot];
        for (uint32_t ti = lane; ti < T; ti += 32) {
            const uint32_t w = ti >> 6, b = ti & 63u;
            s.vc[ti] += (int)((s.ver[(uint64_t)bq * W + w] >> b) & 1u) - (int)((s.ver[(uint64_t)old * W + w] >> b) & 1u);
            s.rc[ti] += (int)((s.rt[(uint64_t)bq * W + w] >> b) & 1u) - (int)((s.rt[(uint64_t)old * W + w] >> b) & 1u);
        }
        __syncwarp();
        if (lane == 0) s.selu[bslot] = bq;
        __syncwarp();
    }
    for (uint32_t t = lane; t < nsel; t += 32) {
        r.sel[t] = s.univ[s.selu[t]];
        r.seld[t] = s.ud[s.selu[t]];
    }
    __syncwarp();
}

__global__ void __launch_bounds__(32 * kPolWarps) policy_prune_kernel(PolicyParams p) {
    __shared__ uint32_t s_sel[kPolWarps][64];
    __shared__ float s_seld[kPolWarps][64];
    const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
    const uint32_t warp = blockIdx.x * kPolWarps + wib;
    RowCtx r;
    r.p = &p;
    r.s = carve(p, warp);
    r.sel = s_sel[wib];
    r.seld = s_seld[wib];
    r.lane = lane;
    r.gw = lane >> 2;
    r.gt = lane & 3u;
    for (;;) {
        uint32_t t = 0;
        if (lane == 0) t = atomicAdd(p.next, 1u);
        t = __shfl_sync(kAll, t, 0);
        if (t >= p.nrows) break;
        const uint64_t i = p.rows ? p.rows[p.row_base + t] : p.row_base + t;
        if (i >= p.n) {
            if (lane == 0) set_error(p.err, kDevBadId);
            continue;
        }
        r.base = i;
        r.nsel = 0;
        // sort_unique_candidates (index.h:225-247): valid ids but the row, by
        // (id, d); the first (smallest d) of each id; by (d, id)
        const uint32_t np = min(p.pool_n[t], p.pool_cap);
        const float* pd = p.pool_d + (uint64_t)t * p.pool_cap;
        const uint32_t* pi = p.pool_i + (uint64_t)t * p.pool_cap;
        uint32_t m = 0;
        for (uint32_t c0 = 0; c0 < np; c0 += 32) {
            const uint32_t c = c0 + lane;
            const uint32_t id = c < np ? pi[c] : kEmpty;
            const bool ok = id < p.n && id != (uint32_t)i;
            const unsigned b = __ballot_sync(kAll, ok);
            if (ok) r.s.key[m + __popc(b & lane_lt_mask())] = ((uint64_t)id << 32) | fkey(pd[c]);
            m += __popc(b);
        }
        const uint32_t m2 = next_pow2(max(m, 2u));
        for (uint32_t c = m + lane; c < m2; c += 32) r.s.key[c] = ~0ull;
        __syncwarp();
        warp_sort_u64(r.s.key, m2);
        uint32_t nc = 0;
        for (uint32_t c0 = 0; c0 < m; c0 += 32) {
            const uint32_t c = c0 + lane;
            const uint64_t k = c < m ? r.s.key[c] : ~0ull;
            const bool first = c < m && (c == 0 || (uint32_t)(r.s.key[c - 1] >> 32) != (uint32_t)(k >> 32));
            const unsigned b = __ballot_sync(kAll, first);
            if (first) r.s.cand[nc + __popc(b & lane_lt_mask())] = (k << 32) | (k >> 32);
            nc += __popc(b);
        }
        const uint32_t n2 = next_pow2(max(nc, 2u));
        for (uint32_t c = nc + lane; c < n2; c += 32) r.s.cand[c] = ~0ull;
        __syncwarp();
        warp_sort_u64(r.s.cand, n2);
        r.nc = nc;
        // prune_pool_to_ids (index.h:772-829)
        const DevPolicyView& q = p.pol;
        const uint32_t M = p.M;
        const uint32_t bud = min(q.budget, M);
        if (q.flags & kPolAuto) {
            rng_extend(r, M);
            bubble(r);
        } else if ((q.flags & kPolLsg) && (q.flags & kPolBall) && q.lsg_alpha != 0.0) {
            lsg_order(r);
            rng_extend_lsg(r, M - bud ? M - bud : M);
            ball_order(r);
            rng_extend_ball(r, M);
            rng_extend_lsg(r, M);
        } else if ((q.flags & kPolLsg) && q.lsg_alpha != 0.0) {
            lsg_order(r);
            rng_extend_lsg(r, M);
        } else if (q.flags & kPolBall) {
            ball_order(r);
            if (q.flags & kPolPure) {
                rng_extend_ball(r, M);
                rng_extend(r, M);
            } else {
                rng_extend(r, M - bud ? M - bud : M);
                rng_extend_ball(r, M);
                rng_extend(r, M);
            }
        } else {
            const uint32_t cover = (q.flags & kPolCover) ? bud : 0u;
            rng_extend(r, M - cover ? M - cover : M);
            residual_cover(r);
            rng_extend(r, M);
        }
        for (uint32_t t2 = lane; t2 < M; t2 += 32) p.out[i * M + t2] = t2 < r.nsel ? r.sel[t2] : kEmpty;
        if (lane == 0) p.out_deg[i] = r.nsel;
        __syncwarp();
    }
}

}  // namespace

int set_edge_policy(Ctx* c, const anqi_edge_policy* pol, uint64_t n) {
    DevPolicy& e = c->edge;
    e.active = false;
    if (!pol || pol->flags == 0) return ANQI_OK;
    if (pol->nks > 8 || pol->flags > 63) return fail(c, ANQI_ERR_ARGS, "invalid edge policy");
    const bool resid = pol->flags & (kPolCover | kPolBall | kPolAuto);
    if (resid && (!pol->resid || pol->nk == 0 || pol->nks == 0))
        return fail(c, ANQI_ERR_ARGS, "edge policy needs its residual table and k values");
    for (uint32_t t = 0; t < pol->nks; t++)
        if (pol->ks[t] == 0 || pol->ks[t] > pol->nk) return fail(c, ANQI_ERR_ARGS, "edge policy k outside 1..nk");
    if ((pol->flags & kPolLsg) && !pol->mu) return fail(c, ANQI_ERR_ARGS, "LSG edge policy needs its mu table");
    int rc;
    if (resid && (rc = h2d(c, e.resid, pol->resid, n * pol->nk * 4))) return rc;
    if ((pol->flags & kPolLsg) && (rc = h2d(c, e.mu, pol->mu, n * 4))) return rc;
    DevPolicyView& v = e.view;
    v.flags = pol->flags;
    v.nks = pol->nks;
    for (uint32_t t = 0; t < 8; t++) v.ks[t] = t < pol->nks ? pol->ks[t] : 0u;
    v.nk = pol->nk;
    v.budget = pol->budget;
    v.occ_all = pol->occlude_all;
    v.auto_cand = pol->auto_candidates ? pol->auto_candidates : 1u;
    v.auto_swaps = pol->auto_max_swaps ? pol->auto_max_swaps : 1u;
    v.lambda = pol->lambda;
    v.scale2 = pol->scale2;
    v.lsg_alpha = pol->lsg_alpha;
    v.resid = resid ? e.resid.as<float>() : nullptr;
    v.mu = (pol->flags & kPolLsg) ? e.mu.as<float>() : nullptr;
    e.active = true;
    return ANQI_OK;
}

void clear_edge_policy(Ctx* c) {
    c->edge.active = false;
    release(c, c->edge.resid);
    release(c, c->edge.mu);
}

int run_policy_prune(Ctx* c, const float* x, const float* norms, uint64_t n, uint32_t stride, uint32_t dim, uint32_t M,
                     float alpha, const float* pool_d, const uint32_t* pool_i, const uint32_t* pool_n,
                     uint32_t pool_cap, const uint32_t* rows, uint64_t row_base, uint32_t nrows, uint32_t* out,
                     uint32_t* out_deg) {
    if (!c->edge.active || nrows == 0) return ANQI_OK;
    if (M > 64) return fail(c, ANQI_ERR_ARGS, "edge policies take M <= 64");
    PolicyParams p{};
    p.x = x;
    p.norms = norms;
    p.n = n;
    p.stride = stride;
    p.dim = dim;
    p.M = M;
    p.alpha = alpha;
    p.pol = c->edge.view;
    p.pool_d = pool_d;
    p.pool_i = pool_i;
    p.pool_n = pool_n;
    p.pool_cap = pool_cap;
    p.rows = rows;
    p.row_base = row_base;
    p.nrows = nrows;
    p.out = out;
    p.out_deg = out_deg;
    p.cap = 1u << (32 - __builtin_clz(std::max(pool_cap, 2u) - 1));
    const bool full = c->edge.view.flags & kPolAutoFull;
    p.umax = M + (full ? p.cap : std::min(p.cap, std::max(1u, c->edge.view.auto_cand)));
    // the lazy targets (the universe) are sorted padded to a power of two
    p.tmax = full ? p.cap : 1u << (32 - __builtin_clz(std::max(p.umax, 2u) - 1));
    p.wmax = (p.tmax + 63) / 64;
    p.warp_bytes = warp_scratch_bytes(p.cap, p.umax, p.tmax, p.wmax);
    // as many warps as fit in about 2 GB of scratch, at most 16 per SM
    uint64_t warps = std::min<uint64_t>((uint64_t)c->sm_count * 16, std::max<uint64_t>(1, (2ull << 30) / p.warp_bytes));
    warps = std::min<uint64_t>(warps, ((uint64_t)nrows + 0) + kPolWarps - 1);
    const uint32_t blocks = (uint32_t)std::max<uint64_t>(1, warps / kPolWarps);
    int rc;
    if ((rc = ensure(c, c->pol_scratch, (size_t)blocks * kPolWarps * p.warp_bytes))) return rc;
    p.scratch = c->pol_scratch.as<unsigned char>();
    p.next = c->counters.as<uint32_t>() + 8;
    p.err = c->err.as<uint32_t>();
    ANQI_CUDA(c, cudaMemsetAsync(p.next, 0, 4, c->stream));
    policy_prune_kernel<<<blocks, 32 * kPolWarps, 0, c->stream>>>(p);
    ANQI_CUDA(c, cudaGetLastError());
    return ANQI_OK;
}

}  // namespace anqi
