/* Test infrastructure only -- the checker the CUDA kernels are compared with.
 * Never linked into, loaded by, or called from the product library.
 *
 * Plain-C restatement of the reference algorithms on the RkNN hot path of
 * Yujian-Fu/anqi-implementation.  Every function names the reference file:line
 * it restates.  Pinned against the reference's own outputs by the golden
 * fixtures in tests/golden/ (see tests/test_oracle_golden.py).
 *
 * Compiled with -ffp-contract=off so no multiply-add is fused except where the
 * reference uses an explicit FMA (the AVX-512 _mm512_fmadd_ps lanes).
 */
#include "anqi_oracle.h"

#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define AO_EMPTY 0xFFFFFFFFu
static const float AO_EPS = 1e-6f; /* distance.h:14 */

/* _mm512_reduce_add_ps as GCC 13 defines it (avx512fintrin.h): fold the upper
 * 256-bit half onto the lower, then the upper 128-bit half, then lanes {2,3}
 * onto {0,1}, then lane 1 onto lane 0. */
static float reduce16(const float* A) {
    float t3[8], t6[4];
    for (int i = 0; i < 8; i++) t3[i] = A[i + 8] + A[i];
    for (int j = 0; j < 4; j++) t6[j] = t3[j + 4] + t3[j];
    float t80 = t6[0] + t6[2];
    float t81 = t6[1] + t6[3];
    return t80 + t81;
}

/* distance.h:58-86 */
float ao_l2sqr(const float* a, const float* b, uint32_t dim) {
    float acc[16] = {0};
    uint32_t q16 = dim / 16, rem = dim % 16;
    for (uint32_t c = 0; c < q16; c++)
        for (int l = 0; l < 16; l++) {
            float df = a[16 * c + l] - b[16 * c + l];
            acc[l] = fmaf(df, df, acc[l]);
        }
    float res = reduce16(acc);
    if (rem) {
        float t[16] = {0};
        for (uint32_t l = 0; l < rem; l++) {
            float df = a[16 * q16 + l] - b[16 * q16 + l];
            t[l] = df * df;
        }
        res += reduce16(t);
    }
    return res;
}

/* distance.h:89-116 (and the free function at distance.h:22-51, identical arithmetic) */
float ao_ip(const float* a, const float* b, uint32_t dim) {
    float acc[16] = {0};
    uint32_t q16 = dim / 16, rem = dim % 16;
    for (uint32_t c = 0; c < q16; c++)
        for (int l = 0; l < 16; l++) acc[l] = fmaf(a[16 * c + l], b[16 * c + l], acc[l]);
    float res = reduce16(acc);
    if (rem) {
        float t[16] = {0};
        for (uint32_t l = 0; l < rem; l++) t[l] = a[16 * q16 + l] * b[16 * q16 + l];
        res += reduce16(t);
    }
    return res;
}

/* distance.h:143-161 -- identical arithmetic to ao_ip(a, a) */
float ao_norm(const float* a, uint32_t dim) { return ao_ip(a, a, dim); }

/* index.h:172-176 */
float ao_d2(const float* a, const float* b, float na, float nb, uint32_t dim) {
    float s = na + nb;
    float t = 2.0f * ao_ip(a, b, dim);
    return s - t;
}

/* distance.h:170-174: the "ip" metric's scalar distance 1 - sum a_i b_i, a
 * sequential sum in index order, as the reference's compiler (GCC 13, -O3,
 * x86-64-v4 / AVX-512 hosts) emits it: the first 8 floor(dim / 8) products are
 * formed in 8-wide vectors and added one by one (each rounded), the remaining
 * dim mod 8 are accumulated by fused multiply-adds.  Pinned against the
 * compiled reference at dimensions 3, 8, 13, 32 and 130 (tests/golden). */
float ao_ip_dist(const float* a, const float* b, uint32_t dim) {
    const uint32_t d8 = dim & ~7u;
    float product = 0.0f;
    for (uint32_t i = 0; i < d8; i++) {
        float t = a[i] * b[i];
        product = product + t;
    }
    for (uint32_t i = d8; i < dim; i++) product = fmaf(a[i], b[i], product);
    return 1.0f - product;
}

/* nndindex::d2 (index.h:172-176): L2 by norms, or the ip metric's distance */
static float metric_d2(const float* a, const float* b, float na, float nb, uint32_t dim, uint32_t ip) {
    return ip ? ao_ip_dist(a, b, dim) : ao_d2(a, b, na, nb, dim);
}

void ao_norms(const float* x, uint64_t n, uint32_t dim, float* out) {
    for (uint64_t i = 0; i < n; i++) out[i] = ao_norm(x + i * dim, dim);
}

/* ------------------------------------------------------------------ LRQ */

/* rknn_query.cpp:482-513, floor policy: last centre <= value, else the first. */
static uint32_t floor_code(double value, const float* c, uint32_t cs) {
    float v = (float)value;
    uint32_t lo = 0, hi = cs; /* upper_bound: first element > v */
    while (lo < hi) {
        uint32_t mid = (lo + hi) / 2;
        if (v < c[mid]) hi = mid;
        else lo = mid + 1;
    }
    return lo == 0 ? 0 : lo - 1;
}

/* rknn_query.cpp:679-720 */
void ao_lrq_encode(const float* keys, uint64_t n, uint32_t nk, uint32_t rankm,
                   const float* mu, const float* basis, const float* codebook,
                   uint32_t code_size, float* coeff, uint8_t* codes) {
    for (uint64_t i = 0; i < n; i++) {
        const float* rk = keys + i * nk;
        float* ci = coeff + i * rankm;
        for (uint32_t m = 0; m < rankm; m++) {
            const float* gm = basis + (uint64_t)m * nk;
            double c = 0.0;
            for (uint32_t k = 0; k < nk; k++) c += ((double)rk[k] - (double)mu[k]) * (double)gm[k];
            ci[m] = (float)c;
        }
        for (uint32_t k = 0; k < nk; k++) {
            double recon = (double)mu[k];
            for (uint32_t m = 0; m < rankm; m++) recon += (double)ci[m] * (double)basis[(uint64_t)m * nk + k];
            double residual = (double)rk[k] - recon;
            codes[i * nk + k] = (uint8_t)floor_code(residual, codebook + (uint64_t)k * code_size, code_size);
        }
    }
}

/* rknn_query.cpp:722-753 (L2: clamp at zero) */
void ao_lrq_materialize(const float* coeff, const uint8_t* codes, uint64_t n, uint32_t nk,
                        uint32_t rankm, const float* mu, const float* basis,
                        const float* codebook, uint32_t code_size, uint32_t k_one_based,
                        double radius_scale, float* thr) {
    uint32_t k = k_one_based - 1;
    for (uint64_t i = 0; i < n; i++) {
        const float* ci = coeff + i * rankm;
        double value = (double)mu[k];
        for (uint32_t m = 0; m < rankm; m++) value += (double)ci[m] * (double)basis[(uint64_t)m * nk + k];
        value += (double)codebook[(uint64_t)k * code_size + codes[i * nk + k]];
        double scaled = radius_scale * value;
        thr[i] = (float)(0.0 < scaled ? scaled : 0.0);
    }
}

/* rknn_query.cpp:482-513 for every policy (0 nearest, 1 floor, 2 ceil):
 * searches with the float value, breaks nearest ties in double. */
static uint32_t policy_code(double value, const float* c, uint32_t cs, uint32_t policy) {
    if (policy == 1) return floor_code(value, c, cs);
    float v = (float)value;
    uint32_t lo = 0, hi = cs; /* lower_bound: first element >= v */
    while (lo < hi) {
        uint32_t mid = (lo + hi) / 2;
        if (c[mid] < v) lo = mid + 1;
        else hi = mid;
    }
    if (policy == 2) return lo == cs ? cs - 1 : lo;
    if (lo == 0) return 0;
    if (lo == cs) return cs - 1;
    double up = (double)c[lo], dn = (double)c[lo - 1];
    return fabs(up - value) < fabs(value - dn) ? lo : lo - 1;
}

/* packed_code_array.h:20-61 */
static void put_code(uint8_t* d, uint64_t idx, uint32_t bits, uint32_t code) {
    if (bits == 2) {
        unsigned sh = (unsigned)(idx & 3u) * 2u;
        d[idx >> 2] = (uint8_t)((d[idx >> 2] & ~(3u << sh)) | ((code & 3u) << sh));
    } else if (bits == 4) {
        if (idx & 1u) d[idx >> 1] = (uint8_t)((d[idx >> 1] & 0x0fu) | ((code & 15u) << 4));
        else d[idx >> 1] = (uint8_t)((d[idx >> 1] & 0xf0u) | (code & 15u));
    } else if (bits == 8) {
        d[idx] = (uint8_t)code;
    } else if (bits == 16) {
        d[2 * idx] = (uint8_t)(code & 255u);
        d[2 * idx + 1] = (uint8_t)(code >> 8);
    }
}

static uint32_t take_code(const uint8_t* d, uint64_t idx, uint32_t bits) {
    if (bits == 2) return (d[idx >> 2] >> ((unsigned)(idx & 3u) * 2u)) & 3u;
    if (bits == 4) return (idx & 1u) ? (uint32_t)(d[idx >> 1] >> 4) : (uint32_t)(d[idx >> 1] & 15u);
    if (bits == 8) return d[idx];
    if (bits == 16) return (uint32_t)d[2 * idx] | ((uint32_t)d[2 * idx + 1] << 8);
    return 0;
}

/* rknn_query.cpp:679-720 for every form: bits 0 (coefficients only), 2/4/8/16
 * (packed codes; the caller zeroes `codes`), 32 (float residuals). */
void ao_lrq_encode_bits(const float* keys, uint64_t n, uint32_t nk, uint32_t rankm, const float* mu,
                        const float* basis, const float* codebook, uint32_t code_size, uint32_t bits,
                        uint32_t policy, float* coeff, uint8_t* codes, float* residual) {
    for (uint64_t i = 0; i < n; i++) {
        const float* rk = keys + i * nk;
        float* ci = coeff + i * rankm;
        for (uint32_t m = 0; m < rankm; m++) {
            const float* gm = basis + (uint64_t)m * nk;
            double c = 0.0;
            for (uint32_t k = 0; k < nk; k++) c += ((double)rk[k] - (double)mu[k]) * (double)gm[k];
            ci[m] = (float)c;
        }
        if (bits == 0) continue;
        for (uint32_t k = 0; k < nk; k++) {
            double recon = (double)mu[k];
            for (uint32_t m = 0; m < rankm; m++) recon += (double)ci[m] * (double)basis[(uint64_t)m * nk + k];
            double r = (double)rk[k] - recon;
            if (bits == 32) residual[i * nk + k] = (float)r;
            else put_code(codes, i * nk + k, bits,
                          policy_code(r, codebook + (uint64_t)k * code_size, code_size, policy));
        }
    }
}

/* rknn_query.cpp:722-753 for every form; signed_keys (IP) skips the clamp. */
void ao_lrq_materialize_bits(const float* coeff, const uint8_t* codes, const float* residual, uint64_t n,
                             uint32_t nk, uint32_t rankm, uint32_t bits, const float* mu, const float* basis,
                             const float* codebook, uint32_t code_size, uint32_t k_one_based,
                             double radius_scale, int signed_keys, float* thr) {
    uint32_t k = k_one_based - 1;
    for (uint64_t i = 0; i < n; i++) {
        const float* ci = coeff + i * rankm;
        double value = (double)mu[k];
        for (uint32_t m = 0; m < rankm; m++) value += (double)ci[m] * (double)basis[(uint64_t)m * nk + k];
        if (bits == 32) value += (double)residual[i * nk + k];
        else if (bits) value += (double)codebook[(uint64_t)k * code_size + take_code(codes, i * nk + k, bits)];
        double scaled = radius_scale * value;
        thr[i] = (float)(signed_keys ? scaled : (0.0 < scaled ? scaled : 0.0));
    }
}

/* rknn_query.cpp:576-600 (AnalyticRankMVerifier::materialize_k) */
void ao_analytic_rankm_materialize(const float* coeff, uint64_t n, uint32_t rankm, uint32_t train_kmax,
                                   uint32_t flags, double b0, uint32_t k_one_based, double radius_scale,
                                   float* thr) {
    double ratio = (flags & 4u) ? (double)k_one_based / (double)train_kmax : (double)k_one_based;
    double logk = log(ratio);
    double b[16];
    b[0] = pow(ratio, b0);
    for (uint32_t m = 1; m < rankm && m < 16; m++) b[m] = b[m - 1] * logk;
    for (uint64_t i = 0; i < n; i++) {
        double value = 0.0;
        for (uint32_t m = 0; m < rankm; m++) value += (double)coeff[i * rankm + m] * b[m];
        double scaled = radius_scale * value;
        thr[i] = (float)(0.0 < scaled ? scaled : 0.0);
    }
}

/* ----------------------------------------------------------------- lift */

/* rknn_query.cpp:2203-2235: anyk_lift, L2, graph radius = the AKNN rank-K cutoff.
 * The sum of squared norms is accumulated row by row in index order (the
 * reference's OpenMP reduction at one thread). */
void ao_lift(const float* base, uint64_t n, uint32_t d, const float* radius,
             float* lifted, double* mstar2, double* scale) {
    ao_lift_metric(base, n, d, radius, 0, lifted, mstar2, scale);
}

/* The same for either metric: the ip lift's coordinate is s^2 r (rknn_query.cpp:2227). */
void ao_lift_metric(const float* base, uint64_t n, uint32_t d, const float* radius, uint32_t ip,
                    float* lifted, double* mstar2, double* scale) {
    double sum_n2 = 0;
    for (uint64_t i = 0; i < n; i++) {
        const float* o = base + i * d;
        double s = 0;
        for (uint32_t j = 0; j < d; j++) s += (double)o[j] * o[j];
        sum_n2 += s;
    }
    double s_scale = 1.0 / sqrt(sum_n2 / (double)n + 1e-12), sc2 = s_scale * s_scale;
    uint32_t dl = d + 1, dout = d + 2;
    double maxn2 = 0;
    for (uint64_t i = 0; i < n; i++) {
        const float* o = base + i * d;
        float* h = lifted + i * dout;
        double nr2 = 0;
        for (uint32_t j = 0; j < d; j++) {
            double v = (double)o[j] * s_scale;
            h[j] = (float)v;
            nr2 += v * v;
        }
        h[d] = ip ? (float)((double)radius[i] * sc2) : (float)(0.5 * ((double)radius[i] * sc2 - nr2));
        double hn2 = nr2 + (double)h[d] * h[d];
        if (hn2 > maxn2) maxn2 = hn2;
    }
    double M2 = maxn2 * 1.0001;
    for (uint64_t i = 0; i < n; i++) {
        float* h = lifted + i * dout;
        double hn2 = 0;
        for (uint32_t j = 0; j < dl; j++) hn2 += (double)h[j] * h[j];
        double pad = M2 - hn2;
        if (pad < 0) pad = 0;
        h[dl] = (float)sqrt(pad);
    }
    *mstar2 = M2;
    *scale = s_scale;
}

/* rknn_query.cpp:2724-2729 */
void ao_lift_query(const float* q, uint32_t d, double scale, float* out) {
    for (uint32_t j = 0; j < d; j++) out[j] = (float)((double)q[j] * scale);
    out[d] = 1.0f;
    out[d + 1] = 0.0f;
}

/* ------------------------------------------------------------ tree entry */

/* rptrees.h:108-124.  Root = last node (post-order) -- callers pass arrays in
 * the reference's post-order.  |margin| <= EPS takes the left child (the
 * reference draws a thread-local random bit there). */
uint32_t ao_tree_entry(uint32_t n_nodes, uint32_t dim, const uint32_t* left,
                       const uint32_t* right, const float* offset, const float* hyperplane,
                       const uint32_t* leaf_first, const float* q) {
    uint32_t v = n_nodes - 1;
    while (left[v] != AO_EMPTY) {
        float margin = ao_ip(hyperplane + (uint64_t)v * dim, q, dim) - offset[v];
        if (margin < -AO_EPS) v = left[v];
        else if (margin > AO_EPS) v = right[v];
        else v = left[v];
    }
    return leaf_first[v] == AO_EMPTY ? 0 : leaf_first[v];
}

/* ---------------------------------------------------- ordered beam queue */

/* neighbor.h:10-27,43-141: (dist, id) total order, bit 31 = expanded. */
typedef struct {
    float d;
    uint32_t id;
} nb_t;
typedef struct {
    nb_t* data;
    uint32_t size, cap, cur;
} queue_t;

static int nb_less(nb_t a, nb_t b) {
    uint32_t ia = a.id & 0x7FFFFFFFu, ib = b.id & 0x7FFFFFFFu;
    return a.d < b.d || (a.d == b.d && ia < ib);
}

static void q_init(queue_t* q, uint32_t cap) {
    q->data = (nb_t*)malloc(sizeof(nb_t) * (cap + 1));
    q->size = 0;
    q->cap = cap;
    q->cur = 0;
}

/* neighbor.h:61-102 */
static void q_insert(queue_t* q, float d, uint32_t id) {
    nb_t x = {d, id};
    if (q->cap == 0 || (q->size == q->cap && nb_less(q->data[q->size - 1], x))) return;
    uint32_t lo = 0, hi = q->size;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (nb_less(x, q->data[mid])) hi = mid;
        else if ((q->data[mid].id & 0x7FFFFFFFu) == id) return;
        else lo = mid + 1;
    }
    if (lo < q->cap) memmove(&q->data[lo + 1], &q->data[lo], (q->size - lo) * sizeof(nb_t));
    q->data[lo] = x;
    if (q->size < q->cap) q->size++;
    if (lo < q->cur) q->cur = lo;
}

/* neighbor.h:105-111 */
static uint32_t q_pop(queue_t* q) {
    q->data[q->cur].id |= 0x80000000u;
    uint32_t pre = q->cur;
    while (q->cur < q->size && (q->data[q->cur].id & 0x80000000u)) q->cur++;
    return q->data[pre].id & 0x7FFFFFFFu;
}

/* --------------------------------------------------------- range search */

/* index.h:1535-1640 with the pinned configuration: eps = 0, radj = null,
 * center beam key, collect threshold = flood threshold = R2.  Followed by the
 * postfilter at rknn_query.cpp:2555-2561,2762-2765. */
int ao_range_search(const ao_index* ix, const float* q, uint32_t L, const float* thr,
                    uint32_t* cand, uint32_t cand_cap, uint32_t* n_cand,
                    uint32_t* pred, uint32_t pred_cap, uint32_t* n_pred, uint32_t* n_dist) {
    const uint32_t dim = ix->dim, d = ix->d;
    float* qb = (float*)malloc(sizeof(float) * dim);
    ao_lift_query(q, d, ix->scale, qb);
    /* rknn_query.cpp:2724-2731: ip adds the lifted query's squared norm */
    double qn2s = 0;
    for (uint32_t j = 0; j < d; j++) {
        double v = (double)q[j] * ix->scale;
        qn2s += v * v;
    }
    double R2 = ix->metric ? (qn2s + 1.0 + ix->mstar2) : (ix->mstar2 + 1.0);
    uint8_t* vis = (uint8_t*)calloc(ix->n, 1);
    uint32_t* flood = (uint32_t*)malloc(sizeof(uint32_t) * (ix->n + 1));
    uint64_t nf = 0, head = 0;
    uint32_t nc = 0, nd = 0;
    int rc = 0;
    queue_t beam;
    q_init(&beam, L);
    uint32_t ep = ao_tree_entry(ix->tree_nodes, dim, ix->tree_left, ix->tree_right, ix->tree_offset,
                                ix->tree_hyperplane, ix->tree_leaf_first, qb);
    float dep = ao_l2sqr(ix->lifted + (uint64_t)ep * dim, qb, dim);
    nd++;
    vis[ep] = 1;
    q_insert(&beam, dep, ep);
    if ((double)dep <= R2) {
        flood[nf++] = ep;
        if (nc < cand_cap) cand[nc] = ep;
        nc++;
    }
    while (beam.cur < beam.size) {
        uint32_t cur = q_pop(&beam);
        const uint32_t* lk = ix->links + (uint64_t)cur * ix->degree;
        for (uint32_t j = 0; j < ix->deg[cur]; j++) {
            uint32_t nb = lk[j];
            if (vis[nb]) continue;
            vis[nb] = 1;
            float dd = ao_l2sqr(ix->lifted + (uint64_t)nb * dim, qb, dim);
            nd++;
            q_insert(&beam, dd, nb);
            if ((double)dd <= R2) {
                flood[nf++] = nb;
                if (nc < cand_cap) cand[nc] = nb;
                nc++;
            }
        }
    }
    while (head < nf) {
        uint32_t cur = flood[head++];
        const uint32_t* lk = ix->links + (uint64_t)cur * ix->degree;
        for (uint32_t j = 0; j < ix->deg[cur]; j++) {
            uint32_t nb = lk[j];
            if (vis[nb]) continue;
            vis[nb] = 1;
            float dd = ao_l2sqr(ix->lifted + (uint64_t)nb * dim, qb, dim);
            nd++;
            if ((double)dd <= R2) {
                if (nc < cand_cap) cand[nc] = nb;
                nc++;
                flood[nf++] = nb;
            }
        }
    }
    uint32_t np = 0;
    if (nc > cand_cap) rc = -1;
    float qn = ao_ip(q, q, d);
    for (uint32_t c = 0; c < nc && c < cand_cap; c++) {
        const float* o = ix->base + (uint64_t)cand[c] * d;
        float ip = ao_ip(o, q, d);
        float on = ao_ip(o, o, d);
        float key = ix->metric ? -ip : (on + qn) - 2.0f * ip;  /* rknn_query.cpp:2555-2561 */
        if ((double)key <= (double)thr[cand[c]]) {
            if (np < pred_cap) pred[np] = cand[c];
            else rc = -1;
            np++;
        }
    }
    *n_cand = nc;
    *n_pred = np;
    *n_dist = nd;
    free(beam.data);
    free(flood);
    free(vis);
    free(qb);
    return rc;
}

/* ------------------------------------------------------- gather / prune */

static float gd2(const ao_knn_graph* g, uint64_t a, uint64_t b) {
    return metric_d2(g->x + a * g->dim, g->x + b * g->dim, g->norms[a], g->norms[b], g->dim, g->metric);
}

/* index.h:1491-1525 */
int64_t ao_gather(const ao_knn_graph* g, uint64_t i, uint32_t ef, uint32_t cap,
                  float* pool_d, uint32_t* pool_id, uint64_t pool_cap) {
    uint8_t* vis = (uint8_t*)calloc(g->n, 1);
    queue_t cand;
    q_init(&cand, ef);
    uint64_t np = 0;
    int over = 0;
#define AO_PUSH(ID, D)                     \
    do {                                   \
        if (np < pool_cap) {               \
            pool_d[np] = (D);              \
            pool_id[np] = (ID);            \
        } else                             \
            over = 1;                      \
        np++;                              \
    } while (0)
    for (uint32_t j = 0; j < g->K; j++) {
        uint32_t id = g->g_ids[i * g->K + j];
        if (id == AO_EMPTY || id >= g->n) continue;
        if (vis[id]) continue;
        vis[id] = 1;
        float d = g->g_vals[i * g->K + j];
        q_insert(&cand, d, id);
        AO_PUSH(id, d);
    }
    while (cand.cur < cand.size) {
        uint32_t cur = q_pop(&cand);
        for (uint32_t j = 0; j < g->K; j++) {
            uint32_t nb = g->g_ids[(uint64_t)cur * g->K + j];
            if (nb == AO_EMPTY || nb >= g->n || vis[nb]) continue;
            vis[nb] = 1;
            float d = gd2(g, i, nb);
            q_insert(&cand, d, nb);
            AO_PUSH(nb, d);
        }
        for (uint64_t p = g->rev_off[cur]; p < g->rev_off[cur + 1]; p++) {
            uint32_t nb = g->rev_ids[p];
            if (nb == AO_EMPTY || nb >= g->n || vis[nb]) continue;
            vis[nb] = 1;
            float d = gd2(g, i, nb);
            q_insert(&cand, d, nb);
            AO_PUSH(nb, d);
        }
        if (np >= cap) break;
    }
#undef AO_PUSH
    free(cand.data);
    free(vis);
    return over ? -1 : (int64_t)np;
}

typedef struct {
    float d;
    uint32_t id;
} pair_t;

static int cmp_dist_id(const void* a, const void* b) {
    const pair_t* x = (const pair_t*)a;
    const pair_t* y = (const pair_t*)b;
    if (x->d < y->d) return -1;
    if (x->d > y->d) return 1;
    return (x->id > y->id) - (x->id < y->id);
}

static int cmp_id_dist(const void* a, const void* b) {
    const pair_t* x = (const pair_t*)a;
    const pair_t* y = (const pair_t*)b;
    if (x->id != y->id) return (x->id > y->id) - (x->id < y->id);
    return (x->d > y->d) - (x->d < y->d);
}

/* index.h:1347-1366 */
void ao_aknn_rows(const ao_knn_graph* g, uint32_t ef, uint32_t cap, uint32_t K,
                  uint32_t* out_ids, float* out_d) {
    uint64_t pool_cap = (uint64_t)cap + (uint64_t)g->K + (g->rev_off[g->n] - g->rev_off[0]) + 1;
    float* pd = (float*)malloc(sizeof(float) * pool_cap);
    uint32_t* pi = (uint32_t*)malloc(sizeof(uint32_t) * pool_cap);
    pair_t* pr = (pair_t*)malloc(sizeof(pair_t) * pool_cap);
    for (uint64_t i = 0; i < g->n; i++) {
        int64_t np = ao_gather(g, i, ef, cap, pd, pi, pool_cap);
        for (int64_t p = 0; p < np; p++) {
            pr[p].d = pd[p];
            pr[p].id = pi[p];
        }
        qsort(pr, (size_t)np, sizeof(pair_t), cmp_dist_id);
        uint32_t c = 0;
        for (int64_t p = 0; p < np && c < K; p++) {
            if (pr[p].id == (uint32_t)i) continue;
            out_ids[i * K + c] = pr[p].id;
            out_d[i * K + c] = pr[p].d;
            c++;
        }
        for (; c < K; c++) {
            out_ids[i * K + c] = AO_EMPTY;
            out_d[i * K + c] = FLT_MAX;
        }
    }
    free(pd);
    free(pi);
    free(pr);
}

/* sort_unique_candidates (index.h:225-248) + rng_extend (index.h:267-281) as
 * prune_pool_to_ids runs them with the default edge policy (index.h:823-828). */
/* ---- edge policies, include/index.h:283-829 ----
 * One prune's state: the pool sorted by (dist, id) without duplicates or the
 * base (sort_unique_candidates, :225-247), and the selected ids. */
typedef struct {
    const float* x;
    const float* norms;
    uint32_t dim;
    uint64_t base;
    float alpha;
    uint32_t M;
    const ao_edge_policy* pol;
    const pair_t* cand;
    uint64_t nc;
    uint32_t* ids;
    uint32_t nids;
} ao_prune_state;

typedef struct {
    double key;
    uint32_t id;
} dpair_t;

static int cmp_dkey_id(const void* a, const void* b) {
    const dpair_t* x = (const dpair_t*)a;
    const dpair_t* y = (const dpair_t*)b;
    if (x->key < y->key) return -1;
    if (x->key > y->key) return 1;
    return (x->id > y->id) - (x->id < y->id);
}

static float ps_d2(const ao_prune_state* st, uint32_t a, uint32_t b) {
    return ao_d2(st->x + (uint64_t)a * st->dim, st->x + (uint64_t)b * st->dim, st->norms[a], st->norms[b], st->dim);
}

static int ps_has(const ao_prune_state* st, uint32_t id) {
    for (uint32_t s = 0; s < st->nids; s++)
        if (st->ids[s] == id) return 1;
    return 0;
}

/* edge_radj, :292-294 */
static double ps_radj(const ao_prune_state* st, uint32_t id, uint32_t k) {
    return st->pol->scale2 * (double)st->pol->resid[(uint64_t)id * st->pol->nk + (k - 1)];
}

/* edge_sort_radj, :296-303 */
static double ps_sort_radj(const ao_prune_state* st, uint32_t id) {
    const ao_edge_policy* p = st->pol;
    if (!p || !(p->flags & AO_EDGE_BALL) || p->nks == 0) return 0.0;
    double best = -INFINITY;
    for (uint32_t t = 0; t < p->nks; t++) {
        const double r = ps_radj(st, id, p->ks[t]);
        best = best > r ? best : r;
    }
    return isfinite(best) ? best : 0.0;
}

/* rng_extend, :264-278 */
static void ps_rng_extend(ao_prune_state* st, uint32_t cap) {
    for (uint64_t q = 0; q < st->nc; q++) {
        if (st->nids >= cap) break;
        const uint32_t cid = st->cand[q].id;
        if (ps_has(st, cid)) continue;
        int occluded = 0;
        for (uint32_t s = 0; s < st->nids && !occluded; s++)
            if (st->alpha * ps_d2(st, st->ids[s], cid) < st->cand[q].d) occluded = 1;
        if (!occluded) st->ids[st->nids++] = cid;
    }
}

/* ball_occludes_distance, :478-495 */
static int ps_ball_occludes(const ao_prune_state* st, uint32_t sid, float dbase_cid, float dsc) {
    const ao_edge_policy* p = st->pol;
    if (!(p->flags & AO_EDGE_BALL) || p->nks == 0) return 0;
    int any = 0, all = 1;
    for (uint32_t t = 0; t < p->nks; t++) {
        const uint32_t k = p->ks[t];
        const double lhs = (double)st->alpha * (double)dsc - p->lambda * ps_radj(st, sid, k);
        const double rhs = (double)dbase_cid - p->lambda * ps_radj(st, (uint32_t)st->base, k);
        const int occ = lhs < rhs;
        any = any || occ;
        all = all && occ;
        if (!p->occlude_all && any) return 1;
        if (p->occlude_all && !all) return 0;
    }
    return p->occlude_all ? all : any;
}

/* ball_sort_candidates, :501-510: the pool by (dist - lambda * sort_radj, id) */
static dpair_t* ps_ball_order(const ao_prune_state* st) {
    dpair_t* o = (dpair_t*)malloc(sizeof(dpair_t) * (st->nc + 1));
    for (uint64_t q = 0; q < st->nc; q++) {
        o[q].id = st->cand[q].id;
        o[q].key = (st->pol->flags & AO_EDGE_BALL)
                       ? (double)st->cand[q].d - st->pol->lambda * ps_sort_radj(st, st->cand[q].id)
                       : (double)st->cand[q].d;
    }
    if (st->pol->flags & AO_EDGE_BALL) qsort(o, (size_t)st->nc, sizeof(dpair_t), cmp_dkey_id);
    return o;
}

static float ps_cand_d(const ao_prune_state* st, uint32_t id) {
    for (uint64_t q = 0; q < st->nc; q++)
        if (st->cand[q].id == id) return st->cand[q].d;
    return 0.0f;
}

/* rng_extend_ball, :512-527 (the occlusion compares the raw distance of the
 * candidate, its pool entry, whatever the order) */
static void ps_rng_extend_ball(ao_prune_state* st, const dpair_t* order, uint32_t cap) {
    for (uint64_t q = 0; q < st->nc; q++) {
        if (st->nids >= cap) break;
        const uint32_t cid = order[q].id;
        if (ps_has(st, cid)) continue;
        const float d2c = ps_cand_d(st, cid);
        int occluded = 0;
        for (uint32_t s = 0; s < st->nids && !occluded; s++)
            if (ps_ball_occludes(st, st->ids[s], d2c, ps_d2(st, st->ids[s], cid))) occluded = 1;
        if (!occluded) st->ids[st->nids++] = cid;
    }
}

/* lsg_distance2, :719-725 */
static double ps_lsg_d2(const ao_prune_state* st, uint32_t a, uint32_t b, double raw) {
    const ao_edge_policy* p = st->pol;
    if (!(p->flags & AO_EDGE_LSG) || p->lsg_alpha == 0.0) return raw;
    const double mu_product = (double)p->mu[a] * (double)p->mu[b];
    const double denom = pow(mu_product, p->lsg_alpha);
    if (!isfinite(denom) || denom <= 0.0) return raw;
    return raw / denom;
}

/* lsg_sort_candidates, :727-737 */
static dpair_t* ps_lsg_order(const ao_prune_state* st) {
    dpair_t* o = (dpair_t*)malloc(sizeof(dpair_t) * (st->nc + 1));
    for (uint64_t q = 0; q < st->nc; q++) {
        o[q].id = st->cand[q].id;
        o[q].key = ps_lsg_d2(st, (uint32_t)st->base, st->cand[q].id, (double)st->cand[q].d);
    }
    qsort(o, (size_t)st->nc, sizeof(dpair_t), cmp_dkey_id);
    return o;
}

/* rng_extend_lsg, :739-754 */
static void ps_rng_extend_lsg(ao_prune_state* st, const dpair_t* order, uint32_t cap) {
    for (uint64_t q = 0; q < st->nc; q++) {
        if (st->nids >= cap) break;
        const uint32_t cid = order[q].id;
        if (ps_has(st, cid)) continue;
        int occluded = 0;
        for (uint32_t s = 0; s < st->nids && !occluded; s++) {
            const double dsc = ps_lsg_d2(st, st->ids[s], cid, (double)ps_d2(st, st->ids[s], cid));
            if ((double)st->alpha * dsc < order[q].key) occluded = 1;
        }
        if (!occluded) st->ids[st->nids++] = cid;
    }
}

/* add_residual_cover_edges, :441-476 */
static void ps_residual_cover(ao_prune_state* st) {
    const ao_edge_policy* p = st->pol;
    if (!(p->flags & AO_EDGE_COVER) || st->nids >= st->M) return;
    uint32_t total = p->budget < st->M - st->nids ? p->budget : st->M - st->nids;
    if (total == 0 || p->nks == 0) return;
    uint32_t per_k = (total + p->nks - 1) / p->nks;
    if (per_k < 1) per_k = 1;
    uint32_t added_total = 0;
    dpair_t* scored = (dpair_t*)malloc(sizeof(dpair_t) * (st->nc + 1));
    for (uint32_t t = 0; t < p->nks; t++) {
        if (added_total >= total || st->nids >= st->M) break;
        const uint32_t k = p->ks[t];
        uint64_t m = 0;
        for (uint64_t q = 0; q < st->nc; q++) {
            const uint32_t cid = st->cand[q].id;
            if (cid == (uint32_t)st->base || ps_has(st, cid)) continue;
            const double residual = (double)p->resid[(uint64_t)cid * p->nk + (k - 1)];
            const double risk = residual > 0.0 ? residual : 0.0;
            if (risk <= 0.0) continue;
            scored[m].key = (double)st->cand[q].d - p->lambda * p->scale2 * risk;
            scored[m].id = cid;
            m++;
        }
        qsort(scored, (size_t)m, sizeof(dpair_t), cmp_dkey_id);
        uint32_t added_k = 0;
        for (uint64_t q = 0; q < m; q++) {
            if (st->nids >= st->M || added_total >= total || added_k >= per_k) break;
            if (ps_has(st, scored[q].id)) continue;
            st->ids[st->nids++] = scored[q].id;
            added_k++;
            added_total++;
        }
    }
    free(scored);
}

/* optimize_verification_constrained_bubble, :531-717 */
static void ps_bubble(ao_prune_state* st) {
    const ao_edge_policy* p = st->pol;
    if (!(p->flags & AO_EDGE_AUTO) || st->nids == 0 || st->nc == 0) return;
    dpair_t* order = ps_ball_order(st);
    const uint64_t ucap = st->nids + st->nc;
    uint32_t* universe = (uint32_t*)malloc(sizeof(uint32_t) * ucap);
    uint64_t nu = 0;
    for (uint32_t s = 0; s < st->nids; s++) universe[nu++] = st->ids[s];
    const uint64_t limit = (p->flags & AO_EDGE_AUTO_FULL) ? st->nc : p->auto_candidates;
    uint64_t alternatives = 0;
    for (uint64_t q = 0; q < st->nc; q++) {
        int dup = 0;
        for (uint64_t u = 0; u < nu && !dup; u++) dup = universe[u] == order[q].id;
        if (dup) continue;
        universe[nu++] = order[q].id;
        if (++alternatives >= limit) break;
    }
    free(order);
    if (alternatives == 0) {
        free(universe);
        return;
    }
    pair_t* targets = (pair_t*)malloc(sizeof(pair_t) * (st->nc + 1));
    uint64_t T = 0;
    if (p->flags & AO_EDGE_AUTO_FULL) {
        for (uint64_t q = 0; q < st->nc; q++) targets[T++] = st->cand[q];
    } else {
        for (uint64_t u = 0; u < nu; u++)
            for (uint64_t q = 0; q < st->nc; q++)
                if (st->cand[q].id == universe[u]) {
                    targets[T++] = st->cand[q];
                    break;
                }
        qsort(targets, (size_t)T, sizeof(pair_t), cmp_dist_id);
    }
    const uint64_t words = (T + 63) / 64;
    uint64_t* verify = (uint64_t*)calloc(nu * words + 1, sizeof(uint64_t));
    uint64_t* route = (uint64_t*)calloc(nu * words + 1, sizeof(uint64_t));
    double* power = (double*)malloc(sizeof(double) * (nu + 1));
    for (uint64_t u = 0; u < nu; u++) {
        const uint32_t id = universe[u];
        const float dbase_u = ps_cand_d(st, id);
        power[u] = (double)dbase_u - p->lambda * ps_sort_radj(st, id);
        for (uint64_t ti = 0; ti < T; ti++) {
            const uint32_t target = targets[ti].id;
            float dsc = 0.0f;
            if (id != target) dsc = ps_d2(st, id, target);
            const uint64_t bit = 1ull << (ti & 63u);
            if (id == target || st->alpha * dsc < targets[ti].d) verify[u * words + (ti >> 6)] |= bit;
            if (ps_ball_occludes(st, id, targets[ti].d, dsc)) route[u * words + (ti >> 6)] |= bit;
        }
    }
    uint64_t* selected = (uint64_t*)malloc(sizeof(uint64_t) * (st->nids + 1));
    uint8_t* is_sel = (uint8_t*)calloc(nu + 1, 1);
    uint64_t nsel = 0;
    for (uint32_t s = 0; s < st->nids; s++)
        for (uint64_t u = 0; u < nu; u++)
            if (universe[u] == st->ids[s]) {
                selected[nsel++] = u;
                is_sel[u] = 1;
                break;
            }
    if (nsel > 0) {
        int32_t* vcount = (int32_t*)calloc(T + 1, sizeof(int32_t));
        int32_t* rcount = (int32_t*)calloc(T + 1, sizeof(int32_t));
        uint8_t* required = (uint8_t*)calloc(T + 1, 1);
#define AO_SIG(u, delta)                                                         \
    for (uint64_t ti = 0; ti < T; ti++) {                                        \
        const uint64_t bit = 1ull << (ti & 63u);                                 \
        if (verify[(u) * words + (ti >> 6)] & bit) vcount[ti] += (delta);        \
        if (route[(u) * words + (ti >> 6)] & bit) rcount[ti] += (delta);         \
    }
        for (uint64_t s = 0; s < nsel; s++) AO_SIG(selected[s], 1);
        for (uint64_t ti = 0; ti < T; ti++) required[ti] = vcount[ti] > 0;
        uint64_t swaps = 0;
        const uint64_t max_swaps = p->auto_max_swaps < alternatives ? p->auto_max_swaps : alternatives;
        while (swaps < max_swaps) {
            long best_gain = LONG_MIN;
            double best_power = -INFINITY;
            uint64_t best_q = UINT64_MAX, best_slot = UINT64_MAX;
            for (uint64_t q = 0; q < nu; q++) {
                if (is_sel[q]) continue;
                long newly = 0;
                for (uint64_t ti = 0; ti < T; ti++)
                    if (rcount[ti] == 0 && (route[q * words + (ti >> 6)] >> (ti & 63u) & 1u)) newly++;
                for (uint64_t slot = 0; slot < nsel; slot++) {
                    const uint64_t old = selected[slot];
                    int feasible = 1;
                    long lost = 0;
                    for (uint64_t ti = 0; ti < T; ti++) {
                        const int ov = (verify[old * words + (ti >> 6)] >> (ti & 63u)) & 1u;
                        const int qv = (verify[q * words + (ti >> 6)] >> (ti & 63u)) & 1u;
                        if (required[ti] && ov && vcount[ti] == 1 && !qv) {
                            feasible = 0;
                            break;
                        }
                        const int orr = (route[old * words + (ti >> 6)] >> (ti & 63u)) & 1u;
                        const int qr = (route[q * words + (ti >> 6)] >> (ti & 63u)) & 1u;
                        if (orr && rcount[ti] == 1 && !qr) lost++;
                    }
                    if (!feasible) continue;
                    const long gain = newly - lost;
                    const double pg = power[old] - power[q];
                    if (gain > best_gain || (gain == best_gain && pg > best_power)) {
                        best_gain = gain;
                        best_power = pg;
                        best_q = q;
                        best_slot = slot;
                    }
                }
            }
            if (best_q == UINT64_MAX || best_gain < 0 || (best_gain == 0 && best_power <= 1e-12)) break;
            const uint64_t old = selected[best_slot];
            AO_SIG(old, -1);
            AO_SIG(best_q, 1);
            is_sel[old] = 0;
            is_sel[best_q] = 1;
            selected[best_slot] = best_q;
            swaps++;
        }
#undef AO_SIG
        for (uint64_t s = 0; s < nsel; s++) st->ids[s] = universe[selected[s]];
        free(vcount);
        free(rcount);
        free(required);
    }
    free(selected);
    free(is_sel);
    free(verify);
    free(route);
    free(power);
    free(targets);
    free(universe);
}

/* prune_pool_to_ids, :772-829 */
uint32_t ao_prune_policy(const float* x, const float* norms, uint32_t dim, uint64_t n, uint64_t i,
                         const float* pool_d, const uint32_t* pool_id, uint64_t pool_n, uint32_t M, float alpha,
                         const ao_edge_policy* pol, uint32_t* out) {
    /* sort_unique_candidates, :225-247 */
    pair_t* c = (pair_t*)malloc(sizeof(pair_t) * (pool_n + 1));
    uint64_t m = 0;
    for (uint64_t p = 0; p < pool_n; p++) {
        uint32_t id = pool_id[p];
        if (id == AO_EMPTY || id >= n || id == (uint32_t)i) continue;
        c[m].d = pool_d[p];
        c[m].id = id;
        m++;
    }
    qsort(c, (size_t)m, sizeof(pair_t), cmp_id_dist);
    uint64_t w = 0;
    for (uint64_t r = 0; r < m;) {
        uint32_t id = c[r].id;
        float best = c[r].d;
        uint64_t e = r + 1;
        while (e < m && c[e].id == id) {
            if (c[e].d < best) best = c[e].d;
            e++;
        }
        c[w].d = best;
        c[w].id = id;
        w++;
        r = e;
    }
    qsort(c, (size_t)w, sizeof(pair_t), cmp_dist_id);
    /* the selection may hold up to M ids and, transiently, no more */
    ao_prune_state st = {x, norms, dim, i, alpha, M, pol, c, w, out, 0};
    const uint32_t f = pol ? pol->flags : 0u;
    if (f & AO_EDGE_AUTO) {
        ps_rng_extend(&st, M);
        ps_bubble(&st);
    } else if ((f & AO_EDGE_LSG) && (f & AO_EDGE_BALL) && pol->lsg_alpha != 0.0) {
        dpair_t* lo = ps_lsg_order(&st);
        uint32_t lsg_cap = M - (pol->budget < M ? pol->budget : M);
        if (lsg_cap == 0) lsg_cap = M;
        ps_rng_extend_lsg(&st, lo, lsg_cap);
        dpair_t* bo = ps_ball_order(&st);
        ps_rng_extend_ball(&st, bo, M);
        ps_rng_extend_lsg(&st, lo, M);
        free(lo);
        free(bo);
    } else if ((f & AO_EDGE_LSG) && pol->lsg_alpha != 0.0) {
        dpair_t* lo = ps_lsg_order(&st);
        ps_rng_extend_lsg(&st, lo, M);
        free(lo);
    } else if (f & AO_EDGE_BALL) {
        dpair_t* bo = ps_ball_order(&st);
        if (f & AO_EDGE_PURE) {
            ps_rng_extend_ball(&st, bo, M);
            ps_rng_extend(&st, M);
        } else {
            uint32_t center_cap = M - (pol->budget < M ? pol->budget : M);
            if (center_cap == 0) center_cap = M;
            ps_rng_extend(&st, center_cap);
            ps_rng_extend_ball(&st, bo, M);
            ps_rng_extend(&st, M);
        }
        free(bo);
    } else {
        const uint32_t cover = (f & AO_EDGE_COVER) ? (pol->budget < M ? pol->budget : M) : 0u;
        uint32_t normal_cap = M - cover;
        if (normal_cap == 0) normal_cap = M;
        ps_rng_extend(&st, normal_cap);
        if (f & AO_EDGE_COVER) ps_residual_cover(&st);
        ps_rng_extend(&st, M);
    }
    free(c);
    return st.nids;
}

uint32_t ao_prune(const float* x, const float* norms, uint32_t dim, uint64_t n, uint64_t i,
                  float* pool_d, uint32_t* pool_id, uint64_t pool_n, uint32_t M, float alpha,
                  uint32_t* out) {
    return ao_prune_policy(x, norms, dim, n, i, pool_d, pool_id, pool_n, M, alpha, NULL, out);
}

/* build_index gather + prune loop, index.h:1248-1257 */
void ao_graph_select_policy(const ao_knn_graph* g, uint32_t ef, uint32_t cap, uint32_t M, float alpha,
                            const ao_edge_policy* pol, uint32_t* O, uint32_t* O_deg) {
    uint64_t pool_cap = (uint64_t)cap + (uint64_t)g->K + (g->rev_off[g->n] - g->rev_off[0]) + 1;
    float* pd = (float*)malloc(sizeof(float) * pool_cap);
    uint32_t* pi = (uint32_t*)malloc(sizeof(uint32_t) * pool_cap);
    for (uint64_t i = 0; i < g->n; i++) {
        int64_t np = ao_gather(g, i, ef, cap, pd, pi, pool_cap);
        uint32_t* row = O + i * M;
        for (uint32_t j = 0; j < M; j++) row[j] = AO_EMPTY;
        O_deg[i] = ao_prune_policy(g->x, g->norms, g->dim, g->n, i, pd, pi, (uint64_t)np, M, alpha, pol, row);
    }
    free(pd);
    free(pi);
}

void ao_graph_select(const ao_knn_graph* g, uint32_t ef, uint32_t cap, uint32_t M, float alpha,
                     uint32_t* O, uint32_t* O_deg) {
    ao_graph_select_policy(g, ef, cap, M, alpha, NULL, O, O_deg);
}

/* One pass of the global Vamana refine (index.h:856-875 greedy_collect,
 * 767-770 append_aknn_edges, 1262-1285): for every row i, a beam of width Lb
 * over the current graph (links n x M, deg) from entry[i] collects every
 * visited node but i with its distance, the row's g0 list (n x K, ANQI_EMPTY
 * skipped) follows with fresh distances, and the pool is pruned as
 * prune_pool_to_ids -> O (n x M, ANQI_EMPTY padded), O_deg. */
/* A Vamana pool of row i (appended to pd/pi, grown as needed): the visits of
 * a beam of width Lb over the current graph (links, deg) from ep but i
 * (greedy_collect / greedy_collect_from_entry, index.h:856-903), the row's g0
 * list (append_aknn_edges, :767-770) and, when cur, the row's current links
 * (append_current_edges, :759-765), each with a fresh distance. */
typedef struct {
    float* d;
    uint32_t* id;
    uint64_t n, cap;
} ao_pool;

static void pool_push(ao_pool* p, uint32_t id, float d) {
    if (p->n == p->cap) {
        p->cap = p->cap ? 2 * p->cap : 1024;
        p->d = (float*)realloc(p->d, sizeof(float) * p->cap);
        p->id = (uint32_t*)realloc(p->id, sizeof(uint32_t) * p->cap);
    }
    p->d[p->n] = d;
    p->id[p->n] = id;
    p->n++;
}

static void vamana_pool(const float* x, const float* norms, uint32_t dim, uint64_t n, const uint32_t* links,
                        const uint32_t* deg, uint32_t M, const uint32_t* g0, uint32_t K, uint64_t i, uint32_t ep,
                        uint32_t Lb, int cur_edges, uint8_t* vis, ao_pool* pool) {
    memset(vis, 0, n);
    pool->n = 0;
    queue_t beam;
    q_init(&beam, Lb);
    if (ep >= n) ep = 0;
    vis[ep] = 1;
    float d0 = ao_d2(x + i * dim, x + (uint64_t)ep * dim, norms[i], norms[ep], dim);
    q_insert(&beam, d0, ep);
    if (ep != (uint32_t)i) pool_push(pool, ep, d0);
    while (beam.cur < beam.size) {
        uint32_t cur = q_pop(&beam);
        for (uint32_t j = 0; j < deg[cur]; j++) {
            uint32_t nb = links[(uint64_t)cur * M + j];
            if (nb >= n || vis[nb]) continue;
            vis[nb] = 1;
            float d = ao_d2(x + i * dim, x + (uint64_t)nb * dim, norms[i], norms[nb], dim);
            q_insert(&beam, d, nb);
            if (nb != (uint32_t)i) pool_push(pool, nb, d);
        }
    }
    free(beam.data);
    for (uint32_t k = 0; k < K; k++) {
        uint32_t j = g0[i * K + k];
        if (j == AO_EMPTY || j >= n || j == (uint32_t)i) continue;
        pool_push(pool, j, ao_d2(x + i * dim, x + (uint64_t)j * dim, norms[i], norms[j], dim));
    }
    if (cur_edges)
        for (uint32_t k = 0; k < deg[i]; k++) {
            uint32_t j = links[i * M + k];
            if (j == AO_EMPTY || j >= n || j == (uint32_t)i) continue;
            pool_push(pool, j, ao_d2(x + i * dim, x + (uint64_t)j * dim, norms[i], norms[j], dim));
        }
}

void ao_vamana_select_policy(const float* x, const float* norms, uint32_t dim, uint64_t n, const uint32_t* links,
                             const uint32_t* deg, uint32_t M, const uint32_t* g0, uint32_t K, const uint32_t* entry,
                             uint32_t Lb, float alpha, const ao_edge_policy* pol, uint32_t* O, uint32_t* O_deg) {
    uint8_t* vis = (uint8_t*)malloc(n);
    ao_pool pool = {0};
    for (uint64_t i = 0; i < n; i++) {
        vamana_pool(x, norms, dim, n, links, deg, M, g0, K, i, entry[i], Lb, 0, vis, &pool);
        uint32_t* row = O + i * M;
        for (uint32_t j = 0; j < M; j++) row[j] = AO_EMPTY;
        O_deg[i] = ao_prune_policy(x, norms, dim, n, i, pool.d, pool.id, pool.n, M, alpha, pol, row);
    }
    free(vis);
    free(pool.d);
    free(pool.id);
}

void ao_vamana_select(const float* x, const float* norms, uint32_t dim, uint64_t n, const uint32_t* links,
                      const uint32_t* deg, uint32_t M, const uint32_t* g0, uint32_t K, const uint32_t* entry,
                      uint32_t Lb, float alpha, uint32_t* O, uint32_t* O_deg) {
    ao_vamana_select_policy(x, norms, dim, n, links, deg, M, g0, K, entry, Lb, alpha, NULL, O, O_deg);
}

/* vamana_batch_refine, index.h:936-1065: per pass, the order shuffled
 * (ao_vamana_batch_order) and cut into batches of 1, b-1, b^2-b, ... rows up
 * to max_batch, then max_batch rows; a batch's rows each prune a pool from
 * the graph as it was at the batch's start (beam from the single entry, g0,
 * current links) and take the result as their links; then every row that a
 * batch row now links to prunes its current links plus those batch rows. */
void ao_vamana_batch_refine(const float* x, const float* norms, uint32_t dim, uint64_t n, uint32_t* links,
                            uint32_t* deg, uint32_t M, const uint32_t* g0, uint32_t K, uint32_t entry, uint32_t Lb,
                            int passes, float final_alpha, float early_alpha, int early_one, double max_frac,
                            uint64_t max_batch_cap, double batch_base, uint64_t seed, const ao_edge_policy* pol) {
    if (n == 0 || passes <= 0) return;
    if (max_frac <= 0.0) max_frac = 0.02;
    double mb = max_frac * (double)n;
    uint64_t max_batch = (uint64_t)(mb > 1.0 ? mb : 1.0);
    if (max_batch > max_batch_cap) max_batch = max_batch_cap;
    if (max_batch == 0) max_batch = n;
    if (batch_base <= 1.0) batch_base = 2.0;
    uint32_t* order = (uint32_t*)malloc(sizeof(uint32_t) * n);
    for (uint64_t i = 0; i < n; i++) order[i] = (uint32_t)i;
    uint8_t* vis = (uint8_t*)malloc(n);
    uint32_t* out = NULL;
    uint32_t* out_deg = NULL;
    uint32_t* rcount = (uint32_t*)calloc(n, sizeof(uint32_t));
    uint64_t* roff = (uint64_t*)calloc(n + 1, sizeof(uint64_t));
    uint32_t* rfill = (uint32_t*)calloc(n, sizeof(uint32_t));
    uint32_t* touched = (uint32_t*)malloc(sizeof(uint32_t) * n);
    uint32_t* rsrc = NULL;
    uint32_t ids[64];
    ao_pool pool = {0};
    for (int pass = 0; pass < passes; pass++) {
        const float alpha = (early_one && pass + 1 < passes) ? early_alpha : final_alpha;
        ao_vamana_batch_order(order, n, seed, pass);
        uint64_t count = 0, inc = 0;
        while (count < n) {
            uint64_t floor_ = count, ceiling;
            const double p0 = pow(batch_base, (double)inc);
            if (p0 <= (double)max_batch) {
                floor_ = (uint64_t)p0 - 1;
                const double p1 = pow(batch_base, (double)(inc + 1));
                ceiling = (uint64_t)p1 - 1;
                if (ceiling > n) ceiling = n;
                count = ceiling;
            } else {
                ceiling = count + max_batch < n ? count + max_batch : n;
                count = ceiling;
            }
            inc++;
            if (ceiling <= floor_ || floor_ >= n) continue;
            const uint64_t bsz = ceiling - floor_;
            out = (uint32_t*)realloc(out, sizeof(uint32_t) * bsz * M);
            out_deg = (uint32_t*)realloc(out_deg, sizeof(uint32_t) * bsz);
            for (uint64_t b = 0; b < bsz; b++) {
                const uint32_t node = order[floor_ + b];
                vamana_pool(x, norms, dim, n, links, deg, M, g0, K, node, entry, Lb, 1, vis, &pool);
                out_deg[b] = ao_prune_policy(x, norms, dim, n, node, pool.d, pool.id, pool.n, M, alpha, pol,
                                             out + b * M);
            }
            for (uint64_t b = 0; b < bsz; b++) {
                const uint32_t node = order[floor_ + b];
                for (uint32_t j = 0; j < M; j++) links[(uint64_t)node * M + j] = j < out_deg[b] ? out[b * M + j] : AO_EMPTY;
                deg[node] = out_deg[b];
            }
            uint64_t nt = 0, tot = 0;
            for (uint64_t b = 0; b < bsz; b++)
                for (uint32_t j = 0; j < out_deg[b]; j++) {
                    const uint32_t dst = out[b * M + j];
                    if (dst >= n) continue;
                    if (rcount[dst]++ == 0) touched[nt++] = dst;
                    tot++;
                }
            rsrc = (uint32_t*)realloc(rsrc, sizeof(uint32_t) * (tot + 1));
            uint64_t acc = 0;
            for (uint64_t t = 0; t < nt; t++) {
                roff[touched[t]] = acc;
                acc += rcount[touched[t]];
            }
            for (uint64_t b = 0; b < bsz; b++)
                for (uint32_t j = 0; j < out_deg[b]; j++) {
                    const uint32_t dst = out[b * M + j];
                    if (dst >= n) continue;
                    rsrc[roff[dst] + rfill[dst]++] = order[floor_ + b];
                }
            for (uint64_t t = 0; t < nt; t++) {
                const uint32_t dst = touched[t];
                pool.n = 0;
                for (uint32_t k = 0; k < deg[dst]; k++) {
                    const uint32_t j = links[(uint64_t)dst * M + k];
                    if (j == AO_EMPTY || j >= n || j == dst) continue;
                    pool_push(&pool, j, ao_d2(x + (uint64_t)dst * dim, x + (uint64_t)j * dim, norms[dst], norms[j], dim));
                }
                for (uint32_t r = 0; r < rcount[dst]; r++) {
                    const uint32_t src = rsrc[roff[dst] + r];
                    if (src == dst || src >= n) continue;
                    pool_push(&pool, src, ao_d2(x + (uint64_t)dst * dim, x + (uint64_t)src * dim, norms[dst], norms[src], dim));
                }
                const uint32_t nd = ao_prune_policy(x, norms, dim, n, dst, pool.d, pool.id, pool.n, M, alpha, pol, ids);
                for (uint32_t j = 0; j < M; j++) links[(uint64_t)dst * M + j] = j < nd ? ids[j] : AO_EMPTY;
                deg[dst] = nd;
            }
            for (uint64_t t = 0; t < nt; t++) {
                rcount[touched[t]] = 0;
                rfill[touched[t]] = 0;
            }
        }
    }
    free(order);
    free(vis);
    free(out);
    free(out_deg);
    free(rcount);
    free(roff);
    free(rfill);
    free(touched);
    free(rsrc);
    free(pool.d);
    free(pool.id);
}

/* commit_edges, index.h:907-930 */
void ao_graph_commit_policy(const float* x, const float* norms, uint32_t dim, uint64_t n, const uint32_t* O,
                            const uint32_t* O_deg, uint32_t M, float alpha, const ao_edge_policy* pol,
                            uint32_t* links, uint32_t* deg) {
    uint64_t* roff = (uint64_t*)calloc(n + 1, sizeof(uint64_t));
    for (uint64_t i = 0; i < n; i++)
        for (uint32_t j = 0; j < O_deg[i]; j++) roff[O[i * M + j] + 1]++;
    for (uint64_t i = 0; i < n; i++) roff[i + 1] += roff[i];
    uint32_t* rids = (uint32_t*)malloc(sizeof(uint32_t) * (roff[n] + 1));
    uint64_t* fill = (uint64_t*)calloc(n, sizeof(uint64_t));
    for (uint64_t i = 0; i < n; i++)
        for (uint32_t j = 0; j < O_deg[i]; j++) {
            uint32_t t = O[i * M + j];
            rids[roff[t] + fill[t]++] = (uint32_t)i;
        }
    uint64_t maxc = 0;
    for (uint64_t i = 0; i < n; i++) {
        uint64_t c = O_deg[i] + (roff[i + 1] - roff[i]);
        if (c > maxc) maxc = c;
    }
    float* pd = (float*)malloc(sizeof(float) * (maxc + 1));
    uint32_t* pi = (uint32_t*)malloc(sizeof(uint32_t) * (maxc + 1));
    for (uint64_t i = 0; i < n; i++) {
        uint64_t c = 0;
        for (uint32_t j = 0; j < O_deg[i]; j++) {
            uint32_t t = O[i * M + j];
            pd[c] = ao_d2(x + i * dim, x + (uint64_t)t * dim, norms[i], norms[t], dim);
            pi[c++] = t;
        }
        for (uint64_t p = roff[i]; p < roff[i + 1]; p++) {
            uint32_t t = rids[p];
            pd[c] = ao_d2(x + i * dim, x + (uint64_t)t * dim, norms[i], norms[t], dim);
            pi[c++] = t;
        }
        uint32_t* row = links + i * M;
        for (uint32_t j = 0; j < M; j++) row[j] = AO_EMPTY;
        deg[i] = ao_prune_policy(x, norms, dim, n, i, pd, pi, c, M, alpha, pol, row);
    }
    free(pd);
    free(pi);
    free(roff);
    free(rids);
    free(fill);
}

void ao_graph_commit(const float* x, const float* norms, uint32_t dim, uint64_t n,
                     const uint32_t* O, const uint32_t* O_deg, uint32_t M, float alpha,
                     uint32_t* links, uint32_t* deg) {
    ao_graph_commit_policy(x, norms, dim, n, O, O_deg, M, alpha, NULL, links, deg);
}

/* -------------------------------------------------------------- heaps */

/* heap.h:162-186 (push_nolock; check_push without reverse edges is identical) */
int ao_heap_push(uint32_t* ids, float* vals, uint32_t K, uint32_t node, float value) {
    if (value > vals[0]) return 0;
    for (uint32_t i = 0; i < K; i++)
        if (ids[i] == node) return 0;
    uint32_t cur = 0, sw;
    for (;;) {
        uint32_t l = 2 * cur + 1, r = l + 1;
        if (l >= K) break;
        else if (r >= K) {
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
    return 1;
}

/* index.h:1210-1217 */
void ao_warm_start(const float* x, const float* norms, uint32_t dim, uint64_t n,
                   const uint32_t* cand, uint32_t stride, uint32_t width, uint32_t K,
                   uint32_t* ids, float* vals) {
    for (uint64_t i = 0; i < n; i++) {
        uint32_t* hi = ids + i * K;
        float* hv = vals + i * K;
        for (uint32_t s = 0; s < K; s++) {
            hi[s] = AO_EMPTY;
            hv[s] = FLT_MAX;
        }
        for (uint32_t k = 0; k < width; k++) {
            uint32_t j = cand[i * stride + k];
            if (j != (uint32_t)i && j < n)
                ao_heap_push(hi, hv, K, j, ao_d2(x + i * dim, x + (uint64_t)j * dim, norms[i], norms[j], dim));
        }
    }
}

/* index.h:1468-1487, snapshot form (see the header). */
uint64_t ao_localjoin_round(const float* x, const float* norms, uint32_t dim, uint64_t n,
                            uint32_t K, uint32_t sample, uint32_t* ids, float* vals) {
    uint32_t* loc = (uint32_t*)malloc(sizeof(uint32_t) * n * sample);
    uint32_t* cnt = (uint32_t*)calloc(n, sizeof(uint32_t));
    for (uint64_t u = 0; u < n; u++)
        for (uint32_t s = 0; s < K && cnt[u] < sample; s++) {
            uint32_t v = ids[u * K + s];
            if (v != AO_EMPTY) loc[u * sample + cnt[u]++] = v;
        }
    /* incoming (source, position) lists per target, sources ascending */
    uint64_t* off = (uint64_t*)calloc(n + 1, sizeof(uint64_t));
    for (uint64_t u = 0; u < n; u++)
        for (uint32_t a = 0; a < cnt[u]; a++) off[loc[u * sample + a] + 1]++;
    for (uint64_t i = 0; i < n; i++) off[i + 1] += off[i];
    uint64_t* fill = (uint64_t*)calloc(n, sizeof(uint64_t));
    uint64_t* inc = (uint64_t*)malloc(sizeof(uint64_t) * (off[n] + 1));
    for (uint64_t u = 0; u < n; u++)
        for (uint32_t a = 0; a < cnt[u]; a++) {
            uint32_t t = loc[u * sample + a];
            inc[off[t] + fill[t]++] = (u << 8) | a;
        }
    uint64_t upd = 0;
    for (uint64_t t = 0; t < n; t++) {
        for (uint64_t p = off[t]; p < off[t + 1]; p++) {
            uint64_t u = inc[p] >> 8;
            uint32_t a = (uint32_t)(inc[p] & 0xFF);
            for (uint32_t b = 0; b < cnt[u]; b++) {
                if (b == a) continue;
                uint32_t w = loc[u * sample + b];
                float dd = ao_d2(x + t * dim, x + (uint64_t)w * dim, norms[t], norms[w], dim);
                upd += (uint64_t)ao_heap_push(ids + t * K, vals + t * K, K, w, dd);
            }
        }
    }
    free(loc);
    free(cnt);
    free(off);
    free(fill);
    free(inc);
    return upd;
}

/* heap.h:190-207 */
void ao_reverse(const uint32_t* ids, uint64_t n, uint32_t K, uint64_t* rev_off, uint32_t* rev_ids) {
    memset(rev_off, 0, sizeof(uint64_t) * (n + 1));
    for (uint64_t i = 0; i < n; i++)
        for (uint32_t j = 0; j < K; j++) {
            uint32_t v = ids[i * K + j];
            if (v != AO_EMPTY && v < n) rev_off[v + 1]++;
        }
    for (uint64_t i = 0; i < n; i++) rev_off[i + 1] += rev_off[i];
    uint64_t* fill = (uint64_t*)calloc(n, sizeof(uint64_t));
    for (uint64_t i = 0; i < n; i++)
        for (uint32_t j = 0; j < K; j++) {
            uint32_t v = ids[i * K + j];
            if (v != AO_EMPTY && v < n) rev_ids[rev_off[v] + fill[v]++] = (uint32_t)i;
        }
    free(fill);
}

/* ------------------------------------------------------------ init_knn */

void ao_init_knn(const float* x, const float* norms, uint32_t dim, uint64_t n, uint32_t K,
                 const uint64_t* leaf_off, const uint32_t* leaf_ids, uint64_t n_leaves,
                 uint32_t* out_ids, float* out_d) {
    ao_init_knn_metric(x, norms, dim, n, K, leaf_off, leaf_ids, n_leaves, 0, out_ids, out_d);
}

void ao_init_knn_metric(const float* x, const float* norms, uint32_t dim, uint64_t n, uint32_t K,
                        const uint64_t* leaf_off, const uint32_t* leaf_ids, uint64_t n_leaves, uint32_t ip,
                        uint32_t* out_ids, float* out_d) {
    /* per row: collect (d, id) of all leaf-mates, dedupe, keep K smallest */
    uint64_t* cnt = (uint64_t*)calloc(n + 1, sizeof(uint64_t));
    for (uint64_t l = 0; l < n_leaves; l++) {
        uint64_t sz = leaf_off[l + 1] - leaf_off[l];
        for (uint64_t a = leaf_off[l]; a < leaf_off[l + 1]; a++) cnt[leaf_ids[a] + 1] += sz - 1;
    }
    for (uint64_t i = 0; i < n; i++) cnt[i + 1] += cnt[i];
    pair_t* all = (pair_t*)malloc(sizeof(pair_t) * (cnt[n] + 1));
    uint64_t* fill = (uint64_t*)calloc(n, sizeof(uint64_t));
    for (uint64_t l = 0; l < n_leaves; l++)
        for (uint64_t a = leaf_off[l]; a < leaf_off[l + 1]; a++)
            for (uint64_t b = leaf_off[l]; b < leaf_off[l + 1]; b++) {
                if (a == b) continue;
                uint32_t p = leaf_ids[a], q = leaf_ids[b];
                pair_t* e = &all[cnt[p] + fill[p]++];
                e->id = q;
                e->d = metric_d2(x + (uint64_t)p * dim, x + (uint64_t)q * dim, norms[p], norms[q], dim, ip);
            }
    for (uint64_t i = 0; i < n; i++) {
        pair_t* r = all + cnt[i];
        uint64_t m = cnt[i + 1] - cnt[i];
        qsort(r, (size_t)m, sizeof(pair_t), cmp_dist_id);
        uint32_t c = 0;
        for (uint64_t p = 0; p < m && c < K; p++) {
            if (p > 0 && r[p].id == r[p - 1].id) continue; /* same pair, same distance */
            int dup = 0;
            for (uint32_t s = 0; s < c; s++)
                if (out_ids[i * K + s] == r[p].id) {
                    dup = 1;
                    break;
                }
            if (dup) continue;
            out_ids[i * K + c] = r[p].id;
            out_d[i * K + c] = r[p].d;
            c++;
        }
        for (; c < K; c++) {
            out_ids[i * K + c] = AO_EMPTY;
            out_d[i * K + c] = FLT_MAX;
        }
    }
    free(cnt);
    free(all);
    free(fill);
}

/* --------------------------------------------------------------- forest */

uint64_t ao_hash64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static uint64_t node_key(uint64_t seed, uint32_t tree, uint32_t node) {
    return ao_hash64(ao_hash64(seed ^ ((uint64_t)tree << 32)) ^ (uint64_t)node);
}

/* rptrees.h:28-84,127-163 in deterministic breadth-first form. */
int64_t ao_rp_tree(const float* x, uint64_t n, uint32_t dim, uint32_t leaf_size,
                   uint32_t max_depth, uint64_t seed, uint32_t tree, ao_tree_out* out) {
    return ao_rp_tree_metric(x, n, dim, leaf_size, max_depth, seed, tree, 0, out);
}

/* angular (the ip metric, rptrees.h:41-52): the hyperplane is the normalized
 * difference of the two unit-scaled points, offset 0. */
int64_t ao_rp_tree_metric(const float* x, uint64_t n, uint32_t dim, uint32_t leaf_size, uint32_t max_depth,
                          uint64_t seed, uint32_t tree, uint32_t angular, ao_tree_out* out) {
    uint32_t* start = (uint32_t*)malloc(sizeof(uint32_t) * out->cap_nodes);
    uint32_t* count = (uint32_t*)malloc(sizeof(uint32_t) * out->cap_nodes);
    uint32_t* depth = (uint32_t*)malloc(sizeof(uint32_t) * out->cap_nodes);
    uint32_t* tmp = (uint32_t*)malloc(sizeof(uint32_t) * (n + 1));
    uint8_t* side = (uint8_t*)malloc(n + 1);
    float* mid = (float*)malloc(sizeof(float) * dim);
    for (uint64_t i = 0; i < n; i++) out->perm[i] = (uint32_t)i;
    start[0] = 0;
    count[0] = (uint32_t)n;
    depth[0] = 0;
    uint32_t n_nodes = 1;
    int64_t rc = 0;
    for (uint32_t v = 0; v < n_nodes; v++) {
        uint32_t s = start[v], c = count[v];
        float* hp = out->hyperplane + (uint64_t)v * dim;
        if (c <= leaf_size || depth[v] >= max_depth) {
            out->left[v] = out->right[v] = AO_EMPTY;
            out->offset[v] = FLT_MAX;
            out->leaf_off[v] = s;
            out->leaf_cnt[v] = c <= leaf_size ? c : leaf_size;
            continue;
        }
        if (n_nodes + 2 > out->cap_nodes) {
            rc = -1;
            break;
        }
        uint64_t key = node_key(seed, tree, v);
        uint32_t r0 = (uint32_t)(ao_hash64(key ^ 1) % c);
        uint32_t r1 = (uint32_t)(ao_hash64(key ^ 2) % c);
        if (r0 == r1) r0 = (r1 + 1) % c;
        const float* x0 = x + (uint64_t)out->perm[s + r0] * dim;
        const float* x1 = x + (uint64_t)out->perm[s + r1] * dim;
        float off = 0.0f;
        if (angular) {
            float n0 = sqrtf(ao_ip(x0, x0, dim));
            float n1 = sqrtf(ao_ip(x1, x1, dim));
            if (fabsf(n0) < AO_EPS) n0 = 1.0f;
            if (fabsf(n1) < AO_EPS) n1 = 1.0f;
            for (uint32_t j = 0; j < dim; j++) hp[j] = x0[j] / n0 - x1[j] / n1;
            float hn = sqrtf(ao_ip(hp, hp, dim));
            if (fabsf(hn) < AO_EPS) hn = 1.0f;
            for (uint32_t j = 0; j < dim; j++) hp[j] /= hn;
        } else {
            for (uint32_t j = 0; j < dim; j++) {
                mid[j] = (x0[j] + x1[j]) / 2;
                hp[j] = x0[j] - x1[j];
            }
            off = ao_ip(hp, mid, dim);
        }
        uint32_t nl = 0;
        for (uint32_t p = 0; p < c; p++) {
            uint32_t id = out->perm[s + p];
            float m = ao_ip(hp, x + (uint64_t)id * dim, dim) - off;
            uint8_t sd;
            if (m < -AO_EPS) sd = 0;
            else if (m > AO_EPS) sd = 1;
            else sd = (uint8_t)(ao_hash64(key ^ ((uint64_t)id << 2 | 3)) & 1);
            side[p] = sd;
            nl += (sd == 0);
        }
        if (nl == 0 || nl == c) {
            nl = 0;
            for (uint32_t p = 0; p < c; p++) {
                uint32_t id = out->perm[s + p];
                side[p] = (uint8_t)(ao_hash64(key ^ ((uint64_t)id << 2 | 2)) & 1);
                nl += (side[p] == 0);
            }
        }
        uint32_t a = 0, b = nl;
        for (uint32_t p = 0; p < c; p++) tmp[side[p] ? b++ : a++] = out->perm[s + p];
        memcpy(out->perm + s, tmp, sizeof(uint32_t) * c);
        uint32_t L = n_nodes, R = n_nodes + 1;
        n_nodes += 2;
        out->left[v] = L;
        out->right[v] = R;
        out->offset[v] = off;
        out->leaf_off[v] = AO_EMPTY;
        out->leaf_cnt[v] = 0;
        start[L] = s;
        count[L] = nl;
        depth[L] = depth[v] + 1;
        start[R] = s + nl;
        count[R] = c - nl;
        depth[R] = depth[v] + 1;
    }
    free(start);
    free(count);
    free(depth);
    free(tmp);
    free(side);
    free(mid);
    return rc < 0 ? rc : (int64_t)n_nodes;
}

/* ---------------------------------------------------------- ground truth */

typedef struct {
    float key;
    uint32_t id;
} kv_t;

static int cmp_kv(const void* a, const void* b) {
    const kv_t* x = (const kv_t*)a;
    const kv_t* y = (const kv_t*)b;
    if (x->key < y->key) return -1;
    if (x->key > y->key) return 1;
    return (x->id > y->id) - (x->id < y->id);
}

/* dataset_gt.cpp:206-248: K smallest (key, id) with the diagonal skipped. */
void ao_exact_topk(const float* base, uint64_t n, uint32_t d, uint32_t K, uint32_t* ids, float* keys) {
    ao_exact_topk_metric(base, n, d, K, 0, ids, keys);
}

/* the ip metric's key is -<a, b> (dataset_gt.cpp:224, 288) */
void ao_exact_topk_metric(const float* base, uint64_t n, uint32_t d, uint32_t K, uint32_t ip, uint32_t* ids,
                          float* keys) {
    float* bn = (float*)malloc(sizeof(float) * n);
    kv_t* row = (kv_t*)malloc(sizeof(kv_t) * n);
    for (uint64_t i = 0; i < n; i++) bn[i] = ao_ip(base + i * d, base + i * d, d);
    for (uint64_t i = 0; i < n; i++) {
        uint64_t m = 0;
        for (uint64_t j = 0; j < n; j++) {
            if (j == i) continue;
            float v = ao_ip(base + i * d, base + j * d, d);
            row[m].key = ip ? -v : (bn[i] + bn[j]) - 2.0f * v;
            row[m].id = (uint32_t)j;
            m++;
        }
        qsort(row, (size_t)m, sizeof(kv_t), cmp_kv);
        for (uint32_t r = 0; r < K; r++) {
            ids[i * K + r] = r < m ? row[r].id : AO_EMPTY;
            keys[i * K + r] = r < m ? row[r].key : FLT_MAX;
        }
    }
    free(bn);
    free(row);
}

/* dataset_gt.cpp:270-299 */
int64_t ao_rknn_gt(const float* base, uint64_t n, const float* query, uint64_t nq, uint32_t d,
                   const float* rk2, uint32_t* off, uint32_t* ids, float* keys, uint64_t cap) {
    return ao_rknn_gt_metric(base, n, query, nq, d, rk2, 0, off, ids, keys, cap);
}

int64_t ao_rknn_gt_metric(const float* base, uint64_t n, const float* query, uint64_t nq, uint32_t d,
                          const float* rk2, uint32_t is_ip, uint32_t* off, uint32_t* ids, float* keys, uint64_t cap) {
    float* bn = (float*)malloc(sizeof(float) * n);
    kv_t* hits = (kv_t*)malloc(sizeof(kv_t) * (n + 1));
    for (uint64_t i = 0; i < n; i++) bn[i] = ao_ip(base + i * d, base + i * d, d);
    uint64_t total = 0;
    int over = 0;
    off[0] = 0;
    for (uint64_t q = 0; q < nq; q++) {
        const float* qv = query + q * d;
        float qn = ao_ip(qv, qv, d);
        uint64_t m = 0;
        for (uint64_t j = 0; j < n; j++) {
            float ip = ao_ip(qv, base + j * d, d);
            float key = is_ip ? -ip : (qn + bn[j]) - 2.0f * ip;
            if (key <= rk2[j]) {
                hits[m].key = key;
                hits[m].id = (uint32_t)j;
                m++;
            }
        }
        qsort(hits, (size_t)m, sizeof(kv_t), cmp_kv);
        for (uint64_t h = 0; h < m; h++) {
            if (total + h < cap) {
                ids[total + h] = hits[h].id;
                keys[total + h] = hits[h].key;
            } else
                over = 1;
        }
        total += m;
        off[q + 1] = (uint32_t)total;
    }
    free(bn);
    free(hits);
    return over ? -1 : (int64_t)total;
}

/* ---- the batched Vamana style's insertion order ---- */
void ao_mt64_seed(ao_mt64* g, uint64_t seed) {
    g->mt[0] = seed;
    for (uint32_t i = 1; i < 312; i++) g->mt[i] = 6364136223846793005ull * (g->mt[i - 1] ^ (g->mt[i - 1] >> 62)) + i;
    g->idx = 312;
}

uint64_t ao_mt64_next(ao_mt64* g) {
    if (g->idx >= 312) {
        for (uint32_t i = 0; i < 312; i++) {
            const uint64_t y = (g->mt[i] & 0xFFFFFFFF80000000ull) | (g->mt[(i + 1) % 312] & 0x7FFFFFFFull);
            g->mt[i] = g->mt[(i + 156) % 312] ^ (y >> 1) ^ ((y & 1ull) ? 0xB5026F5AA96619E9ull : 0ull);
        }
        g->idx = 0;
    }
    uint64_t x = g->mt[g->idx++];
    x ^= (x >> 29) & 0x5555555555555555ull;
    x ^= (x << 17) & 0x71D67FFFEDA60000ull;
    x ^= (x << 37) & 0xFFF7EEE000000000ull;
    x ^= x >> 43;
    return x;
}

/* a uniform draw in [0, range) from full 64-bit outputs: the high half of
 * the 128-bit product, rejecting low halves below 2^64 mod range */
static uint64_t ao_bounded(ao_mt64* g, uint64_t range) {
    unsigned __int128 prod = (unsigned __int128)ao_mt64_next(g) * range;
    uint64_t low = (uint64_t)prod;
    if (low < range) {
        const uint64_t threshold = (0ull - range) % range;
        while (low < threshold) {
            prod = (unsigned __int128)ao_mt64_next(g) * range;
            low = (uint64_t)prod;
        }
    }
    return (uint64_t)(prod >> 64);
}

void ao_shuffle_u32(uint32_t* a, uint64_t n, ao_mt64* g) {
    if (n < 2) return;
    uint64_t i = 1;
    if (n % 2 == 0) {
        const uint64_t j = ao_bounded(g, 2);
        const uint32_t t = a[i];
        a[i] = a[j];
        a[j] = t;
        i++;
    }
    while (i < n) {
        const uint64_t b0 = i + 1, b1 = i + 2;
        const uint64_t x = ao_bounded(g, b0 * b1);
        const uint64_t p0 = x / b1, p1 = x % b1;
        uint32_t t = a[i];
        a[i] = a[p0];
        a[p0] = t;
        i++;
        t = a[i];
        a[i] = a[p1];
        a[p1] = t;
        i++;
    }
}

void ao_vamana_batch_order(uint32_t* order, uint64_t n, uint64_t seed, int pass) {
    ao_mt64 g;
    ao_mt64_seed(&g, seed + 0x9e3779b97f4a7c15ull * (uint64_t)(pass + 1));
    ao_shuffle_u32(order, n, &g);
}
