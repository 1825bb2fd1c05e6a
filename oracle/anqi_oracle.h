/* Test infrastructure only -- never linked into the product library.
 *
 * A plain-C restatement of the reference algorithms on the RkNN hot path
 * (Yujian-Fu/anqi-implementation), used as the parity checker for the CUDA
 * kernels.  Each function cites the reference file:line it restates.  It is
 * pinned against the reference itself through the golden fixtures in
 * tests/golden/ (generated by running the reference's own code).
 *
 * Conventions: row-major float arrays, u32 ids, UINT32_MAX = empty slot.
 */
#ifndef ANQI_ORACLE_H
#define ANQI_ORACLE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- distances, include/distance.h (AVX-512 lane/reduction order) ---- */
float ao_l2sqr(const float* a, const float* b, uint32_t dim);          /* distance.h:58-86  */
float ao_ip(const float* a, const float* b, uint32_t dim);             /* distance.h:89-116 */
float ao_norm(const float* a, uint32_t dim);                           /* distance.h:143-161 */
/* nndindex::d2, index.h:172-176: na + nb - 2 * ip(a, b) */
float ao_d2(const float* a, const float* b, float na, float nb, uint32_t dim);
void ao_norms(const float* x, uint64_t n, uint32_t dim, float* out);

/* ---- LRQ codec, src/rknn_query.cpp:679-753 (floor policy, u8 codes) ---- */
void ao_lrq_encode(const float* keys, uint64_t n, uint32_t nk, uint32_t rankm,
                   const float* mu, const float* basis, const float* codebook,
                   uint32_t code_size, float* coeff, uint8_t* codes);
void ao_lrq_materialize(const float* coeff, const uint8_t* codes, uint64_t n, uint32_t nk,
                        uint32_t rankm, const float* mu, const float* basis,
                        const float* codebook, uint32_t code_size, uint32_t k_one_based,
                        double radius_scale, float* thr);

/* every CompactLrqVerifier form: bits 0 / 2 / 4 / 8 / 16 / 32, policy 0 nearest,
 * 1 floor, 2 ceil; codes packed as include/packed_code_array.h (zeroed by the caller) */
void ao_lrq_encode_bits(const float* keys, uint64_t n, uint32_t nk, uint32_t rankm, const float* mu,
                        const float* basis, const float* codebook, uint32_t code_size, uint32_t bits,
                        uint32_t policy, float* coeff, uint8_t* codes, float* residual);
void ao_lrq_materialize_bits(const float* coeff, const uint8_t* codes, const float* residual, uint64_t n,
                             uint32_t nk, uint32_t rankm, uint32_t bits, const float* mu, const float* basis,
                             const float* codebook, uint32_t code_size, uint32_t k_one_based,
                             double radius_scale, int signed_keys, float* thr);
void ao_analytic_rankm_materialize(const float* coeff, uint64_t n, uint32_t rankm, uint32_t train_kmax,
                                   uint32_t flags, double b0, uint32_t k_one_based, double radius_scale,
                                   float* thr);

/* ---- lift, src/rknn_query.cpp:2203-2235 (anyk_lift, L2) ---- */
void ao_lift(const float* base, uint64_t n, uint32_t d, const float* radius,
             float* lifted /* n x (d+2) */, double* mstar2, double* scale);
void ao_lift_query(const float* q, uint32_t d, double scale, float* out /* d+2 */);
/* ip = 1: the ip metric's lift coordinate s^2 r (rknn_query.cpp:2227) */
void ao_lift_metric(const float* base, uint64_t n, uint32_t d, const float* radius, uint32_t ip,
                    float* lifted, double* mstar2, double* scale);
/* the ip metric's scalar distance 1 - sum a_i b_i (distance.h:170-174) */
float ao_ip_dist(const float* a, const float* b, uint32_t dim);

/* ---- RP tree query descent, include/rptrees.h:108-124 ---- */
uint32_t ao_tree_entry(uint32_t n_nodes, uint32_t dim, const uint32_t* left,
                       const uint32_t* right, const float* offset, const float* hyperplane,
                       const uint32_t* leaf_first, const float* q);

/* ---- range search + postfilter, index.h:1535-1640, rknn_query.cpp:2753-2765 ---- */
typedef struct {
    uint64_t n;
    uint32_t dim;            /* lifted dim d+2 */
    uint32_t d;              /* original dim */
    uint32_t degree;         /* link slots per node */
    const float* lifted;     /* n x dim */
    const uint32_t* deg;     /* n */
    const uint32_t* links;   /* n x degree */
    const float* base;       /* n x d */
    uint32_t tree_nodes;
    const uint32_t* tree_left;
    const uint32_t* tree_right;
    const float* tree_offset;
    const float* tree_hyperplane; /* tree_nodes x dim */
    const uint32_t* tree_leaf_first;
    double scale;
    double mstar2;
    uint32_t metric;         /* 1: ip (per-query R2, key -<o,q>) */
} ao_index;

/* One query: writes candidate ids (visit order), predicted ids, returns counts.
 * Returns 0 on success, -1 if a capacity is exceeded. */
int ao_range_search(const ao_index* ix, const float* q, uint32_t L, const float* thr,
                    uint32_t* cand, uint32_t cand_cap, uint32_t* n_cand,
                    uint32_t* pred, uint32_t pred_cap, uint32_t* n_pred, uint32_t* n_dist);

/* ---- kNN-graph gather (index.h:1491-1525), sort-unique + alpha-RNG prune
 *      (index.h:225-281, 772-829), commit (index.h:907-930) ---- */
typedef struct {
    uint64_t n;
    uint32_t dim;
    const float* x;          /* n x dim */
    const float* norms;      /* n */
    uint32_t K;              /* heap width */
    const uint32_t* g_ids;   /* n x K (heap order) */
    const float* g_vals;     /* n x K */
    const uint64_t* rev_off; /* n+1 */
    const uint32_t* rev_ids;
    uint32_t metric;         /* 1: the ip metric's distance */
} ao_knn_graph;

/* gather_candidates for row i; the pool is written as (dist,id) in visit order.
 * Returns the pool size (or -1 if pool_cap is exceeded). */
int64_t ao_gather(const ao_knn_graph* g, uint64_t i, uint32_t ef, uint32_t cap,
                  float* pool_d, uint32_t* pool_id, uint64_t pool_cap);
/* build_approx_knn tail: gather, sort, first K ids != i (index.h:1347-1366). */
void ao_aknn_rows(const ao_knn_graph* g, uint32_t ef, uint32_t cap, uint32_t K,
                  uint32_t* out_ids, float* out_d);
/* ---- edge policies of the graph prune (include/index.h:283-829) ----
 * The configuration configure_edge_residual_cover (:305-440) leaves, as
 * flags: residual cover, ball occlusion (pure or hybrid), LSG ordering, and
 * the verification-constrained bubble optimizer (lazy or full). */
#define AO_EDGE_COVER 1u
#define AO_EDGE_BALL 2u
#define AO_EDGE_PURE 4u
#define AO_EDGE_LSG 8u
#define AO_EDGE_AUTO 16u
#define AO_EDGE_AUTO_FULL 32u
typedef struct {
    uint32_t flags;
    uint32_t nks;
    uint32_t ks[8];         /* the residual columns' k values, 1 <= k <= nk, in order */
    uint32_t nk;            /* residual table stride */
    uint32_t budget;        /* min(ANQI_EDGE_RESID_BUDGET, M) */
    uint32_t occlude_all;   /* ball occlusion over all k (else any) */
    uint32_t auto_candidates, auto_max_swaps;
    double lambda, scale2, lsg_alpha;
    const float* resid;     /* n x nk */
    const float* mu;        /* n (LSG) */
} ao_edge_policy;
/* prune_pool_to_ids (index.h:772-829) under pol (NULL: the default policy);
 * returns the degree. */
uint32_t ao_prune_policy(const float* x, const float* norms, uint32_t dim, uint64_t n, uint64_t i,
                         const float* pool_d, const uint32_t* pool_id, uint64_t pool_n, uint32_t M, float alpha,
                         const ao_edge_policy* pol, uint32_t* out);
void ao_graph_select_policy(const ao_knn_graph* g, uint32_t ef, uint32_t cap, uint32_t M, float alpha,
                            const ao_edge_policy* pol, uint32_t* O, uint32_t* O_deg);
void ao_graph_commit_policy(const float* x, const float* norms, uint32_t dim, uint64_t n, const uint32_t* O,
                            const uint32_t* O_deg, uint32_t M, float alpha, const ao_edge_policy* pol,
                            uint32_t* links, uint32_t* deg);
/* ---- the batched Vamana style's insertion order ----
 * std::mt19937_64 (the 64-bit Mersenne Twister of Matsumoto and Nishimura,
 * seeded from one value) and std::shuffle as GCC's library performs it on a
 * vector of 32-bit ids: Fisher-Yates from the front, positions drawn two at a
 * time from one bounded draw (Brackett-Rozinsky and Lemire's batched ranged
 * integers), each bounded draw by Lemire's multiply-and-reject.  Checked
 * against the compiler's own std::shuffle (tests/test_vamana_batch.py). */
typedef struct {
    uint64_t mt[312];
    uint32_t idx;
} ao_mt64;
void ao_mt64_seed(ao_mt64* g, uint64_t seed);
uint64_t ao_mt64_next(ao_mt64* g);
void ao_shuffle_u32(uint32_t* a, uint64_t n, ao_mt64* g);
/* index.h:936-1065: pass p's order, shuffled from the previous pass's */
void ao_vamana_batch_order(uint32_t* order, uint64_t n, uint64_t seed, int pass);

/* prune_pool_to_ids with the default edge policy; returns the degree. */
uint32_t ao_prune(const float* x, const float* norms, uint32_t dim, uint64_t n, uint64_t i,
                  float* pool_d, uint32_t* pool_id, uint64_t pool_n, uint32_t M, float alpha,
                  uint32_t* out);
/* gather + prune for all rows -> O (n x M, UINT32_MAX padded) */
void ao_graph_select(const ao_knn_graph* g, uint32_t ef, uint32_t cap, uint32_t M, float alpha,
                     uint32_t* O, uint32_t* O_deg);
/* one pass of the global Vamana refine over the current graph (links, deg):
 * greedy beam from entry[i] + the row's g0 list -> prune -> O, O_deg */
void ao_vamana_select(const float* x, const float* norms, uint32_t dim, uint64_t n, const uint32_t* links,
                      const uint32_t* deg, uint32_t M, const uint32_t* g0, uint32_t K, const uint32_t* entry,
                      uint32_t Lb, float alpha, uint32_t* O, uint32_t* O_deg);
void ao_vamana_select_policy(const float* x, const float* norms, uint32_t dim, uint64_t n, const uint32_t* links,
                             const uint32_t* deg, uint32_t M, const uint32_t* g0, uint32_t K, const uint32_t* entry,
                             uint32_t Lb, float alpha, const ao_edge_policy* pol, uint32_t* O, uint32_t* O_deg);
/* vamana_batch_refine (index.h:936-1065) on links / deg (n x M) in place,
 * from the single entry, with the prunes under pol (NULL: default) */
void ao_vamana_batch_refine(const float* x, const float* norms, uint32_t dim, uint64_t n, uint32_t* links,
                            uint32_t* deg, uint32_t M, const uint32_t* g0, uint32_t K, uint32_t entry, uint32_t Lb,
                            int passes, float final_alpha, float early_alpha, int early_one, double max_frac,
                            uint64_t max_batch_cap, double batch_base, uint64_t seed, const ao_edge_policy* pol);
/* commit_edges: final adjacency (n x M) from O */
void ao_graph_commit(const float* x, const float* norms, uint32_t dim, uint64_t n,
                     const uint32_t* O, const uint32_t* O_deg, uint32_t M, float alpha,
                     uint32_t* links, uint32_t* deg);

/* ---- fixed-capacity max-heap push, heap.h:162-186 ---- */
int ao_heap_push(uint32_t* ids, float* vals, uint32_t K, uint32_t id, float v);
/* warm start, index.h:1210-1217: heaps (n x K) from width candidates per row */
void ao_warm_start(const float* x, const float* norms, uint32_t dim, uint64_t n,
                   const uint32_t* cand, uint32_t stride, uint32_t width, uint32_t K,
                   uint32_t* ids, float* vals);
/* One LocalJoin round (index.h:1468-1487) in its snapshot ("pull") form: every
 * row samples its first <= sample live slots in heap order at round start; each
 * target heap then receives, for each source u in ascending order that sampled
 * it, the other sampled ids of u in sample order.  Returns the update count. */
uint64_t ao_localjoin_round(const float* x, const float* norms, uint32_t dim, uint64_t n,
                            uint32_t K, uint32_t sample, uint32_t* ids, float* vals);
/* push_reverse, heap.h:190-207 (row order, slot order). rev_off has n+1 entries. */
void ao_reverse(const uint32_t* ids, uint64_t n, uint32_t K, uint64_t* rev_off, uint32_t* rev_ids);

/* ---- init_knn from leaves (index.h:1433-1449): per row, the K smallest
 *      unique leaf-mates by (dist, id) ---- */
void ao_init_knn(const float* x, const float* norms, uint32_t dim, uint64_t n, uint32_t K,
                 const uint64_t* leaf_off, const uint32_t* leaf_ids, uint64_t n_leaves,
                 uint32_t* out_ids, float* out_d);
void ao_init_knn_metric(const float* x, const float* norms, uint32_t dim, uint64_t n, uint32_t K,
                        const uint64_t* leaf_off, const uint32_t* leaf_ids, uint64_t n_leaves, uint32_t ip,
                        uint32_t* out_ids, float* out_d);

/* ---- random-projection forest (rptrees.h:28-84,127-163) in this project's
 *      deterministic form: a counter-hash RNG replaces the thread-local mt19937,
 *      nodes are numbered breadth-first.  Returns node count or -1. ---- */
typedef struct {
    uint32_t* left;      /* UINT32_MAX for leaves */
    uint32_t* right;
    float* offset;
    float* hyperplane;   /* cap_nodes x dim */
    uint32_t* leaf_off;  /* leaves: start in perm; internal: UINT32_MAX */
    uint32_t* leaf_cnt;
    uint32_t* perm;      /* n */
    uint32_t cap_nodes;
} ao_tree_out;
int64_t ao_rp_tree(const float* x, uint64_t n, uint32_t dim, uint32_t leaf_size,
                   uint32_t max_depth, uint64_t seed, uint32_t tree, ao_tree_out* out);
int64_t ao_rp_tree_metric(const float* x, uint64_t n, uint32_t dim, uint32_t leaf_size, uint32_t max_depth,
                          uint64_t seed, uint32_t tree, uint32_t angular, ao_tree_out* out);
uint64_t ao_hash64(uint64_t x);

/* ---- exact ground truth, tools/dataset_gt.cpp:206-313 ---- */
void ao_exact_topk(const float* base, uint64_t n, uint32_t d, uint32_t K,
                   uint32_t* ids, float* keys);
/* returns total hits; off has nq+1 entries; ids/keys sized by cap (-1 if exceeded) */
int64_t ao_rknn_gt(const float* base, uint64_t n, const float* query, uint64_t nq, uint32_t d,
                   const float* rk2, uint32_t* off, uint32_t* ids, float* keys, uint64_t cap);
/* the same for either metric (ip = 1: key -<a, b>, dataset_gt.cpp:224, 288) */
void ao_exact_topk_metric(const float* base, uint64_t n, uint32_t d, uint32_t K, uint32_t ip, uint32_t* ids,
                          float* keys);
int64_t ao_rknn_gt_metric(const float* base, uint64_t n, const float* query, uint64_t nq, uint32_t d,
                          const float* rk2, uint32_t is_ip, uint32_t* off, uint32_t* ids, float* keys, uint64_t cap);

#ifdef __cplusplus
}
#endif
#endif
