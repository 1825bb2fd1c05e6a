/* anqi.h -- C ABI of the B200 (sm_100a) implementation of ANQI's reverse-kNN
 * hot path.  Plain pointers and sizes only; every function returns a status.
 *
 * The reference (Yujian-Fu/anqi-implementation) has no FFI: its boundary is
 * three CLIs plus prefix files.  Each entry point below replaces one stage of
 * those CLIs; the comment names the reference code it stands in for.  The CLIs
 * in anqi-implementation_b200/cli/ and the Python host package call only these
 * functions.
 *
 * Ownership: the caller owns every host buffer; a context owns its device
 * memory and one CUDA stream.  Threading: one host thread per context.
 * Errors: no function exits the process; anqi_last_error() describes the last
 * failure of a context.  Unless a function says "device", all array arguments
 * are host memory and the call returns after the results are in host memory.
 */
#ifndef ANQI_H
#define ANQI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes; 2/3/5 match the reference CLIs' exit codes. */
#define ANQI_OK 0
#define ANQI_ERR_ARGS 2        /* bad argument (reference: usage / config error, exit 2) */
#define ANQI_ERR_FORMAT 3      /* bad input contents (reference: exit 3) */
#define ANQI_ERR_INVARIANT 5   /* an output failed validation (reference: exit 5) */
#define ANQI_ERR_DEVICE 7      /* CUDA error or no usable device */
#define ANQI_ERR_TIMEOUT 8     /* a bounded device wait ran out */
#define ANQI_ERR_CAPACITY 9    /* a scratch or output capacity was exceeded; retry with more */

#define ANQI_EMPTY 0xFFFFFFFFu /* empty slot / no neighbour */

/* Metrics (the reference's metric=l2|ip, include/distance.h:170-190).  Under
 * ANQI_METRIC_IP the AKNN source ranks by 1 - <a, b> (a sequential sum, the
 * reference's scalar ip distance), its forest splits angularly through the
 * origin, the exact ground truth keys are -<a, b>, and the query radius and
 * postfilter follow src/rknn_query.cpp:2227, 2555-2561, 2724-2731.  The
 * lifted graph itself is always built in L2. */
#define ANQI_METRIC_L2 0u
#define ANQI_METRIC_IP 1u

typedef struct anqi_ctx anqi_ctx;

/* ---------------------------------------------------------------- context */
int anqi_ctx_create(int device, anqi_ctx** out);
void anqi_ctx_destroy(anqi_ctx* ctx);
const char* anqi_last_error(const anqi_ctx* ctx);
int anqi_version(void);
/* Bytes of device memory the context currently holds. */
uint64_t anqi_device_bytes(const anqi_ctx* ctx);
/* Test hook, no counterpart in the reference: makes the device waits of this
 * context run out without any fault.  ANQI_FAULT_DROP_ROW_COPIES: the search
 * kernel of later anqi_query_run / anqi_rknn_query calls issues no bulk copies
 * of lifted rows, so its bounded waits for them (a fixed number of polls)
 * expire with nothing in flight; the call returns ANQI_ERR_TIMEOUT and the context
 * stays usable.  flags = 0 restores normal operation. */
#define ANQI_FAULT_DROP_ROW_COPIES 1u
int anqi_inject_fault(anqi_ctx* ctx, uint32_t flags);
/* Device timer on the context's stream (CUDA events): start, then stop returns
 * the elapsed milliseconds of everything the context ran in between. */
int anqi_timer_start(anqi_ctx* ctx);
int anqi_timer_stop(anqi_ctx* ctx, float* ms);

/* ------------------------------------------------------- FP32 distances
 * Batch forms of include/distance.h:58-161 in the AVX-512 lane order:
 * out[i] = l2sqr(a_i, b_i) / ip(a_i, b_i) for m pairs of dim floats. */
int anqi_pair_distances(anqi_ctx* ctx, const float* a, const float* b, uint64_t m, uint32_t dim,
                        float* l2sqr, float* ip);
/* The same with `group` = 4, 8 or 16 threads per pair: the forms the kernels
 * use for many short rows, few rows and long rows; identical results.
 * group = 0 (dim 130 only): l2sqr by the d = 128 search's form, 4 threads per
 * pair on rows stored with each 16-float chunk transposed as 4 x 4. */
int anqi_pair_distances_group(anqi_ctx* ctx, const float* a, const float* b, uint64_t m, uint32_t dim,
                              uint32_t group, float* l2sqr, float* ip);

/* ------------------------------------------------------------------ LRQ
 * CompactLrqVerifier::build, floor policy, u8 codes (src/rknn_query.cpp:679-720):
 * keys n x nk (AKNN cutoffs), mu nk, basis rankm x nk, codebook nk x code_size
 * (rows ascending) -> coeff n x rankm, codes n x nk. */
int anqi_lrq_encode(anqi_ctx* ctx, const float* keys, uint64_t n, uint32_t nk, uint32_t rankm,
                    const float* mu, const float* basis, const float* codebook, uint32_t code_size,
                    float* coeff, uint8_t* codes);
/* CompactLrqVerifier::materialize_k (src/rknn_query.cpp:722-753), L2 metric. */
int anqi_lrq_materialize(anqi_ctx* ctx, const float* coeff, const uint8_t* codes, uint64_t n,
                         uint32_t nk, uint32_t rankm, const float* mu, const float* basis,
                         const float* codebook, uint32_t code_size, uint32_t k_one_based,
                         double radius_scale, float* thr);

/* Every CompactLrqVerifier form (src/rknn_query.cpp:144-178, 604-753): bits
 * 0 = rankm_only (no residual), 2 / 4 / 8 / 16 = rankm_resid_u{bits}_lrq_*
 * (codebook of 2^bits sorted centres per rank, codes packed object-major as
 * include/packed_code_array.h:8-63 lays them out: (n * nk * bits + 7) / 8
 * bytes; u2 needs nk % 4 == 0 and u4 nk % 2 == 0, else ANQI_ERR_FORMAT),
 * 32 = rankm_resid_f32 (residual n x nk floats).  policy: the artifact's
 * numbering (encode_learned_residual, :482-513).  codes / residual / codebook
 * may be NULL where the form has none. */
#define ANQI_LRQ_NEAREST 0u
#define ANQI_LRQ_FLOOR 1u
#define ANQI_LRQ_CEIL 2u
int anqi_lrq_encode_bits(anqi_ctx* ctx, const float* keys, uint64_t n, uint32_t nk, uint32_t rankm,
                         const float* mu, const float* basis, const float* codebook, uint32_t code_size,
                         uint32_t bits, uint32_t policy, float* coeff, uint8_t* codes, float* residual);
/* materialize_k for any form; signed_keys != 0 (IP metric, -<q,o> keys) keeps
 * negative thresholds instead of clamping them at zero (:748-751). */
int anqi_lrq_materialize_bits(anqi_ctx* ctx, const float* coeff, const uint8_t* codes, const float* residual,
                              uint64_t n, uint32_t nk, uint32_t rankm, uint32_t bits, const float* mu,
                              const float* basis, const float* codebook, uint32_t code_size,
                              uint32_t k_one_based, double radius_scale, int signed_keys, float* thr);
/* AnalyticRankMVerifier::materialize_k (src/rknn_query.cpp:515-601): the
 * ANQIPW1 model's coefficients (n x rankm) and header fields; thr[i] =
 * max(0, scale * sum_m c_im * ratio^b0 * log(ratio)^m), ratio = k / train_kmax
 * when flags & 4, else k. */
int anqi_analytic_rankm_materialize(anqi_ctx* ctx, const float* coeff, uint64_t n, uint32_t rankm,
                                    uint32_t train_kmax, uint32_t fit_kmin, uint32_t flags, double b0,
                                    uint32_t k_one_based, double radius_scale, float* thr);

/* ----------------------------------------------------------------- lift
 * The anyk_lift of src/rknn_query.cpp:2203-2235 (L2): base n x d and the
 * graph-horizon radius (AKNN rank-K cutoff) -> lifted n x (d+2), M*^2, scale. */
int anqi_lift(anqi_ctx* ctx, const float* base, uint64_t n, uint32_t d, const float* radius,
              float* lifted, double* mstar2, double* scale);
/* Either metric: under ANQI_METRIC_IP the lift coordinate is s^2 * radius
 * (src/rknn_query.cpp:2227) instead of (s^2 * radius - |s o|^2) / 2. */
int anqi_lift_metric(anqi_ctx* ctx, const float* base, uint64_t n, uint32_t d, const float* radius,
                     uint32_t metric, float* lifted, double* mstar2, double* scale);

/* ------------------------------------------------------ random projection
 * RP trees (include/rptrees.h:28-84,127-186) in deterministic breadth-first
 * form: a counter hash of (seed, tree, node) replaces the reference's
 * thread-local mt19937.  Outputs per node (n_nodes <= cap_nodes per tree):
 * left/right child (ANQI_EMPTY on leaves), offset, hyperplane (n_nodes x dim),
 * leaf_off/leaf_cnt into perm (n per tree).  Tree t's arrays start at
 * t * cap_nodes (nodes) and t * n (perm); n_nodes[t] receives its node count. */
int anqi_rp_forest(anqi_ctx* ctx, const float* x, uint64_t n, uint32_t dim, uint32_t trees,
                   uint32_t leaf_size, uint32_t max_depth, uint64_t seed, uint32_t cap_nodes,
                   uint32_t* n_nodes, uint32_t* left, uint32_t* right, float* offset,
                   float* hyperplane, uint32_t* leaf_off, uint32_t* leaf_cnt, uint32_t* perm);
/* The same with the metric's split: ANQI_METRIC_IP splits angularly
 * (include/rptrees.h:41-52), hyperplane x0/|x0| - x1/|x1| normalized, offset 0. */
int anqi_rp_forest_metric(anqi_ctx* ctx, const float* x, uint64_t n, uint32_t dim, uint32_t trees,
                          uint32_t leaf_size, uint32_t max_depth, uint64_t seed, uint32_t cap_nodes, uint32_t metric,
                          uint32_t* n_nodes, uint32_t* left, uint32_t* right, float* offset, float* hyperplane,
                          uint32_t* leaf_off, uint32_t* leaf_cnt, uint32_t* perm);

/* --------------------------------------------------------- AKNN source
 * nndindex::build_approx_knn (include/index.h:1300-1367) as driven by
 * tools/build_aknn_source.cpp: forest -> init_knn -> [LocalJoin x nn_iters]
 * -> reverse lists -> gather (queue ef, pool cap max(K, ef_alpha*ef)) ->
 * per row the K nearest ids != row, ascending.  ids/dists: n x K. */
typedef struct {
    uint32_t k;          /* K = 100 */
    uint32_t leaf;       /* leaf size, 500 */
    uint32_t trees;      /* 64 */
    uint32_t ef;         /* explore range, 600 */
    uint32_t ef_alpha;   /* pool cap multiplier, 8 */
    uint64_t seed;       /* 10 */
    uint32_t nn_iters;   /* ANQI_NNITERS, default 0 */
    uint32_t nn_sample;  /* ANQI_NNSAMPLE, default 20 */
    uint32_t precision;  /* init_knn leaf distances: 0 = FP32 CUDA cores, 1 = BF16 tensor-core
                            tiles with FP32 recheck (identical output; d <= 1024, rows
                            above 256 dimensions in K chunks; larger d runs on the CUDA cores) */
    uint32_t metric;     /* ANQI_METRIC_L2 (0) or ANQI_METRIC_IP (key 1 - <a, b>, either
                            precision); the ip metric takes no LocalJoin (nn_iters = 0) */
} anqi_aknn_params;

typedef struct {
    double total_ms, forest_ms, init_ms, join_ms, reverse_ms, gather_ms;  /* host clock per stage */
    uint64_t join_updates;
    uint64_t pool_total;
    double gather_kernel_ms;  /* device time of the gather kernel launches (CUDA events) */
} anqi_build_stats;

int anqi_aknn_build(anqi_ctx* ctx, const float* base, uint64_t n, uint32_t d,
                    const anqi_aknn_params* p, uint32_t* ids, float* dists, anqi_build_stats* st);
/* Stage entry points (parity tests at stage boundaries). */
/* init_knn given leaves (index.h:1433-1460): K nearest unique leaf-mates by (dist, id). */
int anqi_aknn_init(anqi_ctx* ctx, const float* x, uint64_t n, uint32_t dim, const uint64_t* leaf_off,
                   const uint32_t* leaf_ids, uint64_t n_leaves, uint32_t K, uint32_t* ids, float* dists);
/* gather + top-K given a kNN graph (index.h:1347-1366, 1491-1525). */
int anqi_aknn_gather(anqi_ctx* ctx, const float* x, uint64_t n, uint32_t dim, const uint32_t* g_ids,
                     const float* g_vals, uint32_t K, uint32_t ef, uint32_t cap, uint32_t out_k,
                     uint32_t* ids, float* dists);
/* The two stages in either metric. */
int anqi_aknn_init_metric(anqi_ctx* ctx, const float* x, uint64_t n, uint32_t dim, const uint64_t* leaf_off,
                          const uint32_t* leaf_ids, uint64_t n_leaves, uint32_t K, uint32_t metric, uint32_t* ids,
                          float* dists);
int anqi_aknn_gather_metric(anqi_ctx* ctx, const float* x, uint64_t n, uint32_t dim, const uint32_t* g_ids,
                            const float* g_vals, uint32_t K, uint32_t ef, uint32_t cap, uint32_t out_k,
                            uint32_t metric, uint32_t* ids, float* dists);

/* ----------------------------------------------------------- edge policies
 * The prune of the G48 build under ANQI_EDGE_POLICY (prune_pool_to_ids,
 * include/index.h:772-829, as configure_edge_residual_cover leaves it,
 * :305-440), resolved to flags:
 *   ANQI_EDGE_COVER      residual_cover: RNG to M - budget, residual-cover edges, RNG to M
 *   ANQI_EDGE_BALL       ball occlusion over the pool ordered by d - lambda max_k radj
 *   ANQI_EDGE_PURE       with BALL: ball RNG first (ball_rng, bubble_rng), else RNG to M - budget first
 *   ANQI_EDGE_LSG        the LSG metric d2 / (mu_a mu_b)^lsg_alpha (lsg_rng; with BALL lsg_bubble_hybrid)
 *   ANQI_EDGE_AUTO       RNG, then the verification-constrained bubble optimizer (bubble_auto)
 *   ANQI_EDGE_AUTO_FULL  with AUTO: every pool entry an alternative and a target (bubble_auto_full)
 * radj(id, k) = scale2 * resid[id * nk + k - 1]; flags 0 is the default prune.
 * The tables are host arrays, copied for the build. */
#define ANQI_EDGE_COVER 1u
#define ANQI_EDGE_BALL 2u
#define ANQI_EDGE_PURE 4u
#define ANQI_EDGE_LSG 8u
#define ANQI_EDGE_AUTO 16u
#define ANQI_EDGE_AUTO_FULL 32u
typedef struct {
    uint32_t flags;
    uint32_t nks;              /* ANQI_EDGE_KS values kept (1 <= k <= nk), at most 8 */
    uint32_t ks[8];
    uint32_t nk;               /* ANQI_EDGE_NK: the residual table's stride (100) */
    uint32_t budget;           /* min(ANQI_EDGE_RESID_BUDGET, M) (16) */
    uint32_t occlude_all;      /* ANQI_EDGE_BALL_OCCLUSION != "any" */
    uint32_t auto_candidates;  /* ANQI_EDGE_AUTO_CANDIDATES (M) */
    uint32_t auto_max_swaps;   /* ANQI_EDGE_AUTO_MAX_SWAPS (M) */
    double lambda;             /* ANQI_EDGE_RESID_LAMBDA (1) */
    double scale2;             /* the lift scale squared from <graph folder>_anqi_meta.txt, else 1 */
    double lsg_alpha;          /* ANQI_LSG_ALPHA (1) */
    const float* resid;        /* n x nk (COVER, BALL, AUTO) */
    const float* mu;           /* n, positive (LSG) */
} anqi_edge_policy;

/* ----------------------------------------------------------- G48 graph
 * nndindex::build_index with a flat warm start (include/index.h:1071-1295):
 * entry RP tree (1 tree, leaf p->leaf) -> warm-start heaps (cap nn_k) from the
 * first warm_width ids of each row -> LocalJoin rounds (snapshot form, early
 * exit upd < n/200) -> reverse lists -> gather (queue explore, pool cap
 * max(M, ef_alpha * explore)) -> alpha-RNG prune -> commit_edges.
 * Outputs deg (n), links (n x degree, ANQI_EMPTY padded).  The entry tree is
 * kept in the context; read it with anqi_graph_tree_*. */
typedef struct {
    uint32_t degree;       /* M = 48 */
    uint32_t nn_k;         /* ANQI_LIFTNNK = 50 */
    uint32_t explore;      /* explore_range = 100 */
    uint32_t ef_alpha;     /* 8 */
    uint32_t join_iters;   /* ANQI_GRAPHNND = 6 */
    uint32_t join_sample;  /* ANQI_NNSAMPLE = 20 */
    uint32_t leaf;         /* 100 */
    uint32_t max_depth;    /* 100 */
    uint64_t seed;         /* 10 */
    float alpha;           /* ANQI_ALPHA = 1.2 */
    uint32_t warm_width;   /* 100 */
    uint32_t precision;    /* LocalJoin distances: 0 = FP32 CUDA cores, 1 = BF16 tensor-core tiles
                              filter each round's pairs against the round-start heap tops and
                              only kept pairs are recomputed in FP32 (identical heaps; needs
                              join_sample <= 32 and dim <= 256, else FP32) */
    uint32_t vamana_passes;  /* ANQI_VAMANA (ANQI_VAMANA_PASS, 2): global Vamana refine passes after
                                the commit (include/index.h:1262-1285); 0 = none */
    uint32_t vamana_L;       /* ANQI_VAMANA_L: the refine's beam width (128; 0 = 128) */
    const anqi_edge_policy* edge;  /* the prune's edge policy (select, commit, Vamana); NULL = default */
    /* ANQI_VAMANA_STYLE=batch (include/index.h:936-1065) in place of the global passes: */
    uint32_t vamana_batch;         /* 1: the batched style */
    uint32_t vamana_entry;         /* ANQI_VAMANA_ENTRY resolved to a row (0; "medoid" resolved by the caller) */
    double vamana_batch_frac;      /* ANQI_VAMANA_BATCH_FRAC (0.02) */
    uint64_t vamana_max_batch;     /* ANQI_VAMANA_MAX_BATCH (1000000) */
    double vamana_batch_base;      /* ANQI_VAMANA_BATCH_BASE (2) */
    float vamana_early_alpha;      /* ANQI_VAMANA_EARLY_ALPHA (1): alpha of every pass but the last ... */
    uint32_t vamana_early_alpha_one;  /* ... when ANQI_VAMANA_EARLY_ALPHA_ONE (1) is non-zero */
} anqi_graph_params;

int anqi_graph_build(anqi_ctx* ctx, const float* x, uint64_t n, uint32_t dim, const uint32_t* warm_ids,
                     uint32_t warm_stride, const anqi_graph_params* p, uint32_t* deg, uint32_t* links,
                     anqi_build_stats* st);
/* The same build with the warm start delivered in row chunks, so the host
 * holds one chunk of ids at a time (the reference's streamed warm start,
 * include/index.h:1127-1203, fed by ANQI_PREBUILT_WARM_START_COMMAND or the
 * compacted id file, src/rknn_query.cpp:988-1057).  begin: lifted rows to the
 * device and the entry tree; warm_rows: rows [row0, row0 + rows) of the ids,
 * `stride` per row (the first p->warm_width used), each row exactly once, in
 * any order; finish: LocalJoin, gather + prune, commit, outputs as
 * anqi_graph_build.  A new begin discards a build in progress; finish fails
 * (ANQI_ERR_ARGS) unless every row was delivered.  anqi_graph_build is begin
 * + one warm_rows over all rows + finish. */
int anqi_graph_build_begin(anqi_ctx* ctx, const float* x, uint64_t n, uint32_t dim, const anqi_graph_params* p);
int anqi_graph_build_warm_rows(anqi_ctx* ctx, uint64_t row0, uint64_t rows, const uint32_t* ids, uint32_t stride);
int anqi_graph_build_finish(anqi_ctx* ctx, uint32_t* deg, uint32_t* links, anqi_build_stats* st);
/* Entry tree of the last anqi_graph_build, breadth-first arrays (see anqi_rp_forest). */
int anqi_graph_tree_size(anqi_ctx* ctx, uint32_t* n_nodes, uint64_t* n_points);
int anqi_graph_tree_copy(anqi_ctx* ctx, uint32_t* left, uint32_t* right, float* offset, float* hyperplane,
                         uint32_t* leaf_off, uint32_t* leaf_cnt, uint32_t* perm);
/* Stage entry points. */
int anqi_graph_warm_start(anqi_ctx* ctx, const float* x, uint64_t n, uint32_t dim, const uint32_t* cand,
                          uint32_t stride, uint32_t width, uint32_t K, uint32_t* ids, float* vals);
int anqi_graph_localjoin(anqi_ctx* ctx, const float* x, uint64_t n, uint32_t dim, uint32_t K,
                         uint32_t sample, uint32_t max_rounds, uint32_t* ids, float* vals,
                         uint64_t* updates /* max_rounds entries */, uint32_t* rounds_done);
/* The same with the LocalJoin precision form of anqi_graph_params.precision;
 * join_ms (optional) receives the device time of the rounds. */
int anqi_graph_localjoin_precision(anqi_ctx* ctx, const float* x, uint64_t n, uint32_t dim, uint32_t K,
                                   uint32_t sample, uint32_t max_rounds, uint32_t precision, uint32_t* ids,
                                   float* vals, uint64_t* updates, uint32_t* rounds_done, float* join_ms);
int anqi_graph_select(anqi_ctx* ctx, const float* x, uint64_t n, uint32_t dim, const uint32_t* g_ids,
                      const float* g_vals, uint32_t K, uint32_t M, uint32_t ef, uint32_t cap, float alpha,
                      uint32_t* O, uint32_t* O_deg);
int anqi_graph_commit(anqi_ctx* ctx, const float* x, uint64_t n, uint32_t dim, const uint32_t* O,
                      const uint32_t* O_deg, uint32_t M, float alpha, uint32_t* links, uint32_t* deg);
/* The select and commit stages under an edge policy (NULL: as above). */
int anqi_graph_select_policy(anqi_ctx* ctx, const float* x, uint64_t n, uint32_t dim, const uint32_t* g_ids,
                             const float* g_vals, uint32_t K, uint32_t M, uint32_t ef, uint32_t cap, float alpha,
                             const anqi_edge_policy* edge, uint32_t* O, uint32_t* O_deg);
int anqi_graph_commit_policy(anqi_ctx* ctx, const float* x, uint64_t n, uint32_t dim, const uint32_t* O,
                             const uint32_t* O_deg, uint32_t M, float alpha, const anqi_edge_policy* edge,
                             uint32_t* links, uint32_t* deg);
/* One pass of the global Vamana refine (include/index.h:856-875,
 * 1262-1285), select half: for every row i, a beam of width Lb over the graph
 * (links n x M, deg) from entry[i] collects every visited node, the row's g0
 * list (n x K, ANQI_EMPTY skipped) joins with fresh distances, and the pool is
 * pruned as anqi_graph_select does -> O, O_deg (then anqi_graph_commit).
 * anqi_graph_params.vamana_passes runs whole passes inside anqi_graph_build,
 * the entries from the build's entry tree (ties at the margin to the left). */
/* The batched Vamana refine (include/index.h:936-1065) on a graph (links
 * n x M, deg; refined in place): per pass the rows in a shuffled order
 * (std::mt19937_64 from seed + 0x9e3779b97f4a7c15 (pass + 1), std::shuffle's
 * order restated), cut into batches of growing size; each batch's rows prune
 * a beam from the single entry over the graph as it was at the batch's start,
 * their g0 list (n x K) and current links, take the result as their links,
 * and every row they now link to prunes its links plus those rows.  Uses
 * p->degree (M), alpha, seed, edge, vamana_L, vamana_passes and the
 * vamana_batch* / vamana_entry / vamana_early_alpha* fields. */
int anqi_graph_vamana_batch_refine(anqi_ctx* ctx, const float* x, uint64_t n, uint32_t dim, uint32_t* links,
                                   uint32_t* deg, const uint32_t* g0, uint32_t K, const anqi_graph_params* p);
int anqi_graph_vamana_select(anqi_ctx* ctx, const float* x, uint64_t n, uint32_t dim, const uint32_t* links,
                             const uint32_t* deg, uint32_t M, const uint32_t* g0, uint32_t K, const uint32_t* entry,
                             uint32_t Lb, float alpha, uint32_t* O, uint32_t* O_deg);

/* ------------------------------------------------------- query index
 * A device-resident copy of what rknn_query holds after index load
 * (src/rknn_query.cpp:2283-2322): original vectors, lifted vectors, the
 * fixed-degree adjacency, the entry RP tree, M*^2 and the lift scale. */
typedef struct {
    uint64_t n;
    uint32_t d;                 /* original dimension; lifted is d + 2 */
    uint32_t degree;            /* link slots per node (M) */
    const float* base;          /* n x d */
    const float* lifted;        /* n x (d+2) */
    const uint32_t* deg;        /* n */
    const uint32_t* links;      /* n x degree */
    uint32_t tree_nodes;        /* post-order, root last (the persisted order) */
    const uint32_t* tree_left;  /* ANQI_EMPTY on leaves */
    const uint32_t* tree_right;
    const float* tree_offset;
    const float* tree_hyperplane; /* tree_nodes x (d+2) */
    const uint32_t* tree_leaf_first; /* indices[0] of each leaf, ANQI_EMPTY if empty */
    double scale;
    double mstar2;
    uint32_t metric;            /* ANQI_METRIC_L2 or ANQI_METRIC_IP (the meta file's metric) */
} anqi_index_desc;

int anqi_index_load(anqi_ctx* ctx, const anqi_index_desc* desc);
/* The postfilter verifier (LRQ artifact) -> device; materialize thresholds per k. */
int anqi_verifier_load(anqi_ctx* ctx, const float* coeff, const uint8_t* codes, uint64_t n, uint32_t nk,
                       uint32_t rankm, const float* mu, const float* basis, const float* codebook,
                       uint32_t code_size);
/* The same for any CompactLrqVerifier form (see anqi_lrq_encode_bits), and
 * the analytic Rank-M model; anqi_verifier_materialize then uses it. */
int anqi_verifier_load_bits(anqi_ctx* ctx, const float* coeff, const uint8_t* codes, const float* residual,
                            uint64_t n, uint32_t nk, uint32_t rankm, uint32_t bits, const float* mu,
                            const float* basis, const float* codebook, uint32_t code_size, int signed_keys);
int anqi_verifier_load_analytic(anqi_ctx* ctx, const float* coeff, uint64_t n, uint32_t rankm,
                                uint32_t train_kmax, uint32_t fit_kmin, uint32_t flags, double b0);
int anqi_verifier_materialize(anqi_ctx* ctx, uint32_t k_one_based, double radius_scale);
/* Explicit per-object thresholds for k (e.g. exact_f32 mode). */
int anqi_set_thresholds(anqi_ctx* ctx, uint32_t k_one_based, const float* thr);

/* ------------------------------------------------------------ queries
 * For every query: lift (rknn_query.cpp:2721-2730), entry by RP-tree descent
 * (rptrees.h:108-124), greedy beam of width L then bounded flood over
 * ||q^ - o^||^2 <= M*^2 + 1 (index.h:1535-1640), then the FP32 postfilter
 * against the k-th materialized threshold (rknn_query.cpp:2555-2561,2762-2765).
 * Results are CSR: pred_off (nq+1) into pred_ids.  Per query k and L may
 * differ (k_per_query / L_per_query may be NULL to use k_all / L_all).
 * cand_* (optional, may be NULL) receive the candidate sets in visit order. */
typedef struct {
    uint64_t n_dist;      /* graph distance evaluations, all queries */
    uint64_t n_expand;    /* beam expansions */
    uint64_t n_cand;      /* candidates passed to the verifier */
    uint64_t n_pred;      /* verified results */
    uint64_t n_flood;     /* flood-phase node expansions */
    float search_ms;      /* device time of the search kernel (CUDA events on its stream) */
    float total_ms;       /* device time from first copy to last copy of the call */
    uint64_t h2d_bytes, d2h_bytes;
    uint32_t visited_table;    /* entries of the per-warp shared-memory visited table the search
                                  ran with (chosen by timing; 0 = none) */
    uint32_t visited_l2_table; /* entries of the per-warp L2-resident visited table (0 = none);
                                  beyond both, a per-warp bitmap over all ids */
    uint32_t warps_per_block;  /* block shape of the search launch (2, 4 or 8 warps, one query
                                  each), chosen by timing with the visited-set sizes */
    uint32_t candidate_tile;   /* base rows per postfilter round (8, 4 or 2), chosen by timing */
} anqi_query_stats;

int anqi_rknn_query(anqi_ctx* ctx, const float* queries, uint32_t nq, const uint32_t* k_per_query,
                    uint32_t k_all, const uint32_t* L_per_query, uint32_t L_all, uint32_t* pred_off,
                    uint32_t* pred_ids, uint64_t pred_cap, uint32_t* cand_off, uint32_t* cand_ids,
                    uint64_t cand_cap, uint32_t* n_dist, anqi_query_stats* st);

/* Resident-batch form for callers that keep queries and results in HBM:
 * upload once, run many times (results stay on the device), then download. */
int anqi_query_upload(anqi_ctx* ctx, const float* queries, uint32_t nq, const uint32_t* k_per_query,
                      uint32_t k_all, const uint32_t* L_per_query, uint32_t L_all);
/* st (optional) receives search_ms only; anqi_query_counters sums the
 * per-query counters of the last run (device -> host copies). */
int anqi_query_run(anqi_ctx* ctx, int keep_candidates, anqi_query_stats* st);
/* CUDA-graph form of anqi_query_run for a stream of batches of one shape (same
 * nq, beam-width bound, k/L mode and candidate option; no counterpart in the
 * reference, whose query loop is a host loop).  The first call runs
 * anqi_query_run (autotuning, sizing the outputs) and captures the batch's
 * launch sequence -- lift + tree entry, leaf ordering, search, CSR compaction
 * -- into a graph; later calls replay it on whatever batch anqi_query_upload
 * left resident, with one small copy back of the output fill.  Results equal
 * anqi_query_run's.  A batch whose output outgrows the captured capacity runs
 * the plain path and is captured again. */
int anqi_query_run_graph(anqi_ctx* ctx, int keep_candidates, anqi_query_stats* st);
int anqi_query_counters(anqi_ctx* ctx, anqi_query_stats* st);
int anqi_query_download(anqi_ctx* ctx, uint32_t* pred_off, uint32_t* pred_ids, uint64_t pred_cap,
                        uint32_t* cand_off, uint32_t* cand_ids, uint64_t cand_cap, uint32_t* n_dist);
/* Recall / precision of the resident batch's last results against a
 * ground-truth CSR (rknn_query.cpp:2784-2799), computed on the device. */
int anqi_query_evaluate(anqi_ctx* ctx, const uint32_t* gt_off, const uint32_t* gt_ids, uint64_t gt_total,
                        double* recall_sum, double* precision_sum, double* cand_recall_sum,
                        uint32_t* nonempty);

/* Resident form of the evaluation for timed loops: anqi_gt_load keeps a
 * ground-truth CSR (_rknn_gt.bin layout: nq+1 offsets, ids in any order) on
 * the device for the current batch; anqi_query_evaluate_sums then reduces the
 * last run's per-query metrics on the device, in a fixed order, into sums over
 * the queries with non-empty truth -- the accumulators of
 * rknn_query.cpp:2784-2799 (recall, precision, F1, candidate recall, |C|, |P|,
 * graph distances).  Candidate recall needs a run with keep_candidates. */
typedef struct {
    double recall, precision, f1, cand_recall;
    double cand, pred, graph_dist;
    uint32_t nonempty;
} anqi_eval_sums;
int anqi_gt_load(anqi_ctx* ctx, const uint32_t* gt_off, const uint32_t* gt_ids, uint64_t gt_total);
int anqi_query_evaluate_sums(anqi_ctx* ctx, anqi_eval_sums* out);

/* ------------------------------------------------ allocation-free query
 * No counterpart in the reference: an extra entry point of this library for
 * callers that cannot allocate device memory -- e.g. code inside a host
 * framework whose device memory all comes from its own pool, or a process
 * whose memory budget is fixed up front -- and so cannot use a context (which
 * allocates).  Same search and postfilter as anqi_rknn_query for one k and one
 * L, on index arrays the caller already holds in device memory; it allocates
 * nothing.  Its working memory is a fixed file-scope device array of
 * ANQI_NOALLOC_SCRATCH_BYTES that every GPU loading this library reserves
 * until the process exits.  Each query in flight holds one slot of it (a
 * visited bitmap of n/8 bytes plus 40 KB), so n is at most about 134 million
 * (one slot) and concurrency falls as n grows: at n = 1M about 100 queries run
 * at once, a fraction of what the context path keeps in flight.  All calls on
 * a device share that array: calls that overlap on the GPU race -- serialize
 * them.  The first call on each device looks up the array
 * (cudaGetSymbolAddress).  Every call synchronizes `stream` before it returns
 * (it reads back an error word), so it cannot be called while that stream is
 * being captured.
 * Arrays are device pointers; rows 16-byte aligned, strides multiples of 4
 * floats; queries nq x base_stride.  pred_ids receives up to max_pred ids per
 * query (row q at q * max_pred), pred_count the full count; returns
 * ANQI_ERR_CAPACITY if any count exceeded max_pred or a query's candidate list
 * exceeded 8192 entries, ANQI_ERR_FORMAT for a link or tree child out of
 * range, ANQI_ERR_ARGS for bad sizes or alignment. */
#define ANQI_NOALLOC_SCRATCH_BYTES (16u << 20)
typedef struct {
    uint64_t n;
    uint32_t d, degree;
    const float* base;            /* n x base_stride */
    uint32_t base_stride;
    const float* lifted;          /* n x lifted_stride (>= d + 2) */
    uint32_t lifted_stride;
    const uint32_t* deg;          /* n */
    const uint32_t* links;        /* n x degree */
    uint32_t tree_nodes;          /* post-order, root last */
    const uint32_t* tree_left;
    const uint32_t* tree_right;
    const float* tree_offset;
    const float* tree_hyperplane; /* tree_nodes x lifted_stride */
    const uint32_t* tree_leaf_first;
    double scale, mstar2;
    uint32_t metric;              /* ANQI_METRIC_L2 or ANQI_METRIC_IP */
} anqi_device_index;

int anqi_rknn_query_noalloc(const anqi_device_index* ix, const float* queries, uint32_t nq,
                            const float* thresholds, uint32_t L, uint32_t max_pred, uint32_t* pred_count,
                            uint32_t* pred_ids, uint32_t* n_dist, void* stream);

/* ------------------------------------------- LRQ objective (training)
 * The radius-reconstruction objective the trainer minimises
 * (tools/train_final_m8_u8.py:90-157, 206-218), FP64, on DEVICE pointers,
 * enqueued on `stream` (a cudaStream_t; NULL = legacy default stream); they
 * allocate nothing.  T: n x nk rows; mu: nk; G: m x nk; B: nk x cs, rows
 * ascending.  c = (T - mu) G^T, base = mu + c G, a = nearest code of T - base
 * (decode_nearest, :146-156; or codes_in when given), r = base + B[k,a] - T,
 * *loss = sum(r^2) (divide by n*nk for the mean).  Outputs r (n x nk), c
 * (n x m), a (n x nk).  Limits: nk <= 128, m <= 16, cs <= 256.
 * Backward (codes fixed): g_mu, g_G, g_B = scale * d(sum r^2)/d(mu, G, B)
 * from the forward's r, c, a; the outputs are overwritten.  The B gradient
 * is a segment sum by code; its accumulation order is not fixed (FP64
 * atomics), so repeated calls may differ in the last bits. */
int anqi_lrq_objective_forward(const double* T, uint64_t n, uint32_t nk, uint32_t m, const double* mu,
                               const double* G, const double* B, uint32_t cs, const uint8_t* codes_in, double* r,
                               double* c, uint8_t* a, double* loss, void* stream);
int anqi_lrq_objective_backward(const double* T, uint64_t n, uint32_t nk, uint32_t m, const double* mu,
                                const double* G, const double* r, const double* c, const uint8_t* a, uint32_t cs,
                                double scale, double* g_mu, double* g_G, double* g_B, void* stream);

/* ------------------------------------------- LRQ fit on the device
 * The trainer's rounds (tools/train_final_m8_u8.py:81-258) as FP64 kernels; a
 * host driver keeps the nk x nk eigen-decomposition.  DEVICE pointers, the
 * caller's stream, nothing allocated; scratch sizes are checked
 * (ANQI_ERR_CAPACITY).  keys: cutoff rows (rows x nk, f32, row-major); ids:
 * the rows used (NULL = the first m).  nk <= 128, rank <= 16, cs <= 256.
 * Results agree with the NumPy fit to rounding (sums run in other orders),
 * not bit for bit.
 * stats: mean (nk) and covariance (nk x nk, divided by m) of keys[ids] - sub,
 *   sub nk x m column-major or NULL (fit_basis, :81-89); scratch
 *   ceil(m / 1024) * nk * nk doubles.
 * residual: res = T - (mu + ((T - mu) G^T) G), nk x m column-major
 *   (reconstruct, :90-93); *status |= 1 on a non-finite value.
 * range: lohi[2k], lohi[2k+1] = min, max over all n rows of column k of
 *   the residual (:159-174).
 * codebooks: per column, the sorted residuals' 1-D Lloyd (quantile
 *   centres, prefix-sum cell means, monotone repair, stop below 1e-12;
 *   :97-144); scratch anqi_lrq_fit_codebooks_scratch(m, nk) doubles.
 * decode: dec = nearest centre (lower on ties; :146-156), nk x m; partial
 *   receives *n_partial per-block sums of (dec - res)^2. */
int anqi_lrq_fit_stats(const float* keys, const uint32_t* ids, uint64_t m, uint32_t nk, const double* sub,
                       double* scratch, uint64_t scratch_doubles, double* mean, double* cov, void* stream);
int anqi_lrq_fit_residual(const float* keys, const uint32_t* ids, uint64_t m, uint32_t nk, const double* mu,
                          const double* basis, uint32_t rank, double* res, uint32_t* status, void* stream);
int anqi_lrq_fit_range(const float* keys, uint64_t n, uint32_t nk, const double* mu, const double* basis,
                       uint32_t rank, double* lohi, uint32_t* status, void* stream);
uint64_t anqi_lrq_fit_codebooks_scratch(uint64_t m, uint32_t nk);
int anqi_lrq_fit_codebooks(const double* res, uint64_t m, uint32_t nk, uint32_t cs, uint32_t iters, double* scratch,
                           uint64_t scratch_doubles, double* codebooks, void* stream);
int anqi_lrq_fit_decode(const double* res, uint64_t m, uint32_t nk, const double* codebooks, uint32_t cs, double* dec,
                        double* partial, uint32_t partial_cap, uint32_t* n_partial, void* stream);

/* ------------------------------------------ BF16 tensor-core tiles
 * out[i, j] = <bf16(a_i), bf16(b_j)> accumulated in FP32 on the tcgen05 tensor
 * cores (the tile primitive of the precision-form distance work); a: na x d,
 * b: nb x d, out: na x nb.  d <= 256.  No reference counterpart: the
 * reference computes every distance in FP32 (include/distance.h). */
int anqi_bf16_gram(anqi_ctx* ctx, const float* a, uint64_t na, const float* b, uint64_t nb, uint32_t d, float* out);

/* ---------------------------------------------------- exact ground truth
 * tools/dataset_gt.cpp:206-313 in FP32 with the reference's summation order:
 * per base row the K nearest other rows by (key, id), key = |a|^2+|b|^2-2ab. */
int anqi_exact_topk(anqi_ctx* ctx, const float* base, uint64_t n, uint32_t d, uint32_t K,
                    uint32_t* ids, float* keys);
/* Reverse-kNN membership: for each query, all j with key(q, j) <= rk2[j],
 * ascending (key, id).  off: nq+1.  Returns ANQI_ERR_CAPACITY (and the needed
 * total in *total) when cap is too small. */
int anqi_rknn_ground_truth(anqi_ctx* ctx, const float* base, uint64_t n, const float* query, uint64_t nq,
                           uint32_t d, const float* rk2, uint32_t* off, uint32_t* ids, float* keys,
                           uint64_t cap, uint64_t* total);
/* The same in either metric: ANQI_METRIC_IP keys are -<a, b> in the same lane
 * order (tools/dataset_gt.cpp:224, 288); rk2 may be negative. */
int anqi_exact_topk_metric(anqi_ctx* ctx, const float* base, uint64_t n, uint32_t d, uint32_t K, uint32_t metric,
                           uint32_t* ids, float* keys);
int anqi_rknn_ground_truth_metric(anqi_ctx* ctx, const float* base, uint64_t n, const float* query, uint64_t nq,
                                  uint32_t d, const float* rk2, uint32_t metric, uint32_t* off, uint32_t* ids,
                                  float* keys, uint64_t cap, uint64_t* total);

/* Precision form of the two entry points above: BF16 tcgen05 tiles with FP32
 * accumulation filter every pair by a derived bound on |key~ - key32|; the
 * pairs within it are recomputed in the reference's FP32 order.  Outputs equal
 * anqi_exact_topk / anqi_rknn_ground_truth bit for bit.  d <= 1024: up to 256
 * (padded to 16) the query tile stays in shared memory; above, both operands
 * pass through a ring of 64-wide K chunks accumulating in TMEM.
 * anqi_exact_topk_tc bounds each row's K-th key by the largest FP32 key to K
 * distinct other rows: hints (n x hint_k ids, e.g. the AKNN lists, hint_k >= K)
 * or, when hints is NULL, an AKNN build run here. */
int anqi_exact_topk_tc(anqi_ctx* ctx, const float* base, uint64_t n, uint32_t d, uint32_t K, const uint32_t* hints,
                       uint32_t hint_k, uint32_t* ids, float* keys);
int anqi_rknn_ground_truth_tc(anqi_ctx* ctx, const float* base, uint64_t n, const float* query, uint64_t nq,
                              uint32_t d, const float* rk2, uint32_t* off, uint32_t* ids, float* keys,
                              uint64_t cap, uint64_t* total);
/* The same under either metric (ANQI_METRIC_L2 or ANQI_METRIC_IP: key -<a, b>,
 * as anqi_exact_topk_metric / anqi_rknn_ground_truth_metric, which they equal
 * bit for bit).  Without hints the AKNN build runs under the same metric. */
int anqi_exact_topk_tc_metric(anqi_ctx* ctx, const float* base, uint64_t n, uint32_t d, uint32_t K,
                              const uint32_t* hints, uint32_t hint_k, uint32_t metric, uint32_t* ids, float* keys);
int anqi_rknn_ground_truth_tc_metric(anqi_ctx* ctx, const float* base, uint64_t n, const float* query, uint64_t nq,
                                     uint32_t d, const float* rk2, uint32_t metric, uint32_t* off, uint32_t* ids,
                                     float* keys, uint64_t cap, uint64_t* total);

#ifdef __cplusplus
}
#endif
#endif /* ANQI_H */
