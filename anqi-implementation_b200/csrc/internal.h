// Host-side internals shared by the .cu translation units of libanqi.
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/anqi.h"

namespace anqi {

// A growable device allocation owned by the context.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

struct Ctx;

// Throws nothing: every helper records the error in ctx and returns a status.
int fail(Ctx* c, int status, const char* fmt, ...);
int cuda_check(Ctx* c, cudaError_t e, const char* what);
#define ANQI_CUDA(ctx, call)                                      \
    do {                                                          \
        cudaError_t _e = (call);                                  \
        if (_e != cudaSuccess) return ::anqi::cuda_check((ctx), _e, #call); \
    } while (0)

struct QueryIndex {
    bool loaded = false;
    uint64_t n = 0;
    uint32_t d = 0, dim = 0, degree = 0;
    uint32_t bstride = 0, lstride = 0;  // padded row strides (floats, multiple of 8)
    uint32_t tree_nodes = 0, troot = 0;
    double scale = 0, mstar2 = 0;
    uint32_t metric = 0;  // ANQI_METRIC_L2 / ANQI_METRIC_IP
    DevBuf base, lifted, onorm, deg, links;
    DevBuf tleft, tright, toffset, thyper, tleaf;
    // objects are held renumbered in breadth-first order of the graph:
    // perm[new id] = original id (base, lifted, norms, graph, entries and
    // thresholds are stored by new id; results are returned as original ids)
    DevBuf perm;
};

struct Verifier {
    bool loaded = false;
    uint64_t n = 0;
    uint32_t nk = 0, rankm = 0, code_size = 0;
    uint32_t bits = 8;         // 0 (rank-M only), 2, 4, 8, 16 (codes), 32 (float residuals)
    bool signed_keys = false;  // IP: thresholds are not clamped at zero
    // analytic Rank-M model (coeff only): power-law basis in k
    bool analytic = false;
    uint32_t train_kmax = 0, flags = 0;
    double b0 = 0;
    DevBuf coeff, codes_t /* nk x n4, k-major: u8 / u16 codes or f32 residuals */, mu, basis, codebook;
};

struct Batch {
    uint32_t nq = 0;
    uint32_t L_max = 0;
    bool has_k = false, has_L = false;
    uint32_t k_all = 0, L_all = 0;
    std::vector<uint32_t> k_host;        // distinct k values used (slots)
    DevBuf q, qL, qslot;                 // queries (nq x bstride), per-query L and threshold slot
    DevBuf npred, ncand, ndist, nexp, nflood, pred_at, cand_at;
    DevBuf pred_buf, cand_buf;           // atomic-fill output buffers
    DevBuf pred_off, cand_off;           // CSR offsets (device)
    DevBuf pred_csr, cand_csr;
    DevBuf entry, enode, order, leaf_cnt;  // entry object / leaf node per query, leaf-ordered work list
    DevBuf qr2;                            // ip metric: per-query range radius (float, rounded down)
    uint64_t pred_cap = 0, cand_cap = 0;
    bool have_results = false;
    bool have_cands = false;
    bool ordered = false;  // work list ordered by entry leaf
};

// A G48 build in progress (anqi_graph_build_begin .. _finish): lifted rows,
// norms, the warm-start heaps and the entry tree's row order stay on the
// device between the calls that deliver warm-start rows.
struct GraphBuild {
    bool active = false;
    uint64_t n = 0, rows_done = 0;
    uint32_t dim = 0, xs = 0;
    anqi_graph_params gp{};
    DevBuf dx, dn, hid, hv, order;
    std::vector<uint8_t> seen;  // rows delivered
    double forest_ms = 0, warm_ms = 0;
    // the edge policy of anqi_graph_params.edge, copied at begin
    bool has_edge = false;
    anqi_edge_policy edge{};
    std::vector<float> edge_resid, edge_mu;
};

// The edge policy of the current graph build (anqi_edge_policy on the
// device): the prune of select, commit and Vamana passes runs in
// policy_prune_kernel while active.
struct DevPolicyView {
    uint32_t flags, nks, ks[8], nk, budget, occ_all, auto_cand, auto_swaps;
    double lambda, scale2, lsg_alpha;
    const float* resid;
    const float* mu;
};
struct DevPolicy {
    bool active = false;
    DevPolicyView view{};
    DevBuf resid, mu;
};

struct Ctx {
    int device = 0;
    int sm_count = 0;
    uint32_t inject = 0;  // ANQI_FAULT_* flags (anqi_inject_fault)
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr, ev3 = nullptr;
    cudaEvent_t tev0 = nullptr, tev1 = nullptr;  // anqi_timer_*
    std::string last_error;
    QueryIndex ix;
    Verifier vf;
    Batch batch;
    // scratch
    DevBuf err, counters;
    DevBuf vis_bits, vis_log, cand_scratch;
    uint32_t vis_slots = 0, vis_words = 0, log_cap = 0, cand_cap = 0;
    // resident ground truth (anqi_gt_load) and evaluation scratch
    DevBuf gt_off, gt_ids, eval_rows, eval_sums;
    uint32_t gt_nq = 0;
    // last entry tree from anqi_graph_build
    std::vector<uint32_t> t_left, t_right, t_leaf_off, t_leaf_cnt, t_perm;
    std::vector<float> t_offset, t_hyper;
    uint32_t t_nodes = 0, t_dim = 0;
    // search-kernel autotuning: configuration key -> shared-memory visited table size
    std::unordered_map<uint64_t, uint64_t> tuned;  // value: shared entries | L2 entries << 32
    DevBuf vis_gtab;                               // per-slot L2-resident visited tables
    uint32_t gtab_slots = 0, gtab_cap = 0;
    bool l2_window = false;                        // an L2 persisting window is set on the stream
    // configuration of the last anqi_query_run and the captured graph of it
    uint32_t last_cfg_hash = 0, last_cfg_gcap = 0, last_cfg_blocks = 0;
    size_t last_cfg_smem = 0;
    uint32_t last_cfg_wpb = 4, last_cfg_post = 8;  // block shape and candidate tile
    cudaGraphExec_t qgraph = nullptr;
    DevBuf init_cnt, init_cid, init_key;  // tensor-core init_knn candidate buffers
    GraphBuild gb;                        // staged G48 build
    DevBuf g_bits, g_vlog, g_pd, g_pi, g_gtab;  // gather kernel per-slot scratch
    DevPolicy edge;                              // edge policy of the build in progress
    DevBuf pol_scratch, pol_dump_d, pol_dump_i, pol_dump_n;  // policy prune scratch and pool dumps
    // pinned staging slots for large copies to and from pageable host memory
    static constexpr int kStageSlots = 3;
    void* stage[kStageSlots] = {};
    cudaEvent_t stage_ev[kStageSlots] = {};
    std::vector<uint64_t> qgraph_key;
    uint64_t device_bytes = 0;
    std::vector<DevBuf*> member_bufs() {
        return {&ix.base, &ix.lifted, &ix.onorm, &ix.deg, &ix.links, &ix.tleft, &ix.tright, &ix.toffset,
                &ix.thyper, &ix.tleaf, &ix.perm, &vf.coeff, &vf.codes_t, &vf.mu, &vf.basis, &vf.codebook, &batch.q,
                &batch.qL, &batch.qslot, &batch.npred, &batch.ncand, &batch.ndist, &batch.nexp, &batch.nflood,
                &batch.pred_at, &batch.cand_at, &batch.pred_buf, &batch.cand_buf, &batch.pred_off,
                &batch.cand_off, &batch.pred_csr, &batch.cand_csr, &batch.entry, &batch.enode, &batch.order,
                &batch.leaf_cnt, &batch.qr2, &err, &counters, &vis_bits, &vis_log,
                &cand_scratch, &thr_table, &gt_off, &gt_ids, &eval_rows, &eval_sums, &vis_gtab,
                &init_cnt, &init_cid, &init_key, &g_bits, &g_vlog, &g_pd, &g_pi, &g_gtab, &gb.dx, &gb.dn,
                &edge.resid, &edge.mu, &pol_scratch, &pol_dump_d, &pol_dump_i, &pol_dump_n,
                &gb.hid, &gb.hv, &gb.order};
    }
    // Per-object thresholds for up to kThrSlots values of k: slot s holds
    // thr_k[s] (0 = unused) in thr_table[s * n .. (s+1) * n).
    static constexpr int kThrSlots = 8;
    DevBuf thr_table;
    uint32_t thr_k[kThrSlots] = {0, 0, 0, 0, 0, 0, 0, 0};
    uint64_t thr_n = 0;
};

// Grow buf to at least bytes (contents not preserved).
int ensure(Ctx* c, DevBuf& b, size_t bytes);
void release(Ctx* c, DevBuf& b);

// A temporary device allocation released when it goes out of scope.
struct TmpBuf : DevBuf {
    Ctx* c;
    explicit TmpBuf(Ctx* ctx) : c(ctx) {}
    ~TmpBuf() { release(c, *this); }
    TmpBuf(const TmpBuf&) = delete;
    TmpBuf& operator=(const TmpBuf&) = delete;
};
int h2d(Ctx* c, DevBuf& b, const void* src, size_t bytes);
// Host <-> device copies of raw ranges on the context's stream (large
// pageable ranges through pinned staging slots; d2h_raw then returns with the
// data in place).
int h2d_raw(Ctx* c, void* dst, const void* src, size_t bytes);
int d2h_raw(Ctx* c, void* dst, const void* src, size_t bytes);
int d2h(Ctx* c, void* dst, const DevBuf& b, size_t bytes);
int sync(Ctx* c);
// Reads the device error word, maps it to a status (and clears it).
int check_device_error(Ctx* c, const char* stage);

inline uint32_t round_up(uint32_t x, uint32_t m) { return (x + m - 1) / m * m; }

// Pad rows of a host matrix into a device buffer with stride (floats), zero fill.
int upload_padded(Ctx* c, DevBuf& b, const float* src, uint64_t n, uint32_t d, uint32_t stride);
// Device rows (n x stride) with each of the first `full` columns' 16-float
// chunks stored in chunk column order (common.cuh chunk_col_pos), on the stream.
int chunk_cols(Ctx* c, const float* src, float* dst, uint64_t n, uint32_t stride, uint32_t full);
// dst row i = src row perm[i] (cols_full != 0: in chunk column order over the
// first cols_full columns); dst[i] = src[perm[i]] for one value per row.
__global__ void permute_rows_kernel(const float* __restrict__ src, float* __restrict__ dst,
                                    const uint32_t* __restrict__ perm, uint64_t n, uint32_t stride,
                                    uint32_t cols_full);
__global__ void permute_vals_kernel(const float* __restrict__ src, float* __restrict__ dst,
                                    const uint32_t* __restrict__ perm, uint64_t n);

// A built random-projection forest (breadth-first node numbering per tree; tree
// t's nodes at [t * cap_nodes, ...), its permutation at [t * n, ...)).
struct ForestOut {
    uint32_t trees = 0, cap_nodes = 0, dim = 0, stride = 0;
    uint64_t n = 0;
    std::vector<uint32_t> n_nodes, left, right, leaf_off, leaf_cnt;
    std::vector<float> offset;
    DevBuf perm, hyper;  // device; released by the caller
};
int build_forest(Ctx* c, const float* d_x, uint64_t n, uint32_t dim, uint32_t stride, uint32_t trees, uint32_t leaf,
                 uint32_t max_depth, uint64_t seed, uint32_t cap_nodes, ForestOut& out, int angular = 0);
// Exclusive scan of n u32 counts into n + 1 u64 offsets (device).
int device_scan(Ctx* c, const uint32_t* d_in, uint64_t* d_out, uint64_t n);

// One RP-tree leaf of a forest permutation: members perm[off .. off + cnt).
struct LeafRef {
    uint64_t off;
    uint32_t cnt, pad;
};
// Row block rb (128 rows) of a leaf: one CTA of the tensor-core init_knn filter.
struct LeafTile {
    uint64_t off;
    uint32_t cnt, rb;
};
// Candidate id flag of the tensor-core init_knn filter: the key is the bf16
// approximation and must be recomputed in FP32.
constexpr uint32_t kRecheck = 0x80000000u;

// Rows of a device matrix in the BF16 tensor-core form (tc.cu): bf16 copy
// padded to dp, |x| and |x - bf16(x)| rounded up, exact-integer flags.
struct TcPrep {
    DevBuf bf, nrm, err, xint;
    uint32_t dp = 0;
    float bnorm = 0, berr = 0, bn = 0;  // maxima of |x|, |x - bf16(x)|, the FP32 norm
    int all_exact = 0;                  // every row exact-integer
};
// Padded row length of the tensor path for dimension d: resident query tiles
// up to 256, the wide (K-chunked) form up to 1024; 0 above.
uint32_t tc_padded_dim(uint32_t d);
int tc_prep(Ctx* c, const float* d_x, const float* d_norms, uint64_t n, uint32_t xs, uint32_t d, TcPrep& tp);
void tc_release(Ctx* c, TcPrep& tp);
// LocalJoin precision form: for each source u's samples (samp, scnt; S <= 32)
// the tensor-core Gram tile keeps, per target sample a, the candidates b whose
// key may reach the target's heap top (hval[t * K]); mask[u * S + a] bit b.
int tc_join_filter(Ctx* c, const TcPrep& tp, const float* d_norms, uint64_t n, const uint32_t* samp,
                   const uint32_t* scnt, uint32_t S, const float* hval, uint32_t K, uint32_t* mask);
// init_knn candidates of a batch of one tree's leaves on the tensor cores:
// for every member row, the leaf-mates j != row whose key may be <= the
// row's current K-th list key (any while the list is short), appended to
// out_id / out_key [slot * cap ..] with cnt[slot], slot = the row's position in
// the forest permutation - pos_base (kRecheck marks keys to recompute in FP32).
int tc_leaf_candidates(Ctx* c, const TcPrep& tp, const float* d_x, const float* d_norms, uint64_t n, uint32_t xs,
                       uint32_t d, const uint32_t* d_members, const std::vector<LeafRef>& leaves,
                       const float* list_kd, const uint32_t* list_sz, uint32_t K, uint32_t* cnt, uint32_t cap,
                       uint32_t* out_id, float* out_key, uint64_t pos_base);
// The same in two steps, so that many batches launch without a host round
// trip: the 128-row tiles of a batch's leaves (appended to tiles; a leaf
// longer than cap + 1 is an argument error), then the filter over ntiles
// tiles already on the device (errors are left in the device error word).
// key_mode 0: the l2 key; 1: the ip metric's 1 - <a, b>.
int tc_leaf_tiles(Ctx* c, const std::vector<LeafRef>& leaves, uint32_t cap, std::vector<LeafTile>& tiles);
int tc_leaf_filter(Ctx* c, const TcPrep& tp, const float* d_x, const float* d_norms, uint64_t n, uint32_t xs,
                   uint32_t d, const uint32_t* d_members, const LeafTile* d_tiles, size_t ntiles,
                   const float* list_kd, const uint32_t* list_sz, uint32_t K, uint32_t* cnt, uint32_t cap,
                   uint32_t* out_id, float* out_key, uint64_t pos_base, uint32_t key_mode);

// Edge policy of the next select / commit / Vamana prunes (nullptr or flags 0:
// the default prune; tables copied to the device), and its release.
int set_edge_policy(Ctx* c, const anqi_edge_policy* pol, uint64_t n);
void clear_edge_policy(Ctx* c);
// Prunes the pools of nrows rows (row of entry t: rows[row_base + t], or
// row_base + t; pool t at pool_d / pool_i [t * pool_cap], pool_n[t] entries)
// under the active edge policy into out (n x M) / out_deg.
int run_policy_prune(Ctx* c, const float* x, const float* norms, uint64_t n, uint32_t stride, uint32_t dim, uint32_t M,
                     float alpha, const float* pool_d, const uint32_t* pool_i, const uint32_t* pool_n,
                     uint32_t pool_cap, const uint32_t* rows, uint64_t row_base, uint32_t nrows, uint32_t* out,
                     uint32_t* out_deg);

// L2 persisting window over [p, p + bytes) for kernels on the context's stream.
void set_l2_window(Ctx* c, const void* p, size_t bytes);
void clear_l2_window(Ctx* c);

// Launch helpers implemented in the .cu files.
int lrq_materialize_device(Ctx* c, const Verifier& v, uint32_t k, double scale, float* d_out);
int compute_norms_device(Ctx* c, const float* d_x, uint64_t n, uint32_t dim, uint32_t stride, float* d_out);
int sort_csr_segments(Ctx* c, const uint64_t* d_off, uint64_t nseg, uint32_t* d_ids, float* d_keys, uint64_t maxm);

}  // namespace anqi

struct anqi_ctx {
    anqi::Ctx c;
};
