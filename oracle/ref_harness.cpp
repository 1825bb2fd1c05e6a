// Test infrastructure only: a harness that drives the reference implementation's
// own functions stage by stage and dumps every stage boundary as raw binary.
//
// It is compiled by oracle/Makefile against the reference sources where they lie
// (include/index.h and src/rknn_query.cpp of Yujian-Fu/anqi-implementation); no
// reference source is copied into this repository.  The reference driver's
// main() is renamed so its file-local types (CompactLrqVerifier, the codec
// helpers) become callable here.  Output goes to oracle/_ref/ only.
//
// Subcommands (all single-threaded unless stated, so dumps are reproducible):
//   dist     IN OUT                         distance kernels of include/distance.h
//   verifier PFX OUT [BITS POLICY SIGNED]   CompactLrqVerifier build/materialize (rknn_query.cpp:679-753)
//   analytic MODEL N RANKM OUT              AnalyticRankMVerifier load/materialize (rknn_query.cpp:515-601)
//   graph    LIFTED WARM_REC NNK M OUT      staged lifted-graph build (index.h:1071-1295)
//   aknn     BASE OUT K LEAF TREES EF SEED [METRIC]
//                                           staged AKNN source build (index.h:1300-1461), l2 or ip
//   ipdist   IN OUT                         the ip metric's scalar distance (distance.h:170-174)
//   query    LIFTED GRAPH BASE QUERY META THR L OUT
//                                           range_search + postfilter per query (index.h:1535, rknn_query.cpp:2692-2765)
//   qbench   LIFTED GRAPH BASE QUERY META L THREADS WARMUP STEPS NQ THR GT [THR GT ...]
//                                           the reference's timed query loop body, OpenMP, prints one JSON line
//   qparity  LIFTED GRAPH BASE QUERY META L ENTRY NQ OUT THR [THR ...]
//                                           per-query candidates / verified sets / #dist, entry
//                                           descent as the reference draws it or with ties sent left

#define main anqi_reference_rknn_query_main
#include "src/rknn_query.cpp"
#undef main

#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

namespace {

void die(const char* msg) {
    std::fprintf(stderr, "[ref_harness] %s\n", msg);
    std::exit(3);
}

template <class T>
void write_vec(FILE* f, const std::vector<T>& v) {
    if (!v.empty() && std::fwrite(v.data(), sizeof(T), v.size(), f) != v.size()) die("short write");
}

void write_u64(FILE* f, uint64_t x) { std::fwrite(&x, 8, 1, f); }

FILE* open_out(const std::string& path) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) die(("cannot open output " + path).c_str());
    return f;
}

std::vector<float> read_fbin(const std::string& path, size_t& n, size_t& d) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) die(("cannot open " + path).c_str());
    uint32_t hdr[2];
    if (std::fread(hdr, 4, 2, f) != 2) die("short fbin header");
    n = hdr[0];
    d = hdr[1];
    std::vector<float> x(n * d);
    if (std::fread(x.data(), 4, x.size(), f) != x.size()) die("short fbin body");
    std::fclose(f);
    return x;
}

// Fills an nndindex (vectors already loaded) from a file written by
// nndindex::save_index: header, per-node adjacency, then the RP tree.
void load_graph_file(nndindex& index, const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) die(("cannot open graph " + path).c_str());
    size_t fn = 0, fdim = 0, fM = 0;
    float ctime = 0;
    f.read((char*)&fn, 8);
    f.read((char*)&fdim, 8);
    f.read((char*)&fM, 8);
    f.read((char*)&ctime, 4);
    if (fn != index.n || fdim != index.dim || fM != index.M) die("graph header mismatch");
    for (size_t i = 0; i < index.n; i++) {
        uint32_t d = 0;
        f.read((char*)&d, 4);
        if (d > index.M) die("bad degree");
        f.read((char*)index.lnk(i), d * 4);
        index.deg(i) = d;
    }
    if (!index.load_tree(f)) die("bad tree");
}

Parms lifted_parms(size_t n, size_t dim, size_t nnk, size_t M, const std::string& folder) {
    Parms par;
    par.n = n;
    par.dim = dim;
    par.meric = "l2";
    par.random_seed = 10;
    par.nn_k = nnk;
    par.M = M;
    par.leaf_size = 100;
    par.max_depth = 100;
    par.n_trees = 64;
    par.ef_alpha = 8;
    par.prune_alpha = 1.2f;
    par.explore_range = 100;
    par.n_threads = 1;
    par.folder_path = folder;
    return par;
}

void dump_heaps(HeapList* g0, size_t n, size_t K, const std::string& path) {
    FILE* f = open_out(path);
    for (size_t i = 0; i < n; i++) std::fwrite(g0->indices[i].data(), 4, K, f);
    for (size_t i = 0; i < n; i++) std::fwrite(g0->values[i].data(), 4, K, f);
    std::fclose(f);
}

void dump_csr(const std::vector<std::vector<uint32_t>>& rows, const std::string& path) {
    FILE* f = open_out(path);
    std::vector<uint64_t> off(rows.size() + 1, 0);
    for (size_t i = 0; i < rows.size(); i++) off[i + 1] = off[i] + rows[i].size();
    uint64_t n = rows.size();
    std::fwrite(&n, 8, 1, f);
    write_vec(f, off);
    for (const auto& r : rows) write_vec(f, r);
    std::fclose(f);
}

int cmd_dist(int argc, char** argv) {
    if (argc != 4) return 2;
    FILE* f = std::fopen(argv[2], "rb");
    if (!f) die("cannot open dist input");
    uint32_t m = 0, dim = 0;
    if (std::fread(&m, 4, 1, f) != 1 || std::fread(&dim, 4, 1, f) != 1) die("short dist header");
    std::vector<float> a(dim), b(dim);
    float* al = static_cast<float*>(_mm_malloc(((dim + 15) / 16) * 16 * 4, 64));
    float* bl = static_cast<float*>(_mm_malloc(((dim + 15) / 16) * 16 * 4, 64));
    FILE* o = open_out(argv[3]);
    for (uint32_t i = 0; i < m; i++) {
        if (std::fread(a.data(), 4, dim, f) != dim || std::fread(b.data(), 4, dim, f) != dim) die("short dist body");
        std::memcpy(al, a.data(), dim * 4);
        std::memcpy(bl, b.data(), dim * 4);
        float out[4];
        out[0] = DistCal::L2SqrSIMD16ExtAVX512__(a.data(), b.data(), dim);
        out[1] = DistCal::InnerProductSIMD16ExtAVX512_(a.data(), b.data(), dim);
        out[2] = DistCal::NormSIMD16ExtAVX512__(al, dim);
        // nndindex::d2 (index.h:172): vnorm(a) + vnorm(b) - 2 * IP(a, b)
        out[3] = out[2] + DistCal::NormSIMD16ExtAVX512__(bl, dim) - 2.0f * out[1];
        std::fwrite(out, 4, 4, o);
    }
    _mm_free(al);
    _mm_free(bl);
    std::fclose(o);
    std::fclose(f);
    return 0;
}

// verifier PFX OUT [BITS POLICY SIGNED]: CompactLrqVerifier build + save +
// materialize_k for k = 1, 10, 50, 100.  BITS 0 (rankm_only), 2/4/8/16
// (learned codebook PFX_learned_rq_codebook_M8_u{BITS}.bin), 32 (float
// residuals); POLICY floor / ceil / nearest; SIGNED 1 = IP keys (no clamp).
// ipdist IN OUT: the scalar inner-product distance 1 - sum a_i b_i of the
// "ip" metric (include/distance.h:170-174), per pair.
int cmd_ipdist(int argc, char** argv) {
    if (argc != 4) return 2;
    FILE* f = std::fopen(argv[2], "rb");
    if (!f) die("cannot open ipdist input");
    uint32_t m = 0, dim = 0;
    if (std::fread(&m, 4, 1, f) != 1 || std::fread(&dim, 4, 1, f) != 1) die("short ipdist header");
    std::vector<float> a(dim), b(dim);
    FILE* o = open_out(argv[3]);
    for (uint32_t i = 0; i < m; i++) {
        if (std::fread(a.data(), 4, dim, f) != dim || std::fread(b.data(), 4, dim, f) != dim) die("short ipdist body");
        const float v = DistCal(dim, "ip").calculate(a.data(), b.data());
        std::fwrite(&v, 4, 1, o);
    }
    std::fclose(o);
    std::fclose(f);
    return 0;
}

int cmd_verifier(int argc, char** argv) {
    if (argc != 4 && argc != 7) return 2;
    const std::string pfx = argv[2], out = argv[3];
    const int bits = argc == 7 ? std::atoi(argv[4]) : 8;
    const std::string policy = argc == 7 ? argv[5] : "floor";
    const bool is_ip = argc == 7 && std::atoi(argv[6]) != 0;
    size_t n = 0, d = 0;
    read_fbin(pfx + "_base.bin", n, d);
    const size_t NK = 100;
    const int RANKM = 8;
    std::ifstream bf(pfx + "_radbasis_M8.bin", std::ios::binary);
    int Kb = 0, Mb = 0;
    bf.read((char*)&Kb, 4);
    bf.read((char*)&Mb, 4);
    if (Kb != (int)NK || Mb != RANKM) die("bad basis header");
    std::vector<float> mu(NK), G(NK * RANKM);
    bf.read((char*)mu.data(), NK * 4);
    bf.read((char*)G.data(), NK * RANKM * 4);
    size_t code_size = 0;
    std::vector<float> cb;
    if (anqi::supported_packed_code_bits(bits))
        cb = load_learned_rq_codebook(pfx + "_learned_rq_codebook_M8_u" + std::to_string(bits) + ".bin", NK, RANKM,
                                      bits, code_size);
    std::vector<float> src(n * NK);
    setenv("ANQI_PREBUILT_TOPK_REC", (pfx + "_baseknn_aknn.rec").c_str(), 1);
    setenv("ANQI_PREBUILT_TOPK_K", "100", 1);
    load_threshold_table(pfx, n, NK, is_ip, src);
    CompactLrqVerifier v;
    v.configure(n, NK, RANKM, bits, policy, mu, G, cb, code_size);
    v.build(src);
    v.save(out + "_verifier.bin");
    FILE* f = open_out(out + "_thresholds.bin");
    for (size_t k : {1, 10, 50, 100}) {
        std::vector<float> thr;
        v.materialize_k(k, 1.0, is_ip, thr);
        write_vec(f, thr);
    }
    std::fclose(f);
    return 0;
}

// analytic MODEL N RANKM OUT: AnalyticRankMVerifier::load + materialize_k for
// k = 1, 10, 50, 100 at radius scales 1 and 1.25.
int cmd_analytic(int argc, char** argv) {
    if (argc != 6) return 2;
    AnalyticRankMVerifier a;
    a.load(argv[2], std::strtoull(argv[3], nullptr, 10), std::atoi(argv[4]));
    FILE* f = open_out(std::string(argv[5]) + "_thresholds.bin");
    for (double scale : {1.0, 1.25})
        for (size_t k : {1, 10, 50, 100}) {
            std::vector<float> thr;
            a.materialize_k(k, scale, thr);
            write_vec(f, thr);
        }
    std::fclose(f);
    return 0;
}

int cmd_graph(int argc, char** argv) {
    if (argc != 7) return 2;
    const std::string lifted = argv[2], warm = argv[3], out = argv[6];
    const size_t nnk = std::strtoull(argv[4], nullptr, 10), M = std::strtoull(argv[5], nullptr, 10);
    size_t n = 0, dim = 0;
    read_fbin(lifted, n, dim);
    Parms par = lifted_parms(n, dim, nnk, M, out + "_scratch/");
    nndindex index(lifted, par);
    // the edge policy of the prune from ANQI_EDGE_* / ANQI_LSG_* (none when
    // unset), as build_index configures it before its stages
    index.configure_edge_residual_cover();
    // Warm-start IDs: the interleaved {u32 id, f32 key} top-100 records.
    std::vector<uint32_t> ids(n * 100);
    {
        FILE* f = std::fopen(warm.c_str(), "rb");
        if (!f) die("cannot open warm records");
        std::vector<PrebuiltKnnRecord> rec(n * 100);
        if (std::fread(rec.data(), 8, rec.size(), f) != rec.size()) die("short warm records");
        std::fclose(f);
        for (size_t i = 0; i < rec.size(); i++) ids[i] = rec[i].id;
    }
    performance_recorder rec("harness graph");
    float* cvec = static_cast<float*>(_mm_malloc(n * dim * sizeof(float), 64));
    for (size_t i = 0; i < n; i++) std::memcpy(cvec + i * dim, index.vec(i), dim * sizeof(float));
    std::vector<rptree> forest = make_forest(cvec, n, dim, 1, index.leaf_size, false, index.max_depth, index.random_seed, 1);
    index.search_tree = forest[0];
    _mm_free(cvec);
    HeapList* g0 = new HeapList(n, nnk, false);
    for (size_t i = 0; i < n; i++)
        for (size_t k = 0; k < 100; k++) {
            uint32_t j = ids[i * 100 + k];
            if (j != (uint32_t)i && j < n) g0->push_nolock(i, j, index.d2(i, j));
        }
    dump_heaps(g0, n, nnk, out + "_g0_warm.bin");
    index.nndescent_refine(g0, rec, 6);
    dump_heaps(g0, n, nnk, out + "_g0_join.bin");
    g0->push_reverse(1);
    dump_csr(g0->reverse_indices, out + "_g0_rev.bin");
    std::vector<std::vector<uint32_t>> O(n);
    std::vector<uint32_t> pool_sizes(n);
    size_t cand_cap = std::max<size_t>(M, (size_t)(index.ef_alpha * index.explore_range));
    for (size_t i = 0; i < n; i++) {
        std::vector<std::pair<float, uint32_t>> pool;
        index.gather_candidates(i, g0, pool, cand_cap);
        pool_sizes[i] = (uint32_t)pool.size();
        std::vector<uint32_t> sel;
        index.prune_pool_to_ids(i, pool, sel);
        O[i] = sel;
    }
    dump_csr(O, out + "_O.bin");
    {
        FILE* f = open_out(out + "_pool_sizes.bin");
        write_vec(f, pool_sizes);
        std::fclose(f);
    }
    index.commit_edges(O);
    std::vector<std::vector<uint32_t>> adj(n);
    for (size_t i = 0; i < n; i++) adj[i].assign(index.lnk(i), index.lnk(i) + index.deg(i));
    dump_csr(adj, out + "_adj.bin");
    // the Vamana refine of build_index (index.h:1262-1285) when ANQI_VAMANA is
    // set: global passes from the RP-tree entries, or the batched style
    if (std::getenv("ANQI_VAMANA")) {
        const char* lv = std::getenv("ANQI_VAMANA_L");
        const char* pv = std::getenv("ANQI_VAMANA_PASS");
        const size_t Lb = lv ? (size_t)std::atoi(lv) : 128;
        const int passes = pv ? std::atoi(pv) : 2;
        const char* sv = std::getenv("ANQI_VAMANA_STYLE");
        const std::string style = sv ? sv : "global";
        if (style == "global" || style == "old") {
            for (int pass = 0; pass < passes; pass++) {
                for (size_t i = 0; i < n; i++) {
                    std::vector<std::pair<float, uint32_t>> pool;
                    index.greedy_collect(i, pool, Lb);
                    index.append_aknn_edges(i, g0, pool);
                    std::vector<uint32_t> ids;
                    index.prune_pool_to_ids(i, pool, ids);
                    O[i].assign(ids.begin(), ids.end());
                }
                index.commit_edges(O);
            }
        } else {
            index.vamana_batch_refine(g0, rec, Lb, passes);
        }
        for (size_t i = 0; i < n; i++) adj[i].assign(index.lnk(i), index.lnk(i) + index.deg(i));
        dump_csr(adj, out + "_vam_adj.bin");
    }
    index.construction_time = 0.0f;
    // save_index writes into folder_path + generate_config(); mirror that layout explicitly.
    {
        std::ofstream f(out + "_graph.bin", std::ios::binary);
        f.write((char*)&index.n, 8);
        f.write((char*)&index.dim, 8);
        f.write((char*)&index.M, 8);
        f.write((char*)&index.construction_time, 4);
        for (size_t i = 0; i < n; i++) {
            uint32_t d = index.deg(i);
            f.write((char*)&d, 4);
            f.write((char*)index.lnk(i), d * 4);
        }
        index.save_tree(f);
    }
    delete g0;
    return 0;
}

int cmd_aknn(int argc, char** argv) {
    if (argc != 9 && argc != 10) return 2;
    const std::string base = argv[2], out = argv[3];
    const size_t K = std::strtoull(argv[4], nullptr, 10), leaf = std::strtoull(argv[5], nullptr, 10);
    const size_t trees = std::strtoull(argv[6], nullptr, 10), ef = std::strtoull(argv[7], nullptr, 10);
    const size_t seed = std::strtoull(argv[8], nullptr, 10);
    const std::string metric = argc == 10 ? argv[9] : "l2";
    const bool angular = metric == "ip";
    size_t n = 0, d = 0;
    read_fbin(base, n, d);
    Parms po;
    po.n = n;
    po.dim = d;
    po.meric = metric;
    po.random_seed = seed;
    po.nn_k = K;
    po.M = 32;
    po.leaf_size = leaf;
    po.max_depth = 100;
    po.n_trees = trees;
    po.ef_alpha = 8;
    po.prune_alpha = 1.2f;
    po.explore_range = ef;
    po.n_threads = 1;
    po.folder_path = out + "_scratch/";
    nndindex index(base, po);
    float* cvec = static_cast<float*>(_mm_malloc(n * d * sizeof(float), 64));
    for (size_t i = 0; i < n; i++) std::memcpy(cvec + i * d, index.vec(i), d * sizeof(float));
    std::vector<rptree> forest = make_forest(cvec, n, d, trees, leaf, angular, 100, seed, 1);
    _mm_free(cvec);
    {
        std::vector<std::vector<uint32_t>> leaves;
        std::vector<uint32_t> leaf_tree;
        for (size_t t = 0; t < forest.size(); t++)
            for (const auto& nd : forest[t].nodes)
                if (nd.left == UINT32_MAX && nd.right == UINT32_MAX) {
                    leaves.push_back(nd.indices);
                    leaf_tree.push_back((uint32_t)t);
                }
        dump_csr(leaves, out + "_leaves.bin");
        FILE* f = open_out(out + "_leaf_tree.bin");
        write_vec(f, leaf_tree);
        std::fclose(f);
    }
    HeapList* g0 = new HeapList(n, K, false);
    index.init_knn(forest, g0);
    dump_heaps(g0, n, K, out + "_g0_init.bin");
    g0->push_reverse(1);
    dump_csr(g0->reverse_indices, out + "_g0_rev.bin");
    size_t cand_cap = std::max<size_t>(K, (size_t)(index.ef_alpha * index.explore_range));
    std::vector<uint32_t> rid(n * K, UINT32_MAX);
    std::vector<float> rds(n * K, 0.0f);
    std::vector<uint32_t> pool_sizes(n);
    for (size_t i = 0; i < n; i++) {
        std::vector<std::pair<float, uint32_t>> pool;
        index.gather_candidates(i, g0, pool, cand_cap);
        pool_sizes[i] = (uint32_t)pool.size();
        std::sort(pool.begin(), pool.end());
        size_t c = 0;
        for (auto& pr : pool) {
            if (pr.second == (uint32_t)i) continue;
            rid[i * K + c] = pr.second;
            rds[i * K + c] = pr.first;
            if (++c >= K) break;
        }
    }
    FILE* f = open_out(out + "_final.bin");
    write_vec(f, rid);
    write_vec(f, rds);
    std::fclose(f);
    f = open_out(out + "_pool_sizes.bin");
    write_vec(f, pool_sizes);
    std::fclose(f);
    delete g0;
    return 0;
}

// ANQI_HARNESS_METRIC=ip switches the query modes to the ip metric's lifted
// query and key (rknn_query.cpp:2724-2731, 2555-2558).
struct QueryEnv {
    size_t n = 0, dim = 0, d = 0, nq = 0;
    std::vector<float> base, queries, thr;
    double mstar2 = 0, scale = 0;
    bool is_ip = std::getenv("ANQI_HARNESS_METRIC") && std::string(std::getenv("ANQI_HARNESS_METRIC")) == "ip";
};

void load_query_env(QueryEnv& e, char** a) {
    size_t nl = 0, dl = 0;
    read_fbin(a[0], nl, dl);
    e.n = nl;
    e.dim = dl;
    size_t nb = 0;
    e.base = read_fbin(a[2], nb, e.d);
    size_t dq = 0;
    e.queries = read_fbin(a[3], e.nq, dq);
    if (nb != nl || dq != e.d || dl != e.d + 2) die("query input shapes disagree");
    std::ifstream mf(a[4]);
    if (!(mf >> e.mstar2 >> e.scale)) die("bad meta");
    e.thr.resize(e.n);
    FILE* f = std::fopen(a[5], "rb");
    if (!f || std::fread(e.thr.data(), 4, e.n, f) != e.n) die("bad threshold file");
    std::fclose(f);
}

void lift_query(const QueryEnv& e, const float* q, std::vector<float>& qb, double& R2) {
    double qn2s = 0;
    for (size_t j = 0; j < e.d; j++) {
        const double v = (double)q[j] * e.scale;
        qb[j] = (float)v;
        qn2s += v * v;
    }
    qb[e.d] = 1.0f;
    qb[e.d + 1] = 0.0f;
    R2 = e.is_ip ? (qn2s + 1.0 + e.mstar2) : (e.mstar2 + 1.0);
}

float recheck_key(const QueryEnv& e, size_t id, const float* q) {
    const float* o = e.base.data() + id * e.d;
    float ip = DistCal::InnerProductSIMD16ExtAVX512_(o, q, (uint32_t)e.d);
    if (e.is_ip) return -ip;
    float on = DistCal::InnerProductSIMD16ExtAVX512_(o, o, (uint32_t)e.d);
    float qn = DistCal::InnerProductSIMD16ExtAVX512_(q, q, (uint32_t)e.d);
    return on + qn - 2.0f * ip;
}

// query LIFTED GRAPH BASE QUERY META THR L OUT
int cmd_query(int argc, char** argv) {
    if (argc != 10) return 2;
    QueryEnv e;
    load_query_env(e, argv + 2);
    const size_t L = std::strtoull(argv[8], nullptr, 10);
    const std::string out = argv[9];
    Parms par = lifted_parms(e.n, e.dim, 50, 48, out + "_scratch/");
    nndindex index(argv[2], par);
    load_graph_file(index, argv[3]);
    std::vector<uint16_t> mark(e.n, 0);
    uint16_t ver = 0;
    std::vector<float> qb(e.dim);
    std::vector<std::vector<uint32_t>> cands(e.nq), preds(e.nq);
    std::vector<uint32_t> ndists(e.nq);
    for (size_t i = 0; i < e.nq; i++) {
        const float* q = e.queries.data() + i * e.d;
        double R2 = 0;
        lift_query(e, q, qb, R2);
        if (++ver == 0) {
            std::fill(mark.begin(), mark.end(), 0);
            ver = 1;
        }
        std::vector<uint32_t> cand;
        size_t nd = 0;
        index.range_search(qb.data(), R2, 0.0f, L, cand, nd, mark.data(), ver, nullptr, 0.5f, false);
        ndists[i] = (uint32_t)nd;
        for (uint32_t id : cand)
            if (recheck_key(e, id, q) <= (double)e.thr[id]) preds[i].push_back(id);
        cands[i] = cand;
    }
    dump_csr(cands, out + "_cand.bin");
    dump_csr(preds, out + "_pred.bin");
    FILE* f = open_out(out + "_ndist.bin");
    write_vec(f, ndists);
    std::fclose(f);
    return 0;
}

// The reference's entry descent (rptrees.h:108-124) with ties (|margin| <= EPS)
// sent left instead of to a random side; *tie reports whether any node on the
// path had such a margin (where the reference's own descent may go right).
uint32_t entry_ties_left(nndindex& index, const float* qb, bool* tie) {
    const rptree& t = index.search_tree;
    size_t v = t.nodes.size() - 1;
    *tie = false;
    while (t.nodes[v].left != UINT32_MAX) {
        const std::vector<float>& h = t.nodes[v].hyperplane;
        const float margin = DistCal::InnerProductSIMD16ExtAVX512_(h.data(), qb, h.size()) - t.nodes[v].offset;
        if (!(margin < -EPS) && !(margin > EPS)) *tie = true;
        v = margin > EPS ? t.nodes[v].right : t.nodes[v].left;
    }
    return t.nodes[v].indices.empty() ? 0u : t.nodes[v].indices[0];
}

// qparity LIFTED GRAPH BASE QUERY META L ENTRY NQ OUT THR1 [THR2 ...]
// Per-query outputs of the reference's range_search + FP32 postfilter for the
// first NQ queries (one thread), for comparison with another implementation
// query by query.  ENTRY "tree": the reference's own entry descent, which draws
// a random side at margin ties; ENTRY "left": the same descent with ties sent
// left (the entry handed to range_search through its single-entry switch).
// Writes OUT_entry.bin (per query: u32 tie-left entry, u32 1 if the tie-left
// path met a tie), OUT_cand.bin (CSR, visit order), OUT_ndist.bin (u32), and
// per threshold file t: OUT_pred{t}.bin (CSR, candidate order).
int cmd_qparity(int argc, char** argv) {
    if (argc < 12) return 2;
    char* env_args[6] = {argv[2], argv[3], argv[4], argv[5], argv[6], argv[11]};
    QueryEnv e;
    load_query_env(e, env_args);
    const size_t L = std::strtoull(argv[7], nullptr, 10);
    const std::string mode = argv[8];
    if (mode != "tree" && mode != "left") return 2;
    const size_t nq = std::min(e.nq, (size_t)std::strtoull(argv[9], nullptr, 10));
    const std::string out = argv[10];
    const int nt = argc - 11;
    std::vector<std::vector<float>> thr(nt);
    for (int t = 0; t < nt; t++) {
        thr[t].resize(e.n);
        FILE* f = std::fopen(argv[11 + t], "rb");
        if (!f || std::fread(thr[t].data(), 4, e.n, f) != e.n) die("bad threshold file");
        std::fclose(f);
    }
    if (mode == "left") setenv("ANQI_QUERY_SINGLE_ENTRY", "1", 1);
    else unsetenv("ANQI_QUERY_SINGLE_ENTRY");
    unsetenv("ANQI_VAMANA_QUERY_ENTRY");
    Parms par = lifted_parms(e.n, e.dim, 50, 48, out + "_scratch/");
    nndindex index(argv[2], par);
    load_graph_file(index, argv[3]);
    std::vector<uint16_t> mark(e.n, 0);
    uint16_t ver = 0;
    std::vector<float> qb(e.dim);
    std::vector<std::vector<uint32_t>> cands(nq);
    std::vector<std::vector<std::vector<uint32_t>>> preds(nt, std::vector<std::vector<uint32_t>>(nq));
    std::vector<uint32_t> ndists(nq), entry(2 * nq);
    for (size_t i = 0; i < nq; i++) {
        const float* q = e.queries.data() + i * e.d;
        double R2 = 0;
        lift_query(e, q, qb, R2);
        bool tie = false;
        entry[2 * i] = entry_ties_left(index, qb.data(), &tie);
        entry[2 * i + 1] = tie ? 1u : 0u;
        index.graph_entry_ = entry[2 * i];
        if (++ver == 0) {
            std::fill(mark.begin(), mark.end(), 0);
            ver = 1;
        }
        size_t nd = 0;
        index.range_search(qb.data(), R2, 0.0f, L, cands[i], nd, mark.data(), ver, nullptr, 0.5f, false);
        ndists[i] = (uint32_t)nd;
        for (uint32_t id : cands[i]) {
            const float key = recheck_key(e, id, q);
            for (int t = 0; t < nt; t++)
                if (key <= (double)thr[t][id]) preds[t][i].push_back(id);
        }
    }
    dump_csr(cands, out + "_cand.bin");
    for (int t = 0; t < nt; t++) dump_csr(preds[t], out + "_pred" + std::to_string(t) + ".bin");
    FILE* f = open_out(out + "_ndist.bin");
    write_vec(f, ndists);
    std::fclose(f);
    f = open_out(out + "_entry.bin");
    write_vec(f, entry);
    std::fclose(f);
    return 0;
}

// qbench LIFTED GRAPH BASE QUERY META L THREADS WARMUP STEPS NQ THR1 GT1 [THR2 GT2 ...]
// Times the reference's own per-query work (rknn_query.cpp:2714-2803): query
// lift, nndindex::range_search, the FP32 postfilter into an unordered_set, and
// the recall/precision evaluation against the ground-truth CSR, OpenMP over
// queries (schedule dynamic, 16).  One step runs the first NQ queries once for
// every (thresholds, ground truth) pair; prints one JSON line.
int cmd_qbench(int argc, char** argv) {
    if (argc < 14 || (argc - 12) % 2 != 0) return 2;
    const size_t L = std::strtoull(argv[7], nullptr, 10);
    const int threads = std::atoi(argv[8]);
    const int warmup = std::atoi(argv[9]);
    const int steps = std::atoi(argv[10]);
    const size_t nq_limit = std::strtoull(argv[11], nullptr, 10);
    const int nk = (argc - 12) / 2;
    char* env_args[6] = {argv[2], argv[3], argv[4], argv[5], argv[6], argv[12]};
    QueryEnv e;
    load_query_env(e, env_args);
    const size_t nq = std::min(e.nq, nq_limit ? nq_limit : e.nq);
    std::vector<std::vector<float>> thr(nk);
    std::vector<std::vector<uint32_t>> goff(nk), gids(nk);
    for (int k = 0; k < nk; k++) {
        thr[k].resize(e.n);
        FILE* f = std::fopen(argv[12 + 2 * k], "rb");
        if (!f || std::fread(thr[k].data(), 4, e.n, f) != e.n) die("bad threshold file");
        std::fclose(f);
        f = std::fopen(argv[13 + 2 * k], "rb");
        uint32_t gnq = 0;
        if (!f || std::fread(&gnq, 4, 1, f) != 1 || gnq != e.nq) die("bad GT header");
        goff[k].resize(gnq + 1);
        if (std::fread(goff[k].data(), 4, goff[k].size(), f) != goff[k].size()) die("short GT offsets");
        gids[k].resize(goff[k].back());
        if (std::fread(gids[k].data(), 4, gids[k].size(), f) != gids[k].size()) die("short GT ids");
        std::fclose(f);
    }
    Parms par = lifted_parms(e.n, e.dim, 50, 48, "/tmp/anqi_harness_work/");
    par.n_threads = threads;
    nndindex index(argv[2], par);
    load_graph_file(index, argv[3]);
    omp_set_num_threads(threads);
    std::vector<double> step_s;
    std::vector<double> rec(nk, 0), prec(nk, 0), cand(nk, 0), dist(nk, 0);
    std::vector<size_t> nonempty(nk, 0);
    for (int st = 0; st < warmup + steps; st++) {
        const bool timed = st >= warmup;
        auto t0 = std::chrono::steady_clock::now();
        for (int k = 0; k < nk; k++) {
            double s_rec = 0, s_prec = 0, s_cand = 0, s_nd = 0;
            size_t s_ne = 0;
            #pragma omp parallel reduction(+ : s_rec, s_prec, s_cand, s_nd, s_ne)
            {
                std::vector<uint16_t> mark(e.n, 0);
                uint16_t ver = 0;
                std::vector<float> qb(e.dim);
                #pragma omp for schedule(dynamic, 16)
                for (size_t i = 0; i < nq; i++) {
                    const float* q = e.queries.data() + i * e.d;
                    double R2 = 0;
                    lift_query(e, q, qb, R2);
                    if (++ver == 0) {
                        std::fill(mark.begin(), mark.end(), 0);
                        ver = 1;
                    }
                    std::vector<uint32_t> cd;
                    size_t nd = 0;
                    index.range_search(qb.data(), R2, 0.0f, L, cd, nd, mark.data(), ver, nullptr, 0.5f, false);
                    std::unordered_set<uint32_t> pred;
                    for (uint32_t id : cd)
                        if (recheck_key(e, id, q) <= (double)thr[k][id]) pred.insert(id);
                    nd += cd.size();
                    std::unordered_set<uint32_t> truth(gids[k].begin() + goff[k][i], gids[k].begin() + goff[k][i + 1]);
                    if (truth.empty()) continue;
                    s_ne++;
                    size_t hit = 0;
                    for (uint32_t id : pred) hit += truth.count(id);
                    s_rec += (double)hit / truth.size();
                    s_prec += pred.empty() ? 1.0 : (double)hit / pred.size();
                    s_cand += cd.size();
                    s_nd += nd;
                }
            }
            if (timed) {
                rec[k] += s_rec;
                prec[k] += s_prec;
                cand[k] += s_cand;
                dist[k] += s_nd;
                nonempty[k] += s_ne;
            }
        }
        const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (timed) step_s.push_back(secs);
    }
    double tot = 0;
    for (double x : step_s) tot += x;
    std::printf("{\"threads\": %d, \"L\": %zu, \"queries_per_step\": %zu, \"steps\": %d, \"seconds\": %.6f, "
                "\"qps\": %.3f, \"step_seconds\": [",
                threads, L, nq * (size_t)nk, steps, tot, steps ? (double)nq * nk * steps / tot : 0.0);
    for (size_t i = 0; i < step_s.size(); i++) std::printf("%s%.6f", i ? ", " : "", step_s[i]);
    std::printf("], \"per_k\": [");
    for (int k = 0; k < nk; k++) {
        const double dn = nonempty[k] ? (double)nonempty[k] : 1.0;
        std::printf("%s{\"recall\": %.6f, \"precision\": %.6f, \"avg_cand\": %.3f, \"avg_dist\": %.3f, "
                    "\"nonempty\": %zu}",
                    k ? ", " : "", rec[k] / dn, prec[k] / dn, cand[k] / dn, dist[k] / dn, nonempty[k]);
    }
    std::printf("]}\n");
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: ref_harness dist|verifier|analytic|graph|aknn|query|qbench|qparity ...\n");
        return 2;
    }
    const std::string cmd = argv[1];
    int rc = 2;
    if (cmd == "dist") rc = cmd_dist(argc, argv);
    else if (cmd == "verifier") rc = cmd_verifier(argc, argv);
    else if (cmd == "analytic") rc = cmd_analytic(argc, argv);
    else if (cmd == "ipdist") rc = cmd_ipdist(argc, argv);
    else if (cmd == "graph") rc = cmd_graph(argc, argv);
    else if (cmd == "aknn") rc = cmd_aknn(argc, argv);
    else if (cmd == "query") rc = cmd_query(argc, argv);
    else if (cmd == "qbench") rc = cmd_qbench(argc, argv);
    else if (cmd == "qparity") rc = cmd_qparity(argc, argv);
    if (rc == 2) std::fprintf(stderr, "[ref_harness] bad arguments for %s\n", cmd.c_str());
    return rc;
}
