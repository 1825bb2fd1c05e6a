// rknn_query: ANQI's shared-index reverse-kNN benchmark with the G48 graph
// build, the LRQ postfilter verifier and the query loop on the GPU.
//
//   rknn_query L_DESCENT_LIST PREFIX [GRAPH_DEGREE=48] [LEAF_SIZE=1000]
//              [TREE_COUNT=64] [BUILD_EF=400] [QUERY_K]
//
// Mirrors src/rknn_query.cpp:1547-2956 for the anyk_lift geometry with the
// postfilter placement -- the configuration scripts/run_final.sh pins -- under
// either metric (the prefix's meta file names l2 or ip) and every independent
// verifier (compact LRQ forms, rank-M only, float32 residuals, exact_f32,
// analytic rank-M): the same argv, environment, prefix files, caches (file
// names and identity keys, so a cache written by either program is found by
// the other), stdout result lines and exit codes.  The Vamana refine
// (ANQI_VAMANA, the global passes and the batched style) and the edge policies
// of the prune (ANQI_EDGE_POLICY and its options) run on the device too.
// Configurations outside that path (rank-M or original geometry, integrated
// verifier, fixed-k lift, recheck) exit 2 with a message naming the setting.
//
// Differences of mechanism, not of result: the graph build, lift, LRQ
// encode/materialize, search, postfilter and evaluation run on the device;
// one "batch" of the timed loop is one device pass over all queries (search,
// postfilter, result compaction, evaluation), queries resident on the device
// as they are resident in host memory in the reference loop.
#include "cli_common.h"
#include "graph_file.h"

#include <fcntl.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <iomanip>
#include <iostream>
#include <memory>
#include <sstream>

using namespace anqi_cli;
using Clock = std::chrono::steady_clock;

static double since(Clock::time_point t0) { return std::chrono::duration<double>(Clock::now() - t0).count(); }

// ------------------------------------------------------------ mode names
static bool is_learned_rq_mode(const std::string& m) {
    return m.rfind("rankm_resid_u2_lrq_", 0) == 0 || m.rfind("rankm_resid_u4_lrq_", 0) == 0 ||
           m.rfind("rankm_resid_u8_lrq_", 0) == 0 || m.rfind("rankm_resid_u16_lrq_", 0) == 0;
}

// ------------------------------------------------------------ prefix data
static Fbin load_fbin_or_die(const std::string& p) {
    Fbin f;
    std::string why;
    if (!read_fbin(p, f, why)) {
        if (why == "cannot open") die(3, "[rknn] cannot open fbin: %s", p.c_str());
        die(3, "[rknn] %s: %s", why.c_str(), p.c_str());
    }
    return f;
}

static std::string prebuilt_topk_path() { return env_or("ANQI_PREBUILT_TOPK_REC", ""); }

static uint64_t prebuilt_topk_width(uint64_t fallback) {
    const char* v = std::getenv("ANQI_PREBUILT_TOPK_K");
    if (!v || !*v) return fallback;
    uint64_t w = 0;
    if (!parse_positive(v, w) || w > 10000) die(2, "[rknn] invalid ANQI_PREBUILT_TOPK_K=%s", v);
    return w;
}

static void validate_prebuilt_topk(const std::string& path, uint64_t n, uint64_t source_k, uint64_t required_k) {
    if (source_k < required_k)
        die(3, "[rknn] prebuilt top-k width=%" PRIu64 " is smaller than required K=%" PRIu64, source_k, required_k);
    struct stat st {};
    const uint64_t expected = n * source_k * sizeof(TopKRecord);
    const bool ok = ::stat(path.c_str(), &st) == 0;
    if (!ok || (uint64_t)st.st_size != expected)
        die(3, "[rknn] bad prebuilt top-k table %s: bytes=%lld expected=%llu", path.c_str(),
            (long long)(ok ? st.st_size : -1), (unsigned long long)expected);
}

// The interleaved top-k records of ANQI_PREBUILT_TOPK_REC (n x source_k).
static std::vector<TopKRecord> read_prebuilt(const std::string& path, uint64_t n, uint64_t source_k) {
    std::vector<TopKRecord> rec(n * source_k);
    std::ifstream in(path, std::ios::binary);
    if (!in.read(reinterpret_cast<char*>(rec.data()), (std::streamsize)(rec.size() * sizeof(TopKRecord))))
        die(3, "[rknn] truncated prebuilt radius table at row=0");
    return rec;
}

// Keys n x NK (load_threshold_table, rknn_query.cpp:1101-1157): the prebuilt
// records' keys, else a PFX_baseknn_aknn.bin table [n][K][ids][keys].
static std::vector<float> load_threshold_table(const std::string& pfx, uint64_t n, uint64_t NK) {
    std::vector<float> out(n * NK);
    const std::string topk = prebuilt_topk_path();
    if (!topk.empty()) {
        const uint64_t sk = prebuilt_topk_width(NK);
        validate_prebuilt_topk(topk, n, sk, NK);
        const std::vector<TopKRecord> rec = read_prebuilt(topk, n, sk);
        for (uint64_t i = 0; i < n; i++)
            for (uint64_t k = 0; k < NK; k++) out[i * NK + k] = rec[i * sk + k].key;
        printf("[rknn] loaded AKNN cutoffs from interleaved top-k %s (n=%" PRIu64 " K=%" PRIu64 ")\n", topk.c_str(), n,
               NK);
        return out;
    }
    const std::string path = pfx + "_baseknn_aknn.bin";
    std::ifstream gf(path, std::ios::binary);
    if (!gf) die(3, "[rknn] missing threshold table %s", path.c_str());
    uint32_t gn = 0, gk = 0;
    gf.read(reinterpret_cast<char*>(&gn), 4);
    gf.read(reinterpret_cast<char*>(&gk), 4);
    if (gn != n || gk < NK)
        die(3, "[rknn] bad threshold table %s: n=%u K=%u expected n=%" PRIu64 " K>=%" PRIu64, path.c_str(), gn, gk, n,
            NK);
    gf.seekg((std::streamoff)gn * gk * 4, std::ios::cur);
    std::vector<float> row(gk);
    for (uint64_t i = 0; i < n; i++) {
        gf.read(reinterpret_cast<char*>(row.data()), (std::streamsize)gk * 4);
        std::copy(row.begin(), row.begin() + NK, out.begin() + i * NK);
    }
    if (!gf) die(3, "[rknn] truncated threshold table %s", path.c_str());
    printf("[rknn] loaded threshold table %s (n=%" PRIu64 " K=%" PRIu64 ")\n", path.c_str(), n, NK);
    return out;
}

static std::vector<float> load_threshold_column(const std::string& pfx, uint64_t n, uint64_t k1) {
    std::vector<float> out(n);
    const std::string topk = prebuilt_topk_path();
    if (!topk.empty()) {
        const uint64_t sk = prebuilt_topk_width(k1);
        validate_prebuilt_topk(topk, n, sk, k1);
        const std::vector<TopKRecord> rec = read_prebuilt(topk, n, sk);
        for (uint64_t i = 0; i < n; i++) out[i] = rec[i * sk + k1 - 1].key;
        printf("[rknn] loaded AKNN cutoff column from interleaved top-k %s (n=%" PRIu64 " k=%" PRIu64 ")\n",
               topk.c_str(), n, k1);
        return out;
    }
    const std::string path = pfx + "_baseknn_aknn.bin";
    std::ifstream gf(path, std::ios::binary);
    if (!gf) die(3, "[rknn] missing threshold table %s", path.c_str());
    uint32_t gn = 0, gk = 0;
    gf.read(reinterpret_cast<char*>(&gn), 4);
    gf.read(reinterpret_cast<char*>(&gk), 4);
    if (gn != n || k1 < 1 || k1 > gk)
        die(3, "[rknn] bad threshold column request %s: n=%u K=%u expected n=%" PRIu64 " k=%" PRIu64, path.c_str(), gn,
            gk, n, k1);
    gf.seekg((std::streamoff)gn * gk * 4, std::ios::cur);
    std::vector<float> row(gk);
    for (uint64_t i = 0; i < n; i++) {
        gf.read(reinterpret_cast<char*>(row.data()), (std::streamsize)gk * 4);
        out[i] = row[k1 - 1];
    }
    if (!gf) die(3, "[rknn] truncated threshold table %s", path.c_str());
    printf("[rknn] loaded threshold column %s (n=%" PRIu64 " k=%" PRIu64 ")\n", path.c_str(), n, k1);
    return out;
}

static std::string threshold_source_identity(const std::string& pfx) {
    const std::string topk = prebuilt_topk_path();
    return topk.empty() ? file_stat_identity(pfx + "_baseknn_aknn.bin")
                        : file_stat_identity(topk) + ":interleaved_k" + std::to_string(prebuilt_topk_width(100));
}

// ------------------------------------------------------------------ keys
// graph_cache_key (rknn_query.cpp:301-341) for the supported configuration.
static std::string graph_cache_key(uint64_t M, uint64_t leaf, uint64_t nt, uint64_t ef) {
    std::string k = "M" + std::to_string(M) + "_leaf" + std::to_string(leaf) + "_nt" + std::to_string(nt) + "_ef" +
                    std::to_string(ef) + "_geomanyk_lift_rankm0_specific0_alpha" + env_or("ANQI_ALPHA", "1.2") +
                    "_liftnnk" + env_or("ANQI_LIFTNNK", "50") + "_graphnnd" + env_or("ANQI_GRAPHNND", "6");
    // rknn_query.cpp:314-324
    if (std::getenv("ANQI_EDGE_POLICY")) {
        k += "_edge" + env_or("ANQI_EDGE_POLICY", "none") + "_eks" + env_or("ANQI_EDGE_KS", "10,50,100") + "_enk" +
             env_or("ANQI_EDGE_NK", "100") + "_erb" + env_or("ANQI_EDGE_RESID_BUDGET", "16") + "_erl" +
             env_or("ANQI_EDGE_RESID_LAMBDA", "1.0") + "_ebo" + env_or("ANQI_EDGE_BALL_OCCLUSION", "all");
        if (std::getenv("ANQI_EDGE_RESID_FILE"))
            k += "_erf" + hash16(file_fingerprint(env_or("ANQI_EDGE_RESID_FILE", "")));
    }
    if (std::getenv("ANQI_VAMANA")) {
        const std::string style = env_or("ANQI_VAMANA_STYLE", "global");
        k += "_vam1_style" + style + "_L" + env_or("ANQI_VAMANA_L", "128") + "_P" + env_or("ANQI_VAMANA_PASS", "2") +
             "_bf" + env_or("ANQI_VAMANA_BATCH_FRAC", "0.02") + "_mb" + env_or("ANQI_VAMANA_MAX_BATCH", "1000000") +
             "_bb" + env_or("ANQI_VAMANA_BATCH_BASE", "2") + "_ea" + env_or("ANQI_VAMANA_EARLY_ALPHA", "1.0") +
             "_eao" + env_or("ANQI_VAMANA_EARLY_ALPHA_ONE", "1") + "_entry" + env_or("ANQI_VAMANA_ENTRY", "0");
        if (style == "batch") k += "_implcsr1";
    } else {
        k += "_vam0";
    }
    return sanitize_tag(k);
}

// ANQI_EDGE_POLICY and its options, resolved for the device prune as
// configure_edge_residual_cover (include/index.h:305-440) configures the
// reference's: the same defaults, atoi / atof parsing, filters and exit-2
// errors.  folder: the graph's folder prefix (its lift meta and default
// residual table).  Resolved only when the graph is built, as there.
struct EdgePolicyHost {
    anqi_edge_policy p{};
    std::vector<float> resid, mu;
};

static std::vector<int> parse_int_list(const std::string& s) {
    std::vector<int> out;
    std::stringstream ss(s);
    std::string tok;
    while (std::getline(ss, tok, ',')) {
        if (tok.empty()) continue;
        const int v = std::atoi(tok.c_str());
        if (v > 0) out.push_back(v);
    }
    return out;
}

static bool read_table(const std::string& path, size_t floats, std::vector<float>& out, long long& got) {
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    got = -1;
    if (!f) return false;
    got = (long long)f.tellg();
    if (got != (long long)(floats * 4)) return true;
    f.seekg(0);
    out.resize(floats);
    f.read(reinterpret_cast<char*>(out.data()), (std::streamsize)(floats * 4));
    if (!f) got = -2;
    return true;
}

static void resolve_edge_policy(EdgePolicyHost& e, uint64_t n, uint32_t M, const std::string& folder) {
    const char* pol_c = std::getenv("ANQI_EDGE_POLICY");
    if (!pol_c || !*pol_c) return;
    const std::string pol = pol_c;
    anqi_edge_policy& p = e.p;
    auto envd = [](const char* k, double d) { const char* v = std::getenv(k); return v ? std::atof(v) : d; };
    auto envi = [](const char* k, int d) { const char* v = std::getenv(k); return v ? std::atoi(v) : d; };
    if (pol == "lsg_rng" || pol == "lsg_bubble_hybrid") {
        p.lsg_alpha = envd("ANQI_LSG_ALPHA", 1.0);
        if (!std::isfinite(p.lsg_alpha) || p.lsg_alpha < 0.0)
            die(2, "[edge-policy] invalid ANQI_LSG_ALPHA=%.17g", p.lsg_alpha);
        const char* mp = std::getenv("ANQI_LSG_MU_FILE");
        const std::string mu_path = mp ? mp : "";
        if (mu_path.empty()) die(2, "[edge-policy] lsg_rng requires ANQI_LSG_MU_FILE");
        long long got = 0;
        if (!read_table(mu_path, n, e.mu, got)) die(2, "[edge-policy] lsg_rng cannot open mu table %s", mu_path.c_str());
        if (got != (long long)(n * 4))
            die(2, "[edge-policy] lsg mu size mismatch %s: expected %zu bytes, got %lld", mu_path.c_str(),
                (size_t)(n * 4), got);
        for (uint64_t i = 0; i < n; i++)
            if (!std::isfinite((double)e.mu[i]) || e.mu[i] <= 0.0f)
                die(2, "[edge-policy] invalid lsg mu[%zu]=%.9g", (size_t)i, (double)e.mu[i]);
        p.flags |= ANQI_EDGE_LSG;
        fprintf(stderr, "[edge-policy] %s lsg enabled alpha=%.6g mu=%s\n", pol.c_str(), p.lsg_alpha, mu_path.c_str());
        if (pol == "lsg_rng") return;
    }
    static const char* kResidual[] = {"residual_cover", "ball_rng", "ball_hybrid", "ball_multik", "bubble_rng",
                                      "bubble_hybrid", "bubble_multik", "bubble_auto", "bubble_auto_full",
                                      "lsg_bubble_hybrid"};
    bool needs = false;
    for (const char* r : kResidual) needs = needs || pol == r;
    if (!needs) return;
    int nk = envi("ANQI_EDGE_NK", 100);
    if (nk == 0) nk = 100;
    if (nk < 0) die(2, "[edge-policy] invalid ANQI_EDGE_NK=%d", nk);
    p.nk = (uint32_t)nk;
    p.budget = (uint32_t)std::min<long long>(std::max(0, envi("ANQI_EDGE_RESID_BUDGET", 16)), M);
    p.auto_candidates = (uint32_t)std::max(1, envi("ANQI_EDGE_AUTO_CANDIDATES", (int)M));
    p.auto_max_swaps = (uint32_t)std::max(1, envi("ANQI_EDGE_AUTO_MAX_SWAPS", (int)M));
    p.lambda = envd("ANQI_EDGE_RESID_LAMBDA", 1.0);
    p.scale2 = 1.0;
    const char* ks_c = std::getenv("ANQI_EDGE_KS");
    std::vector<int> ks;
    for (int k : parse_int_list(ks_c ? ks_c : "10,50,100"))
        if (k >= 1 && k <= nk) ks.push_back(k);
    if (ks.empty()) return;
    if (ks.size() > 8) die(2, "[edge-policy] at most 8 values in ANQI_EDGE_KS are supported here");
    p.nks = (uint32_t)ks.size();
    for (size_t t = 0; t < ks.size(); t++) p.ks[t] = (uint32_t)ks[t];
    const bool autop = pol == "bubble_auto" || pol == "bubble_auto_full";
    if (p.budget == 0 && pol != "ball_rng" && !autop) return;
    {
        std::ifstream mf(folder + "_anqi_meta.txt");
        double mstar = 0.0, sc = 1.0;
        if (mf >> mstar >> sc) p.scale2 = sc * sc;
    }
    const char* rf = std::getenv("ANQI_EDGE_RESID_FILE");
    const std::string resid_path = rf ? rf : folder + "_anqi_rankm_residual.bin";
    long long got = 0;
    if (!read_table(resid_path, n * (size_t)nk, e.resid, got))
        die(2, "[edge-policy] residual_cover requested but missing %s", resid_path.c_str());
    if (got == -2) die(2, "[edge-policy] bad residual table %s", resid_path.c_str());
    if (got != (long long)(n * (size_t)nk * 4))
        die(2, "[edge-policy] residual table stride/size mismatch %s: expected %zu bytes (n=%zu edge_nk=%d), got %lld "
               "bytes; set ANQI_EDGE_NK to the table stride",
            resid_path.c_str(), (size_t)(n * (size_t)nk * 4), (size_t)n, nk, got);
    if (pol == "residual_cover") {
        p.flags |= ANQI_EDGE_COVER;
    } else {
        p.flags |= ANQI_EDGE_BALL;
        if (pol == "ball_rng" || pol == "bubble_rng") p.flags |= ANQI_EDGE_PURE;
        const char* oc = std::getenv("ANQI_EDGE_BALL_OCCLUSION");
        p.occlude_all = std::string(oc ? oc : "all") != "any";
    }
    if (autop) p.flags |= ANQI_EDGE_AUTO | (pol == "bubble_auto_full" ? ANQI_EDGE_AUTO_FULL : 0u);
    p.resid = e.resid.data();
    p.mu = e.mu.empty() ? nullptr : e.mu.data();
    fprintf(stderr, "[edge-policy] %s enabled budget=%u lambda=%.4g scale2=%.6g nk=%d\n", pol.c_str(), p.budget,
            p.lambda, p.scale2, nk);
}

// nndindex::generate_config (include/index.h:1703-1769) with ANQI_GRAPH_CACHE_KEY set;
// ef_alpha and prune_alpha are floats there, printed by std::to_string.
static std::string graph_file_name(uint64_t M, uint64_t nn_k, uint64_t n, uint64_t dim, float alpha,
                                   const std::string& graph_key) {
    std::string cfg = "fd_metric_l2_M_" + std::to_string(M) + "_nnk_" + std::to_string(nn_k) + "_ntrees_64_n_" +
                      std::to_string(n) + "_dim_" + std::to_string(dim) + "_efa_" + std::to_string(8.0f) + "_pa_" + std::to_string(alpha) +
                      "_er_100_graphnnd_" + env_or("ANQI_GRAPHNND", "6") + "_gk_" + hash16(graph_key);
    // the edge policy's part of the name (index.h:1741-1764)
    if (std::getenv("ANQI_EDGE_POLICY")) {
        const std::string pol = env_or("ANQI_EDGE_POLICY", "none");
        cfg += "_edge_" + pol;
        if (pol == "lsg_rng" || pol == "lsg_bubble_hybrid") {
            std::string mu_key = env_or("ANQI_LSG_CACHE_KEY", "");
            if (mu_key.empty()) mu_key = env_or("ANQI_LSG_MU_FILE", "");
            cfg += "_lsa_" + env_or("ANQI_LSG_ALPHA", "1.0") + "_lsgmu_" + hash16(mu_key);
        }
        if (pol != "lsg_rng") {
            cfg += "_eks_" + env_or("ANQI_EDGE_KS", "10,50,100") + "_enk_" + env_or("ANQI_EDGE_NK", "100") + "_erb_" +
                   env_or("ANQI_EDGE_RESID_BUDGET", "16") + "_erl_" + env_or("ANQI_EDGE_RESID_LAMBDA", "1.0") + "_ebo_" +
                   env_or("ANQI_EDGE_BALL_OCCLUSION", "all");
            if (pol == "bubble_auto" || pol == "bubble_auto_full")
                cfg += "_eac_" + env_or("ANQI_EDGE_AUTO_CANDIDATES", "M") + "_eas_" +
                       env_or("ANQI_EDGE_AUTO_MAX_SWAPS", "M");
        }
    }
    return sanitize_tag(cfg);
}

// ANQI_BASE_U8BIN (rknn_query.cpp:55-123): a uint8 base, [u32 n][u32 d][n*d
// u8], read in place of PREFIX_base.bin and widened to float (exact), so every
// later stage sees the same values; the caches name the uint8 file.
static std::string base_vector_source(const std::string& fbin_path) {
    const char* u8 = std::getenv("ANQI_BASE_U8BIN");
    return (u8 && *u8) ? std::string(u8) : fbin_path;
}

static Fbin load_base_or_die(const std::string& fbin_path) {
    const char* u8 = std::getenv("ANQI_BASE_U8BIN");
    if (!(u8 && *u8)) return load_fbin_or_die(fbin_path);
    const std::string path = u8;
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    if (!f) die(3, "[rknn] cannot open uint8 base %s: %s", path.c_str(), std::strerror(errno));
    const std::streamoff bytes = f.tellg();
    f.seekg(0);
    uint32_t shape[2] = {0, 0};
    if (bytes < 8 || !f.read(reinterpret_cast<char*>(shape), 8))
        die(3, "[rknn] cannot read uint8 base header %s", path.c_str());
    const uint64_t values = (uint64_t)shape[0] * shape[1];
    if (shape[0] == 0 || shape[1] == 0 || (uint64_t)bytes != 8 + values)
        die(3, "[rknn] bad uint8 base %s: n=%u d=%u bytes=%lld expected=%llu", path.c_str(), shape[0], shape[1],
            (long long)bytes, (unsigned long long)(8 + values));
    std::vector<uint8_t> raw(values);
    if (!f.read(reinterpret_cast<char*>(raw.data()), (std::streamsize)values))
        die(3, "[rknn] cannot read uint8 base header %s", path.c_str());
    Fbin out;
    out.n = shape[0];
    out.d = shape[1];
    out.x.resize(values);
    for (uint64_t i = 0; i < values; i++) out.x[i] = (float)raw[i];
    printf("[rknn] loaded uint8 base directly as float: %s n=%u d=%u %.3fGB\n", path.c_str(), out.n, out.d,
           values * 4.0 / 1e9);
    return out;
}

// ANQI_COMPACT_PREBUILT_TOPK_IDS_INPLACE (rknn_query.cpp:988-1057): the
// prebuilt {id, key} table becomes an n x width id table in place, in 64 MB
// chunks, then is truncated; an id >= n exits 3.
static void compact_topk_ids_in_place(const std::string& path, uint64_t n, uint64_t source_k, uint64_t width) {
    validate_prebuilt_topk(path, n, source_k, width);
    const int fd = ::open(path.c_str(), O_RDWR);
    if (fd < 0) die(3, "[rknn] cannot open prebuilt top-k for compaction %s: %s", path.c_str(), std::strerror(errno));
    const uint64_t rows_per_chunk = std::max<uint64_t>(1, (64ull << 20) / (source_k * sizeof(TopKRecord)));
    std::vector<TopKRecord> rec(rows_per_chunk * source_k);
    std::vector<uint32_t> ids(rows_per_chunk * width);
    auto io = [&](bool write, void* buf, uint64_t bytes, uint64_t off) {
        uint8_t* p = static_cast<uint8_t*>(buf);
        while (bytes) {
            const ssize_t got = write ? ::pwrite(fd, p, bytes, (off_t)off) : ::pread(fd, p, bytes, (off_t)off);
            if (got < 0 && errno == EINTR) continue;
            if (got <= 0)
                die(3, write ? "[rknn] cannot write compact warm-start IDs %s offset=%llu: %s"
                             : "[rknn] cannot read prebuilt top-k during compaction %s offset=%llu: %s",
                    path.c_str(), (unsigned long long)off, got == 0 ? "unexpected EOF" : std::strerror(errno));
            p += got;
            bytes -= (uint64_t)got;
            off += (uint64_t)got;
        }
    };
    const uint64_t step = std::max<uint64_t>(1, n / 20);
    uint64_t next = step;
    for (uint64_t r0 = 0; r0 < n; r0 += rows_per_chunk) {
        const uint64_t rows = std::min(rows_per_chunk, n - r0);
        io(false, rec.data(), rows * source_k * sizeof(TopKRecord), r0 * source_k * sizeof(TopKRecord));
        for (uint64_t r = 0; r < rows; r++)
            for (uint64_t k = 0; k < width; k++) {
                const uint32_t id = rec[r * source_k + k].id;
                if (id >= n)
                    die(3, "[rknn] invalid warm-start id at row=%llu k=%u", (unsigned long long)(r0 + r), (unsigned)k);
                ids[r * width + k] = id;
            }
        // the rows written never pass the rows read: the ids table is smaller
        io(true, ids.data(), rows * width * 4, r0 * width * 4);
        if (r0 + rows >= next || r0 + rows == n) {
            printf("[rknn] compact warm-start IDs: %.1f%%\n", 100.0 * (double)(r0 + rows) / (double)n);
            next = r0 + rows + step;
        }
    }
    if (::ftruncate(fd, (off_t)(n * width * 4)) != 0 || ::fsync(fd) != 0 || ::close(fd) != 0)
        die(3, "[rknn] cannot finalize compact warm-start IDs %s: %s", path.c_str(), std::strerror(errno));
    printf("[rknn] compacted regenerable prebuilt top-k to IDs in place: %s source_k=%" PRIu64 " width=%" PRIu64
           " bytes=%.3fGB\n",
           path.c_str(), source_k, width, n * width * 4 / 1e9);
}

// The streamed warm start (include/index.h:1127-1203): n rows of `stride`
// records ({u32 id, f32 key}, or u32 ids when ids_only) read in 64 MB chunks
// from a command's stdout or a file, each chunk handed to the device build;
// the stream must hold exactly n rows.
static void stream_warm_rows(anqi_ctx* ctx, FILE* in, bool is_command, uint64_t n, uint64_t stride, uint64_t width,
                             bool ids_only) {
    const uint64_t rec_bytes = ids_only ? 4 : sizeof(TopKRecord);
    const uint64_t rows_per_chunk = std::max<uint64_t>(1, (64ull << 20) / (stride * rec_bytes));
    std::vector<uint8_t> buf(rows_per_chunk * stride * rec_bytes);
    std::vector<uint32_t> ids(rows_per_chunk * width);
    bool ok = true;
    for (uint64_t r0 = 0; r0 < n && ok; r0 += rows_per_chunk) {
        const uint64_t rows = std::min(rows_per_chunk, n - r0);
        if (std::fread(buf.data(), rec_bytes, rows * stride, in) != rows * stride) {
            ok = false;
            break;
        }
        for (uint64_t r = 0; r < rows; r++)
            for (uint64_t k = 0; k < width; k++) {
                uint32_t id;
                std::memcpy(&id, buf.data() + (r * stride + k) * rec_bytes, 4);
                ids[r * width + k] = id;
            }
        const int rc = anqi_graph_build_warm_rows(ctx, r0, rows, ids.data(), (uint32_t)width);
        if (rc) die(rc, "[rknn] graph warm start failed: %s", anqi_last_error(ctx));
    }
    if (ok && std::fgetc(in) != EOF) ok = false;
    const int status = is_command ? ::pclose(in) : std::fclose(in);
    if (!ok || status != 0) die(3, "[rknn] streamed warm-start ended early, produced extra data, or failed");
}

// ------------------------------------------------------------- verifier
// CompactLrqVerifier state (rknn_query.cpp:604-753): bits 0 (rank-M only),
// 2 / 4 / 8 / 16 (packed codes, learned codebook), 32 (float residuals).
struct Lrq {
    uint64_t n = 0;
    uint32_t nk = 0, rankm = 0, bits = 0, code_size = 0;
    std::string policy = "floor";
    std::vector<float> mu, basis, codebook, coeff, residual;
    std::vector<uint8_t> codes;  // packed, object-major
    uint32_t policy_code() const { return policy == "floor" ? 1u : (policy == "ceil" ? 2u : 0u); }
    uint64_t code_bytes() const {
        return (bits == 2 || bits == 4 || bits == 8 || bits == 16) ? (n * nk * bits + 7) / 8 : 0;
    }
    uint64_t persistent_bytes() const {
        return coeff.size() * 4 + codes.size() + residual.size() * 4 + mu.size() * 4 + basis.size() * 4 +
               codebook.size() * 4 + 36 + 8 + (bits ? 24 : 0);
    }
};

static void load_basis(const std::string& rb, uint64_t NK, int RANKM, Lrq& v) {
    std::ifstream bf(rb, std::ios::binary | std::ios::ate);
    const std::streamoff bytes = bf ? (std::streamoff)bf.tellg() : (std::streamoff)-1;
    bf.seekg(0);
    int32_t Kb = 0, Mb = 0;
    if (!bf || !bf.read(reinterpret_cast<char*>(&Kb), 4) || !bf.read(reinterpret_cast<char*>(&Mb), 4) || Kb <= 0 ||
        Mb <= 0 || (uint64_t)Kb != NK || Mb != RANKM)
        die(3, "[rknn] missing or invalid rank-M basis %s (K=%d M=%d, expected K=%" PRIu64 " M=%d)", rb.c_str(), Kb, Mb,
            NK, RANKM);
    if ((uint64_t)bytes != 8 + (uint64_t)Kb * 4 + (uint64_t)Mb * Kb * 4)
        die(3, "[rknn] invalid rank-M basis size: %s", rb.c_str());
    v.mu.resize(Kb);
    v.basis.resize((size_t)Mb * Kb);
    if (!bf.read(reinterpret_cast<char*>(v.mu.data()), (std::streamsize)Kb * 4) ||
        !bf.read(reinterpret_cast<char*>(v.basis.data()), (std::streamsize)Mb * Kb * 4))
        die(3, "[rknn] truncated rank-M basis: %s", rb.c_str());
}

static void load_codebook(const std::string& path, uint64_t NK, int RANKM, int bits, Lrq& v) {
    std::ifstream f(path, std::ios::binary);
    if (!f) die(3, "[rknn] missing learned RQ codebook %s", path.c_str());
    char magic[8];
    f.read(magic, 8);
    if (f.gcount() != 8 || std::memcmp(magic, "ANQIRQ1\0", 8) != 0)
        die(3, "[rknn] bad learned RQ codebook magic %s", path.c_str());
    int32_t nk = 0, rankm = 0, b = 0, cs = 0;
    f.read(reinterpret_cast<char*>(&nk), 4);
    f.read(reinterpret_cast<char*>(&rankm), 4);
    f.read(reinterpret_cast<char*>(&b), 4);
    f.read(reinterpret_cast<char*>(&cs), 4);
    if (!f || nk != (int)NK || rankm != RANKM || b != bits || cs <= 0)
        die(3,
            "[rknn] bad learned RQ codebook header %s: nk=%d rankm=%d bits=%d code_size=%d expected nk=%" PRIu64
            " rankm=%d bits=%d",
            path.c_str(), nk, rankm, b, cs, NK, RANKM, bits);
    v.code_size = (uint32_t)cs;
    v.codebook.resize((size_t)nk * cs);
    f.read(reinterpret_cast<char*>(v.codebook.data()), (std::streamsize)v.codebook.size() * 4);
    if (f.gcount() != (std::streamsize)v.codebook.size() * 4) die(3, "[rknn] truncated learned RQ codebook %s", path.c_str());
    char extra;
    if (f.read(&extra, 1)) die(3, "[rknn] oversized learned RQ codebook %s", path.c_str());
    for (int k = 0; k < nk; k++)
        for (int j = 1; j < cs; j++)
            if (v.codebook[(size_t)k * cs + j] < v.codebook[(size_t)k * cs + j - 1])
                die(3, "[rknn] LRQ codebook row %d is not sorted: %s", k, path.c_str());
}

// ANQIVF2 artifact, CompactLrqVerifier::save/load (rknn_query.cpp:755-838).
static void save_verifier(const std::string& path, const Lrq& v) {
    const std::string tmp = path + ".tmp";
    std::ofstream f(tmp, std::ios::binary | std::ios::trunc);
    if (!f) die(3, "[rknn] cannot write LRQ verifier artifact %s", tmp.c_str());
    const uint32_t hdr[5] = {v.nk, v.rankm, v.bits, v.code_size, v.policy_code()};
    f.write("ANQIVF2\0", 8);
    f.write(reinterpret_cast<const char*>(&v.n), 8);
    f.write(reinterpret_cast<const char*>(hdr), sizeof(hdr));
    f.write(reinterpret_cast<const char*>(v.coeff.data()), (std::streamsize)v.coeff.size() * 4);
    f.write(reinterpret_cast<const char*>(v.codes.data()), (std::streamsize)v.codes.size());
    f.write(reinterpret_cast<const char*>(v.residual.data()), (std::streamsize)v.residual.size() * 4);
    if (!f) die(3, "[rknn] failed while writing LRQ verifier artifact %s", tmp.c_str());
    f.close();
    if (!f || std::rename(tmp.c_str(), path.c_str()) != 0) die(3, "[rknn] cannot publish LRQ verifier artifact %s", path.c_str());
}

static void load_verifier(const std::string& path, Lrq& v) {
    std::ifstream f(path, std::ios::binary);
    if (!f) die(3, "[rknn] missing LRQ verifier artifact %s", path.c_str());
    char magic[8] = {};
    uint64_t n64 = 0;
    uint32_t hdr[5] = {0, 0, 0, 0, 0};
    f.read(magic, 8);
    f.read(reinterpret_cast<char*>(&n64), 8);
    f.read(reinterpret_cast<char*>(hdr), sizeof(hdr));
    if (!f || std::memcmp(magic, "ANQIVF2\0", 8) != 0 || n64 != v.n || hdr[0] != v.nk || hdr[1] != v.rankm ||
        hdr[2] != v.bits || hdr[3] != v.code_size || hdr[4] != v.policy_code())
        die(3, "[rknn] LRQ verifier artifact header mismatch %s", path.c_str());
    v.coeff.resize(v.n * v.rankm);
    v.codes.resize(v.code_bytes());
    v.residual.resize(v.bits == 32 ? v.n * v.nk : 0);
    f.read(reinterpret_cast<char*>(v.coeff.data()), (std::streamsize)v.coeff.size() * 4);
    if (f.gcount() != (std::streamsize)v.coeff.size() * 4) die(3, "[rknn] truncated LRQ verifier coefficients %s", path.c_str());
    f.read(reinterpret_cast<char*>(v.codes.data()), (std::streamsize)v.codes.size());
    if (f.gcount() != (std::streamsize)v.codes.size()) die(3, "[rknn] truncated LRQ verifier codes %s", path.c_str());
    f.read(reinterpret_cast<char*>(v.residual.data()), (std::streamsize)v.residual.size() * 4);
    if (f.gcount() != (std::streamsize)v.residual.size() * 4)
        die(3, "[rknn] truncated float32 residuals %s", path.c_str());
    char extra;
    if (f.read(&extra, 1)) die(3, "[rknn] oversized LRQ verifier artifact %s", path.c_str());
}

// ANQIPW1 analytic Rank-M model, AnalyticRankMVerifier::load (rknn_query.cpp:528-573).
struct AnalyticModel {
    uint32_t train_kmax = 0, fit_kmin = 0, flags = 0;
    double b0 = 0;
    std::vector<float> coeff;
};

static AnalyticModel read_analytic_model(const std::string& path, uint64_t n, int rankm) {
    std::ifstream f(path, std::ios::binary);
    if (!f) die(3, "[rknn] missing analytic Rank-M model %s", path.c_str());
    char magic[8] = {};
    uint64_t n64 = 0;
    uint32_t h[4] = {0, 0, 0, 0};
    AnalyticModel m;
    f.read(magic, 8);
    f.read(reinterpret_cast<char*>(&n64), 8);
    f.read(reinterpret_cast<char*>(h), sizeof(h));
    f.read(reinterpret_cast<char*>(&m.b0), 8);
    m.train_kmax = h[0];
    m.fit_kmin = h[2];
    m.flags = h[3];
    if (!f || std::memcmp(magic, "ANQIPW1\0", 8) != 0 || n64 != n || h[1] != (uint32_t)rankm || h[0] < 1 ||
        h[2] < 1 || h[2] > h[0] || (h[3] != 3u && h[3] != 7u) || !std::isfinite(m.b0))
        die(3,
            "[rknn] analytic Rank-M header mismatch %s: n=%llu train_kmax=%u rankm=%u fit_kmin=%u flags=%u b0=%.9g "
            "expected n=%" PRIu64 " rankm=%d",
            path.c_str(), (unsigned long long)n64, h[0], h[1], h[2], h[3], m.b0, n, rankm);
    m.coeff.resize(n * (uint64_t)rankm);
    f.read(reinterpret_cast<char*>(m.coeff.data()), (std::streamsize)m.coeff.size() * 4);
    if (f.gcount() != (std::streamsize)m.coeff.size() * 4)
        die(3, "[rknn] truncated analytic Rank-M coefficients %s", path.c_str());
    char extra;
    if (f.read(&extra, 1)) die(3, "[rknn] oversized analytic Rank-M model %s", path.c_str());
    return m;
}

// ------------------------------------------------------------------ main
struct PointStats {
    double recall = 0, prec = 0, f1 = 0, cand_recall = 0, cand = 0, pred = 0, graph_dist = 0;
    uint64_t nonempty = 0, tasks = 0, batches = 0;
    double secs = 0;
    void add(const PointStats& o) {
        recall += o.recall;
        prec += o.prec;
        f1 += o.f1;
        cand_recall += o.cand_recall;
        cand += o.cand;
        pred += o.pred;
        graph_dist += o.graph_dist;
        nonempty += o.nonempty;
        tasks += o.tasks;
        batches += o.batches;
        secs += o.secs;
    }
};

static int run(int argc, char** argv) {
    if (argc < 3 || argc > 8) {
        fprintf(stderr,
                "usage: %s L_DESCENT_LIST PREFIX [GRAPH_DEGREE] [LEAF_SIZE] "
                "[TREE_COUNT] [BUILD_EF] [QUERY_K]\n",
                argv[0]);
        return 2;
    }
    auto size_arg = [](const char* text, const char* name) {
        uint64_t v = 0;
        if (!text || !*text) die(2, "[rknn] invalid %s (expected a positive integer)", name);
        if (!parse_positive(text, v)) die(2, "[rknn] invalid %s=%s (expected a positive integer)", name, text);
        return v;
    };
    std::vector<uint64_t> Lds;
    {
        const std::string list(argv[1]);
        size_t start = 0;
        while (start <= list.size()) {
            const size_t comma = list.find(',', start);
            const std::string item = list.substr(start, comma == std::string::npos ? std::string::npos : comma - start);
            Lds.push_back(size_arg(item.c_str(), "L_DESCENT"));
            if (comma == std::string::npos) break;
            start = comma + 1;
        }
    }
    const uint64_t Marg = argc > 3 ? size_arg(argv[3], "GRAPH_DEGREE") : 48;
    const uint64_t leafA = argc > 4 ? size_arg(argv[4], "LEAF_SIZE") : 1000;
    const uint64_t ntA = argc > 5 ? size_arg(argv[5], "TREE_COUNT") : 64;
    const uint64_t efA = argc > 6 ? size_arg(argv[6], "BUILD_EF") : 400;
    const std::string PFX(argv[2]);
    const std::string meta_p = PFX + "_lifted.meta";
    std::string gt_p = PFX + "_rknn_gt.bin";

    // Metadata: Mstar^2, dimension, rank horizon, metric, scale (rknn_query.cpp:1603-1619).
    double Mstar2 = 0, scale = 0;
    uint64_t d0 = 0, kk = 0;
    std::string metric;
    {
        std::ifstream mf(meta_p);
        if (!(mf >> Mstar2 >> d0 >> kk >> metric >> scale) || !std::isfinite(Mstar2) || Mstar2 < 0 || d0 == 0 ||
            kk == 0 || (metric != "l2" && metric != "ip") || !std::isfinite(scale) || scale <= 0)
            die(3, "[rknn] invalid or missing lift metadata: %s", meta_p.c_str());
    }
    printf("[rknn] metric=%s M*^2=%.6g d=%" PRIu64 " k=%" PRIu64 " L_descent_points=%zu\n", metric.c_str(), Mstar2, d0,
           kk, Lds.size());
    auto env_rank = [](const char* name, uint64_t dflt) {
        const char* v = std::getenv(name);
        if (!v) return dflt;
        uint64_t x = 0;
        if (!parse_positive(v, x) || x > 10000) die(2, "[rknn] invalid %s=%s (expected integer in [1,10000])", name, v);
        return x;
    };
    const uint64_t NK = env_rank("ANQI_NK", 100);
    const uint64_t GRAPH_NK = env_rank("ANQI_GRAPH_NK", NK);
    const uint64_t Kq = argc > 7 ? size_arg(argv[7], "QUERY_K") : kk;
    if (Kq < 1 || Kq > NK)
        die(2, "[rknn] requested Kq=%" PRIu64 " is outside the represented rank range [1,%" PRIu64 "]", Kq, NK);
    {
        const std::string gp = PFX + "_rknn_gt_k" + std::to_string(Kq) + ".bin";
        if (file_exists(gp)) gt_p = gp;
        else if (Kq != kk)
            die(3,
                "[rknn] missing k-specific reverse-kNN GT %s; the generic GT is only valid for metadata k=%" PRIu64,
                gp.c_str(), kk);
        else if (!file_exists(gt_p))
            die(3, "[rknn] missing reverse-kNN GT %s", gt_p.c_str());
    }
    printf("[rknn] shared-index query: Kq=%" PRIu64 " NK=%" PRIu64 " graph_NK=%" PRIu64 " GT=%s\n", Kq, NK, GRAPH_NK,
           gt_p.c_str());

    Fbin base = load_base_or_die(PFX + "_base.bin");
    Fbin query = load_fbin_or_die(PFX + "_query.bin");
    const uint64_t n = base.n, d = base.d, nq = query.n;
    if (d != d0 || query.d != d0)
        die(3, "[rknn] vector dimension does not match lift metadata: base=%" PRIu64 " query=%u metadata=%" PRIu64, d,
            query.d, d0);

    // Reverse-kNN ground truth, CSR + one key per id (rknn_query.cpp:1676-1718).
    std::vector<uint32_t> goff, gids;
    {
        std::ifstream gf(gt_p, std::ios::binary | std::ios::ate);
        const std::streamoff gt_bytes = gf ? (std::streamoff)gf.tellg() : (std::streamoff)-1;
        gf.seekg(0);
        uint32_t gnq = 0;
        if (!gf || !gf.read(reinterpret_cast<char*>(&gnq), 4) || gnq != nq)
            die(3, "[rknn] invalid reverse-kNN GT header: %s", gt_p.c_str());
        goff.resize((size_t)gnq + 1);
        if (!gf.read(reinterpret_cast<char*>(goff.data()), (std::streamsize)goff.size() * 4) || goff.front() != 0 ||
            !std::is_sorted(goff.begin(), goff.end()))
            die(3, "[rknn] invalid reverse-kNN GT offsets: %s", gt_p.c_str());
        const uint64_t expected = 4 + goff.size() * 4 + (uint64_t)goff.back() * 8;
        if (gt_bytes < 0 || (uint64_t)gt_bytes != expected) die(3, "[rknn] invalid reverse-kNN GT size: %s", gt_p.c_str());
        gids.resize(goff.back());
        if (!gf.read(reinterpret_cast<char*>(gids.data()), (std::streamsize)gids.size() * 4) ||
            std::any_of(gids.begin(), gids.end(), [n](uint32_t id) { return id >= n; }))
            die(3, "[rknn] invalid reverse-kNN GT ids: %s", gt_p.c_str());
    }

    const std::string DSDIR = PFX.substr(0, PFX.rfind('/') + 1);
    auto cache_dir = [&](const char* key) {
        std::string p = env_or(key, DSDIR.c_str());
        if (p.empty() || p.back() != '/') p.push_back('/');
        return p;
    };
    const std::string graph_cache_dir = cache_dir("ANQI_GRAPH_CACHE_DIR");
    const std::string verifier_cache_dir = cache_dir("ANQI_VERIFIER_CACHE_DIR");
    const auto tb0 = Clock::now();

    // ---- configuration: the pinned shared-index path only
    const std::string radius_mode = env_or("ANQI_RADIUS_MODE", "approx");
    int RANKM = 0;
    if (const char* r = std::getenv("ANQI_RANKM")) {
        char* end = nullptr;
        errno = 0;
        const long v = std::strtol(r, &end, 10);
        if (!*r || errno == ERANGE || end == r || *end != '\0' || v < 0 || v > 1024)
            die(2, "[rknn] invalid ANQI_RANKM=%s (expected integer in [0,1024])", r);
        RANKM = (int)v;
    }
    std::string geometry = env_or("ANQI_GRAPH_GEOMETRY", RANKM > 0 ? "rankm" : "anyk_lift");
    if (geometry == "anyk" || geometry == "lift") geometry = "anyk_lift";
    if (geometry == "raw" || geometry == "no_lift" || geometry == "nolift") geometry = "original";
    if (geometry != "anyk_lift" && geometry != "rankm" && geometry != "original")
        die(2, "[rknn] unsupported ANQI_GRAPH_GEOMETRY=%s (expected anyk_lift, original, or rankm)", geometry.c_str());
    auto not_here = [](const std::string& what) {
        die(2, "[rknn] %s is not implemented on the GPU path (supported: the scripts/run_final.sh configuration)",
            what.c_str());
    };
    const bool is_ip = metric == "ip";
    if (geometry != "anyk_lift") not_here("ANQI_GRAPH_GEOMETRY=" + geometry);
    // the independent postfilter verifiers (rknn_query.cpp:1771-1792): learned
    // LRQ (u2 / u4 / u8 / u16, floor / ceil / nearest), float32 residuals,
    // rank-M only, exact source thresholds, analytic rank-M
    enum class VMode { Compact, Exact, Analytic };
    VMode vmode = VMode::Compact;
    int bits = 0;
    std::string lrq_policy = "floor";
    std::string vmode_label;
    if (is_learned_rq_mode(radius_mode)) {
        bits = radius_mode.rfind("rankm_resid_u2_", 0) == 0 ? 2
               : radius_mode.rfind("rankm_resid_u4_", 0) == 0 ? 4
               : radius_mode.rfind("rankm_resid_u8_", 0) == 0 ? 8 : 16;
        const bool fl = radius_mode.size() >= 6 && radius_mode.compare(radius_mode.size() - 6, 6, "_floor") == 0;
        const bool ce = radius_mode.size() >= 5 && radius_mode.compare(radius_mode.size() - 5, 5, "_ceil") == 0;
        lrq_policy = fl ? "floor" : (ce ? "ceil" : "nearest");
        vmode_label = "rank-M+LRQ";
    } else if (radius_mode == "rankm_resid_f32") {
        bits = 32;
        vmode_label = "rank-M+float32-residual";
    } else if (radius_mode == "rankm_only") {
        bits = 0;
        vmode_label = "rank-M-only";
    } else if (radius_mode == "exact_f32") {
        vmode = VMode::Exact;
        vmode_label = "exact_f32";
    } else if (radius_mode == "analytic_rankm") {
        vmode = VMode::Analytic;
        vmode_label = "analytic-rank-M";
    } else {
        not_here("ANQI_RADIUS_MODE=" + radius_mode);
    }
    const std::string placement = env_or("ANQI_VERIFIER_PLACEMENT", "postfilter");
    if (placement != "integrated" && placement != "postfilter")
        die(2, "[rknn] unsupported ANQI_VERIFIER_PLACEMENT=%s (expected integrated or postfilter)", placement.c_str());
    if (placement != "postfilter") not_here("ANQI_VERIFIER_PLACEMENT=" + placement);
    if (RANKM <= 0 && vmode == VMode::Compact) die(2, "[rknn] the rank-M verifier requires ANQI_RANKM>0");
    if (RANKM <= 0 && vmode == VMode::Analytic) die(2, "[rknn] analytic_rankm requires ANQI_RANKM>0");
    if (std::getenv("ANQI_SPECIFIC"))
        die(2, "[rknn] independent postfilter verifier requires a shared graph; unset ANQI_SPECIFIC");
    // analytic_rankm defaults to the verifier envelope (rknn_query.cpp:1816-1818)
    const std::string envelope =
        env_or("ANQI_CANDIDATE_ENVELOPE", vmode == VMode::Analytic ? "verifier" : "graph_horizon");
    if (envelope != "graph_horizon" && envelope != "verifier")
        die(2, "[rknn] unsupported ANQI_CANDIDATE_ENVELOPE=%s (expected graph_horizon or verifier)", envelope.c_str());
    if (envelope != "graph_horizon") not_here("ANQI_CANDIDATE_ENVELOPE=" + envelope);
    if (env_or("ANQI_RQ_OBJECTIVE", "radius_reconstruction") != "radius_reconstruction")
        die(2, "[rknn] unsupported ANQI_RQ_OBJECTIVE=%s (implemented: radius_reconstruction; reserved: "
               "predicate_boundary)",
            env_or("ANQI_RQ_OBJECTIVE", "").c_str());
    if (env_flag("ANQI_RECHECK"))
        die(2, "[rknn] ANQI_RECHECK cannot be mixed with an independent postfilter verifier; select "
               "ANQI_RADIUS_MODE=exact_f32 for the exact component comparison");
    if (std::getenv("ANQI_REUSE_ORIG_KNN")) not_here("ANQI_REUSE_ORIG_KNN");
    // the Vamana refine (index.h:1262-1285): global passes, or the batched style (:936-1065)
    uint32_t vamana_passes = 0, vamana_L = 128;
    bool vamana_batch = false;
    if (std::getenv("ANQI_VAMANA")) {
        const char* sv = std::getenv("ANQI_VAMANA_STYLE");
        const std::string style = sv ? sv : "global";
        vamana_batch = style != "global" && style != "old";
        vamana_passes = (uint32_t)std::max(0, std::atoi(env_or("ANQI_VAMANA_PASS", "2").c_str()));
        vamana_L = (uint32_t)std::max(1, std::atoi(env_or("ANQI_VAMANA_L", "128").c_str()));
        if (vamana_L > 1024) die(2, "[rknn] ANQI_VAMANA_L=%u exceeds the device beam limit 1024", vamana_L);
    }
    if (env_or("ANQI_SEARCH_SCORE", "center") != "center") not_here("ANQI_SEARCH_SCORE=" + env_or("ANQI_SEARCH_SCORE", ""));
    if (std::getenv("ANQI_RCEPS") && std::atof(std::getenv("ANQI_RCEPS")) != 0.0) not_here("ANQI_RCEPS!=0");
    if (std::getenv("ANQI_RADIUS_RELAX") && std::atof(std::getenv("ANQI_RADIUS_RELAX")) != 0.0)
        die(2, "[rknn] postfilter verifier uses ANQI_RANKM_SLACK; ANQI_RADIUS_RELAX is not accepted");
    const double rankm_slack = std::getenv("ANQI_RANKM_SLACK") ? std::atof(std::getenv("ANQI_RANKM_SLACK")) : 0.0;
    const double slack_factor = 1.0 + rankm_slack;
    if (slack_factor <= 0.0)
        die(2, "[rknn] ANQI_RANKM_SLACK=%.6g makes non-positive radius scale", rankm_slack);
    if (vmode == VMode::Exact && rankm_slack != 0.0)
        die(2, "[rknn] exact_f32 postfilter does not accept ANQI_RANKM_SLACK");
    // rknn_query.cpp:1812-1816, 2417-2422
    if (vmode == VMode::Analytic && is_ip)
        die(2, "[rknn] analytic_rankm uses the L2 LID power law and does not support IP");
    if (vmode == VMode::Compact && is_ip && rankm_slack != 0.0)
        die(2, "[rknn] IP compact postfilter currently requires ANQI_RANKM_SLACK=0; multiplicative scaling is not "
               "monotone for signed -ip thresholds");

    // ---- cache identities (rknn_query.cpp:1840-1872, 1217-1241)
    const std::string basis_path = PFX + "_radbasis_M" + std::to_string(RANKM) + ".bin";
    const std::string cb_path = env_or("ANQI_RQ_CODEBOOK", (PFX + "_learned_rq_codebook_M" + std::to_string(RANKM) +
                                                            "_u" + std::to_string(bits) + ".bin").c_str());
    const std::string model_path =
        env_or("ANQI_ANALYTIC_RANKM_MODEL", (PFX + "_analytic_rankm_M" + std::to_string(RANKM) + ".bin").c_str());
    std::string radius_key;
    if (vmode == VMode::Compact) {
        radius_key = radius_mode + ":M" + env_or("ANQI_RANKM", "0") + ":b" +
                     (std::getenv("ANQI_RESID_BIAS") ? std::getenv("ANQI_RESID_BIAS") : "0") + ":obj" +
                     env_or("ANQI_RQ_OBJECTIVE", "radius_reconstruction") + ":basis" +
                     (std::getenv("ANQI_RQ_BASIS_ID") && *std::getenv("ANQI_RQ_BASIS_ID")
                          ? std::string(std::getenv("ANQI_RQ_BASIS_ID"))
                          : file_fingerprint(basis_path));
        if (is_learned_rq_mode(radius_mode))
            radius_key += ":cb" + (std::getenv("ANQI_RQ_CODEBOOK_ID") && *std::getenv("ANQI_RQ_CODEBOOK_ID")
                                       ? std::string(std::getenv("ANQI_RQ_CODEBOOK_ID"))
                                       : file_fingerprint(cb_path));
        const std::string radius_source_id = std::getenv("ANQI_RADIUS_SOURCE_ID")
                                                 ? env_or("ANQI_RADIUS_SOURCE_ID", "missing_radius_source_id")
                                                 : threshold_source_identity(PFX);
        radius_key += ":src" + hash16(radius_source_id) + ":rqpred_v3";
    } else if (vmode == VMode::Analytic) {
        radius_key = radius_mode + ":M" + std::to_string(RANKM) + ":model" + hash16(file_fingerprint(model_path));
    } else {
        radius_key = radius_mode;
    }
    std::string graph_key = graph_cache_key(Marg, leafA, ntA, efA);
    const std::string graph_radius_source = env_or("ANQI_GRAPH_RADIUS_SOURCE_PFX", PFX.c_str());
    const std::string graph_radius_id =
        std::getenv("ANQI_GRAPH_RADIUS_ID")
            ? env_or("ANQI_GRAPH_RADIUS_ID", "aknn_k100_v1")
            : file_stat_identity(base_vector_source(graph_radius_source + "_base.bin")) + "|" +
                  threshold_source_identity(graph_radius_source) + ":k" + std::to_string(GRAPH_NK) + ":v2";
    graph_key += "_graph_cutoff_k" + std::to_string(GRAPH_NK) + "_" + hash16(graph_radius_id);
    graph_key = sanitize_tag(graph_key);
    const std::string tag = hash16(graph_key);
    const std::string approxlift = graph_cache_dir + "_approxlift_graph_" + tag + ".bin";
    const std::string meta_file = graph_cache_dir + "_anqi_meta_graph_" + tag + ".txt";
    const std::string state_file = graph_cache_dir + "_anqi_graph_state_" + tag + ".txt";
    const std::string marker = graph_cache_dir + "_anqi_" + graph_key + ".built";
    const std::string cache_state_key = "graph=" + graph_key;
    uint64_t lift_nnk = 50;
    if (const char* v = std::getenv("ANQI_LIFTNNK"))
        if (!parse_positive(v, lift_nnk)) die(2, "[rknn] invalid ANQI_LIFTNNK=%s (expected a positive integer)", v);
    const float alpha = std::getenv("ANQI_ALPHA") ? (float)std::atof(std::getenv("ANQI_ALPHA")) : 1.2f;
    const uint64_t dim = d + 2;
    const std::string graph_path = graph_cache_dir + graph_file_name(Marg, lift_nnk, n, dim, alpha, graph_key);
    printf("[rknn] graph geometry=anyk_lift graph_rankm=0 verification_rankm=%d radius_mode=%s placement=postfilter\n",
           RANKM, radius_mode.c_str());
    printf("[rknn] graph cache key=%s\n", graph_key.c_str());
    auto first_line = [](const std::string& p) {
        std::ifstream f(p);
        std::string s;
        std::getline(f, s);
        return s;
    };
    bool can_load = file_exists(state_file) && first_line(state_file) == cache_state_key && file_exists(marker) &&
                    file_exists(approxlift) && file_exists(meta_file);
    printf("[rknn] component caches: graph=%s verifier=%s\n", graph_cache_dir.c_str(), verifier_cache_dir.c_str());
    if (env_flag("ANQI_REQUIRE_GRAPH_CACHE") && !can_load)
        die(3, "[rknn] required graph cache is incomplete or incompatible: dir=%s key=%s", graph_cache_dir.c_str(),
            graph_key.c_str());
    mkdir_p(graph_cache_dir);
    mkdir_p(verifier_cache_dir);

    Lrq lrq;
    lrq.n = n;
    lrq.nk = (uint32_t)NK;
    lrq.rankm = (uint32_t)RANKM;
    lrq.bits = (uint32_t)bits;
    lrq.policy = is_learned_rq_mode(radius_mode) ? lrq_policy : (bits == 32 ? "float32" : "rankm");
    std::unique_ptr<Device> device;  // created when the first device stage runs
    auto dev = [&]() -> Device& {
        if (!device) device = std::make_unique<Device>("[rknn]");
        return *device;
    };
    double verifier_load_ms = 0, verifier_encode_save_ms = 0;
    AnalyticModel model;
    if (vmode == VMode::Analytic) {
        const auto t0 = Clock::now();
        model = read_analytic_model(model_path, n, RANKM);
        verifier_load_ms = since(t0) * 1e3;
        if (model.train_kmax != GRAPH_NK)
            die(2, "[rknn] analytic Rank-M training horizon=%u must match graph horizon=%" PRIu64
                   " for the controlled multi-rank experiment", model.train_kmax, GRAPH_NK);
        printf("[rknn] loaded analytic Rank-M verifier %s (train_kmax=%u fit_kmin=%u M=%d b0=%.9g flags=%u "
               "persistent=%.3fGB load_ms=%.3f)\n",
               model_path.c_str(), model.train_kmax, model.fit_kmin, RANKM, model.b0, model.flags,
               (40.0 + model.coeff.size() * 4.0) / 1e9, verifier_load_ms);
    }
    if (vmode == VMode::Compact) {
        load_basis(basis_path, NK, RANKM, lrq);
        printf("[rknn] loaded rank-M basis: M=%d path=%s\n", RANKM, basis_path.c_str());
        if (is_learned_rq_mode(radius_mode)) {
            load_codebook(cb_path, NK, RANKM, bits, lrq);
            if (lrq.code_size != (1u << bits)) die(3, "[rknn] invalid CompactLrqVerifier configuration");
        }
        if ((bits == 2 && NK % 4 != 0) || (bits == 4 && NK % 2 != 0))
            die(3, "[rknn] packed u%d verifier requires NK divisible by %d, got %" PRIu64, bits, bits == 2 ? 4 : 2, NK);
    }
    const std::string lrq_file = verifier_cache_dir + "_anqi_verifier_" + hash16(radius_key) + ".bin";
    bool lrq_ready = vmode != VMode::Compact;
    if (vmode == VMode::Compact && file_exists(lrq_file)) {
        const auto t0 = Clock::now();
        load_verifier(lrq_file, lrq);
        lrq_ready = true;
        verifier_load_ms = since(t0) * 1e3;
        printf("[rknn] loaded independent compact verifier mode=%s bits=%d %s (persistent=%.3fGB "
               "load_ms=%.3f)\n",
               vmode_label.c_str(), bits, lrq_file.c_str(), lrq.persistent_bytes() / 1e9, verifier_load_ms);
    }
    auto ensure_lrq = [&]() {
        if (lrq_ready) return;
        const std::vector<float> keys = load_threshold_table(PFX, n, NK);
        const auto t0 = Clock::now();
        lrq.coeff.resize(n * lrq.rankm);
        lrq.codes.assign(lrq.code_bytes(), 0);
        lrq.residual.resize(bits == 32 ? n * NK : 0);
        dev().check(anqi_lrq_encode_bits(dev().get(), keys.data(), n, lrq.nk, lrq.rankm, lrq.mu.data(),
                                         lrq.basis.data(), lrq.codebook.empty() ? nullptr : lrq.codebook.data(),
                                         lrq.code_size, lrq.bits, lrq.policy_code(), lrq.coeff.data(),
                                         lrq.codes.empty() ? nullptr : lrq.codes.data(),
                                         lrq.residual.empty() ? nullptr : lrq.residual.data()),
                    "LRQ encode");
        save_verifier(lrq_file, lrq);
        verifier_encode_save_ms = since(t0) * 1e3;
        lrq_ready = true;
        printf("[rknn] built independent compact verifier mode=%s bits=%d %s (persistent=%.3fGB "
               "encode_save_ms=%.3f)\n",
               vmode_label.c_str(), bits, lrq_file.c_str(), lrq.persistent_bytes() / 1e9, verifier_encode_save_ms);
    };
    // bytes the reference reports for the verification structure (rknn_query.cpp:2015-2020, 1243-1264)
    auto verification_bytes = [&]() -> uint64_t {
        return vmode == VMode::Compact ? lrq.persistent_bytes()
                                       : (vmode == VMode::Analytic ? 40 + n * (uint64_t)RANKM * 4 : n * NK * 4);
    };

    std::vector<float> lifted;
    std::vector<uint32_t> deg, links;
    PostTree tree;
    double source_prepare_s = 0, lift_verifier_prepare_s = 0, graph_index_s = 0;
    if (can_load) {
        {
            std::ifstream f(meta_file);
            if (!(f >> Mstar2 >> scale)) die(3, "[rknn] bad meta cache %s", meta_file.c_str());
        }
        ensure_lrq();
        printf("[rknn] loaded cached index (M=%" PRIu64 "): M*^2=%.6g scale=%.4g radius=%s:postfilter\n", Marg, Mstar2,
               scale, radius_key.c_str());
        Fbin lf = load_fbin_or_die(approxlift);
        if (lf.n != n || lf.d != dim) die(3, "[rknn] lifted cache %s has shape %ux%u", approxlift.c_str(), lf.n, lf.d);
        lifted = std::move(lf.x);
        printf("[rknn] graph degree M=%" PRIu64 "\n", Marg);
        std::cout << "Index config: " << graph_path.substr(graph_cache_dir.size()) << "\n";
        std::cout << "Loading index from: " << graph_path << "\n" << std::flush;
        const auto t0 = Clock::now();
        float ctime = 0;
        std::string why;
        if (!read_graph(graph_path, n, dim, Marg, deg, links, tree, ctime, why)) {
            fprintf(stderr, "%s\n", why.c_str());
            can_load = false;  // rebuilt below from the warm start
        }
        graph_index_s = since(t0);
    }
    if (!can_load) {
        // warm start: prebuilt records, or an AKNN build over the base here
        const auto t_src = Clock::now();
        std::vector<uint32_t> warm;
        const uint64_t width = 100;
        const std::string topk = prebuilt_topk_path();
        // where the graph's warm-start ids come from (rknn_query.cpp:2092-2131)
        const char* stream_command = std::getenv("ANQI_PREBUILT_WARM_START_COMMAND");
        const bool streamed_cmd = !topk.empty() && stream_command && *stream_command;
        const bool compact_ids = !topk.empty() && env_flag("ANQI_COMPACT_PREBUILT_TOPK_IDS_INPLACE");
        const uint64_t sk = topk.empty() ? width : prebuilt_topk_width(width);
        if (compact_ids && streamed_cmd)
            die(2, "[rknn] compact local warm-start IDs cannot be combined with ANQI_PREBUILT_WARM_START_COMMAND");
        if (compact_ids || streamed_cmd) {
            validate_prebuilt_topk(topk, n, sk, width);
            printf(compact_ids ? "[rknn] deferred original KNN IDs to compact local graph warm-start (source_k=%" PRIu64
                                 " width=%" PRIu64 ")\n"
                               : "[rknn] deferred original KNN IDs to streamed graph warm-start (source_k=%" PRIu64
                                 " width=%" PRIu64 ")\n",
                   sk, width);
        } else if (!topk.empty()) {
            validate_prebuilt_topk(topk, n, sk, width);
            const std::vector<TopKRecord> rec = read_prebuilt(topk, n, sk);
            warm.resize(n * width);
            for (uint64_t i = 0; i < n; i++)
                for (uint64_t j = 0; j < width; j++) warm[i * width + j] = rec[i * sk + j].id;
        } else {
            printf("[rknn] original-space AKNN: leaf=%" PRIu64 " n_trees=%" PRIu64 " ef=%" PRIu64 " metric=%s\n",
                   leafA, ntA, efA, metric.c_str());
            anqi_aknn_params ap{};
            ap.k = (uint32_t)width;
            ap.leaf = (uint32_t)leafA;
            ap.trees = (uint32_t)ntA;
            ap.ef = (uint32_t)efA;
            ap.ef_alpha = 8;
            ap.seed = 10;
            ap.nn_iters = (uint32_t)std::max(0, std::atoi(env_or("ANQI_NNITERS", "0").c_str()));
            ap.nn_sample = (uint32_t)std::min(std::max(0, std::atoi(env_or("ANQI_NNSAMPLE", "20").c_str())), 120);
            ap.precision = env_or("ANQI_B200_PRECISION", "bf16") == "fp32" ? 0u : 1u;
            ap.metric = is_ip ? ANQI_METRIC_IP : ANQI_METRIC_L2;
            if (is_ip && ap.nn_iters > 0)
                die(2, "[rknn] ANQI_NNITERS > 0 is implemented for metric l2 only on this path");
            warm.resize(n * width);
            std::vector<float> wd(n * width);
            dev().check(anqi_aknn_build(dev().get(), base.x.data(), n, (uint32_t)d, &ap, warm.data(), wd.data(), nullptr),
                      "original-space AKNN");
        }
        source_prepare_s = since(t_src);
        printf("[rknn] original-space AKNN warm start ready: rows=%" PRIu64 " source=%s\n", n,
               (compact_ids || streamed_cmd) ? "prebuilt-stream" : (topk.empty() ? "internal" : "prebuilt-contiguous"));
        const auto t_prep = Clock::now();
        ensure_lrq();
        const std::vector<float> radius = load_threshold_column(graph_radius_source, n, GRAPH_NK);
        printf("[rknn] RADIUS_MODE=%s:postfilter conceptual_radius_store=%.3fGB\n", radius_key.c_str(),
               verification_bytes() / 1e9);
        lifted.resize(n * dim);
        dev().check(anqi_lift_metric(dev().get(), base.x.data(), n, (uint32_t)d, radius.data(),
                                     is_ip ? ANQI_METRIC_IP : ANQI_METRIC_L2, lifted.data(), &Mstar2, &scale),
                    "lift");
        {
            const uint32_t hdr[2] = {(uint32_t)n, (uint32_t)dim};
            write_file_or_die(approxlift, {{hdr, 8}, {lifted.data(), lifted.size() * 4}}, 3, "[rknn]");
        }
        {
            std::ofstream f(meta_file);
            f << std::setprecision(17) << Mstar2 << " " << scale << "\n";
        }
        {
            std::ofstream f(state_file);
            f << cache_state_key << "\n";
        }
        printf("[rknn] BUILD lift M*^2=%.6g scale=%.4g (graph radius=aknn_k%" PRIu64 "; verifier=%s:postfilter)\n",
               Mstar2, scale, GRAPH_NK, radius_key.c_str());
        // the prebuilt table's keys are read (verifier, radius): it can now be
        // compacted to ids or released (rknn_query.cpp:2170-2186)
        if (compact_ids) {
            compact_topk_ids_in_place(topk, n, sk, width);
        } else if (!topk.empty() && env_flag("ANQI_RELEASE_PREBUILT_TOPK_AFTER_PREP")) {
            if (::unlink(topk.c_str()) != 0)
                die(3, "[rknn] cannot release regenerable prebuilt top-k %s: %s", topk.c_str(), std::strerror(errno));
            printf("[rknn] released regenerable prebuilt top-k after verifier/lift preparation: %s\n", topk.c_str());
        }
        lift_verifier_prepare_s = since(t_prep);

        printf("[rknn] graph degree M=%" PRIu64 "\n", Marg);
        std::cout << "Index config: " << graph_path.substr(graph_cache_dir.size()) << "\n" << std::flush;
        const auto t_graph = Clock::now();
        anqi_graph_params gp{};
        gp.degree = (uint32_t)Marg;
        gp.nn_k = (uint32_t)lift_nnk;
        gp.explore = 100;
        gp.ef_alpha = 8;
        gp.join_iters = (uint32_t)std::max(0, std::atoi(env_or("ANQI_GRAPHNND", "6").c_str()));
        gp.join_sample = (uint32_t)std::min(std::max(0, std::atoi(env_or("ANQI_NNSAMPLE", "20").c_str())), 120);
        gp.leaf = 100;
        gp.max_depth = 100;
        gp.seed = 10;
        gp.alpha = alpha;
        gp.warm_width = (uint32_t)width;
        gp.precision = env_or("ANQI_B200_PRECISION", "bf16") == "fp32" ? 0u : 1u;
        gp.vamana_passes = vamana_passes;
        gp.vamana_L = vamana_L;
        if (vamana_batch) {
            // vamana_batch_refine's settings (index.h:939-951) and entry (choose_vamana_entry, :190-222)
            auto envd = [](const char* k, double d) { const char* v = std::getenv(k); return v ? std::atof(v) : d; };
            auto envi = [](const char* k, int d) { const char* v = std::getenv(k); return v ? std::atoi(v) : d; };
            gp.vamana_batch = 1;
            gp.vamana_batch_frac = envd("ANQI_VAMANA_BATCH_FRAC", 0.02);
            gp.vamana_max_batch = (uint64_t)(int64_t)envi("ANQI_VAMANA_MAX_BATCH", 1000000);
            gp.vamana_batch_base = envd("ANQI_VAMANA_BATCH_BASE", 2.0);
            const char* ea = std::getenv("ANQI_VAMANA_EARLY_ALPHA");
            gp.vamana_early_alpha = ea ? (float)std::atof(ea) : 1.0f;
            gp.vamana_early_alpha_one = envi("ANQI_VAMANA_EARLY_ALPHA_ONE", 1) != 0;
            const char* ev = std::getenv("ANQI_VAMANA_ENTRY");
            uint32_t entry = 0;
            if (ev && *ev) {
                const std::string es(ev);
                if (es == "medoid" || es == "centroid") {
                    size_t sample = (size_t)envi("ANQI_VAMANA_ENTRY_SAMPLE", (int)std::min<uint64_t>(n, 100000));
                    sample = std::max<size_t>(1, std::min<size_t>(sample, n));
                    std::vector<double> mean(dim, 0.0);
                    const size_t step = std::max<size_t>(1, n / sample);
                    for (size_t t = 0; t < sample; t++)
                        for (size_t j = 0; j < dim; j++) mean[j] += (double)lifted[((t * step) % n) * dim + j];
                    for (size_t j = 0; j < dim; j++) mean[j] /= (double)sample;
                    double bestd = std::numeric_limits<double>::infinity();
                    for (size_t t = 0; t < sample; t++) {
                        const size_t id = (t * step) % n;
                        double dd = 0.0;
                        for (size_t j = 0; j < dim; j++) {
                            const double z = (double)lifted[id * dim + j] - mean[j];
                            dd += z * z;
                        }
                        if (dd < bestd) {
                            bestd = dd;
                            entry = (uint32_t)id;
                        }
                    }
                } else {
                    char* endp = nullptr;
                    const unsigned long long id = std::strtoull(ev, &endp, 10);
                    if (endp != ev && n > 0) entry = (uint32_t)(id % n);
                }
            }
            gp.vamana_entry = entry;
        }
        // the edge policy of the prunes (the graph folder of the postfilter
        // placement is the graph cache directory, rknn_query.cpp:1947)
        EdgePolicyHost edge;
        resolve_edge_policy(edge, n, (uint32_t)Marg, graph_cache_dir);
        if (edge.p.flags) gp.edge = &edge.p;
        deg.resize(n);
        links.resize(n * Marg);
        anqi_build_stats gs{};
        if (compact_ids || streamed_cmd) {
            dev().check(anqi_graph_build_begin(dev().get(), lifted.data(), n, (uint32_t)dim, &gp), "graph build");
            FILE* in = streamed_cmd ? ::popen(stream_command, "r") : std::fopen(topk.c_str(), "rb");
            if (!in) die(3, "[rknn] cannot start streamed warm-start %s", streamed_cmd ? "command" : topk.c_str());
            stream_warm_rows(dev().get(), in, streamed_cmd, n, compact_ids ? width : sk, width, compact_ids);
            if (compact_ids && ::unlink(topk.c_str()) != 0)
                die(3, "[rknn] cannot release consumed streamed warm-start file %s", topk.c_str());
            printf(compact_ids ? "[rknn] init: streamed compact KNN IDs warm-start (recompute lifted d2)\n"
                               : "[rknn] init: streamed original KNN warm-start (recompute lifted d2)\n");
            dev().check(anqi_graph_build_finish(dev().get(), deg.data(), links.data(), &gs), "graph build");
        } else {
            dev().check(anqi_graph_build(dev().get(), lifted.data(), n, (uint32_t)dim, warm.data(), (uint32_t)width,
                                         &gp, deg.data(), links.data(), &gs),
                        "graph build");
        }
        uint32_t tn = 0;
        uint64_t tp = 0;
        dev().check(anqi_graph_tree_size(dev().get(), &tn, &tp), "entry tree size");
        std::vector<uint32_t> tl(tn), tr(tn), lo(tn), lc(tn), perm(tp);
        std::vector<float> to(tn), th((size_t)tn * dim);
        dev().check(anqi_graph_tree_copy(dev().get(), tl.data(), tr.data(), to.data(), th.data(), lo.data(), lc.data(),
                                       perm.data()),
                  "entry tree copy");
        tree = bfs_to_postorder(tl, tr, to, th, lo, lc, perm, 100, (uint32_t)dim);
        graph_index_s = since(t_graph);
        std::cout << "Index saved to: " << graph_path << "\n";
        if (!write_graph(graph_path, n, dim, Marg, (float)graph_index_s, deg, links, tree))
            die(3, "[rknn] failed writing graph cache %s", graph_path.c_str());
        std::ofstream(marker) << "1\n";
    }
    {
        uint64_t sum = 0;
        uint32_t mn = UINT32_MAX, mx = 0;
        for (uint32_t v : deg) {
            sum += v;
            mn = std::min(mn, v);
            mx = std::max(mx, v);
        }
        std::cout << "Degree: Max=" << mx << " Min=" << mn << " Avg=" << (double)sum / (double)n
                  << " (fixed cap M=" << Marg << ")\n";
    }

    // ---- device index + verifier
    const std::vector<uint32_t> leaf_first = tree.leaf_first();
    anqi_index_desc desc{};
    desc.n = n;
    desc.d = (uint32_t)d;
    desc.degree = (uint32_t)Marg;
    desc.base = base.x.data();
    desc.lifted = lifted.data();
    desc.deg = deg.data();
    desc.links = links.data();
    desc.tree_nodes = tree.nodes();
    desc.tree_left = tree.left.data();
    desc.tree_right = tree.right.data();
    desc.tree_offset = tree.offset.data();
    desc.tree_hyperplane = tree.hyper.data();
    desc.tree_leaf_first = leaf_first.data();
    desc.scale = scale;
    desc.mstar2 = Mstar2;
    desc.metric = is_ip ? ANQI_METRIC_IP : ANQI_METRIC_L2;
    dev().check(anqi_index_load(dev().get(), &desc), "index load");
    if (vmode == VMode::Compact)
        dev().check(anqi_verifier_load_bits(dev().get(), lrq.coeff.data(), lrq.codes.empty() ? nullptr : lrq.codes.data(),
                                            lrq.residual.empty() ? nullptr : lrq.residual.data(), n, lrq.nk, lrq.rankm,
                                            lrq.bits, lrq.mu.data(), lrq.basis.data(),
                                            lrq.codebook.empty() ? nullptr : lrq.codebook.data(), lrq.code_size,
                                            is_ip ? 1 : 0),
                    "verifier load");
    else if (vmode == VMode::Analytic)
        dev().check(anqi_verifier_load_analytic(dev().get(), model.coeff.data(), n, (uint32_t)RANKM, model.train_kmax,
                                                model.fit_kmin, model.flags, model.b0),
                    "verifier load");
    const double build_s = since(tb0);
    auto external_seconds = [](const char* name) {
        const char* raw = std::getenv(name);
        if (!raw || !*raw) return 0.0;
        char* end = nullptr;
        errno = 0;
        const double v = std::strtod(raw, &end);
        if (errno != 0 || end == raw || *end != '\0' || !std::isfinite(v) || v < 0.0)
            die(2, "[rknn] invalid %s=%s", name, raw);
        return v;
    };
    const double aknn_build_s = external_seconds("ANQI_AKNN_BUILD_SECONDS");
    const double verifier_train_s = external_seconds("ANQI_VERIFIER_TRAIN_SECONDS");
    const double end_to_end_s = aknn_build_s + verifier_train_s + build_s;
    const double verification_gb = verification_bytes() / 1e9;
    const double idx_gb = ((double)n * Marg * 4 + (double)n * dim * 4 + (double)verification_bytes()) / 1e9;
    if (can_load) {
        printf("[rknn] INDEX_LOAD_TIME=%.1fs INDEX_SIZE=%.2fGB (graph M=%" PRIu64 " + graph dim=%" PRIu64
               " + verification=%.3fGB + envelope=%.3fGB)\n",
               build_s, idx_gb, Marg, dim, verification_gb, 0.0);
    } else {
        printf("[rknn] BUILD_TIME=%.1fs INDEX_SIZE=%.2fGB (aknn_source=%.1fs + verifier_training=%.1fs + "
               "index=%.1fs, graph M=%" PRIu64 " + graph dim=%" PRIu64 " + verification=%.3fGB + envelope=%.3fGB)\n",
               end_to_end_s, idx_gb, aknn_build_s, verifier_train_s, build_s, Marg, dim, verification_gb, 0.0);
    }
    if (env_flag("ANQI_BUILD_BREAKDOWN")) {
        if (can_load)
            printf("[rknn] LOAD_BREAKDOWN index_load_s=%.6f verifier_load_ms=%.3f\n", build_s, verifier_load_ms);
        else
            printf("[rknn] BUILD_BREAKDOWN aknn_source_s=%.6f verifier_train_s=%.6f source_prepare_s=%.6f "
                   "lift_verifier_prepare_s=%.6f graph_index_s=%.6f index_total_s=%.6f end_to_end_s=%.6f "
                   "verifier_encode_save_ms=%.3f\n",
                   aknn_build_s, verifier_train_s, source_prepare_s, lift_verifier_prepare_s, graph_index_s, build_s,
                   end_to_end_s, verifier_encode_save_ms);
    }
    const auto t_mat = Clock::now();
    if (vmode == VMode::Exact) {
        // exact_f32: the rank-Kq column of the source thresholds (load_threshold_column)
        const std::vector<float> col = load_threshold_column(PFX, n, Kq);
        dev().check(anqi_set_thresholds(dev().get(), (uint32_t)Kq, col.data()), "verifier thresholds");
    } else {
        dev().check(anqi_verifier_materialize(dev().get(), (uint32_t)Kq, slack_factor), "verifier materialize");
    }
    const double materialize_ms = since(t_mat) * 1e3;
    printf("[rknn] independent verifier ready: mode=%s k=%" PRIu64 " slack=%.6g persistent=%.3fGB "
           "temporary_thresholds=%.3fGB materialize_ms=%.3f bits=%d\n",
           vmode_label.c_str(), Kq, rankm_slack, verification_gb, n * 4 / 1e9, materialize_ms,
           vmode == VMode::Compact ? bits : 0);
    const float beta = std::getenv("ANQI_BETA") ? (float)std::atof(std::getenv("ANQI_BETA")) : 0.5f;
    printf("[rknn] k-adaptive flood: Kq=%" PRIu64 " radj=off beta=%.2f\n", Kq, beta);
    printf("[rknn] candidate generator: AKNN-k%" PRIu64 " envelope, center graph search; verifier is post-filter only\n",
           GRAPH_NK);
    printf("[rknn] search score: mode=center lambda=%s\n", env_or("ANQI_SEARCH_SCORE_LAMBDA", "1.0").c_str());
    const std::string visited_mode = env_or("ANQI_QUERY_VISITED", "stamps");
    if (visited_mode != "stamps" && visited_mode != "bitset")
        die(2, "[rknn] invalid ANQI_QUERY_VISITED=%s (expected stamps or bitset)", visited_mode.c_str());
    printf("[rknn] query visited mode=device (per-warp shared-memory table, spilling to a per-warp bitmap; "
           "ANQI_QUERY_VISITED=%s has no effect)\n",
           visited_mode.c_str());

    // ---- timed loop (rknn_query.cpp:2692-2956)
    uint64_t bench_repeats = 1;
    if (const char* r = std::getenv("ANQI_BENCH_REPEATS")) {
        bool digits = *r != '\0';
        for (const char* p = r; *p; p++) digits = digits && std::isdigit((unsigned char)*p);
        uint64_t v = 0;
        if (!digits || !parse_positive(r, v) || v > std::numeric_limits<uint64_t>::max() / std::max<uint64_t>(1, nq))
            die(2, "[rknn] invalid ANQI_BENCH_REPEATS=%s", r);
        bench_repeats = v;
    }
    const bool calibrated = env_flag("ANQI_BENCH_CALIBRATED_TIMING");
    auto positive_seconds = [](const char* name, double fallback) {
        const char* v = std::getenv(name);
        if (!v || !*v) return fallback;
        char* end = nullptr;
        errno = 0;
        const double x = std::strtod(v, &end);
        if (errno == ERANGE || end == v || *end != '\0' || !std::isfinite(x) || x <= 0.0)
            die(2, "[rknn] invalid %s=%s", name, v);
        return x;
    };
    const double min_total_s = positive_seconds("ANQI_BENCH_MIN_TOTAL_S", 30.0);
    const double min_repeat_s = positive_seconds("ANQI_BENCH_MIN_REPEAT_S", 10.0);
    printf("[rknn] benchmark repeats=%" PRIu64 " calibrated=%s (timing uses steady_clock sub-millisecond precision)\n",
           bench_repeats, calibrated ? "on" : "off");
    printf("[rknn] query parallelism: nq=%" PRIu64 " device=cuda:0 (one warp per query)\n", nq);
    if (calibrated)
        printf("[rknn] calibrated timing: min_total_s=%.3f min_repeat_s=%.3f windows=%" PRIu64 "\n", min_total_s,
               min_repeat_s, bench_repeats);
    else
        printf("[rknn] flattened_repeats=1 tasks=%" PRIu64 "\n", nq * bench_repeats);
    if (env_flag("ANQI_TIME_BREAKDOWN"))
        printf("[rknn] query stage timing is not split per query on the device (ANQI_TIME_BREAKDOWN ignored)\n");
    fflush(stdout);

    auto run_point = [&](uint64_t L, uint64_t batches) {
        PointStats s;
        const auto t0 = Clock::now();
        for (uint64_t b = 0; b < batches; b++) {
            dev().check(anqi_query_run(dev().get(), 1, nullptr), "query run");
            anqi_eval_sums e{};
            dev().check(anqi_query_evaluate_sums(dev().get(), &e), "evaluation");
            s.recall += e.recall;
            s.prec += e.precision;
            s.f1 += e.f1;
            s.cand_recall += e.cand_recall;
            s.cand += e.cand;
            s.pred += e.pred;
            s.graph_dist += e.graph_dist;
            s.nonempty += e.nonempty;
        }
        s.secs = since(t0);
        s.tasks = nq * batches;
        s.batches = batches;
        (void)L;
        return s;
    };
    auto print_point = [&](uint64_t L, const PointStats& s, double qps) {
        if (s.nonempty == 0 || s.tasks == 0 || s.secs <= 0.0)
            die(3, "[rknn] empty benchmark statistics for L_descent=%" PRIu64, L);
        const double dn = (double)s.nonempty;
        const double total_dist = s.graph_dist + s.cand;
        printf("[rknn] L_descent=%-5" PRIu64 " | recall=%.4f precision=%.4f F1=%.4f | avg cand=%.0f pred=%.0f "
               "#dist=%.0f | QPS=%.0f (parallel)\n",
               L, s.recall / dn, s.prec / dn, s.f1 / dn, s.cand / dn, s.pred / dn, total_dist / dn, qps);
        printf("[rknn] DIST_BREAKDOWN L_descent=%" PRIu64 " #graph_dist=%.0f #verify_dist=%.0f #total_dist=%.0f\n", L,
               s.graph_dist / dn, s.cand / dn, total_dist / dn);
        printf("[rknn] CANDIDATE_RECALL L_descent=%" PRIu64 " recall=%.6f\n", L, s.cand_recall / dn);
    };

    for (uint64_t L : Lds) {
        dev().check(anqi_query_upload(dev().get(), query.x.data(), (uint32_t)nq, nullptr, (uint32_t)Kq, nullptr,
                                    (uint32_t)L),
                  "query upload");
        dev().check(anqi_gt_load(dev().get(), goff.data(), gids.data(), gids.size()), "ground-truth load");
        if (!calibrated) {
            const PointStats s = run_point(L, bench_repeats);
            print_point(L, s, (double)s.tasks / s.secs);
            fflush(stdout);
            continue;
        }
        const PointStats warm = run_point(L, 1);
        const PointStats calib = run_point(L, 1);
        const double target = std::max(min_repeat_s, min_total_s / (double)bench_repeats);
        const uint64_t planned = std::max<uint64_t>(1, (uint64_t)std::ceil(target / std::max(calib.secs, 1e-9)));
        PointStats agg;
        std::vector<double> qps;
        double min_repeat = std::numeric_limits<double>::infinity();
        for (uint64_t rep = 0; rep < bench_repeats; rep++) {
            uint64_t actual = planned;
            PointStats m;
            for (int attempt = 0; attempt < 4; attempt++) {
                m = run_point(L, actual);
                if (m.secs + 1e-9 >= target) break;
                const double scaled = (double)actual * target / std::max(m.secs, 1e-9) * 1.05;
                const uint64_t next = std::max<uint64_t>(actual + 1, (uint64_t)std::ceil(scaled));
                printf("[rknn] HOT_RETRY L_descent=%" PRIu64 " repeat=%" PRIu64 " seconds=%.6f target_s=%.6f "
                       "batches=%" PRIu64 " next_batches=%" PRIu64 "\n",
                       L, rep + 1, m.secs, target, actual, next);
                actual = next;
            }
            if (m.secs + 1e-9 < target)
                die(3, "[rknn] calibrated repeat too short for L_descent=%" PRIu64 " repeat=%" PRIu64
                       " seconds=%.6f target_s=%.6f",
                    L, rep + 1, m.secs, target);
            const double q = (double)m.tasks / m.secs;
            qps.push_back(q);
            min_repeat = std::min(min_repeat, m.secs);
            agg.add(m);
            printf("[rknn] HOT_REPEAT L_descent=%" PRIu64 " repeat=%" PRIu64 "/%" PRIu64 " batches=%" PRIu64
                   " tasks=%" PRIu64 " seconds=%.6f QPS=%.3f\n",
                   L, rep + 1, bench_repeats, m.batches, m.tasks, m.secs, q);
        }
        std::vector<double> sorted = qps;
        std::sort(sorted.begin(), sorted.end());
        const size_t mid = sorted.size() / 2;
        const double median = sorted.size() % 2 ? sorted[mid] : 0.5 * (sorted[mid - 1] + sorted[mid]);
        print_point(L, agg, median);
        printf("[rknn] HOT_TIMING L_descent=%" PRIu64 " warm_s=%.6f calibration_s=%.6f measured_s=%.6f repeats=%" PRIu64
               " planned_batches_per_repeat=%" PRIu64 " actual_batches_total=%" PRIu64
               " min_repeat_s=%.6f qps_median=%.3f qps_samples=",
               L, warm.secs, calib.secs, agg.secs, bench_repeats, planned, agg.batches, min_repeat, median);
        for (size_t i = 0; i < qps.size(); i++) printf("%s%.3f", i ? "," : "", qps[i]);
        printf("\n");
        fflush(stdout);
    }
    return 0;
}

int main(int argc, char** argv) {
    try {
        return run(argc, argv);
    } catch (const Exit& e) {
        fflush(stdout);
        fprintf(stderr, "%s\n", e.what());
        return e.code;
    }
}
