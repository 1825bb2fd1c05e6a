// dataset_gt: exact base-to-base top-K thresholds and reverse-kNN ground truth
// on the GPU.
//
//   dataset_gt --base BASE.bin [--query QUERY.bin] --out_prefix PREFIX
//              [--K 100] [--rk_k 10] [--tile 512] [--metric l2|ip]
//              [--threads N] [--mode both|thresholds|ground-truth]
//              [--threshold-table FILE]
//
// Same options, files, stdout lines and exit codes as tools/dataset_gt.cpp
// (2 usage, 3 bad input or write failure; 7/8/9 device failure).  Outputs:
//   PREFIX_baseknn_gt.bin     [u32 n][u32 K][n*K u32 ids][n*K f32 keys]
//   PREFIX_rknn_gt.bin.rk     [u32 n][u32 rk_k][n f32 rank-k keys]
//   PREFIX_rknn_gt.bin        [u32 nq][(nq+1) u32 off][ids][f32 keys]
//   PREFIX_threshold_build_time.meta
// Keys are the reference's FP32 |a|^2 + |b|^2 - 2<a,b> (--metric l2) or
// -<a,b> (--metric ip) in its summation order, so the files are bit-identical.
// --tile and --threads are accepted and reported; the device tiles on its own.
#include "cli_common.h"

#include <chrono>
#include <memory>
#include <iostream>

using namespace anqi_cli;

static uint64_t positive_or_die(const char* text, const char* name) {
    uint64_t v = 0;
    if (!text || !*text) die(2, "[dgt] missing value for %s", name);
    if (!parse_positive(text, v)) die(2, "[dgt] invalid %s=%s", name, text);
    return v;
}

static Fbin load_fbin_or_die(const std::string& p) {
    Fbin f;
    std::string why;
    if (!read_fbin(p, f, why)) {
        if (why == "cannot open") die(3, "[dgt] cannot open %s", p.c_str());
        die(3, "[dgt] %s: %s", why.c_str(), p.c_str());
    }
    return f;
}

// Column rank_one_based of a _baseknn_gt.bin table (tools/dataset_gt.cpp:73-116).
static std::vector<float> load_threshold_column(const std::string& path, uint64_t expected_n, uint64_t rank) {
    std::ifstream in(path, std::ios::binary | std::ios::ate);
    const std::streamoff bytes = in ? (std::streamoff)in.tellg() : (std::streamoff)-1;
    in.seekg(0);
    uint32_t n = 0, k = 0;
    if (!in.read(reinterpret_cast<char*>(&n), 4) || !in.read(reinterpret_cast<char*>(&k), 4) || n != expected_n ||
        rank == 0 || rank > k)
        die(3, "[dgt] invalid threshold table: %s", path.c_str());
    const uint64_t cells = (uint64_t)n * k;
    if (8 + 2 * cells * 4 != (uint64_t)bytes) die(3, "[dgt] invalid threshold-table size: %s", path.c_str());
    in.seekg((std::streamoff)(8 + cells * 4));
    std::vector<float> keys(cells);
    if (!in.read(reinterpret_cast<char*>(keys.data()), (std::streamsize)(cells * 4)))
        die(3, "[dgt] truncated threshold table: %s", path.c_str());
    std::vector<float> col(n);
    for (uint64_t i = 0; i < n; i++) col[i] = keys[i * k + rank - 1];
    return col;
}

static void write_rk(const std::string& prefix, uint64_t n, uint64_t rk_k, const std::vector<float>& rk2) {
    const std::string path = prefix + "_rknn_gt.bin.rk";
    const uint32_t un = (uint32_t)n, uk = (uint32_t)rk_k;
    write_file_or_die(path, {{&un, 4}, {&uk, 4}, {rk2.data(), n * 4}}, 3, "[dgt]");
    std::cout << "[dgt] wrote " << path << " (rank-k threshold array)\n";
}

static int run(int argc, char** argv) {
    std::string base_p, query_p, prefix, metric = "l2", mode = "both", threshold_table;
    uint64_t K = 100, rk_k = 10, tile = 512, nthreads = 0;
    auto next_value = [&](int& i, const std::string& option) -> const char* {
        if (i + 1 >= argc) die(2, "[dgt] missing value for %s", option.c_str());
        return argv[++i];
    };
    for (int i = 1; i < argc; i++) {
        const std::string a = argv[i];
        if (a == "--base") base_p = next_value(i, a);
        else if (a == "--query") query_p = next_value(i, a);
        else if (a == "--K") K = positive_or_die(next_value(i, a), "K");
        else if (a == "--rk_k") rk_k = positive_or_die(next_value(i, a), "rk_k");
        else if (a == "--out_prefix") prefix = next_value(i, a);
        else if (a == "--tile") tile = positive_or_die(next_value(i, a), "tile");
        else if (a == "--metric") metric = next_value(i, a);
        else if (a == "--threads") nthreads = positive_or_die(next_value(i, a), "threads");
        else if (a == "--mode") mode = next_value(i, a);
        else if (a == "--threshold-table") threshold_table = next_value(i, a);
        else die(2, "[dgt] unknown option: %s", a.c_str());
    }
    if (mode != "both" && mode != "thresholds" && mode != "ground-truth")
        die(2, "[dgt] mode must be both, thresholds, or ground-truth");
    const bool build_thresholds = mode != "ground-truth";
    const bool build_ground_truth = mode != "thresholds";
    if (base_p.empty() || prefix.empty() || (build_ground_truth && query_p.empty())) {
        std::cerr << "usage: " << argv[0]
                  << " --base BASE.bin [--query QUERY.bin] --out_prefix PREFIX"
                  << " [--K 100] [--rk_k 10] [--tile 512] [--metric l2|ip]"
                  << " [--threads N] [--mode both|thresholds|ground-truth]"
                  << " [--threshold-table FILE]\n";
        return 2;
    }
    if (metric != "l2" && metric != "ip") die(2, "[dgt] metric must be l2 or ip");
    const uint32_t metric_code = metric == "ip" ? ANQI_METRIC_IP : ANQI_METRIC_L2;
    if (nthreads > (uint64_t)std::numeric_limits<int>::max()) die(2, "[dgt] thread count is too large");
    const int T = nthreads ? (int)nthreads : 1;
    const auto t_all = std::chrono::steady_clock::now();

    Fbin base = load_fbin_or_die(base_p);
    const uint64_t n = base.n, D = base.d;
    if (K >= n || rk_k > K) die(2, "[dgt] require rk_k <= K < base vector count");
    std::cout << "[dgt] mode=" << mode << " n=" << n << " D=" << D << " K=" << K << " rk_k=" << rk_k
              << " tile=" << tile << " threads=" << T << "\n";
    std::unique_ptr<Device> device;  // created when the first device stage runs
    auto dev = [&]() -> Device& {
        if (!device) device = std::make_unique<Device>("[dgt]");
        return *device;
    };

    std::vector<float> rk2(n);
    double threshold_build_s = 0.0;
    // From 20,000 rows the BF16 tensor-core tiles with FP32 recheck (outputs
    // equal to the FP32 CUDA-core path bit for bit); ANQI_B200_GT_TENSOR=0
    // keeps the FP32 path.
    const char* tenv = std::getenv("ANQI_B200_GT_TENSOR");
    const bool tensor = D <= 1024 && n >= 20000 && !(tenv && std::strcmp(tenv, "0") == 0);
    if (build_thresholds) {
        std::vector<uint32_t> ids(n * K);
        std::vector<float> keys(n * K);
        const auto t1 = std::chrono::steady_clock::now();
        dev().check(tensor ? anqi_exact_topk_tc_metric(dev().get(), base.x.data(), n, (uint32_t)D, (uint32_t)K, nullptr,
                                                       0, metric_code, ids.data(), keys.data())
                           : anqi_exact_topk_metric(dev().get(), base.x.data(), n, (uint32_t)D, (uint32_t)K,
                                                    metric_code, ids.data(), keys.data()),
                    "exact top-K");
        std::cout << "[dgt] base-to-base top-K done in "
                  << std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count() << "s\n";
        for (uint64_t i = 0; i < n; i++) rk2[i] = keys[i * K + rk_k - 1];
        {
            const std::string path = prefix + "_baseknn_gt.bin";
            const uint32_t un = (uint32_t)n, uk = (uint32_t)K;
            write_file_or_die(path, {{&un, 4}, {&uk, 4}, {ids.data(), n * K * 4}, {keys.data(), n * K * 4}}, 3,
                              "[dgt]");
            std::cout << "[dgt] wrote " << path << " (n*K = " << n << "*" << K << ")\n";
        }
        write_rk(prefix, n, rk_k, rk2);
        threshold_build_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_all).count();
        const std::string meta = prefix + "_threshold_build_time.meta";
        write_timing(meta, "ANQI_THRESHOLD_BUILD_V1",
                     {{"seconds", g17(threshold_build_s)},
                      {"metric", metric},
                      {"n", std::to_string(n)},
                      {"d", std::to_string(D)},
                      {"k", std::to_string(K)},
                      {"threads", std::to_string(T)}},
                     3, "[dgt]");
        std::cout << "[dgt] wrote " << meta << "\n";
        std::cout << "[dgt] THRESHOLD_BUILD_TIME=" << threshold_build_s << "s\n";
    } else {
        if (threshold_table.empty()) threshold_table = prefix + "_baseknn_gt.bin";
        rk2 = load_threshold_column(threshold_table, n, rk_k);
        std::cout << "[dgt] loaded rank-" << rk_k << " threshold column from " << threshold_table << "\n";
    }

    double ground_truth_s = 0.0;
    if (build_ground_truth) {
        Fbin query = load_fbin_or_die(query_p);
        if (query.d != D) die(3, "[dgt] base/query dimension mismatch: %" PRIu64 " != %u", D, query.d);
        const uint64_t nq = query.n;
        std::cout << "[dgt] nq=" << nq << "\n";
        const auto t2 = std::chrono::steady_clock::now();
        std::vector<uint32_t> off(nq + 1);
        uint64_t cap = std::max<uint64_t>(1 << 20, nq * 64), total = 0;
        std::vector<uint32_t> ids;
        std::vector<float> keys;
        for (int attempt = 0; attempt < 2; attempt++) {
            ids.resize(cap);
            keys.resize(cap);
            const int rc =
                tensor ? anqi_rknn_ground_truth_tc_metric(dev().get(), base.x.data(), n, query.x.data(), nq, (uint32_t)D,
                                                          rk2.data(), metric_code, off.data(), ids.data(), keys.data(),
                                                          cap, &total)
                       : anqi_rknn_ground_truth_metric(dev().get(), base.x.data(), n, query.x.data(), nq, (uint32_t)D,
                                                       rk2.data(), metric_code, off.data(), ids.data(), keys.data(), cap,
                                                       &total);
            if (rc == ANQI_ERR_CAPACITY && attempt == 0) {
                cap = total;
                continue;
            }
            dev().check(rc, "reverse-kNN ground truth");
            break;
        }
        ground_truth_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t2).count();
        std::cout << "[dgt] reverse-kNN membership done in " << ground_truth_s << "s\n";
        if (total > std::numeric_limits<uint32_t>::max()) die(3, "[dgt] reverse-kNN output exceeds uint32 CSR capacity");
        {
            const std::string path = prefix + "_rknn_gt.bin";
            const uint32_t unq = (uint32_t)nq;
            write_file_or_die(path, {{&unq, 4}, {off.data(), (nq + 1) * 4}, {ids.data(), total * 4},
                                     {keys.data(), total * 4}},
                              3, "[dgt]");
            std::cout << "[dgt] wrote " << path << " (total_pairs=" << off[nq]
                      << ", mean |R|=" << (double)off[nq] / (double)nq << ")\n";
        }
        if (!build_thresholds) write_rk(prefix, n, rk_k, rk2);
    }
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_all).count();
    std::cout << "[dgt] summary mode=" << mode << " threads=" << T << " threshold_build_time=" << threshold_build_s
              << "s ground_truth_time=" << ground_truth_s << "s total_time=" << secs << "s\n";
    return 0;
}

int main(int argc, char** argv) {
    try {
        return run(argc, argv);
    } catch (const Exit& e) {
        std::cerr << e.what() << "\n";
        return e.code;
    }
}
