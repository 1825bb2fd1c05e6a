// build_aknn_source: the approximate base-space top-K source shared by ANQI's
// graph and verifier, built on the GPU.
//
//   build_aknn_source BASE.fbin OUTPUT_PREFIX [K=100] [leaf=500] [trees=64]
//                     [ef=600] [threads=64] [seed=10] [metric=l2]
//
// Same arguments, outputs and exit codes as tools/build_aknn_source.cpp:
//   2  usage / bad argument            3  unreadable base file or n <= K
//   4  row-count mismatch              5  invalid neighbour row
//   6  output write failure            7/8/9  device failure (library status)
// Outputs: PREFIX_baseknn_aknn.rec (n x K x {u32 id, f32 key}, key = max(0, d)
// for l2 and d - 1 = -<a, b> for ip, written to .part then renamed) and
// PREFIX_aknn_build_time.meta.  `threads` is recorded in the metadata; the
// device decides its own parallelism.  ANQI_NNITERS / ANQI_NNSAMPLE select
// NN-Descent rounds as in include/index.h:1312-1316 (metric l2 only: with ip
// and ANQI_NNITERS > 0 the tool exits 2).
#include "cli_common.h"

#include <algorithm>
#include <chrono>
#include <iostream>

using namespace anqi_cli;

static int run(int argc, char** argv) {
    if (argc < 3 || argc > 10) {
        std::cerr << "usage: " << argv[0]
                  << " BASE.fbin OUTPUT_PREFIX [K=100] [leaf=500]"
                     " [trees=64] [ef=600] [threads=64] [seed=10] [metric=l2]\n";
        return 2;
    }
    const std::string base_path = argv[1];
    const std::string prefix = argv[2];
    uint64_t k = 100, leaf = 500, trees = 64, ef = 600, threads = 64, seed = 10;
    uint64_t* slots[] = {&k, &leaf, &trees, &ef, &threads, &seed};
    for (int i = 3; i < argc && i < 9; i++)
        if (!parse_count(argv[i], *slots[i - 3])) die(2, "[aknn] invalid argument %d: %s", i, argv[i]);
    const std::string metric = argc > 9 ? argv[9] : "l2";
    if (metric != "l2" && metric != "ip") die(2, "[aknn] metric must be l2 or ip");
    if (k == 0 || leaf == 0 || trees == 0 || ef == 0) die(2, "[aknn] K, leaf, trees and ef must be positive");

    uint32_t hn = 0, hd = 0;
    if (!fbin_header(base_path, hn, hd) || hn <= k || hd == 0 || k > std::numeric_limits<uint32_t>::max())
        die(3, "[aknn] invalid base file or K: %s", base_path.c_str());

    const auto started = std::chrono::steady_clock::now();
    Fbin base;
    std::string why;
    if (!read_fbin(base_path, base, why)) die(3, "[aknn] invalid base file or K: %s (%s)", base_path.c_str(), why.c_str());
    const uint64_t n = base.n;
    const uint32_t d = base.d;

    Device dev("[aknn]");
    anqi_aknn_params p{};
    p.k = (uint32_t)k;
    p.leaf = (uint32_t)leaf;
    p.trees = (uint32_t)trees;
    p.ef = (uint32_t)ef;
    p.ef_alpha = 8;
    p.seed = seed;
    p.nn_iters = (uint32_t)std::max(0, std::atoi(env_or("ANQI_NNITERS", "0").c_str()));
    p.nn_sample = (uint32_t)std::min(std::max(0, std::atoi(env_or("ANQI_NNSAMPLE", "20").c_str())), 120);
    // init_knn distances: BF16 tensor-core tiles with FP32 recheck (default) or
    // FP32 CUDA cores; the lists are identical either way
    p.precision = env_or("ANQI_B200_PRECISION", "bf16") == "fp32" ? 0u : 1u;
    p.metric = metric == "ip" ? ANQI_METRIC_IP : ANQI_METRIC_L2;
    if (p.metric == ANQI_METRIC_IP && p.nn_iters > 0)
        die(2, "[aknn] ANQI_NNITERS > 0 is implemented for metric l2 only on this path");
    std::vector<uint32_t> ids(n * k);
    std::vector<float> dists(n * k);
    anqi_build_stats st{};
    dev.check(anqi_aknn_build(dev.get(), base.x.data(), n, d, &p, ids.data(), dists.data(), &st), "AKNN build");

    // Row validation, tools/build_aknn_source.cpp:94-116.
    for (uint64_t row = 0; row < n; ++row) {
        const uint32_t* r = ids.data() + row * k;
        const float* dr = dists.data() + row * k;
        for (uint64_t rank = 0; rank < k; ++rank) {
            if (r[rank] >= n || r[rank] == row) {
                std::cerr << "[aknn] invalid neighbor at row=" << row << " rank=" << rank << "\n";
                return 5;
            }
            for (uint64_t prev = 0; prev < rank; ++prev)
                if (r[prev] == r[rank]) {
                    std::cerr << "[aknn] duplicate neighbor at row=" << row << " rank=" << rank << "\n";
                    return 5;
                }
            if (rank != 0 && dr[rank] < dr[rank - 1]) {
                std::cerr << "[aknn] unsorted row=" << row << "\n";
                return 5;
            }
        }
    }

    const std::string record_path = prefix + "_baseknn_aknn.rec";
    const std::string record_tmp = record_path + ".part";
    {
        std::vector<TopKRecord> recs(n * k);
        // build_aknn_source.cpp:125-126
        for (uint64_t i = 0; i < n * k; i++)
            recs[i] = {ids[i], p.metric == ANQI_METRIC_IP ? dists[i] - 1.0f : std::max(0.0f, dists[i])};
        write_file_or_die(record_tmp, {{recs.data(), recs.size() * sizeof(TopKRecord)}}, 6, "[aknn]");
    }
    if (std::rename(record_tmp.c_str(), record_path.c_str()) != 0) {
        std::perror("rename");
        return 6;
    }

    const double elapsed = std::chrono::duration<double>(std::chrono::steady_clock::now() - started).count();
    const std::string timing_path = prefix + "_aknn_build_time.meta";
    write_timing(timing_path, "ANQI_AKNN_BUILD_V1",
                 {{"seconds", g17(elapsed)},
                  {"metric", metric},
                  {"n", std::to_string(n)},
                  {"d", std::to_string(d)},
                  {"k", std::to_string(k)},
                  {"leaf", std::to_string(leaf)},
                  {"trees", std::to_string(trees)},
                  {"ef", std::to_string(ef)},
                  {"threads", std::to_string(threads)},
                  {"seed", std::to_string(seed)}},
                 6, "[aknn]");

    std::cout << "[aknn] DONE n=" << n << " d=" << d << " K=" << k << " leaf=" << leaf << " trees=" << trees
              << " ef=" << ef << " threads=" << threads << " seed=" << seed << " metric=" << metric
              << " elapsed_s=" << elapsed << " peak_gb=" << peak_gb() << " source=" << record_path << "\n";
    std::cout << "[aknn] DEVICE_BREAKDOWN forest_ms=" << st.forest_ms << " init_ms=" << st.init_ms
              << " join_ms=" << st.join_ms << " reverse_ms=" << st.reverse_ms << " gather_ms=" << st.gather_ms
              << " total_ms=" << st.total_ms << "\n";
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
