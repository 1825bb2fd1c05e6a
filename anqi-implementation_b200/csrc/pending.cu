// Entry points whose kernels are still being written report ANQI_ERR_ARGS.
#include "internal.h"

using namespace anqi;

extern "C" {
#define PENDING(name, ...) \
    int name(anqi_ctx* h, __VA_ARGS__) { return h ? fail(&h->c, ANQI_ERR_ARGS, #name " is not available in this build") : ANQI_ERR_ARGS; }
PENDING(anqi_rp_forest, const float*, uint64_t, uint32_t, uint32_t, uint32_t, uint32_t, uint64_t, uint32_t, uint32_t*, uint32_t*, uint32_t*, float*, float*, uint32_t*, uint32_t*, uint32_t*)
PENDING(anqi_aknn_build, const float*, uint64_t, uint32_t, const anqi_aknn_params*, uint32_t*, float*, anqi_build_stats*)
PENDING(anqi_aknn_init, const float*, uint64_t, uint32_t, const uint64_t*, const uint32_t*, uint64_t, uint32_t, uint32_t*, float*)
PENDING(anqi_aknn_gather, const float*, uint64_t, uint32_t, const uint32_t*, const float*, uint32_t, uint32_t, uint32_t, uint32_t, uint32_t*, float*)
PENDING(anqi_graph_build, const float*, uint64_t, uint32_t, const uint32_t*, uint32_t, const anqi_graph_params*, uint32_t*, uint32_t*, anqi_build_stats*)
PENDING(anqi_graph_tree_size, uint32_t*, uint64_t*)
PENDING(anqi_graph_tree_copy, uint32_t*, uint32_t*, float*, float*, uint32_t*, uint32_t*, uint32_t*)
PENDING(anqi_graph_warm_start, const float*, uint64_t, uint32_t, const uint32_t*, uint32_t, uint32_t, uint32_t, uint32_t*, float*)
PENDING(anqi_graph_localjoin, const float*, uint64_t, uint32_t, uint32_t, uint32_t, uint32_t, uint32_t*, float*, uint64_t*, uint32_t*)
PENDING(anqi_graph_select, const float*, uint64_t, uint32_t, const uint32_t*, const float*, uint32_t, uint32_t, uint32_t, uint32_t, float, uint32_t*, uint32_t*)
PENDING(anqi_graph_commit, const float*, uint64_t, uint32_t, const uint32_t*, const uint32_t*, uint32_t, float, uint32_t*, uint32_t*)
PENDING(anqi_exact_topk, const float*, uint64_t, uint32_t, uint32_t, uint32_t*, float*)
PENDING(anqi_rknn_ground_truth, const float*, uint64_t, const float*, uint64_t, uint32_t, const float*, uint32_t*, uint32_t*, float*, uint64_t, uint64_t*)
}
