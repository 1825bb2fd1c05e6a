// Random-projection forest, built level by level on the device.
//
// Reference: random_projection_split / build_rptree_recursively / make_forest,
// include/rptrees.h:28-84,127-186.  Differences by design: the two pivot points
// and the tie sides come from a counter hash of (seed, tree, node, point) instead
// of a thread-local mt19937, so a forest is reproducible for any parallelism, and
// nodes are numbered breadth-first (the persisted post-order is produced on the
// host).  Everything else follows the reference: hyperplane x0 - x1 through the
// midpoint, margin = ip(h, x) - h.mid in the AVX lane order, |margin| <= 1e-6
// takes a hashed side, an all-one-side split falls back to hashed halves, a
// segment of <= leaf points (or at max_depth, truncated to leaf points) is a
// leaf, and partitions are stable.
//
// All trees advance together: per level, one warp per splitting node builds
// its hyperplane; 4-thread groups compute point margins over fixed-size chunks
// of the segments; a stable partition per chunk places points using per-chunk
// prefix counts.  The host only keeps the small per-node records.
#include <algorithm>
#include <cfloat>

#include "internal.h"
#include "util.cuh"

namespace anqi {

constexpr uint32_t kChunk = 2048;

struct SplitNode {
    uint32_t tree, local, start, count;
};
struct Chunk {
    uint32_t node, begin, len, pad;
};

__device__ __forceinline__ uint64_t node_key(uint64_t seed, uint32_t tree, uint32_t node) {
    return hash64(hash64(seed ^ ((uint64_t)tree << 32)) ^ (uint64_t)node);
}

// One warp per splitting node: pivots, hyperplane, midpoint, offset.  The
// angular form (the ip metric, rptrees.h:41-52) splits through the origin by
// the normalized difference of the unit-scaled pivots: x0/|x0| - x1/|x1|,
// divided by its norm; a norm below 1e-6 counts as 1.
__global__ void forest_hyperplane_kernel(const float* __restrict__ x, uint32_t stride, uint32_t dim, uint64_t n,
                                         const uint32_t* __restrict__ perm, const SplitNode* __restrict__ nodes,
                                         uint32_t n_split, uint64_t seed, uint32_t cap_nodes,
                                         float* __restrict__ hyper, float* __restrict__ mid,
                                         float* __restrict__ offset, int angular) {
    const uint32_t lane = threadIdx.x & 31u, gt = lane & 3u;
    const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (w >= n_split) return;
    const SplitNode nd = nodes[w];
    const uint64_t key = node_key(seed, nd.tree, nd.local);
    uint32_t r0 = (uint32_t)(hash64(key ^ 1) % nd.count);
    const uint32_t r1 = (uint32_t)(hash64(key ^ 2) % nd.count);
    if (r0 == r1) r0 = (r1 + 1) % nd.count;
    const uint32_t* pt = perm + (uint64_t)nd.tree * n + nd.start;
    const float* x0 = x + (uint64_t)pt[r0] * stride;
    const float* x1 = x + (uint64_t)pt[r1] * stride;
    float* hp = hyper + ((uint64_t)nd.tree * cap_nodes + nd.local) * stride;
    float* md = mid + (uint64_t)w * stride;
    if (angular) {
        float n0 = __fsqrt_rn(group_ip(x0, x0, dim, gt, kAll));
        float n1 = __fsqrt_rn(group_ip(x1, x1, dim, gt, kAll));
        if (fabsf(n0) < kSplitEps) n0 = 1.0f;
        if (fabsf(n1) < kSplitEps) n1 = 1.0f;
        for (uint32_t j = lane; j < stride; j += 32)
            hp[j] = j < dim ? __fsub_rn(__fdiv_rn(x0[j], n0), __fdiv_rn(x1[j], n1)) : 0.f;
        __syncwarp();
        float hn = __fsqrt_rn(group_ip(hp, hp, dim, gt, kAll));
        if (fabsf(hn) < kSplitEps) hn = 1.0f;
        __syncwarp();
        for (uint32_t j = lane; j < dim; j += 32) hp[j] = __fdiv_rn(hp[j], hn);
        if (lane == 0) offset[w] = 0.0f;
        return;
    }
    for (uint32_t j = lane; j < stride; j += 32) {
        const bool in = j < dim;
        hp[j] = in ? __fsub_rn(x0[j], x1[j]) : 0.f;
        md[j] = in ? __fdiv_rn(__fadd_rn(x0[j], x1[j]), 2.0f) : 0.f;
    }
    __syncwarp();
    const float off = group_ip(hp, md, dim, gt, kAll);
    if (lane == 0) offset[w] = off;
}

// Sides for every point of every chunk; counts lefts per chunk.
__global__ void forest_sides_kernel(const float* __restrict__ x, uint32_t stride, uint32_t dim, uint64_t n,
                                    const uint32_t* __restrict__ perm, const SplitNode* __restrict__ nodes,
                                    const Chunk* __restrict__ chunks, uint64_t seed, uint32_t cap_nodes,
                                    const float* __restrict__ hyper, const float* __restrict__ offset,
                                    uint8_t* __restrict__ side, uint32_t* __restrict__ chunk_left, int fallback) {
    __shared__ uint32_t s_cnt;
    const Chunk ch = chunks[blockIdx.x];
    const SplitNode nd = nodes[ch.node];
    const uint64_t key = node_key(seed, nd.tree, nd.local);
    const uint32_t* pt = perm + (uint64_t)nd.tree * n + nd.start;
    uint8_t* sd = side + (uint64_t)nd.tree * n + nd.start;
    const float* hp = hyper + ((uint64_t)nd.tree * cap_nodes + nd.local) * stride;
    const float off = offset[ch.node];
    if (threadIdx.x == 0) s_cnt = 0;
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31u, gt = lane & 3u;
    const uint32_t group = threadIdx.x >> 2, ngroups = blockDim.x >> 2;
    uint32_t lefts = 0;
    // all lanes of a warp iterate together (group shuffles need convergence)
    const uint32_t iters = (ch.len + ngroups - 1) / ngroups;
    for (uint32_t it = 0; it < iters; it++) {
        const uint32_t p = ch.begin + it * ngroups + group;
        const bool ok = p < ch.begin + ch.len;
        const uint32_t id = pt[ok ? p : ch.begin];
        uint8_t s;
        if (fallback) {
            s = (uint8_t)(hash64(key ^ (((uint64_t)id << 2) | 2)) & 1);
        } else {
            const float ip = group_ip(hp, x + (uint64_t)id * stride, dim, gt, kAll);
            const float m = __fsub_rn(ip, off);
            if (m < -kSplitEps) s = 0;
            else if (m > kSplitEps) s = 1;
            else s = (uint8_t)(hash64(key ^ (((uint64_t)id << 2) | 3)) & 1);
        }
        if (ok && gt == 0) {
            sd[p] = s;
            lefts += (s == 0);
        }
    }
    for (int o = 16; o > 0; o >>= 1) lefts += __shfl_xor_sync(kAll, lefts, o);
    if (lane == 0) atomicAdd(&s_cnt, lefts);
    __syncthreads();
    if (threadIdx.x == 0) chunk_left[blockIdx.x] = s_cnt;
}

// Stable partition of each chunk into tmp; lprefix = lefts in earlier chunks
// of the node, nleft = lefts of the node.
__global__ void forest_partition_kernel(uint64_t n, const uint32_t* __restrict__ perm, const SplitNode* __restrict__ nodes,
                                        const Chunk* __restrict__ chunks, const uint32_t* __restrict__ lprefix,
                                        const uint32_t* __restrict__ nleft, const uint8_t* __restrict__ side,
                                        uint32_t* __restrict__ tmp) {
    __shared__ uint32_t s_warp[32];
    __shared__ uint32_t s_run;
    const Chunk ch = chunks[blockIdx.x];
    const SplitNode nd = nodes[ch.node];
    const uint32_t* pt = perm + (uint64_t)nd.tree * n + nd.start;
    const uint8_t* sd = side + (uint64_t)nd.tree * n + nd.start;
    uint32_t* out = tmp + (uint64_t)nd.tree * n + nd.start;
    const uint32_t nl = nleft[ch.node];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (threadIdx.x == 0) s_run = 0;
    __syncthreads();
    for (uint32_t b0 = 0; b0 < ch.len; b0 += blockDim.x) {
        const uint32_t p = ch.begin + b0 + threadIdx.x;
        const bool ok = p < ch.begin + ch.len;
        const bool is_left = ok && sd[p] == 0;
        const unsigned bal = __ballot_sync(kAll, is_left);
        if (lane == 0) s_warp[warp] = __popc(bal);
        __syncthreads();
        uint32_t before = 0, total = 0;
        for (uint32_t w = 0; w < nw; w++) {
            if (w < warp) before += s_warp[w];
            total += s_warp[w];
        }
        const uint32_t run = s_run;
        const uint32_t lrank = run + before + __popc(bal & lane_lt_mask());
        if (ok) {
            const uint32_t lbefore = lprefix[blockIdx.x] + lrank;  // lefts before p within the node
            const uint32_t rbefore = (p - 0) - lbefore;              // rights before p within the node
            const uint32_t dst = is_left ? lbefore : nl + rbefore;
            out[dst] = pt[p];
        }
        __syncthreads();
        if (threadIdx.x == 0) s_run = run + total;
        __syncthreads();
    }
}

__global__ void forest_copyback_kernel(uint64_t n, uint32_t* __restrict__ perm, const SplitNode* __restrict__ nodes,
                                       const Chunk* __restrict__ chunks, const uint32_t* __restrict__ tmp) {
    const Chunk ch = chunks[blockIdx.x];
    const SplitNode nd = nodes[ch.node];
    const uint64_t base = (uint64_t)nd.tree * n + nd.start;
    for (uint32_t p = ch.begin + threadIdx.x; p < ch.begin + ch.len; p += blockDim.x) perm[base + p] = tmp[base + p];
}

__global__ void iota_trees_kernel(uint32_t* perm, uint64_t n, uint32_t trees) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < n * trees;
         t += (uint64_t)gridDim.x * blockDim.x)
        perm[t] = (uint32_t)(t % n);
}

int build_forest(Ctx* c, const float* d_x, uint64_t n, uint32_t dim, uint32_t stride, uint32_t trees,
                 uint32_t leaf, uint32_t max_depth, uint64_t seed, uint32_t cap_nodes, ForestOut& out, int angular) {
    if (n == 0 || trees == 0 || leaf == 0 || cap_nodes < 1) return fail(c, ANQI_ERR_ARGS, "invalid forest arguments");
    if (n >= 0xFFFFFFFFull) return fail(c, ANQI_ERR_ARGS, "forest needs n < 2^32");
    out.trees = trees;
    out.cap_nodes = cap_nodes;
    out.n = n;
    out.dim = dim;
    out.stride = stride;
    const size_t tot_nodes = (size_t)trees * cap_nodes;
    out.left.assign(tot_nodes, kEmpty);
    out.right.assign(tot_nodes, kEmpty);
    out.offset.assign(tot_nodes, FLT_MAX);
    out.leaf_off.assign(tot_nodes, kEmpty);
    out.leaf_cnt.assign(tot_nodes, 0);
    out.n_nodes.assign(trees, 1);
    int rc;
    if ((rc = ensure(c, out.perm, (size_t)trees * n * 4)) || (rc = ensure(c, out.hyper, tot_nodes * stride * 4)))
        return rc;
    TmpBuf tmp(c), side(c), dnodes(c), dchunks(c), dmid(c), doff(c), dleft(c), dpre(c), dnl(c);
    if ((rc = ensure(c, tmp, (size_t)trees * n * 4)) || (rc = ensure(c, side, (size_t)trees * n)))
        return rc;
    iota_trees_kernel<<<c->sm_count * 8, 256, 0, c->stream>>>(out.perm.as<uint32_t>(), n, trees);
    ANQI_CUDA(c, cudaGetLastError());
    struct Active {
        uint32_t tree, local, start, count, depth;
    };
    std::vector<Active> active;
    for (uint32_t t = 0; t < trees; t++) active.push_back({t, 0, 0, (uint32_t)n, 0});
    std::vector<uint32_t> next_local(trees, 1);
    for (uint32_t level = 0; !active.empty(); level++) {
        std::vector<SplitNode> split;
        std::vector<uint32_t> split_depth;
        for (const Active& a : active) {
            const size_t g = (size_t)a.tree * cap_nodes + a.local;
            if (a.count <= leaf || a.depth >= max_depth) {
                out.left[g] = out.right[g] = kEmpty;
                out.offset[g] = FLT_MAX;
                out.leaf_off[g] = a.start;
                out.leaf_cnt[g] = std::min(a.count, leaf);
            } else {
                if (next_local[a.tree] + 2 > cap_nodes)
                    return fail(c, ANQI_ERR_CAPACITY, "RP tree node capacity %u exceeded", cap_nodes);
                split.push_back({a.tree, a.local, a.start, a.count});
                split_depth.push_back(a.depth);
            }
        }
        if (split.empty()) break;
        const uint32_t ns = (uint32_t)split.size();
        std::vector<Chunk> chunks;
        for (uint32_t s = 0; s < ns; s++)
            for (uint32_t b = 0; b < split[s].count; b += kChunk)
                chunks.push_back({s, b, std::min(kChunk, split[s].count - b), 0});
        const uint32_t nc = (uint32_t)chunks.size();
        if ((rc = h2d(c, dnodes, split.data(), ns * sizeof(SplitNode))) ||
            (rc = h2d(c, dchunks, chunks.data(), nc * sizeof(Chunk))) ||
            (rc = ensure(c, dmid, (size_t)ns * stride * 4)) || (rc = ensure(c, doff, ns * 4)) ||
            (rc = ensure(c, dleft, nc * 4)) || (rc = ensure(c, dpre, nc * 4)) || (rc = ensure(c, dnl, ns * 4)))
            return rc;
        forest_hyperplane_kernel<<<(ns + 3) / 4, 128, 0, c->stream>>>(
            d_x, stride, dim, n, out.perm.as<uint32_t>(), dnodes.as<SplitNode>(), ns, seed, cap_nodes,
            out.hyper.as<float>(), dmid.as<float>(), doff.as<float>(), angular);
        forest_sides_kernel<<<nc, 256, 0, c->stream>>>(d_x, stride, dim, n, out.perm.as<uint32_t>(),
                                                       dnodes.as<SplitNode>(), dchunks.as<Chunk>(), seed, cap_nodes,
                                                       out.hyper.as<float>(), doff.as<float>(), side.as<uint8_t>(),
                                                       dleft.as<uint32_t>(), 0);
        ANQI_CUDA(c, cudaGetLastError());
        std::vector<uint32_t> cl(nc);
        std::vector<float> offs(ns);
        if ((rc = d2h(c, cl.data(), dleft, nc * 4)) || (rc = d2h(c, offs.data(), doff, ns * 4)) || (rc = sync(c)))
            return rc;
        std::vector<uint32_t> nl(ns, 0);
        for (uint32_t k = 0; k < nc; k++) nl[chunks[k].node] += cl[k];
        std::vector<Chunk> fb;
        std::vector<uint32_t> fb_idx;
        for (uint32_t k = 0; k < nc; k++) {
            const uint32_t s = chunks[k].node;
            if (nl[s] == 0 || nl[s] == split[s].count) {
                fb.push_back(chunks[k]);
                fb_idx.push_back(k);
            }
        }
        if (!fb.empty()) {
            TmpBuf dfb(c), dfl(c);
            if ((rc = h2d(c, dfb, fb.data(), fb.size() * sizeof(Chunk))) || (rc = ensure(c, dfl, fb.size() * 4)))
                return rc;
            forest_sides_kernel<<<(unsigned)fb.size(), 256, 0, c->stream>>>(
                d_x, stride, dim, n, out.perm.as<uint32_t>(), dnodes.as<SplitNode>(), dfb.as<Chunk>(), seed, cap_nodes,
                out.hyper.as<float>(), doff.as<float>(), side.as<uint8_t>(), dfl.as<uint32_t>(), 1);
            ANQI_CUDA(c, cudaGetLastError());
            std::vector<uint32_t> fl(fb.size());
            if ((rc = d2h(c, fl.data(), dfl, fb.size() * 4)) || (rc = sync(c))) return rc;
            for (size_t k = 0; k < fb.size(); k++) cl[fb_idx[k]] = fl[k];
            std::fill(nl.begin(), nl.end(), 0);
            for (uint32_t k = 0; k < nc; k++) nl[chunks[k].node] += cl[k];
        }
        std::vector<uint32_t> pre(nc);
        {
            std::vector<uint32_t> run(ns, 0);
            for (uint32_t k = 0; k < nc; k++) {
                pre[k] = run[chunks[k].node];
                run[chunks[k].node] += cl[k];
            }
        }
        if ((rc = h2d(c, dpre, pre.data(), nc * 4)) || (rc = h2d(c, dnl, nl.data(), ns * 4))) return rc;
        forest_partition_kernel<<<nc, 256, 0, c->stream>>>(n, out.perm.as<uint32_t>(), dnodes.as<SplitNode>(),
                                                           dchunks.as<Chunk>(), dpre.as<uint32_t>(),
                                                           dnl.as<uint32_t>(), side.as<uint8_t>(), tmp.as<uint32_t>());
        forest_copyback_kernel<<<nc, 256, 0, c->stream>>>(n, out.perm.as<uint32_t>(), dnodes.as<SplitNode>(),
                                                          dchunks.as<Chunk>(), tmp.as<uint32_t>());
        ANQI_CUDA(c, cudaGetLastError());
        std::vector<Active> next;
        for (uint32_t s = 0; s < ns; s++) {
            const SplitNode& sn = split[s];
            const size_t g = (size_t)sn.tree * cap_nodes + sn.local;
            const uint32_t L = next_local[sn.tree]++, R = next_local[sn.tree]++;
            out.left[g] = L;
            out.right[g] = R;
            out.offset[g] = offs[s];
            out.leaf_off[g] = kEmpty;
            out.leaf_cnt[g] = 0;
            next.push_back({sn.tree, L, sn.start, nl[s], split_depth[s] + 1});
            next.push_back({sn.tree, R, sn.start + nl[s], sn.count - nl[s], split_depth[s] + 1});
        }
        // `next` is already in (tree, local) order, breadth-first per tree: the
        // splits come in that order and each takes the next two numbers of its tree
        active.swap(next);
    }
    for (uint32_t t = 0; t < trees; t++) out.n_nodes[t] = next_local[t];
    return sync(c);
}

}  // namespace anqi

using namespace anqi;

extern "C" int anqi_rp_forest(anqi_ctx* h, const float* x, uint64_t n, uint32_t dim, uint32_t trees,
                              uint32_t leaf_size, uint32_t max_depth, uint64_t seed, uint32_t cap_nodes,
                              uint32_t* n_nodes, uint32_t* left, uint32_t* right, float* offset, float* hyperplane,
                              uint32_t* leaf_off, uint32_t* leaf_cnt, uint32_t* perm) {
    return anqi_rp_forest_metric(h, x, n, dim, trees, leaf_size, max_depth, seed, cap_nodes, ANQI_METRIC_L2, n_nodes,
                                 left, right, offset, hyperplane, leaf_off, leaf_cnt, perm);
}

extern "C" int anqi_rp_forest_metric(anqi_ctx* h, const float* x, uint64_t n, uint32_t dim, uint32_t trees,
                                     uint32_t leaf_size, uint32_t max_depth, uint64_t seed, uint32_t cap_nodes,
                                     uint32_t metric, uint32_t* n_nodes, uint32_t* left, uint32_t* right,
                                     float* offset, float* hyperplane, uint32_t* leaf_off, uint32_t* leaf_cnt,
                                     uint32_t* perm) {
    if (!h || !x || !n_nodes || !left || !right || !offset || !hyperplane || !leaf_off || !leaf_cnt || !perm ||
        dim == 0 || metric > ANQI_METRIC_IP)
        return ANQI_ERR_ARGS;
    Ctx* c = &h->c;
    cudaSetDevice(c->device);
    const uint32_t stride = round_up(dim, 8);
    TmpBuf dx(c);
    int rc = upload_padded(c, dx, x, n, dim, stride);
    if (rc) return rc;
    ForestOut f;
    rc = build_forest(c, dx.as<float>(), n, dim, stride, trees, leaf_size, max_depth, seed, cap_nodes, f,
                      metric == ANQI_METRIC_IP);
    if (rc) {
        release(c, f.perm);
        release(c, f.hyper);
        return rc;
    }
    std::memcpy(n_nodes, f.n_nodes.data(), trees * 4);
    std::memcpy(left, f.left.data(), f.left.size() * 4);
    std::memcpy(right, f.right.data(), f.right.size() * 4);
    std::memcpy(offset, f.offset.data(), f.offset.size() * 4);
    std::memcpy(leaf_off, f.leaf_off.data(), f.leaf_off.size() * 4);
    std::memcpy(leaf_cnt, f.leaf_cnt.data(), f.leaf_cnt.size() * 4);
    ANQI_CUDA(c, cudaMemcpy2DAsync(hyperplane, dim * 4, f.hyper.p, stride * 4, dim * 4, (size_t)trees * cap_nodes,
                                   cudaMemcpyDeviceToHost, c->stream));
    rc = d2h(c, perm, f.perm, (size_t)trees * n * 4);
    if (!rc) rc = sync(c);
    // internal (never written) hyperplane rows of leaves are zero on the host side
    for (size_t g = 0; g < (size_t)trees * cap_nodes; g++)
        if (f.left[g] == kEmpty) std::memset(hyperplane + g * dim, 0, dim * 4);
    release(c, f.perm);
    release(c, f.hyper);
    return rc;
}
