// The persisted G48 graph + entry RP tree (nndindex::save_index / load_index /
// save_tree / load_tree, include/index.h:1810-1915) and the conversion of the
// device's breadth-first entry tree into the reference's post-order.
#pragma once

#include "cli_common.h"

#include <utility>

namespace anqi_cli {

// Entry tree in the persisted post-order (left subtree, right subtree, node;
// include/rptrees.h:127-152): children before parents, root last.  Leaves
// have left = right = ANQI_EMPTY and keep their member list.
struct PostTree {
    uint64_t leaf_size = 0;
    uint32_t dim = 0;
    std::vector<uint32_t> left, right;
    std::vector<float> offset;
    std::vector<float> hyper;          // nodes x dim, zero rows on leaves
    std::vector<uint64_t> leaf_off;    // nodes + 1 into indices
    std::vector<uint32_t> indices;
    uint32_t nodes() const { return (uint32_t)left.size(); }
    uint64_t leaves() const {
        uint64_t c = 0;
        for (uint32_t v : left) c += v == ANQI_EMPTY;
        return c;
    }
    std::vector<uint32_t> leaf_first() const {
        std::vector<uint32_t> f(nodes(), ANQI_EMPTY);
        for (uint32_t i = 0; i < nodes(); i++)
            if (leaf_off[i + 1] > leaf_off[i]) f[i] = indices[leaf_off[i]];
        return f;
    }
};

// Breadth-first arrays from anqi_graph_tree_copy -> post-order.
inline PostTree bfs_to_postorder(const std::vector<uint32_t>& left, const std::vector<uint32_t>& right,
                                 const std::vector<float>& offset, const std::vector<float>& hyper,
                                 const std::vector<uint32_t>& leaf_off, const std::vector<uint32_t>& leaf_cnt,
                                 const std::vector<uint32_t>& perm, uint64_t leaf_size, uint32_t dim) {
    const uint32_t nn = (uint32_t)left.size();
    std::vector<uint32_t> order;
    order.reserve(nn);
    std::vector<std::pair<uint32_t, bool>> stack{{0u, false}};
    while (!stack.empty()) {
        const auto [v, done] = stack.back();
        stack.pop_back();
        if (left[v] == ANQI_EMPTY || done) {
            order.push_back(v);
            continue;
        }
        stack.push_back({v, true});
        stack.push_back({right[v], false});
        stack.push_back({left[v], false});
    }
    std::vector<uint32_t> newid(nn, ANQI_EMPTY);
    for (uint32_t i = 0; i < (uint32_t)order.size(); i++) newid[order[i]] = i;
    PostTree t;
    t.leaf_size = leaf_size;
    t.dim = dim;
    const uint32_t m = (uint32_t)order.size();
    t.left.resize(m);
    t.right.resize(m);
    t.offset.resize(m);
    t.hyper.assign((size_t)m * dim, 0.0f);
    t.leaf_off.assign(m + 1, 0);
    for (uint32_t j = 0; j < m; j++) {
        const uint32_t o = order[j];
        const bool leaf = left[o] == ANQI_EMPTY;
        t.left[j] = leaf ? ANQI_EMPTY : newid[left[o]];
        t.right[j] = leaf ? ANQI_EMPTY : newid[right[o]];
        t.offset[j] = leaf ? std::numeric_limits<float>::max() : offset[o];
        if (!leaf) std::copy(hyper.begin() + (size_t)o * dim, hyper.begin() + (size_t)(o + 1) * dim,
                             t.hyper.begin() + (size_t)j * dim);
        t.leaf_off[j + 1] = t.leaf_off[j] + (leaf ? leaf_cnt[o] : 0);
    }
    t.indices.resize(t.leaf_off[m]);
    for (uint32_t j = 0; j < m; j++) {
        const uint32_t o = order[j];
        if (left[o] != ANQI_EMPTY) continue;
        std::copy(perm.begin() + leaf_off[o], perm.begin() + leaf_off[o] + leaf_cnt[o],
                  t.indices.begin() + t.leaf_off[j]);
    }
    return t;
}

// [size_t n, dim, M][f32 ctime]{u32 deg, deg x u32}, then the tree:
// [size_t leaf_size, n_leaves, n_nodes] and per node
// [size_t left, right][f32 offset][size_t hs][hs f32][size_t is][is u32].
inline bool write_graph(const std::string& path, uint64_t n, uint64_t dim, uint64_t M, float ctime,
                        const std::vector<uint32_t>& deg, const std::vector<uint32_t>& links, const PostTree& t) {
    std::ofstream f(path, std::ios::binary | std::ios::trunc);
    if (!f) return false;
    auto put = [&](const void* p, size_t b) { f.write(static_cast<const char*>(p), (std::streamsize)b); };
    put(&n, 8);
    put(&dim, 8);
    put(&M, 8);
    put(&ctime, 4);
    for (uint64_t i = 0; i < n; i++) {
        put(&deg[i], 4);
        put(links.data() + i * M, deg[i] * 4ull);
    }
    const uint64_t ls = t.leaf_size, nl = t.leaves(), ns = t.nodes();
    put(&ls, 8);
    put(&nl, 8);
    put(&ns, 8);
    for (uint32_t i = 0; i < t.nodes(); i++) {
        const bool leaf = t.left[i] == ANQI_EMPTY;
        const uint64_t l = leaf ? 0xFFFFFFFFull : t.left[i], r = leaf ? 0xFFFFFFFFull : t.right[i];
        put(&l, 8);
        put(&r, 8);
        put(&t.offset[i], 4);
        const uint64_t hs = leaf ? 0 : t.dim;
        put(&hs, 8);
        if (hs) put(t.hyper.data() + (size_t)i * t.dim, hs * 4);
        const uint64_t is = t.leaf_off[i + 1] - t.leaf_off[i];
        put(&is, 8);
        if (is) put(t.indices.data() + t.leaf_off[i], is * 4);
    }
    f.close();
    return (bool)f;
}

// load_index + load_tree with the reference's validation; why names the failure.
inline bool read_graph(const std::string& path, uint64_t n, uint64_t dim, uint64_t M, std::vector<uint32_t>& deg,
                       std::vector<uint32_t>& links, PostTree& t, float& ctime, std::string& why) {
    std::ifstream f(path, std::ios::binary);
    if (!f.good()) {
        why = "no cached index: " + path;
        return false;
    }
    auto get = [&](void* p, size_t b) { return (bool)f.read(static_cast<char*>(p), (std::streamsize)b); };
    uint64_t fn = 0, fdim = 0, fM = 0;
    if (!get(&fn, 8) || !get(&fdim, 8) || !get(&fM, 8) || !get(&ctime, 4) || fn != n || fdim != dim || fM != M ||
        !std::isfinite(ctime)) {
        why = "incompatible or truncated cached index: " + path;
        return false;
    }
    deg.assign(n, 0);
    links.assign(n * M, ANQI_EMPTY);
    for (uint64_t i = 0; i < n; i++) {
        uint32_t d = 0;
        if (!get(&d, 4) || d > M || !get(links.data() + i * M, d * 4ull)) {
            why = "invalid adjacency data in cached index: " + path;
            return false;
        }
        for (uint32_t j = 0; j < d; j++)
            if (links[i * M + j] >= n) {
                why = "invalid neighbor id in cached index: " + path;
                return false;
            }
        deg[i] = d;
    }
    uint64_t leaf_size = 0, n_leaves = 0, ns = 0;
    const std::string bad = "invalid RP tree in cached index: " + path;
    if (!get(&leaf_size, 8) || !get(&n_leaves, 8) || !get(&ns, 8) || leaf_size == 0 || leaf_size > 1000000 ||
        n_leaves == 0 || n_leaves > n || ns == 0 || ns > 2 * n) {
        why = bad;
        return false;
    }
    t = PostTree{};
    t.leaf_size = leaf_size;
    t.dim = (uint32_t)dim;
    t.left.resize(ns);
    t.right.resize(ns);
    t.offset.resize(ns);
    t.hyper.assign(ns * dim, 0.0f);
    t.leaf_off.assign(ns + 1, 0);
    for (uint64_t i = 0; i < ns; i++) {
        uint64_t l = 0, r = 0, hs = 0, is = 0;
        float off = 0;
        if (!get(&l, 8) || !get(&r, 8) || !get(&off, 4) || !get(&hs, 8) || hs > dim || !std::isfinite(off)) {
            why = bad;
            return false;
        }
        if (hs && !get(t.hyper.data() + i * dim, hs * 4)) {
            why = bad;
            return false;
        }
        if (!get(&is, 8) || is > n) {
            why = bad;
            return false;
        }
        const size_t at = t.indices.size();
        t.indices.resize(at + is);
        if (is && !get(t.indices.data() + at, is * 4)) {
            why = bad;
            return false;
        }
        const bool leaf = l == 0xFFFFFFFFull && r == 0xFFFFFFFFull;
        const bool internal = l < i && r < i;
        if ((!leaf && !internal) || (leaf && is == 0) || (internal && hs != dim)) {
            why = bad;
            return false;
        }
        for (size_t j = at; j < at + is; j++)
            if (t.indices[j] >= n) {
                why = bad;
                return false;
            }
        t.left[i] = leaf ? ANQI_EMPTY : (uint32_t)l;
        t.right[i] = leaf ? ANQI_EMPTY : (uint32_t)r;
        t.offset[i] = off;
        t.leaf_off[i + 1] = t.leaf_off[i] + is;
    }
    return true;
}

}  // namespace anqi_cli
