"""GPU parity of the index-construction stages (sm_100a, via the C ABI).

Bit-exact against the reference goldens where the reference is deterministic
given its stage inputs (warm start, gather + prune, commit, AKNN gather, exact
ground truth), bit-exact against the oracle's restatement for the GPU's own
deterministic forms (forest, snapshot LocalJoin, init_knn), and statistical
for the end-to-end builds (the reference itself is nondeterministic there)."""
from pathlib import Path

import numpy as np
import pytest

import oracle_lib as ol
from anqi import formats
from anqi._lib import Context, AknnParams, GraphParams, BuildStats
import ctypes as C

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
EMPTY = 0xFFFFFFFF


@pytest.fixture(scope="module")
def ctx():
    with Context(0) as c:
        yield c


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def csr_rows(off, ids):
    return [ids[int(off[i]):int(off[i + 1])] for i in range(len(off) - 1)]


def f32(a):
    return np.ascontiguousarray(a, np.float32)


def u32(a):
    return np.ascontiguousarray(a, np.uint32)


def warm_start(ctx, x, cand, width, K):
    x = f32(x)
    cand = u32(cand)
    n, dim = x.shape
    ids = np.empty((n, K), np.uint32)
    vals = np.empty((n, K), np.float32)
    ctx._check(ctx.lib.anqi_graph_warm_start(ctx.h, x, n, dim, cand, cand.shape[1], width, K, ids, vals), "warm")
    return ids, vals


def localjoin(ctx, x, ids, vals, sample=20, rounds=6):
    x = f32(x)
    ids = u32(ids).copy()
    vals = f32(vals).copy()
    n, dim = x.shape
    up = np.zeros(rounds, np.uint64)
    done = C.c_uint32()
    ctx._check(ctx.lib.anqi_graph_localjoin(ctx.h, x, n, dim, ids.shape[1], sample, rounds, ids, vals, up,
                                            C.byref(done)), "localjoin")
    return ids, vals, [int(u) for u in up[:done.value]]


def select(ctx, x, ids, vals, M=48, ef=100, cap=800, alpha=1.2):
    x = f32(x)
    n, dim = x.shape
    O = np.empty((n, M), np.uint32)
    Od = np.empty(n, np.uint32)
    ctx._check(ctx.lib.anqi_graph_select(ctx.h, x, n, dim, u32(ids), f32(vals), ids.shape[1], M, ef, cap, alpha, O,
                                         Od), "select")
    return O, Od


def commit(ctx, x, O, Od, alpha=1.2):
    x = f32(x)
    n, dim = x.shape
    M = O.shape[1]
    links = np.empty((n, M), np.uint32)
    deg = np.empty(n, np.uint32)
    ctx._check(ctx.lib.anqi_graph_commit(ctx.h, x, n, dim, u32(O), u32(Od), M, alpha, links, deg), "commit")
    return links, deg


def aknn_gather(ctx, x, ids, vals, ef, cap, out_k=100):
    x = f32(x)
    n, dim = x.shape
    oi = np.empty((n, out_k), np.uint32)
    od = np.empty((n, out_k), np.float32)
    ctx._check(ctx.lib.anqi_aknn_gather(ctx.h, x, n, dim, u32(ids), f32(vals), ids.shape[1], ef, cap, out_k, oi, od),
               "gather")
    return oi, od


def aknn_init(ctx, x, leaf_off, leaves, K):
    x = f32(x)
    n, dim = x.shape
    oi = np.empty((n, K), np.uint32)
    od = np.empty((n, K), np.float32)
    ctx._check(ctx.lib.anqi_aknn_init(ctx.h, x, n, dim, np.ascontiguousarray(leaf_off, np.uint64), u32(leaves),
                                      len(leaf_off) - 1, K, oi, od), "init")
    return oi, od


def test_warm_start_bit_exact(ctx, sample):
    ids, vals = warm_start(ctx, sample["lifted"], sample["rec_ids"], 100, 50)
    assert np.array_equal(ids, sample["g_warm_ids"])
    assert np.array_equal(bits(vals), bits(sample["g_warm_vals"]))


def test_localjoin_matches_oracle_snapshot_form(ctx, sample):
    x = sample["lifted"]
    ids, vals, ups = localjoin(ctx, x, sample["g_warm_ids"], sample["g_warm_vals"])
    oi, ov, oups = ol.localjoin(x, ol.norms(x), sample["g_warm_ids"], sample["g_warm_vals"])
    assert ups == oups
    assert np.array_equal(ids, oi)
    assert np.array_equal(bits(vals), bits(ov))


def test_select_commit_bit_exact(ctx, sample):
    x = sample["lifted"]
    O, Od = select(ctx, x, sample["g_join_ids"], sample["g_join_vals"])
    ref_O = csr_rows(sample["g_O_off"], sample["g_O"])
    for i in range(256):
        assert list(O[i, :Od[i]]) == list(ref_O[i]), i
    links, deg = commit(ctx, x, O, Od)
    ref_adj = csr_rows(sample["g_adj_off"], sample["g_adj"])
    for i in range(256):
        assert list(links[i, :deg[i]]) == list(ref_adj[i]), i


def test_aknn_gather_bit_exact(ctx, sample):
    # sample: ef = 64 < K + 1 -> pool top-K path
    ids, d = aknn_gather(ctx, sample["base"], sample["a_init_ids"], sample["a_init_vals"], 64, 512)
    assert np.array_equal(ids, sample["a_final_ids"])
    assert np.array_equal(bits(d), bits(sample["a_final_d"]))


def test_init_knn_given_reference_leaves(ctx, sample):
    x = sample["base"]
    gi, gd = aknn_init(ctx, x, sample["a_leaf_off"], sample["a_leaves"], 100)
    oi, od = ol.init_knn(x, ol.norms(x), sample["a_leaf_off"], sample["a_leaves"], 100)
    assert np.array_equal(gi, oi)
    assert np.array_equal(bits(gd), bits(od))


def test_exact_ground_truth_bit_exact(ctx, sample):
    base = f32(sample["base"])
    n, d = base.shape
    ids = np.empty((n, 100), np.uint32)
    keys = np.empty((n, 100), np.float32)
    ctx._check(ctx.lib.anqi_exact_topk(ctx.h, base, n, d, 100, ids, keys), "exact_topk")
    assert np.array_equal(ids, sample["exact_ids"])
    assert np.array_equal(bits(keys), bits(sample["exact_keys"]))
    q = f32(sample["query"])
    for k in (10, 50, 100):
        off = np.empty(len(q) + 1, np.uint32)
        cap = n * len(q)
        gid = np.empty(cap, np.uint32)
        gkey = np.empty(cap, np.float32)
        tot = C.c_uint64()
        ctx._check(ctx.lib.anqi_rknn_ground_truth(ctx.h, base, n, q, len(q), d, f32(keys[:, k - 1]), off, gid, gkey,
                                                  cap, C.byref(tot)), "gt")
        assert np.array_equal(off, sample[f"gt_off_{k}"])
        assert np.array_equal(gid[:tot.value], sample[f"gt_ids_{k}"])
        assert np.array_equal(bits(gkey[:tot.value]), bits(sample[f"gt_keys_{k}"]))


# ------------------------------------------------------------ random, larger

def clustered(n, d, seed, nc=50, spread=1.0):
    rng = np.random.default_rng(seed)
    centers = rng.normal(scale=4.0, size=(nc, d))
    lab = rng.integers(0, nc, size=n)
    return (centers[lab] + rng.normal(scale=spread, size=(n, d))).astype(np.float32)


def rp_forest(ctx, x, trees, leaf, max_depth=100, seed=10):
    x = f32(x)
    n, dim = x.shape
    cap = 4 * n + 8
    nn = np.empty(trees, np.uint32)
    left = np.empty(trees * cap, np.uint32)
    right = np.empty(trees * cap, np.uint32)
    off = np.empty(trees * cap, np.float32)
    hyp = np.empty(trees * cap * dim, np.float32)
    lo = np.empty(trees * cap, np.uint32)
    lc = np.empty(trees * cap, np.uint32)
    perm = np.empty(trees * n, np.uint32)
    ctx._check(ctx.lib.anqi_rp_forest(ctx.h, x, n, dim, trees, leaf, max_depth, seed, cap, nn, left, right, off, hyp,
                                      lo, lc, perm), "forest")
    return nn, cap, left, right, off, hyp.reshape(-1, dim), lo, lc, perm.reshape(trees, n)


def test_rp_forest_bit_exact_vs_oracle(ctx):
    x = clustered(5000, 34, 21)
    nn, cap, left, right, off, hyp, lo, lc, perm = rp_forest(ctx, x, 4, 60)
    for t in range(4):
        o = ol.rp_tree(x, 60, 100, 10, t)
        m = int(nn[t])
        assert m == o["n_nodes"]
        s = slice(t * cap, t * cap + m)
        assert np.array_equal(left[s], o["left"])
        assert np.array_equal(right[s], o["right"])
        internal = o["left"] != EMPTY
        assert np.array_equal(bits(off[s][internal]), bits(o["offset"][internal]))
        assert np.array_equal(bits(hyp[s][internal]), bits(o["hyperplane"][internal]))
        leafm = ~internal
        assert np.array_equal(lo[s][leafm], o["leaf_off"][leafm])
        assert np.array_equal(lc[s][leafm], o["leaf_cnt"][leafm])
        assert np.array_equal(perm[t], o["perm"])


def test_localjoin_and_select_random_vs_oracle(ctx):
    x = clustered(3000, 18, 31)
    n = len(x)
    nrm = ol.norms(x)
    rng = np.random.default_rng(4)
    cand = rng.integers(0, n, size=(n, 100)).astype(np.uint32)
    gi, gv = warm_start(ctx, x, cand, 100, 50)
    oi, ov = ol.warm_start(x, nrm, cand, 100, 50)
    assert np.array_equal(gi, oi) and np.array_equal(bits(gv), bits(ov))
    gi, gv, gu = localjoin(ctx, x, gi, gv)
    oi, ov, ou = ol.localjoin(x, nrm, oi, ov)
    assert gu == ou and np.array_equal(gi, oi) and np.array_equal(bits(gv), bits(ov))
    O, Od = select(ctx, x, gi, gv)
    O2, Od2 = ol.graph_select(x, nrm, oi, ov)
    assert np.array_equal(Od, Od2)
    for i in range(n):
        assert np.array_equal(O[i, :Od[i]], O2[i, :Od2[i]]), i
    L1, D1 = commit(ctx, x, O, Od)
    L2, D2 = ol.graph_commit(x, nrm, O2, Od2)
    assert np.array_equal(D1, D2)
    for i in range(n):
        assert np.array_equal(L1[i, :D1[i]], L2[i, :D2[i]]), i


def test_vamana_pass_vs_oracle(ctx):
    """One global Vamana pass (index.h:856-875, 1262-1285): per row a beam of
    width 64 over the current graph from a given entry, plus the row's g0
    list, pruned -> O; then commit.  Bit-exact against the oracle."""
    x = clustered(3000, 18, 41)
    n = len(x)
    nrm = ol.norms(x)
    rng = np.random.default_rng(8)
    cand = rng.integers(0, n, size=(n, 100)).astype(np.uint32)
    gi, gv = ol.warm_start(x, nrm, cand, 100, 50)
    gi, gv, _ = ol.localjoin(x, nrm, gi, gv)
    O, Od = ol.graph_select(x, nrm, gi, gv, M=24)
    links, deg = ol.graph_commit(x, nrm, O, Od)
    entry = rng.integers(0, n, size=n).astype(np.uint32)
    for Lb in (16, 64):
        Og = np.empty((n, 24), np.uint32)
        Odg = np.empty(n, np.uint32)
        ctx._check(ctx.lib.anqi_graph_vamana_select(ctx.h, f32(x), n, x.shape[1], u32(links), u32(deg), 24, u32(gi),
                                                    gi.shape[1], entry, Lb, 1.2, Og, Odg), "vamana_select")
        Oo, Odo = ol.vamana_select(x, nrm, links, deg, gi, entry, Lb)
        assert np.array_equal(Odg, Odo), Lb
        for i in range(n):
            assert np.array_equal(Og[i, :Odg[i]], Oo[i, :Odo[i]]), (Lb, i)
    L1, D1 = commit(ctx, x, Og, Odg)
    L2, D2 = ol.graph_commit(x, nrm, Oo, Odo)
    assert np.array_equal(D1, D2)


def test_graph_build_with_vamana_passes(ctx):
    """anqi_graph_build with two global Vamana passes (beam 64) on 4,000 rows:
    a valid degree-capped graph (ids in range, no self edge, no duplicate),
    changed by the passes."""
    x = clustered(4000, 24, 12)
    n, dim = x.shape
    warm = np.random.default_rng(3).integers(0, n, size=(n, 100)).astype(np.uint32)
    out = {}
    for passes in (0, 2):
        gp = GraphParams(24, 50, 100, 8, 6, 20, 100, 100, 10, 1.2, 100, 0, passes, 64)
        deg = np.empty(n, np.uint32)
        links = np.empty((n, 24), np.uint32)
        st = BuildStats()
        ctx._check(ctx.lib.anqi_graph_build(ctx.h, f32(x), n, dim, warm, 100, C.byref(gp), deg, links, C.byref(st)),
                   "graph_build")
        assert (deg <= 24).all() and (deg > 0).all()
        for i in range(n):
            row = links[i, :deg[i]]
            assert (row < n).all() and (row != i).all() and len(set(row.tolist())) == deg[i]
        out[passes] = (links.copy(), deg.copy())
    assert not np.array_equal(out[0][0], out[2][0])


def test_aknn_gather_beam_path_vs_oracle(ctx):
    # ef >= K + 1 -> the beam holds the answer
    x = clustered(4000, 24, 41)
    nrm = ol.norms(x)
    leaves_t = []
    for t in range(3):
        o = ol.rp_tree(x, 80, 100, 10, t)
        for v in range(o["n_nodes"]):
            if o["left"][v] == EMPTY and o["leaf_cnt"][v] > 0:
                s = int(o["leaf_off"][v])
                leaves_t.append(o["perm"][s:s + int(o["leaf_cnt"][v])])
    leaf_off = np.concatenate([[0], np.cumsum([len(l) for l in leaves_t])]).astype(np.uint64)
    leaves = np.concatenate(leaves_t).astype(np.uint32)
    gi, gd = aknn_init(ctx, x, leaf_off, leaves, 40)
    oi, od = ol.init_knn(x, nrm, leaf_off, leaves, 40)
    assert np.array_equal(gi, oi) and np.array_equal(bits(gd), bits(od))
    ids, d = aknn_gather(ctx, x, gi, gd, ef=120, cap=960, out_k=40)
    ri, rd = ol.aknn_rows(x, nrm, oi, od, K=40, ef=120)
    assert np.array_equal(ids, ri)
    assert np.array_equal(bits(d), bits(rd))


def test_aknn_build_recall(ctx):
    """End-to-end AKNN source build: recall@K vs exact, as the reference's own
    build_aknn_source gets on such data (0.98 at 50k on the reference recipe)."""
    x = clustered(20000, 32, 51, nc=200)
    n, d = x.shape
    K = 50
    p = AknnParams(K, 200, 16, 200, 8, 10, 0, 20)
    ids = np.empty((n, K), np.uint32)
    dist = np.empty((n, K), np.float32)
    st = BuildStats()
    ctx._check(ctx.lib.anqi_aknn_build(ctx.h, x, n, d, C.byref(p), ids, dist, C.byref(st)), "aknn_build")
    assert not np.any(ids == np.arange(n)[:, None])
    assert np.all(np.diff(dist, axis=1) >= 0)
    rng = np.random.default_rng(0)
    rows = rng.choice(n, 300, replace=False)
    nrm = (x.astype(np.float64) ** 2).sum(1)
    hit = 0
    for r in rows:
        dd = nrm + nrm[r] - 2 * x.astype(np.float64) @ x[r].astype(np.float64)
        dd[r] = np.inf
        true = set(np.argsort(dd)[:K].tolist())
        hit += len(true & set(ids[r].tolist()))
    assert hit / (300 * K) > 0.97, (hit / (300 * K), st.as_dict())


def test_graph_build_query_recall(ctx, sample):
    """Full G48 build on the reference sample, then queries: recall/precision
    within 0.2 points of the reference's own result lines (same L, k)."""
    x = sample["lifted"]
    n, dim = x.shape
    gp = GraphParams(48, 50, 100, 8, 6, 20, 100, 100, 10, 1.2, 100, 0)
    deg = np.empty(n, np.uint32)
    links = np.empty((n, 48), np.uint32)
    st = BuildStats()
    warm = u32(sample["rec_ids"])
    ctx._check(ctx.lib.anqi_graph_build(ctx.h, f32(x), n, dim, warm, 100, C.byref(gp), deg, links, C.byref(st)),
               "graph_build")
    nn = C.c_uint32()
    npt = C.c_uint64()
    ctx._check(ctx.lib.anqi_graph_tree_size(ctx.h, C.byref(nn), C.byref(npt)), "tree_size")
    m = nn.value
    t = {k: np.empty(m, np.uint32) for k in ("left", "right", "leaf_off", "leaf_cnt")}
    off = np.empty(m, np.float32)
    hyp = np.empty((m, dim), np.float32)
    perm = np.empty(npt.value, np.uint32)
    ctx._check(ctx.lib.anqi_graph_tree_copy(ctx.h, t["left"], t["right"], off, hyp, t["leaf_off"], t["leaf_cnt"],
                                            perm), "tree_copy")
    tree = formats.bfs_tree_to_postorder(t["left"], t["right"], off, hyp, t["leaf_off"], t["leaf_cnt"], perm, 100,
                                        dim)
    ctx.index_load(sample["base"], x, deg, links, tree, float(sample["scale"]), float(sample["mstar2"]))
    for ki, k in enumerate((1, 10, 50, 100)):
        if k == 1:
            continue
        ctx.set_thresholds(k, sample["thresholds"][ki])
        off_gt, ids_gt = sample[f"gt_off_{k}"], sample[f"gt_ids_{k}"]
        for L in (16, 32, 64, 128):
            r = ctx.rknn_query(sample["query"], k, L)
            rec, prec, ne = 0.0, 0.0, 0
            for i in range(len(sample["query"])):
                truth = set(ids_gt[off_gt[i]:off_gt[i + 1]].tolist())
                if not truth:
                    continue
                pred = set(r.pred(i).tolist())
                hit = len(pred & truth)
                rec += hit / len(truth)
                prec += 1.0 if not pred else hit / len(pred)
                ne += 1
            sel = [j for j, kl in enumerate(sample["ref_lines_k_L"]) if kl[0] == k and kl[1] == L][0]
            ref_rec, ref_prec = sample["ref_lines"][sel][:2]
            assert rec / ne >= ref_rec - 0.002, (k, L, rec / ne, ref_rec)
            assert prec / ne >= ref_prec - 0.002, (k, L, prec / ne, ref_prec)


def _aknn(ctx, x, precision, K=50, leaf=300, trees=8, ef=150):
    n, d = x.shape
    p = AknnParams(K, leaf, trees, ef, 8, 10, 0, 20, precision)
    ids = np.empty((n, K), np.uint32)
    dist = np.empty((n, K), np.float32)
    st = BuildStats()
    ctx._check(ctx.lib.anqi_aknn_build(ctx.h, f32(x), n, d, C.byref(p), ids, dist, C.byref(st)), "aknn_build")
    return ids, dist


@pytest.mark.parametrize("kind", ["integer", "float", "duplicates", "batched"])
def test_aknn_build_tensor_init_identical(ctx, kind, monkeypatch):
    """init_knn on BF16 tensor-core leaf tiles (exact keys on integer rows, FP32
    recheck otherwise) gives the FP32 path's AKNN lists bit for bit; leaves of
    up to 300 rows span several 128-row tiles; "batched" runs each tree's
    leaves in batches of candidate slots."""
    rng = np.random.default_rng(17)
    if kind in ("integer", "batched"):
        from anqi import pipeline
        x, _ = pipeline.mixture(12000, 64, 1, centers=40, seed=5)
        if kind == "batched":  # leaves in batches of about 1,500 rows per tree
            monkeypatch.setenv("ANQI_B200_INIT_BATCH_ROWS", "1500")
    elif kind == "float":
        x = clustered(12000, 48, 9, nc=60)
    else:
        x = clustered(6000, 40, 4, nc=30)
        x = np.concatenate([x, x[:3000]])  # exact duplicate rows: ties at distance 0
    a_ids, a_d = _aknn(ctx, x, 0)
    b_ids, b_d = _aknn(ctx, x, 1)
    assert np.array_equal(a_ids, b_ids)
    assert np.array_equal(bits(a_d), bits(b_d))



@pytest.mark.parametrize("kind", ["integer128", "float40", "duplicates", "islands"])
def test_aknn_gather_renumbered_identical(ctx, kind, monkeypatch):
    """The AKNN gather over rows renumbered for locality (components of the
    list graph, tree-0 order inside; the per-warp window bitmap) gives the
    original numbering's lists bit for bit: ties at equal distances (integer
    rows, duplicate rows) break on the original ids."""
    from anqi import pipeline
    if kind == "integer128":
        x, _ = pipeline.mixture(20000, 128, 1, centers=50, seed=7)
    elif kind == "float40":
        x = clustered(12000, 40, 11, nc=60)
    elif kind == "duplicates":
        x = clustered(6000, 24, 4, nc=30)
        x = np.concatenate([x, x[:3000], x[:500]])
    else:  # well-separated clusters of about 90 rows (K = 50): the list graph falls into components
        x, _ = pipeline.mixture(9000, 128, 1, centers=100, sigma=2.0, seed=3)
    got = []
    for ren in ("1", "0"):
        monkeypatch.setenv("ANQI_B200_GATHER_RENUMBER", ren)
        got.append(_aknn(ctx, x, 1))
    assert np.array_equal(got[0][0], got[1][0])
    assert np.array_equal(bits(got[0][1]), bits(got[1][1]))


def localjoin_precision(ctx, x, ids, vals, precision, sample=20, rounds=6):
    x = f32(x)
    ids = u32(ids).copy()
    vals = f32(vals).copy()
    n, dim = x.shape
    up = np.zeros(rounds, np.uint64)
    done = C.c_uint32()
    ms = C.c_float()
    ctx._check(ctx.lib.anqi_graph_localjoin_precision(ctx.h, x, n, dim, ids.shape[1], sample, rounds, precision, ids,
                                                      vals, up, C.byref(done), C.byref(ms)), "localjoin")
    return ids, vals, [int(u) for u in up[:done.value]], ms.value


@pytest.mark.parametrize("kind", ["lifted_mixture", "clustered_float", "duplicates"])
def test_localjoin_tensor_tiles_identical(ctx, kind):
    """The LocalJoin precision form (BF16 tcgen05 tiles filter each round's
    pairs against the round-start heap tops, the kept pairs are recomputed in
    FP32) leaves the heaps and per-round update counts bit-identical to the FP32
    form, on lifted (non-integer) vectors as the graph build sees them."""
    from anqi import pipeline
    if kind == "lifted_mixture":
        base, _ = pipeline.mixture(6000, 128, 0, centers=30, seed=5)
        radius = np.random.default_rng(8).uniform(2000.0, 8000.0, 6000).astype(np.float32)
        x, _, _ = ol.lift(base, radius)
    elif kind == "clustered_float":
        x = clustered(5000, 40, 9)
    else:
        x = clustered(4000, 24, 12)
        x[100:140] = x[7]
    n = len(x)
    rng = np.random.default_rng(3)
    cand = rng.integers(0, n, size=(n, 100)).astype(np.uint32)
    gi, gv = warm_start(ctx, x, cand, 100, 50)
    a = localjoin_precision(ctx, x, gi, gv, 0)
    b = localjoin_precision(ctx, x, gi, gv, 1)
    assert a[2] == b[2], (a[2], b[2])
    assert np.array_equal(a[0], b[0]) and np.array_equal(bits(a[1]), bits(b[1]))
    assert sum(a[2]) > 0


def test_aknn_build_d128_vs_oracle_stages(ctx):
    """A whole AKNN build at d = 128, where the gather reads its rows in chunk
    column order (group_ip_cols), equals the oracle's forest -> init_knn ->
    gather on the same seed, bit for bit (every row has K leaf-mates, so no
    random fill)."""
    from anqi import pipeline
    x = clustered(3000, 128, 77)
    n = len(x)
    K, leaf, trees, ef = 20, 100, 4, 40
    for precision in ("bf16", "fp32"):
        ids, keys, _ = pipeline.aknn_build(ctx, x, k=K, leaf=leaf, trees=trees, ef=ef, precision=precision)
        nrm = ol.norms(x)
        leaf_off, leaves = [0], []
        for t in range(trees):
            o = ol.rp_tree(x, leaf, 100, 10, t)
            for v in np.flatnonzero(o["left"] == EMPTY):
                a, c = int(o["leaf_off"][v]), int(o["leaf_cnt"][v])
                leaves.extend(o["perm"][a:a + c].tolist())
                leaf_off.append(len(leaves))
        ii, iv = ol.init_knn(x, nrm, np.array(leaf_off, np.uint64), np.array(leaves, np.uint32), K)
        assert not np.any(ii == EMPTY)
        ref_i, ref_d = ol.aknn_rows(x, nrm, ii, iv, K=K, ef=ef)
        assert np.array_equal(ids, ref_i), precision
        assert np.array_equal(bits(keys), bits(np.maximum(ref_d, np.float32(0.0)))), precision
