"""GPU parity of the ip metric (the reference's metric=ip) through the C ABI:
the reference's own outputs on the d = 32 ip sample (tests/golden/sample_ip_d32.npz)
for init_knn, the AKNN gather, the exact thresholds and RkNN sets (key -<a, b>),
the ip lift and the query path (per-query radius, key -<o, q>); the oracle for
the angular forest and for a whole AKNN build on random data.  Bit-exact."""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

import oracle_lib as ol
from anqi import formats, pipeline
from anqi._lib import METRICS, AknnParams, BuildStats, Context

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
EMPTY = 0xFFFFFFFF
IP = METRICS["ip"]


@pytest.fixture(scope="module")
def ctx():
    with Context(0) as c:
        yield c


@pytest.fixture(scope="module")
def ipz():
    return dict(np.load(GOLDEN / "sample_ip_d32.npz"))


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def f32(a):
    return np.ascontiguousarray(a, np.float32)


def u32(a):
    return np.ascontiguousarray(a, np.uint32)


def csr_rows(off, ids):
    return [ids[int(off[i]):int(off[i + 1])] for i in range(len(off) - 1)]


def test_ip_init_knn_from_reference_leaves(ctx, ipz):
    x = f32(ipz["base"])
    n, d = x.shape
    K = 100
    oi = np.empty((n, K), np.uint32)
    od = np.empty((n, K), np.float32)
    leaf_off = np.ascontiguousarray(ipz["a_leaf_off"], np.uint64)
    ctx._check(ctx.lib.anqi_aknn_init_metric(ctx.h, x, n, d, leaf_off, u32(ipz["a_leaves"]), len(leaf_off) - 1, K, IP,
                                             oi, od), "init")
    zero = np.zeros(n, np.float32)
    ref_i, ref_d = ol.init_knn(x, zero, ipz["a_leaf_off"], ipz["a_leaves"], K, metric=1)
    assert np.array_equal(oi, ref_i)
    assert np.array_equal(bits(od), bits(ref_d))
    # and the reference's own lists, up to its tie order at the K-th key
    gi, gv = ipz["a_init_ids"], ipz["a_init_vals"]
    for i in range(n):
        ours = {int(a): float(b) for a, b in zip(oi[i], od[i]) if a != EMPTY}
        ref = {int(a): float(b) for a, b in zip(gi[i], gv[i]) if a != EMPTY}
        kth = max(ref.values())
        assert {a for a, b in ours.items() if b < kth} == {a for a, b in ref.items() if b < kth}


def test_ip_aknn_gather_bit_exact(ctx, ipz):
    x = f32(ipz["base"])
    n, d = x.shape
    gi, gv = u32(ipz["a_init_ids"]), f32(ipz["a_init_vals"])
    oi = np.empty((n, 100), np.uint32)
    od = np.empty((n, 100), np.float32)
    ctx._check(ctx.lib.anqi_aknn_gather_metric(ctx.h, x, n, d, gi, gv, gi.shape[1], 64, 8 * 64, 100, IP, oi, od),
               "gather")
    assert np.array_equal(oi, ipz["a_final_ids"])
    assert np.array_equal(bits(od), bits(ipz["a_final_d"]))


def test_ip_exact_ground_truth_bit_exact(ctx, ipz):
    ids, keys = pipeline.exact_thresholds(ctx, ipz["base"], 100, metric="ip")
    assert np.array_equal(ids, ipz["exact_ids"])
    assert np.array_equal(bits(keys), bits(ipz["exact_keys"]))
    for k in (10, 50, 100):
        off, gid, gkey = pipeline.rknn_ground_truth(ctx, ipz["base"], ipz["query"], keys[:, k - 1], metric="ip")
        assert np.array_equal(off, ipz[f"gt_off_{k}"])
        assert np.array_equal(gid, ipz[f"gt_ids_{k}"])
        assert np.array_equal(bits(gkey), bits(ipz[f"gt_keys_{k}"]))


def test_ip_lift_bit_exact(ctx, ipz):
    lifted, m2, sc = ctx.lift(ipz["base"], ipz["rec_keys"][:, 99], metric="ip")
    assert sc == float(ipz["scale"]) and m2 == float(ipz["mstar2"])
    assert np.array_equal(bits(lifted), bits(ipz["lifted"]))


def test_ip_query_bit_exact_vs_reference(ctx, ipz, tmp_path):
    """Candidates (visit order), #graph_dist and verified ids equal the
    reference's range search + postfilter under metric=ip, with its signed
    thresholds, on its own graph."""
    p = tmp_path / "g.bin"
    p.write_bytes(ipz["graph_file"].tobytes())
    g = formats.read_graph(p)
    ctx.index_load(ipz["base"], ipz["lifted"], g.deg, g.links, g.tree, float(ipz["scale"]), float(ipz["mstar2"]),
                   metric="ip")
    for ki, k in enumerate((1, 10, 50, 100)):
        if k == 1:
            continue
        ctx.set_thresholds(k, ipz["thresholds"][ki])
        for L in (16, 32, 64, 128):
            r = ctx.rknn_query(ipz["query"], k, L, keep_candidates=True)
            ref_c = csr_rows(ipz[f"q_cand_off_{k}_{L}"], ipz[f"q_cand_{k}_{L}"])
            ref_p = csr_rows(ipz[f"q_pred_off_{k}_{L}"], ipz[f"q_pred_{k}_{L}"])
            assert np.array_equal(r.n_dist, ipz[f"q_ndist_{k}_{L}"]), (k, L)
            for i in range(len(ref_c)):
                assert list(r.cand(i)) == list(ref_c[i]), (k, L, i)
                assert list(r.pred(i)) == list(ref_p[i]), (k, L, i)


def test_ip_angular_forest_bit_exact_vs_oracle(ctx):
    rng = np.random.default_rng(5)
    x = rng.normal(size=(4000, 34)).astype(np.float32)
    x[:50] *= np.float32(1e-8)  # near-zero rows take the unit-norm fallback
    n, dim = x.shape
    trees, leaf = 3, 50
    cap = 4 * n + 8
    nn = np.empty(trees, np.uint32)
    left = np.empty(trees * cap, np.uint32)
    right = np.empty(trees * cap, np.uint32)
    off = np.empty(trees * cap, np.float32)
    hyp = np.empty(trees * cap * dim, np.float32)
    lo = np.empty(trees * cap, np.uint32)
    lc = np.empty(trees * cap, np.uint32)
    perm = np.empty(trees * n, np.uint32)
    ctx._check(ctx.lib.anqi_rp_forest_metric(ctx.h, x, n, dim, trees, leaf, 100, 10, cap, IP, nn, left, right, off,
                                             hyp, lo, lc, perm), "forest")
    hyp = hyp.reshape(-1, dim)
    perm = perm.reshape(trees, n)
    for t in range(trees):
        o = ol.rp_tree(x, leaf, 100, 10, t, angular=1)
        m = int(nn[t])
        assert m == o["n_nodes"]
        s = slice(t * cap, t * cap + m)
        assert np.array_equal(left[s], o["left"])
        internal = o["left"] != EMPTY
        assert np.all(off[s][internal] == 0.0)
        assert np.array_equal(bits(hyp[s][internal]), bits(o["hyperplane"][internal]))
        assert np.array_equal(perm[t], o["perm"])


def test_ip_aknn_build_vs_oracle_stages(ctx):
    """A whole ip AKNN build equals the oracle's angular forest -> init_knn ->
    gather on the same seed (every row has K leaf-mates, so no random fill)."""
    rng = np.random.default_rng(9)
    x = rng.normal(size=(3000, 24)).astype(np.float32)
    n = x.shape[0]
    K, leaf, trees, ef = 20, 100, 4, 40
    ids, keys, _ = pipeline.aknn_build(ctx, x, k=K, leaf=leaf, trees=trees, ef=ef, metric="ip")
    leaf_off, leaves = [0], []
    for t in range(trees):
        o = ol.rp_tree(x, leaf, 100, 10, t, angular=1)
        for v in np.flatnonzero(o["left"] == EMPTY):
            a, c = int(o["leaf_off"][v]), int(o["leaf_cnt"][v])
            leaves.extend(o["perm"][a:a + c].tolist())
            leaf_off.append(len(leaves))
    zero = np.zeros(n, np.float32)
    ii, iv = ol.init_knn(x, zero, np.array(leaf_off, np.uint64), np.array(leaves, np.uint32), K, metric=1)
    assert not np.any(ii == EMPTY)
    ref_i, ref_d = ol.aknn_rows(x, zero, ii, iv, K=K, ef=ef, metric=1)
    assert np.array_equal(ids, ref_i)
    assert np.array_equal(bits(keys), bits(ref_d - np.float32(1.0)))


@pytest.mark.parametrize("data", ["normalized", "integers", "wide"])
def test_ip_aknn_build_tensor_init_equals_fp32(ctx, data):
    """init_knn under ip on BF16 tcgen05 tiles (key~ = 1 - <q~, x~>, eps bound,
    FP32 recheck in the sequential order) gives the FP32 path's lists and keys:
    L2-normalised rows (every pair near the bound rechecked), integer rows (the
    exact path, no recheck) and rows wider than the resident tile (K chunks)."""
    rng = np.random.default_rng(17)
    if data == "normalized":
        x = rng.normal(size=(6000, 96))
        x /= np.linalg.norm(x, axis=1, keepdims=True)
    elif data == "integers":
        x = rng.integers(-6, 7, size=(6000, 64))
    else:
        x = rng.normal(size=(2500, 300))
    x = x.astype(np.float32)
    kw = dict(k=50, leaf=200, trees=6, ef=100, metric="ip")
    i16, k16, st = pipeline.aknn_build(ctx, x, precision="bf16", **kw)
    i32, k32, _ = pipeline.aknn_build(ctx, x, precision="fp32", **kw)
    assert np.array_equal(i16, i32)
    assert np.array_equal(bits(k16), bits(k32))


def test_ip_rejects_localjoin_rounds(ctx):
    x = np.random.default_rng(1).normal(size=(500, 8)).astype(np.float32)
    p = AknnParams(10, 50, 2, 20, 8, 10, 2, 20, 0, IP)
    ids = np.empty((500, 10), np.uint32)
    dist = np.empty((500, 10), np.float32)
    st = BuildStats()
    assert ctx.lib.anqi_aknn_build(ctx.h, x, 500, 8, C.byref(p), ids, dist, C.byref(st)) == 2
