"""GPU parity of the query path, LRQ codec, lift and distances (sm_100a kernels
through the C ABI) against the reference's golden outputs and the C oracle.
Bit-exact: every compared integer is equal and every float has the same bits."""
import tempfile
from pathlib import Path

import numpy as np
import pytest

import oracle_lib as ol
from anqi import formats
from anqi._lib import AnqiError, Context

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def ctx():
    with Context(0) as c:
        yield c


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def csr_rows(off, ids):
    return [ids[int(off[i]):int(off[i + 1])] for i in range(len(off) - 1)]


@pytest.mark.parametrize("group", [4, 8, 16])
def test_pair_distances_bit_exact(ctx, group):
    """The reference's AVX-512 order with 4, 8 or 16 threads per pair."""
    z = np.load(GOLDEN / "dist.npz")
    for dim in (8, 10, 16, 32, 34, 128, 130, 962):
        l2, ip = ctx.pair_distances(z[f"a_{dim}"], z[f"b_{dim}"], group)
        assert np.array_equal(bits(l2), bits(z[f"l2_{dim}"])), dim
        assert np.array_equal(bits(ip), bits(z[f"ip_{dim}"])), dim


def test_pair_distances_chunk_columns(ctx):
    """The d = 128 search's distance on transposed 16-float chunks (registers
    fold AVX lanes i + 8 and i + 4): same bits as the golden vectors, and on
    random rows with large and tiny magnitudes."""
    z = np.load(GOLDEN / "dist.npz")
    l2, ip = ctx.pair_distances(z["a_130"], z["b_130"], 0)
    assert np.array_equal(bits(l2), bits(z["l2_130"]))
    assert np.array_equal(bits(ip), bits(z["ip_130"]))
    rng = np.random.default_rng(11)
    a = (rng.normal(size=(4099, 130)) * 10.0 ** rng.integers(-6, 6, size=(4099, 1))).astype(np.float32)
    b = (a + rng.normal(size=a.shape).astype(np.float32) * 1e-3).astype(np.float32)
    a[:7] = b[:7]  # zero distances
    l2c, _ = ctx.pair_distances(a, b, 0)
    l2r, _ = ctx.pair_distances(a, b, 4)
    assert np.array_equal(bits(l2c), bits(l2r))
    ref = np.array([ol.LIB.ao_l2sqr(a[i], b[i], 130) for i in range(0, len(a), 37)], np.float32)
    assert np.array_equal(bits(l2c[::37]), bits(ref))


def test_lrq_bit_exact(ctx, sample):
    coeff, codes = ctx.lrq_encode(sample["rec_keys"], sample["mu"], sample["basis"], sample["codebook"])
    assert np.array_equal(bits(coeff), bits(sample["coeff"]))
    assert np.array_equal(codes, sample["codes"])
    for i, k in enumerate((1, 10, 50, 100)):
        thr = ctx.lrq_materialize(coeff, codes, sample["mu"], sample["basis"], sample["codebook"], k)
        assert np.array_equal(bits(thr), bits(sample["thresholds"][i])), k


def test_lrq_random_vs_oracle(ctx):
    rng = np.random.default_rng(3)
    n, nk, m = 5003, 100, 8
    keys = np.sort(rng.gamma(2.0, 10.0, size=(n, nk)).astype(np.float32), axis=1)
    mu = keys.mean(0).astype(np.float32)
    basis = np.linalg.qr(rng.normal(size=(nk, m)))[0].T.astype(np.float32)
    cb = np.sort(rng.normal(scale=3.0, size=(nk, 256)).astype(np.float32), axis=1)
    c_gpu, k_gpu = ctx.lrq_encode(keys, mu, basis, cb)
    c_or, k_or = ol.lrq_encode(keys, mu, basis, cb)
    assert np.array_equal(bits(c_gpu), bits(c_or))
    assert np.array_equal(k_gpu, k_or)
    for k in (1, 10, 50, 100):
        for scale in (1.0, 1.05):
            a = ctx.lrq_materialize(c_gpu, k_gpu, mu, basis, cb, k, scale)
            b = ol.lrq_materialize(c_or, k_or, mu, basis, cb, k, scale)
            assert np.array_equal(bits(a), bits(b))


def test_lift_bit_exact(ctx, sample):
    lifted, m2, sc = ctx.lift(sample["base"], sample["rec_keys"][:, 99])
    assert sc == float(sample["scale"]) and m2 == float(sample["mstar2"])
    assert np.array_equal(bits(lifted), bits(sample["lifted"]))


def test_lift_random_vs_oracle(ctx):
    rng = np.random.default_rng(5)
    base = np.round(rng.uniform(0, 255, size=(20011, 128))).astype(np.float32)
    radius = rng.gamma(3.0, 1000.0, size=20011).astype(np.float32)
    a = ctx.lift(base, radius)
    b = ol.lift(base, radius)
    assert a[1] == b[1] and a[2] == b[2]
    assert np.array_equal(bits(a[0]), bits(b[0]))


def _load_sample_index(ctx, sample, tmp_path):
    p = tmp_path / "g.bin"
    p.write_bytes(sample["graph_file"].tobytes())
    g = formats.read_graph(p)
    ctx.index_load(sample["base"], sample["lifted"], g.deg, g.links, g.tree, float(sample["scale"]),
                   float(sample["mstar2"]))
    return g


def test_query_bit_exact_vs_reference(ctx, sample, tmp_path):
    """Candidate lists (visit order), #graph_dist and verified lists equal the
    reference's range_search + postfilter on the reference's own graph."""
    _load_sample_index(ctx, sample, tmp_path)
    for ki, k in enumerate((1, 10, 50, 100)):
        if k == 1:
            continue
        ctx.set_thresholds(k, sample["thresholds"][ki])
        for L in (16, 32, 64, 128):
            r = ctx.rknn_query(sample["query"], k, L, keep_candidates=True)
            ref_c = csr_rows(sample[f"q_cand_off_{k}_{L}"], sample[f"q_cand_{k}_{L}"])
            ref_p = csr_rows(sample[f"q_pred_off_{k}_{L}"], sample[f"q_pred_{k}_{L}"])
            assert np.array_equal(r.n_dist, sample[f"q_ndist_{k}_{L}"]), (k, L)
            for i in range(len(ref_c)):
                assert list(r.cand(i)) == list(ref_c[i]), (k, L, i)
                assert list(r.pred(i)) == list(ref_p[i]), (k, L, i)


def test_query_verifier_materialized_on_device(ctx, sample, tmp_path):
    _load_sample_index(ctx, sample, tmp_path)
    ctx.verifier_load(sample["coeff"], sample["codes"], sample["mu"], sample["basis"], sample["codebook"])
    for k in (10, 50, 100):
        ctx.verifier_materialize(k)
    ks = np.array([10, 50, 100] * 11, np.uint32)[:32]
    Ls = np.array([16, 32, 64, 128] * 8, np.uint32)
    r = ctx.rknn_query(sample["query"], ks, Ls, keep_candidates=True)
    for i in range(32):
        k, L = int(ks[i]), int(Ls[i])
        ref_p = csr_rows(sample[f"q_pred_off_{k}_{L}"], sample[f"q_pred_{k}_{L}"])
        assert list(r.pred(i)) == list(ref_p[i]), (i, k, L)


def _random_index(n=6000, d=32, nq=300, seed=11):
    """A G48 index built by the C oracle from an exact-kNN warm start."""
    rng = np.random.default_rng(seed)
    centers = rng.normal(scale=4.0, size=(40, d))
    lab = rng.integers(0, 40, size=n + nq)
    x = (centers[lab] + rng.normal(size=(n + nq, d))).astype(np.float32)
    base, query = x[:n], x[n:]
    nrm = ol.norms(base)
    d2 = nrm[:, None] + nrm[None, :] - 2.0 * (base.astype(np.float64) @ base.T)
    np.fill_diagonal(d2, np.inf)
    knn = np.argsort(d2, axis=1)[:, :100].astype(np.uint32)
    radius = np.take_along_axis(d2, knn[:, 99:100].astype(np.int64), 1)[:, 0].astype(np.float32)
    lifted, m2, sc = ol.lift(base, radius)
    ln = ol.norms(lifted)
    ids, vals = ol.warm_start(lifted, ln, knn, 100, 50)
    ids, vals, _ = ol.localjoin(lifted, ln, ids, vals)
    O, Od = ol.graph_select(lifted, ln, ids, vals)
    links, deg = ol.graph_commit(lifted, ln, O, Od)
    t = ol.rp_tree(lifted, 100)
    tree = formats.bfs_tree_to_postorder(t["left"], t["right"], t["offset"], t["hyperplane"], t["leaf_off"],
                                        t["leaf_cnt"], t["perm"], 100, d + 2)
    thr = {k: np.take_along_axis(d2, np.argsort(d2, axis=1)[:, k - 1:k], 1)[:, 0].astype(np.float32)
           for k in (10, 50, 100)}
    return base, query, lifted, links, deg, tree, sc, m2, thr


@pytest.fixture(scope="module")
def random_index():
    return _random_index()


_ORACLE_CACHE = {}


@pytest.mark.parametrize("renumber", ["1", "0"])
@pytest.mark.parametrize("table", [None, "0", "1024", "4096", "0,4096", "512,4096", "1024,4096"])
def test_query_bit_exact_vs_oracle_random(ctx, random_index, table, renumber, monkeypatch):
    """Every visited-set form (autotuned; bitmap only; shared-memory tables of
    1024 / 4096 entries; an L2-resident table alone or behind a shared one)
    returns the oracle's candidates, #dist and verified lists.  With the
    objects in their given (random) order, a third of the visits fall outside
    the 4,096-id window and L=1000 pushes each table through every migration
    up to the bitmap; with the graph-order numbering most visits stay in the
    window."""
    monkeypatch.setenv("ANQI_B200_RENUMBER", renumber)
    if table is not None:
        monkeypatch.setenv("ANQI_B200_HASH", table)
    base, query, lifted, links, deg, tree, sc, m2, thr = random_index
    ctx.index_load(base, lifted, deg, links, tree, sc, m2)
    ta = ol.TreeArrays(tree.left, tree.right, tree.offset, tree.hyperplane, tree.leaf_first())
    for k in (10, 100):
        ctx.set_thresholds(k, thr[k])
        for L in (8, 48, 200, 1000):
            r = ctx.rknn_query(query, k, L, keep_candidates=True)
            if table is not None:
                sh, _, l2 = table.partition(",")
                assert r.stats["visited_table"] == int(sh)
                assert r.stats["visited_l2_table"] == int(l2 or 0)
            if (k, L) not in _ORACLE_CACHE:
                _ORACLE_CACHE[k, L] = ol.range_search_all(lifted, links, deg, base, ta, sc, m2, query, thr[k], L)
            cands, preds, nds = _ORACLE_CACHE[k, L]
            assert np.array_equal(r.n_dist, nds), (k, L)
            for i in range(len(query)):
                assert np.array_equal(r.cand(i), cands[i]), (k, L, i)
                assert np.array_equal(r.pred(i), preds[i]), (k, L, i)


def _gpu_built_index(ctx, n, d, nq, seed):
    """L2-normalised N(0,1) rows (the 960-d shape); the G48 graph and entry tree
    built by the GPU builders (their parity is tested on their own); the
    query stage is then compared with the oracle on that index."""
    from anqi import pipeline
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(n + nq, d)).astype(np.float32)
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    base, query = np.ascontiguousarray(x[:n]), np.ascontiguousarray(x[n:])
    nrm = ol.norms(base)
    d2 = nrm[:, None] + nrm[None, :] - 2.0 * (base.astype(np.float64) @ base.T)
    np.fill_diagonal(d2, np.inf)
    knn = np.argsort(d2, axis=1)[:, :100].astype(np.uint32)
    radius = np.take_along_axis(d2, knn[:, 99:100].astype(np.int64), 1)[:, 0].astype(np.float32)
    lifted, m2, sc = ctx.lift(base, radius)
    deg, links, tree, _ = pipeline.graph_build(ctx, lifted, knn)
    thr = {k: np.take_along_axis(d2, np.argsort(d2, axis=1)[:, k - 1:k], 1)[:, 0].astype(np.float32)
           for k in (10, 50, 100)}
    return base, query, lifted, links, deg, tree, sc, m2, thr


@pytest.fixture(scope="module", params=[128, 960])
def random_index_wide(request, ctx):
    d = request.param
    if d == 128:
        return _random_index(n=4000, d=d, nq=200, seed=23)
    return _gpu_built_index(ctx, 3000, d, 100, seed=29)


def test_query_bit_exact_vs_oracle_wide(ctx, random_index_wide):
    """d = 128 (lifted dimension 130) runs the search kernel instance whose
    distance loops are unrolled at compile time; d = 960 stages two long rows
    per round, reduced by 16-thread groups: same candidates, #dist and
    verified lists as the oracle."""
    base, query, lifted, links, deg, tree, sc, m2, thr = random_index_wide
    ctx.index_load(base, lifted, deg, links, tree, sc, m2)
    ta = ol.TreeArrays(tree.left, tree.right, tree.offset, tree.hyperplane, tree.leaf_first())
    for k in (10, 100):
        ctx.set_thresholds(k, thr[k])
        for L in (32, 128, 400):
            r = ctx.rknn_query(query, k, L, keep_candidates=True)
            cands, preds, nds = ol.range_search_all(lifted, links, deg, base, ta, sc, m2, query, thr[k], L)
            assert np.array_equal(r.n_dist, nds), (k, L)
            for i in range(len(query)):
                assert np.array_equal(r.cand(i), cands[i]), (k, L, i)
                assert np.array_equal(r.pred(i), preds[i]), (k, L, i)


def test_query_graph_replay_equals_plain(ctx, random_index):
    """anqi_query_run_graph: the first call runs the plain path and captures
    the launch sequence; replays on newly uploaded batches of the same shape
    return exactly what anqi_query_run returns for them."""
    base, query, lifted, links, deg, tree, sc, m2, thr = random_index
    ctx.index_load(base, lifted, deg, links, tree, sc, m2)
    for k in (10, 50, 100):
        ctx.set_thresholds(k, thr[k])
    rng = np.random.default_rng(7)
    nq = len(query)

    def batch(seed):
        r = np.random.default_rng(seed)
        q = query[r.permutation(nq)]
        return q, r.choice([10, 50, 100], nq).astype(np.uint32), r.integers(16, 400, nq).astype(np.uint32)

    for seed in (1, 2, 3):
        q, ks, Ls = batch(seed)
        Ls[0] = 400  # same beam-width bound in every batch
        ctx.query_upload(q, ks, Ls)
        ctx.query_run(keep_candidates=True)
        want = ctx.query_download(with_candidates=True)
        ctx.query_upload(q, ks, Ls)
        for _ in range(2):
            st = ctx.query_run_graph(keep_candidates=True)
            got = ctx.query_download(with_candidates=True)
            assert np.array_equal(got.pred_off, want.pred_off) and np.array_equal(got.pred_ids, want.pred_ids)
            assert np.array_equal(got.cand_off, want.cand_off) and np.array_equal(got.cand_ids, want.cand_ids)
            assert np.array_equal(got.n_dist, want.n_dist)
            assert st["search_ms"] > 0


def test_rknn_query_into_caller_buffers(ctx, random_index):
    """out=: results copied straight into caller-owned buffers reused across
    calls (views returned), and a pred buffer too small for the results is
    replaced by a larger one; same results as the allocating call."""
    base, query, lifted, links, deg, tree, sc, m2, thr = random_index
    ctx.index_load(base, lifted, deg, links, tree, sc, m2)
    ctx.set_thresholds(10, thr[10])
    want = ctx.rknn_query(query, 10, 64)
    nq = len(query)
    out = (np.empty(nq + 1, np.uint32), np.empty(int(want.pred_off[-1]) + 10, np.uint32), np.empty(nq, np.uint32))
    for _ in range(2):
        got = ctx.rknn_query(query, 10, 64, out=out)
        assert np.shares_memory(got.pred_ids, out[1]) and got.pred_off is out[0]
        assert np.array_equal(got.pred_off, want.pred_off) and np.array_equal(got.pred_ids, want.pred_ids)
        assert np.array_equal(got.n_dist, want.n_dist)
    small = (np.empty(nq + 1, np.uint32), np.empty(3, np.uint32), np.empty(nq, np.uint32))
    got = ctx.rknn_query(query, 10, 64, out=small)
    assert np.array_equal(got.pred_off, want.pred_off) and np.array_equal(got.pred_ids, want.pred_ids)


def test_query_upload_rejects_bad_k_and_L(ctx, random_index):
    """Per-query k without materialized thresholds, a zero beam width and a
    beam width above 4,096 are argument errors (status 2) naming the value;
    the context then runs a valid batch as before."""
    base, query, lifted, links, deg, tree, sc, m2, thr = random_index
    ctx.index_load(base, lifted, deg, links, tree, sc, m2)
    ctx.set_thresholds(10, thr[10])
    want = ctx.rknn_query(query, 10, 64)
    nq = len(query)
    ks = np.full(nq, 10, np.uint32)
    ks[nq // 2] = 77
    with pytest.raises(AnqiError, match="k=77") as e:
        ctx.query_upload(query, ks, 64)
    assert e.value.status == 2
    Ls = np.full(nq, 64, np.uint32)
    Ls[5] = 0
    with pytest.raises(AnqiError, match="positive") as e:
        ctx.query_upload(query, 10, Ls)
    assert e.value.status == 2
    Ls[5] = 5000
    with pytest.raises(AnqiError, match="4096") as e:
        ctx.rknn_query(query, 10, Ls)
    assert e.value.status == 2
    got = ctx.rknn_query(query, np.full(nq, 10, np.uint32), 64)
    assert np.array_equal(got.pred_off, want.pred_off) and np.array_equal(got.pred_ids, want.pred_ids)


def test_resident_batch_and_evaluate(ctx, random_index):
    base, query, lifted, links, deg, tree, sc, m2, thr = random_index
    ctx.index_load(base, lifted, deg, links, tree, sc, m2)
    ctx.set_thresholds(10, thr[10])
    ctx.query_upload(query, 10, 64)
    st1 = ctx.query_run(keep_candidates=True)
    r1 = ctx.query_download(with_candidates=True)
    st2 = ctx.query_run(keep_candidates=True)
    r2 = ctx.query_download(with_candidates=True)
    assert st1["n_dist"] == st2["n_dist"] and np.array_equal(r1.pred_ids, r2.pred_ids)
    off, ids, _ = ol.rknn_gt(base, query, thr[10])
    ev = ctx.query_evaluate(off, ids)
    # host recomputation
    rec, prec, ne = 0.0, 0.0, 0
    for i in range(len(query)):
        truth = set(ids[off[i]:off[i + 1]].tolist())
        if not truth:
            continue
        pred = set(r1.pred(i).tolist())
        hit = len(pred & truth)
        rec += hit / len(truth)
        prec += 1.0 if not pred else hit / len(pred)
        ne += 1
    assert ev["nonempty"] == ne
    assert abs(ev["recall"] - rec / ne) < 1e-12 and abs(ev["precision"] - prec / ne) < 1e-12
    assert ev["recall"] > 0.3
    # resident ground truth + device sums (the accumulators of rknn_query.cpp:2784-2799)
    ctx.gt_load(off, ids)
    ctx.query_run(keep_candidates=True)
    sums = ctx.query_evaluate_sums()
    h = dict(recall=0.0, precision=0.0, f1=0.0, cand_recall=0.0, cand=0.0, pred=0.0, graph_dist=0.0)
    for i in range(len(query)):
        truth = set(ids[off[i]:off[i + 1]].tolist())
        if not truth:
            continue
        pred = set(r1.pred(i).tolist())
        cand = r1.cand(i)
        hit = len(pred & truth)
        r, p = hit / len(truth), (1.0 if not pred else hit / len(pred))
        h["recall"] += r
        h["precision"] += p
        h["f1"] += 2 * r * p / (r + p) if r + p > 0 else 0.0
        h["cand_recall"] += len(set(cand.tolist()) & truth) / len(truth)
        h["cand"] += len(cand)
        h["pred"] += len(pred)
        h["graph_dist"] += int(r1.n_dist[i])
    assert sums["nonempty"] == ne
    for key, v in h.items():
        assert abs(sums[key] - v) <= 1e-9 * max(1.0, abs(v)), (key, sums[key], v)
    # a new batch invalidates the resident ground truth
    ctx.query_upload(query, 10, 64)
    ctx.query_run()
    with pytest.raises(Exception):
        ctx.query_evaluate_sums()


def test_bounded_wait_runs_out_without_a_fault(sample):
    """Failure detection without a GPU fault: with the search's row copies
    withheld (anqi_inject_fault), every bounded wait for them expires after
    a fixed number of polls with nothing in flight; the call returns ANQI_ERR_TIMEOUT,
    and the same context then answers the same batch exactly as before."""
    import time
    from anqi._lib import ANQI_ERR_TIMEOUT, AnqiError
    z = sample
    with tempfile.TemporaryDirectory() as td:
        p = Path(td) / "g.bin"
        p.write_bytes(z["graph_file"].tobytes())
        g = formats.read_graph(p)
    with Context(0) as ctx:
        ctx.index_load(z["base"], z["lifted"], g.deg, g.links, g.tree, float(z["scale"]), float(z["mstar2"]))
        ctx.set_thresholds(10, z["thresholds"][1])
        before = ctx.rknn_query(z["query"], 10, 32)
        ctx.inject_fault(1)
        t0 = time.time()
        with pytest.raises(AnqiError) as e:
            ctx.rknn_query(z["query"], 10, 32)
        assert e.value.status == ANQI_ERR_TIMEOUT, e.value
        waited = time.time() - t0
        print(f"bounded row waits ran out after {waited:.2f} s")
        assert waited < 60
        ctx.inject_fault(0)
        after = ctx.rknn_query(z["query"], 10, 32)
        assert np.array_equal(before.pred_off, after.pred_off) and np.array_equal(before.pred_ids, after.pred_ids)
        assert np.array_equal(before.n_dist, after.n_dist)
