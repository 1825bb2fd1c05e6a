"""Pins the oracle's ip-metric forms against the reference's own outputs on the
d = 32 sample under the ip metric (tests/golden/sample_ip_d32.npz, made by
make_golden.py): the scalar ip distance, init_knn and the AKNN gather in the
ip metric, the exact thresholds and RkNN sets with key -<a, b>, the ip lift,
the verifier's signed thresholds and the query path (per-query R2, key
-<o, q>)."""
from pathlib import Path

import numpy as np
import pytest

import oracle_lib as ol
from anqi import formats

GOLDEN = Path(__file__).resolve().parent / "golden"
EMPTY = 0xFFFFFFFF


@pytest.fixture(scope="module")
def ipz():
    return dict(np.load(GOLDEN / "sample_ip_d32.npz"))


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def csr_rows(off, ids):
    return [ids[int(off[i]):int(off[i + 1])] for i in range(len(off) - 1)]


def test_ip_distance_bit_exact(ipz):
    for dim in (3, 8, 13, 32, 130):
        a, b = ipz[f"ipd_a_{dim}"], ipz[f"ipd_b_{dim}"]
        got = np.array([ol.LIB.ao_ip_dist(a[i], b[i], dim) for i in range(len(a))], np.float32)
        assert np.array_equal(bits(got), bits(ipz[f"ipd_{dim}"])), dim


def test_ip_init_knn_from_reference_leaves(ipz):
    x = ipz["base"]
    zero = np.zeros(len(x), np.float32)  # the ip metric keeps no norms (index.h:164)
    ids, d = ol.init_knn(x, zero, ipz["a_leaf_off"], ipz["a_leaves"], 100, metric=1)
    ref_i, ref_v = ipz["a_init_ids"], ipz["a_init_vals"]
    for i in range(len(x)):
        ours = {int(a): float(b) for a, b in zip(ids[i], d[i]) if a != EMPTY}
        ref = {int(a): float(b) for a, b in zip(ref_i[i], ref_v[i]) if a != EMPTY}
        kth = max(ref.values())
        assert {a for a, b in ours.items() if b < kth} == {a for a, b in ref.items() if b < kth}
        for a in set(ours) & set(ref):
            assert ours[a] == ref[a]


def test_ip_aknn_gather_bit_exact(ipz):
    x = ipz["base"]
    zero = np.zeros(len(x), np.float32)
    ids, d = ol.aknn_rows(x, zero, ipz["a_init_ids"], ipz["a_init_vals"], K=100, ef=64, metric=1)
    assert np.array_equal(ids, ipz["a_final_ids"])
    assert np.array_equal(bits(d), bits(ipz["a_final_d"]))


def test_ip_exact_ground_truth_bit_exact(ipz):
    ids, keys = ol.exact_topk(ipz["base"], 100, metric=1)
    assert np.array_equal(ids, ipz["exact_ids"])
    assert np.array_equal(bits(keys), bits(ipz["exact_keys"]))
    for k in (10, 50, 100):
        off, gid, gkey = ol.rknn_gt(ipz["base"], ipz["query"], keys[:, k - 1], metric=1)
        assert np.array_equal(off, ipz[f"gt_off_{k}"])
        assert np.array_equal(gid, ipz[f"gt_ids_{k}"])
        assert np.array_equal(bits(gkey), bits(ipz[f"gt_keys_{k}"]))


def test_ip_lift_and_signed_thresholds_bit_exact(ipz):
    lifted, m2, sc = ol.lift(ipz["base"], ipz["rec_keys"][:, 99], metric=1)
    assert sc == float(ipz["scale"]) and m2 == float(ipz["mstar2"])
    assert np.array_equal(bits(lifted), bits(ipz["lifted"]))
    coeff, codes = ol.lrq_encode(ipz["rec_keys"], ipz["mu"], ipz["basis"], ipz["codebook"])
    assert np.array_equal(codes, ipz["codes"]) and np.array_equal(bits(coeff), bits(ipz["coeff"]))
    for i, k in enumerate((1, 10, 50, 100)):
        thr = ol.lrq_materialize_bits(coeff, codes, None, 256, 100, ipz["mu"], ipz["basis"], ipz["codebook"], 8, k,
                                      1.0, True)
        assert np.array_equal(bits(thr), bits(ipz["thresholds"][i])), k
    assert (ipz["thresholds"] < 0).any()  # signed keys survive unclamped


def test_ip_range_search_and_postfilter_bit_exact(ipz, tmp_path):
    p = tmp_path / "g.bin"
    p.write_bytes(ipz["graph_file"].tobytes())
    g = formats.read_graph(p)
    t = g.tree
    tree = ol.TreeArrays(t.left, t.right, t.offset, t.hyperplane, t.leaf_first())
    for ki, k in enumerate((1, 10, 50, 100)):
        if k == 1:
            continue
        thr = ipz["thresholds"][ki]
        for L in (16, 32, 64, 128):
            cands, preds, nds = ol.range_search_all(ipz["lifted"], g.links, g.deg, ipz["base"], tree,
                                                    float(ipz["scale"]), float(ipz["mstar2"]), ipz["query"], thr, L,
                                                    metric=1)
            ref_c = csr_rows(ipz[f"q_cand_off_{k}_{L}"], ipz[f"q_cand_{k}_{L}"])
            ref_p = csr_rows(ipz[f"q_pred_off_{k}_{L}"], ipz[f"q_pred_{k}_{L}"])
            assert np.array_equal(nds, ipz[f"q_ndist_{k}_{L}"]), (k, L)
            for i in range(len(cands)):
                assert list(cands[i]) == list(ref_c[i]), (k, L, i)
                assert list(preds[i]) == list(ref_p[i]), (k, L, i)


def test_ip_angular_forest_splits(ipz):
    """The deterministic forest in its angular form: unit-norm hyperplanes
    through the origin (offset 0), leaves partition the rows."""
    x = ipz["base"]
    t = ol.rp_tree(x, 16, angular=1)
    internal = t["left"] != EMPTY
    assert internal.any()
    assert np.all(t["offset"][internal] == 0.0)
    hn = np.linalg.norm(t["hyperplane"][internal].astype(np.float64), axis=1)
    assert np.allclose(hn, 1.0, atol=1e-5)
    assert sorted(t["perm"].tolist()) == list(range(len(x)))
