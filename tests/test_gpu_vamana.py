"""GPU parity of the Vamana refine against the reference's own refined graphs
(tests/golden/vamana.npz): the batched style through
anqi_graph_vamana_batch_refine (every option set, with and without an edge
policy) and the global passes through anqi_graph_vamana_select +
anqi_graph_commit, each from the reference's committed graph.  Bit-exact."""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as ol
import test_vamana_batch as tv
from anqi import pipeline
from anqi._lib import Context, GraphParams, edge_policy_c

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    with Context(0) as c:
        yield c


def start_graph(fx, pol):
    _, s, e = fx
    if pol is None:
        return tv.as_matrix(s["g_adj_off"], s["g_adj"])
    return tv.as_matrix(e[f"{pol.name}_adj_off"], e[f"{pol.name}_adj"])


@pytest.mark.parametrize("name", tv.NAMES)
def test_vamana_refine_vs_reference(ctx, name, tmp_path):
    fx = (dict(np.load(tv.GOLDEN / "vamana.npz")), dict(np.load(tv.GOLDEN / "sample_d32.npz")),
          dict(np.load(tv.GOLDEN / "edge_policies.npz")))
    z, s, _ = fx
    vp, pol = tv.config(fx, name, tmp_path)
    x = np.ascontiguousarray(s["lifted"], np.float32)
    n, dim = x.shape
    links, deg = start_graph(fx, pol)
    g0 = np.ascontiguousarray(s["g_join_ids"], np.uint32)
    if vp.style in ("global", "old"):
        if pol is not None:
            pytest.skip("the global pass's stage entry takes the default prune")
        entry = tv.tree_entries(s)
        for _ in range(vp.passes):
            O = np.empty((n, 48), np.uint32)
            Od = np.empty(n, np.uint32)
            ctx._check(ctx.lib.anqi_graph_vamana_select(ctx.h, x, n, dim, links, deg, 48, g0, g0.shape[1], entry,
                                                        vp.L, 1.2, O, Od), "vamana_select")
            links = np.empty((n, 48), np.uint32)
            deg = np.empty(n, np.uint32)
            ctx._check(ctx.lib.anqi_graph_commit(ctx.h, x, n, dim, O, Od, 48, 1.2, links, deg), "commit")
    else:
        gp = GraphParams(48, 50, 100, 8, 6, 20, 100, 100, 10, 1.2, 100, 0)
        pipeline.vamana_params(gp, vp)
        e = edge_policy_c(pol)
        if e is not None:
            gp.edge = C.addressof(e)
        links = np.ascontiguousarray(links)
        deg = np.ascontiguousarray(deg)
        ctx._check(ctx.lib.anqi_graph_vamana_batch_refine(ctx.h, x, n, dim, links, deg, g0, g0.shape[1],
                                                          C.byref(gp)), "vamana_batch_refine")
    ref = tv.rows(z[f"{name}_off"], z[f"{name}_adj"])
    for i in range(n):
        assert list(links[i, :deg[i]]) == ref[i], (name, i)


def test_vamana_batch_chunked_policy_vs_oracle(ctx, tmp_path, monkeypatch):
    """The batched style over 3,000 rows (batches up to 60 rows, then the
    reverse updates of hundreds of rows) under ball_hybrid, its prunes in
    chunks of 100 rows, against the oracle."""
    from anqi import edge_policy as ep, vamana
    rng = np.random.default_rng(12)
    c = rng.normal(scale=4.0, size=(30, 20))
    x = (c[rng.integers(0, 30, size=3000)] + rng.normal(size=(3000, 20))).astype(np.float32)
    n = len(x)
    nrm = ol.norms(x)
    cand = rng.integers(0, n, size=(n, 60)).astype(np.uint32)
    gi, gv = ol.warm_start(x, nrm, cand, 60, 30)
    gi, gv, _ = ol.localjoin(x, nrm, gi, gv)
    O, Od = ol.graph_select(x, nrm, gi, gv, M=24)
    links, deg = ol.graph_commit(x, nrm, O, Od)
    rf = tmp_path / "r.bin"
    rng.normal(0.0, 3.0, size=(n, 100)).astype(np.float32).tofile(rf)
    pol = ep.from_env({"ANQI_EDGE_POLICY": "ball_hybrid", "ANQI_EDGE_RESID_FILE": str(rf)}, n, 24,
                      folder=str(tmp_path / "none"))
    vp = vamana.from_env({"ANQI_VAMANA": "1", "ANQI_VAMANA_STYLE": "batch", "ANQI_VAMANA_L": "24",
                          "ANQI_VAMANA_PASS": "2", "ANQI_VAMANA_ENTRY": "5"}, x)
    ol_links, ol_deg = ol.vamana_batch_refine(x, nrm, links, deg, gi, vp, pol)
    monkeypatch.setenv("ANQI_B200_POLICY_CHUNK_ROWS", "100")
    gp = GraphParams(24, 30, 100, 8, 6, 20, 100, 100, 10, 1.2, 60, 0)
    pipeline.vamana_params(gp, vp)
    e = edge_policy_c(pol)
    gp.edge = C.addressof(e)
    gl, gd = links.copy(), deg.copy()
    ctx._check(ctx.lib.anqi_graph_vamana_batch_refine(ctx.h, x, n, x.shape[1], gl, gd, gi, gi.shape[1], C.byref(gp)),
               "vamana_batch_refine")
    assert np.array_equal(gd, ol_deg)
    for i in range(n):
        assert list(gl[i, :gd[i]]) == list(ol_links[i, :ol_deg[i]]), i
