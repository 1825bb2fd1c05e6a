"""GPU parity of the edge policies of the G48 prune (policy_prune_kernel
behind anqi_graph_select_policy / anqi_graph_commit_policy and
anqi_graph_params.edge): the reference's own select and commit outputs under
every policy (tests/golden/edge_policies.npz), and the oracle on larger random
pools, in chunks of rows as at scale.  Bit-exact."""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

import oracle_lib as ol
from anqi import edge_policy as ep
from anqi import pipeline
from anqi._lib import Context, edge_policy_c

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
NAMES = [str(n) for n in np.load(GOLDEN / "edge_policies.npz")["names"]]


@pytest.fixture(scope="module")
def ctx():
    with Context(0) as c:
        yield c


@pytest.fixture(scope="module")
def fx():
    return dict(np.load(GOLDEN / "edge_policies.npz")), dict(np.load(GOLDEN / "sample_d32.npz"))


def rows(off, ids):
    return [list(ids[int(off[i]):int(off[i + 1])]) for i in range(len(off) - 1)]


def policy_for(z, name, tmp_path, n=256, M=48):
    rf = tmp_path / "resid.bin"
    mf = tmp_path / "mu.bin"
    z["resid"].tofile(rf)
    z["mu"].tofile(mf)
    env = dict(kv.split("=", 1) for kv in z[f"{name}_env"])
    env.update(ANQI_EDGE_RESID_FILE=str(rf), ANQI_LSG_MU_FILE=str(mf))
    return ep.from_env(env, n, M, folder=str(tmp_path / "none"), scale2=float(z[f"{name}_scale"]) ** 2)


def select(ctx, x, ids, vals, pol, M=48, ef=100, cap=800, alpha=1.2):
    x = np.ascontiguousarray(x, np.float32)
    n, dim = x.shape
    O = np.empty((n, M), np.uint32)
    Od = np.empty(n, np.uint32)
    e = edge_policy_c(pol)
    ctx._check(ctx.lib.anqi_graph_select_policy(ctx.h, x, n, dim, np.ascontiguousarray(ids, np.uint32),
                                                np.ascontiguousarray(vals, np.float32), ids.shape[1], M, ef, cap,
                                                alpha, C.byref(e) if e is not None else None, O, Od), "select")
    return O, Od


def commit(ctx, x, O, Od, pol, alpha=1.2):
    x = np.ascontiguousarray(x, np.float32)
    n, dim = x.shape
    M = O.shape[1]
    links = np.empty((n, M), np.uint32)
    deg = np.empty(n, np.uint32)
    e = edge_policy_c(pol)
    ctx._check(ctx.lib.anqi_graph_commit_policy(ctx.h, x, n, dim, np.ascontiguousarray(O, np.uint32),
                                                np.ascontiguousarray(Od, np.uint32), M, alpha,
                                                C.byref(e) if e is not None else None, links, deg), "commit")
    return links, deg


@pytest.mark.parametrize("name", NAMES)
def test_select_commit_policy_vs_reference(ctx, fx, name, tmp_path):
    z, s = fx
    pol = policy_for(z, name, tmp_path)
    x = s["lifted"]
    O, Od = select(ctx, x, s["g_join_ids"], s["g_join_vals"], pol)
    ref_O = rows(z[f"{name}_O_off"], z[f"{name}_O"])
    for i in range(256):
        assert list(O[i, :Od[i]]) == ref_O[i], (name, i)
    # commit from the reference's own O
    ref_Od = np.diff(z[f"{name}_O_off"]).astype(np.uint32)
    Oref = np.full((256, 48), 0xFFFFFFFF, np.uint32)
    for i, r in enumerate(ref_O):
        Oref[i, :len(r)] = r
    links, deg = commit(ctx, x, Oref, ref_Od, pol)
    ref_adj = rows(z[f"{name}_adj_off"], z[f"{name}_adj"])
    for i in range(256):
        assert list(links[i, :deg[i]]) == ref_adj[i], (name, i)


def clustered(n, d, seed, nc=40):
    rng = np.random.default_rng(seed)
    c = rng.normal(scale=4.0, size=(nc, d))
    return (c[rng.integers(0, nc, size=n)] + rng.normal(size=(n, d))).astype(np.float32)


@pytest.mark.parametrize("name,n", [("residual_cover", 2500), ("ball_hybrid", 2500), ("bubble_rng", 2500),
                                    ("lsg_rng", 2500), ("lsg_bubble_hybrid", 2500), ("bubble_auto_small", 2500),
                                    ("bubble_auto_full", 120)])
def test_select_commit_policy_vs_oracle_chunked(ctx, fx, name, n, tmp_path, monkeypatch):
    """Larger pools (hundreds of candidates) than the sample's, pruned in
    chunks of 300 rows; the oracle's select and commit under the same policy."""
    z, _ = fx
    x = clustered(n, 24, 5)
    nrm = ol.norms(x)
    rng = np.random.default_rng(8)
    env = dict(kv.split("=", 1) for kv in z[f"{name}_env"])
    rf = tmp_path / "r.bin"
    mf = tmp_path / "m.bin"
    med = 2.0 * 24
    rng.normal(0.0, 0.3 * med, size=(n, 100)).astype(np.float32).tofile(rf)
    np.exp(rng.normal(0.0, 0.35, size=n)).astype(np.float32).tofile(mf)
    env.update(ANQI_EDGE_RESID_FILE=str(rf), ANQI_LSG_MU_FILE=str(mf))
    pol = ep.from_env(env, n, 32, folder=str(tmp_path / "none"), scale2=1.3)
    # warm heaps: the oracle's warm start from exact neighbour lists
    ids, _ = pipeline.exact_thresholds(ctx, x, 40)
    wi, wv = ol.warm_start(x, nrm, ids, 40, 30)
    monkeypatch.setenv("ANQI_B200_POLICY_CHUNK_ROWS", "300")
    O, Od = select(ctx, x, wi, wv, pol, M=32, ef=60, cap=480)
    oO, oOd = ol.graph_select_policy(x, nrm, wi, wv, pol, M=32, ef=60, cap=480)
    assert np.array_equal(Od, oOd)
    for i in range(n):
        assert list(O[i, :Od[i]]) == list(oO[i, :oOd[i]]), (name, i)
    links, deg = commit(ctx, x, O, Od, pol)
    ol_links, ol_deg = ol.graph_commit_policy(x, nrm, O, Od, pol)
    assert np.array_equal(deg, ol_deg)
    for i in range(n):
        assert list(links[i, :deg[i]]) == list(ol_links[i, :ol_deg[i]]), (name, i)


def test_graph_build_with_policy_equals_stages(ctx, fx, tmp_path):
    """anqi_graph_params.edge reaches the build's prunes: the sample's G48
    build under ball_rng differs from the default build and equals warm start
    -> LocalJoin -> select -> commit run as stages under the policy."""
    z, s = fx
    pol = policy_for(z, "ball_rng", tmp_path)
    x = s["lifted"]
    d0, l0, _, _ = pipeline.graph_build(ctx, x, s["rec_ids"], degree=48)
    d1, l1, _, _ = pipeline.graph_build(ctx, x, s["rec_ids"], degree=48, edge=pol)
    assert not np.array_equal(l0, l1)
    wi, wv = pipeline.graph_warm_start(ctx, x, s["rec_ids"])
    ji, jv, _, _ = pipeline.graph_localjoin(ctx, x, wi, wv)
    O, Od = select(ctx, x, ji, jv, pol)
    links, deg = commit(ctx, x, O, Od, pol)
    assert np.array_equal(deg, d1)
    for i in range(256):
        assert list(links[i, :deg[i]]) == list(l1[i, :d1[i]]), i
