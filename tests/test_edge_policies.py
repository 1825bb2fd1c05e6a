"""Edge policies of the G48 prune (include/index.h:283-829): the policy
resolution from the environment (anqi.edge_policy, configure_edge_residual_cover
:305-440) and the oracle's select and commit stages under every policy,
against the reference's own outputs (tests/golden/edge_policies.npz, made by
oracle/ref_harness graph with ANQI_EDGE_* set).  Bit-exact."""
from pathlib import Path

import numpy as np
import pytest

import oracle_lib as ol
from anqi import edge_policy as ep

GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def fx():
    return dict(np.load(GOLDEN / "edge_policies.npz")), dict(np.load(GOLDEN / "sample_d32.npz"))


def rows(off, ids):
    return [list(ids[int(off[i]):int(off[i + 1])]) for i in range(len(off) - 1)]


def policy_for(fx, name, tmp_path):
    z, _ = fx
    rf = tmp_path / "resid.bin"
    mf = tmp_path / "mu.bin"
    z["resid"].tofile(rf)
    z["mu"].tofile(mf)
    env = dict(kv.split("=", 1) for kv in z[f"{name}_env"])
    env.update(ANQI_EDGE_RESID_FILE=str(rf), ANQI_LSG_MU_FILE=str(mf))
    return ep.from_env(env, 256, 48, folder=str(tmp_path / "none"), scale2=float(z[f"{name}_scale"]) ** 2)


NAMES = [str(n) for n in np.load(GOLDEN / "edge_policies.npz")["names"]]


@pytest.mark.parametrize("name", NAMES)
def test_oracle_select_commit_under_policy(fx, name, tmp_path):
    z, s = fx
    pol = policy_for(fx, name, tmp_path)
    x = s["lifted"]
    nrm = ol.norms(x)
    O, Od = ol.graph_select_policy(x, nrm, s["g_join_ids"], s["g_join_vals"], pol)
    ref_O = rows(z[f"{name}_O_off"], z[f"{name}_O"])
    for i in range(256):
        assert list(O[i, :Od[i]]) == ref_O[i], (name, i)
    links, deg = ol.graph_commit_policy(np.ascontiguousarray(x, np.float32), nrm, O, Od, pol)
    ref_adj = rows(z[f"{name}_adj_off"], z[f"{name}_adj"])
    for i in range(256):
        assert list(links[i, :deg[i]]) == ref_adj[i], (name, i)


def test_policy_resolution(tmp_path):
    n, M = 10, 48
    r = tmp_path / "r.bin"
    np.zeros((n, 100), np.float32).tofile(r)
    m = tmp_path / "m.bin"
    np.ones(n, np.float32).tofile(m)
    base = {"ANQI_EDGE_RESID_FILE": str(r), "ANQI_LSG_MU_FILE": str(m)}
    assert ep.from_env({}, n, M) is None
    assert ep.from_env({"ANQI_EDGE_POLICY": ""}, n, M) is None
    assert not ep.from_env({"ANQI_EDGE_POLICY": "nope", **base}, n, M).active
    p = ep.from_env({"ANQI_EDGE_POLICY": "residual_cover", **base}, n, M)
    assert p.flags == ep.COVER and p.ks == [10, 50, 100] and p.budget == 16 and p.scale2 == 1.0
    # budget 0 disables every residual policy except ball_rng and the optimizer
    assert not ep.from_env({"ANQI_EDGE_POLICY": "residual_cover", "ANQI_EDGE_RESID_BUDGET": "0", **base}, n, M).active
    assert ep.from_env({"ANQI_EDGE_POLICY": "ball_rng", "ANQI_EDGE_RESID_BUDGET": "0", **base}, n, M).flags == \
        ep.BALL | ep.PURE
    assert ep.from_env({"ANQI_EDGE_POLICY": "bubble_auto", "ANQI_EDGE_RESID_BUDGET": "0", **base}, n, M).flags == \
        ep.BALL | ep.AUTO
    p = ep.from_env({"ANQI_EDGE_POLICY": "bubble_multik", "ANQI_EDGE_BALL_OCCLUSION": "any", **base}, n, M)
    assert p.flags == ep.BALL and not p.occlude_all
    # ks outside 1..nk are dropped; none left: no policy
    assert ep.from_env({"ANQI_EDGE_POLICY": "ball_hybrid", "ANQI_EDGE_KS": "0,-3,7x,500", **base}, n, M).ks == [7]
    assert not ep.from_env({"ANQI_EDGE_POLICY": "ball_hybrid", "ANQI_EDGE_KS": "200", **base}, n, M).active
    # the budget is at most M
    assert ep.from_env({"ANQI_EDGE_POLICY": "ball_hybrid", "ANQI_EDGE_RESID_BUDGET": "99", **base}, n, M).budget == M
    p = ep.from_env({"ANQI_EDGE_POLICY": "lsg_bubble_hybrid", "ANQI_LSG_ALPHA": "0.5", **base}, n, M)
    assert p.flags == ep.LSG | ep.BALL and p.lsg_alpha == 0.5
    meta = tmp_path / "g_anqi_meta.txt"
    meta.write_text("2.5 3\n")
    assert ep.from_env({"ANQI_EDGE_POLICY": "ball_rng", **base}, n, M, folder=str(tmp_path / "g")).scale2 == 9.0


@pytest.mark.parametrize("env,msg", [
    ({"ANQI_EDGE_POLICY": "residual_cover", "ANQI_EDGE_RESID_FILE": "/nonexistent/r.bin"}, "missing"),
    ({"ANQI_EDGE_POLICY": "ball_rng", "ANQI_EDGE_NK": "50"}, "stride/size mismatch"),
    ({"ANQI_EDGE_POLICY": "lsg_rng"}, "requires ANQI_LSG_MU_FILE"),
    ({"ANQI_EDGE_POLICY": "lsg_rng", "ANQI_LSG_MU_FILE": "MU", "ANQI_LSG_ALPHA": "-1"}, "invalid ANQI_LSG_ALPHA"),
    ({"ANQI_EDGE_POLICY": "lsg_rng", "ANQI_LSG_MU_FILE": "BADMU"}, "invalid lsg mu"),
])
def test_policy_errors(tmp_path, env, msg):
    n = 10
    r = tmp_path / "r.bin"
    np.zeros((n, 100), np.float32).tofile(r)
    (tmp_path / "mu.bin").write_bytes(np.ones(n, np.float32).tobytes())
    bad = np.ones(n, np.float32)
    bad[3] = 0.0
    (tmp_path / "bad.bin").write_bytes(bad.tobytes())
    env = dict(env)
    env.setdefault("ANQI_EDGE_RESID_FILE", str(r))
    if env.get("ANQI_LSG_MU_FILE") == "MU":
        env["ANQI_LSG_MU_FILE"] = str(tmp_path / "mu.bin")
    if env.get("ANQI_LSG_MU_FILE") == "BADMU":
        env["ANQI_LSG_MU_FILE"] = str(tmp_path / "bad.bin")
    with pytest.raises(ep.PolicyError, match=msg):
        ep.from_env(env, n, 48)
