"""The three command-line drivers end to end on the GPU, on the reference's own
sample (scripts/run_sample.sh): dataset_gt bit-exact against the reference's
files, build_aknn_source valid and deterministic, and rknn_query printing the
reference's own result lines when it runs on the reference's graph (cache
interoperability both ways)."""
import os
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from anqi import formats

import test_cli as tc

pytestmark = pytest.mark.gpu
RESULT_RE = re.compile(r"\[rknn\] L_descent=(\d+)\s+\| recall=([\d.]+) precision=([\d.]+) F1=([\d.]+) \| "
                       r"avg cand=(\d+) pred=(\d+) #dist=(\d+) \| QPS=(\d+)")


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def lines(stdout):
    return {int(m.group(1)): [float(m.group(i)) for i in range(2, 8)] for m in RESULT_RE.finditer(stdout)}


@pytest.mark.parametrize("d", [8, 32])
def test_dataset_gt_cli_bit_exact(tmp_path, d):
    z = dict(np.load(tc.GOLDEN / f"sample_d{d}.npz"))
    base, query = tmp_path / "b.bin", tmp_path / "q.bin"
    formats.write_fbin(base, z["base"])
    formats.write_fbin(query, z["query"])
    thr = tmp_path / "thr"
    rc, out, err = tc.run("dataset_gt", "--base", base, "--K", 100, "--rk_k", 100, "--threads", 4, "--tile", 64,
                          "--mode", "thresholds", "--out_prefix", thr)
    assert rc == 0, err
    assert "[dgt] THRESHOLD_BUILD_TIME=" in out
    raw = Path(f"{thr}_baseknn_gt.bin").read_bytes()
    assert raw[:8] == np.array([256, 100], np.uint32).tobytes()
    ids = np.frombuffer(raw[8:8 + 256 * 400], np.uint32).reshape(256, 100)
    keys = np.frombuffer(raw[8 + 256 * 400:], np.float32).reshape(256, 100)
    assert np.array_equal(ids, z["exact_ids"]) and np.array_equal(bits(keys), bits(z["exact_keys"]))
    assert Path(f"{thr}_threshold_build_time.meta").read_text().startswith("ANQI_THRESHOLD_BUILD_V1\n")
    for k in (10, 50, 100):
        t = tmp_path / f"gt{k}"
        rc, out, err = tc.run("dataset_gt", "--base", base, "--query", query, "--K", 100, "--rk_k", k,
                              "--mode", "ground-truth", "--threshold-table", f"{thr}_baseknn_gt.bin",
                              "--out_prefix", t)
        assert rc == 0, err
        off, gids, gkeys = formats.read_rknn_csr(f"{t}_rknn_gt.bin")
        assert np.array_equal(off, z[f"gt_off_{k}"]) and np.array_equal(gids, z[f"gt_ids_{k}"])
        assert np.array_equal(bits(gkeys), bits(z[f"gt_keys_{k}"]))


def test_build_aknn_source_cli(tmp_path):
    z = dict(np.load(tc.GOLDEN / "sample_d32.npz"))
    base = tmp_path / "b.bin"
    formats.write_fbin(base, z["base"])
    outs = []
    for rep in range(2):
        pfx = tmp_path / f"p{rep}"
        rc, out, err = tc.run("build_aknn_source", base, pfx, 100, 64, 8, 64, 4, 10, "l2")
        assert rc == 0, err
        assert re.search(r"\[aknn\] DONE n=256 d=32 K=100 leaf=64 trees=8 ef=64 threads=4 seed=10 metric=l2", out)
        ids, keys = formats.read_rec(f"{pfx}_baseknn_aknn.rec", 256, 100)
        outs.append((ids, keys))
        meta = Path(f"{pfx}_aknn_build_time.meta").read_text().splitlines()
        assert meta[0] == "ANQI_AKNN_BUILD_V1" and meta[1].startswith("seconds ")
        assert not Path(f"{pfx}_baseknn_aknn.rec.part").exists()
    ids, keys = outs[0]
    assert np.array_equal(ids, outs[1][0]) and np.array_equal(bits(keys), bits(outs[1][1]))
    n = 256
    assert (ids < n).all() and (ids != np.arange(n)[:, None]).all()
    assert all(len(set(r.tolist())) == 100 for r in ids)
    assert (np.diff(keys, axis=1) >= 0).all() and (keys >= 0).all()
    # recall@100 against the exact table (the reference reaches 0.98+ on such data)
    hit = np.mean([len(set(ids[i]) & set(z["exact_ids"][i])) / 100 for i in range(n)])
    assert hit > 0.95, hit


@pytest.mark.parametrize("d", [8, 32])
def test_rknn_query_cli_matches_reference_lines(tmp_path, d):
    pfx, env, z = tc.sample_prefix(tmp_path, d)
    ref_lines = {(int(k), int(L)): list(v) for (k, L), v in zip(z["ref_lines_k_L"], z["ref_lines"])}
    # 1) cold: the graph is built on the device from the reference's AKNN warm start
    built = {}
    for k in (10, 50, 100):
        rc, out, err = tc.run("rknn_query", "16,32,64,128", pfx, 48, 500, 64, 600, k, env=env)
        assert rc == 0, err
        assert ("[rknn] BUILD_TIME=" in out) == (k == 10) and ("[rknn] INDEX_LOAD_TIME=" in out) == (k != 10)
        got = lines(out)
        assert sorted(got) == [16, 32, 64, 128]
        for L, v in got.items():
            built[k, L] = v
            r = ref_lines[k, L]
            assert abs(v[0] - r[0]) < 0.02 and v[1] >= 0.99, (k, L, v, r)   # recall, precision
        for tag in ("DIST_BREAKDOWN", "CANDIDATE_RECALL"):
            assert out.count(f"[rknn] {tag} L_descent=") == 4
    # 2) the reference's own graph in the same cache slot: its printed lines exactly
    gdir = Path(env["ANQI_GRAPH_CACHE_DIR"])
    gfiles = list(gdir.glob("fd_metric_*"))
    assert len(gfiles) == 1
    gfiles[0].write_bytes(z["graph_file"].tobytes())
    for k in (10, 50, 100):
        rc, out, err = tc.run("rknn_query", "16,32,64,128", pfx, 48, 500, 64, 600, k, env=env)
        assert rc == 0, err
        assert "[rknn] loaded cached index" in out
        for L, v in lines(out).items():
            assert v == ref_lines[k, L], (k, L, v, ref_lines[k, L])


@pytest.mark.skipif(not tc.REF_BIN.exists(), reason="reference binaries not built")
def test_reference_loads_the_caches_this_driver_writes(tmp_path):
    pfx, env, z = tc.sample_prefix(tmp_path, 8)
    rc, ours, err = tc.run("rknn_query", "16,32,64,128", pfx, 48, 500, 64, 600, 50, env=env)
    assert rc == 0, err
    e = {k: v for k, v in os.environ.items() if not k.startswith("ANQI_")}
    e.update(env)
    e["OMP_NUM_THREADS"] = "4"
    ref = subprocess.run([str(tc.REF_BIN), "16,32,64,128", str(pfx), "48", "500", "64", "600", "50"], env=e,
                         capture_output=True, text=True, timeout=300)
    assert ref.returncode == 0, ref.stderr
    assert "[rknn] loaded cached index" in ref.stdout and "Loading index from:" in ref.stdout
    assert "[rknn] loaded independent compact verifier" in ref.stdout
    assert lines(ref.stdout) == lines(ours)


VERIFIER_MODES = ["rankm_resid_u2_lrq_floor", "rankm_resid_u4_lrq_nearest", "rankm_resid_u8_lrq_ceil",
                  "rankm_resid_u16_lrq_floor", "rankm_resid_f32", "rankm_only", "exact_f32", "analytic_rankm"]


@pytest.mark.skipif(not tc.REF_BIN.exists(), reason="reference binaries not built")
@pytest.mark.parametrize("mode", VERIFIER_MODES)
def test_rknn_query_verifier_modes_match_reference(tmp_path, mode):
    """Every independent postfilter verifier of the reference (rknn_query.cpp:
    1771-1792) through this driver: the verifier artifact it writes equals the
    one the reference writes byte for byte, and on the reference's graph it
    prints the reference's result lines exactly."""
    import lrq_forms as lf
    pfx, env, z = tc.sample_prefix(tmp_path, 32)
    f, _ = lf.load()
    env = dict(env, ANQI_RADIUS_MODE=mode)
    for b in (2, 4, 8, 16):
        formats.write_codebook(f"{pfx}_learned_rq_codebook_M8_u{b}.bin", lf.codebook(f, b), 8, b)
    if mode == "analytic_rankm":
        formats.write_analytic(f"{pfx}_analytic_rankm_M8.bin",
                               formats.AnalyticModel(100, 8, 10, 7, float(f["pw_b0_7"][0]), f["pw_coeff_7"]))
        env["ANQI_CANDIDATE_ENVELOPE"] = "graph_horizon"
    ref_env = {k: v for k, v in os.environ.items() if not k.startswith("ANQI_")}
    ref_env.update(env, OMP_NUM_THREADS="1", ANQI_GRAPH_CACHE_DIR=str(tmp_path / "ref" / "graph"),
                   ANQI_VERIFIER_CACHE_DIR=str(tmp_path / "ref" / "verifier"))
    for sub in ("graph", "verifier"):
        (tmp_path / "ref" / sub).mkdir(parents=True)
    ref = subprocess.run([str(tc.REF_BIN), "16,32,64", str(pfx), "48", "500", "64", "600", "50"], env=ref_env,
                         capture_output=True, text=True, timeout=300)
    assert ref.returncode == 0, ref.stderr
    rc, ours, err = tc.run("rknn_query", "16,32,64", pfx, 48, 500, 64, 600, 50, env=env)
    assert rc == 0, err
    ref_vf = sorted((tmp_path / "ref" / "verifier").glob("_anqi_verifier_*.bin"))
    our_vf = sorted(Path(env["ANQI_VERIFIER_CACHE_DIR"]).glob("_anqi_verifier_*.bin"))
    assert [p.name for p in our_vf] == [p.name for p in ref_vf]
    for a, b in zip(our_vf, ref_vf):
        assert a.read_bytes() == b.read_bytes(), mode
    # the reference's graph in this driver's cache slot: its printed lines exactly
    gref = list((tmp_path / "ref" / "graph").glob("fd_metric_*"))
    gours = list(Path(env["ANQI_GRAPH_CACHE_DIR"]).glob("fd_metric_*"))
    assert len(gref) == 1 and len(gours) == 1 and gref[0].name == gours[0].name
    gours[0].write_bytes(gref[0].read_bytes())
    for suffix in ("_approxlift_graph_", "_anqi_meta_graph_"):
        for p in (tmp_path / "ref" / "graph").glob(suffix + "*"):
            (Path(env["ANQI_GRAPH_CACHE_DIR"]) / p.name).write_bytes(p.read_bytes())
    rc, ours, err = tc.run("rknn_query", "16,32,64", pfx, 48, 500, 64, 600, 50, env=env)
    assert rc == 0, err
    assert "[rknn] loaded cached index" in ours
    assert lines(ours) == lines(ref.stdout), (mode, lines(ours), lines(ref.stdout))


def ip_prefix(tmp_path):
    """The reference sample under metric=ip (tests/golden/sample_ip_d32.npz):
    its prefix files, the reference's own .rec (keys d - 1), basis, codebook and
    RkNN ground truth."""
    z = dict(np.load(tc.GOLDEN / "sample_ip_d32.npz"))
    pfx = tmp_path / "ipsample"
    formats.write_fbin(f"{pfx}_base.bin", z["base"])
    formats.write_fbin(f"{pfx}_query.bin", z["query"])
    Path(f"{pfx}_lifted.meta").write_text("0 32 100 ip 1.0\n")
    formats.write_rec(f"{pfx}_baseknn_aknn.rec", z["rec_ids"], z["rec_keys"])
    formats.write_basis(f"{pfx}_radbasis_M8.bin", z["mu"], z["basis"])
    formats.write_codebook(f"{pfx}_learned_rq_codebook_M8_u8.bin", z["codebook"])
    for k in (10, 50, 100):
        formats.write_rknn_csr(f"{pfx}_rknn_gt_k{k}.bin", z[f"gt_off_{k}"], z[f"gt_ids_{k}"], z[f"gt_keys_{k}"])
    env = dict(tc.RUN_FINAL_ENV)
    env["ANQI_PREBUILT_TOPK_REC"] = f"{pfx}_baseknn_aknn.rec"
    env["ANQI_GRAPH_CACHE_DIR"] = str(tmp_path / "cache" / "graph")
    env["ANQI_VERIFIER_CACHE_DIR"] = str(tmp_path / "cache" / "verifier")
    return pfx, env, z


def test_dataset_gt_cli_ip_bit_exact(tmp_path):
    """--metric ip: thresholds and RkNN CSR with keys -<a, b>, the reference's files bit for bit."""
    z = dict(np.load(tc.GOLDEN / "sample_ip_d32.npz"))
    base, query = tmp_path / "b.bin", tmp_path / "q.bin"
    formats.write_fbin(base, z["base"])
    formats.write_fbin(query, z["query"])
    thr = tmp_path / "thr"
    rc, out, err = tc.run("dataset_gt", "--base", base, "--K", 100, "--rk_k", 100, "--metric", "ip",
                          "--mode", "thresholds", "--out_prefix", thr)
    assert rc == 0, err
    raw = Path(f"{thr}_baseknn_gt.bin").read_bytes()
    ids = np.frombuffer(raw[8:8 + 256 * 400], np.uint32).reshape(256, 100)
    keys = np.frombuffer(raw[8 + 256 * 400:], np.float32).reshape(256, 100)
    assert np.array_equal(ids, z["exact_ids"]) and np.array_equal(bits(keys), bits(z["exact_keys"]))
    assert "metric ip" in Path(f"{thr}_threshold_build_time.meta").read_text()
    for k in (10, 50, 100):
        t = tmp_path / f"gt{k}"
        rc, out, err = tc.run("dataset_gt", "--base", base, "--query", query, "--K", 100, "--rk_k", k,
                              "--metric", "ip", "--mode", "ground-truth", "--threshold-table",
                              f"{thr}_baseknn_gt.bin", "--out_prefix", t)
        assert rc == 0, err
        off, gids, gkeys = formats.read_rknn_csr(f"{t}_rknn_gt.bin")
        assert np.array_equal(off, z[f"gt_off_{k}"]) and np.array_equal(gids, z[f"gt_ids_{k}"])
        assert np.array_equal(bits(gkeys), bits(z[f"gt_keys_{k}"]))


@pytest.mark.parametrize("metric", ["l2", "ip"])
def test_dataset_gt_cli_tensor_path_equals_fp32(tmp_path, metric):
    """From 20,000 rows dataset_gt runs the BF16 tensor path (its own AKNN
    lists bound the thresholds); its files equal the FP32 path's
    (ANQI_B200_GT_TENSOR=0) byte for byte."""
    rng = np.random.default_rng(3)
    x = rng.normal(size=(20500, 48))
    if metric == "ip":
        x /= np.linalg.norm(x, axis=1, keepdims=True)
    base, query = tmp_path / "b.bin", tmp_path / "q.bin"
    formats.write_fbin(base, x[:20000].astype(np.float32))
    formats.write_fbin(query, x[20000:].astype(np.float32))
    files = {}
    for mode, env in (("tensor", {}), ("fp32", {"ANQI_B200_GT_TENSOR": "0"})):
        thr = tmp_path / f"thr_{mode}"
        rc, out, err = tc.run("dataset_gt", "--base", base, "--K", 100, "--rk_k", 50, "--metric", metric,
                              "--mode", "thresholds", "--out_prefix", thr, env=env)
        assert rc == 0, err
        t = tmp_path / f"gt_{mode}"
        rc, out, err = tc.run("dataset_gt", "--base", base, "--query", query, "--K", 100, "--rk_k", 50,
                              "--metric", metric, "--mode", "ground-truth", "--threshold-table",
                              f"{thr}_baseknn_gt.bin", "--out_prefix", t, env=env)
        assert rc == 0, err
        files[mode] = (Path(f"{thr}_baseknn_gt.bin").read_bytes(), Path(f"{t}_rknn_gt.bin").read_bytes())
    assert files["tensor"][0] == files["fp32"][0]
    assert files["tensor"][1] == files["fp32"][1]


def test_build_aknn_source_cli_ip(tmp_path):
    """metric=ip: .rec keys are d - 1 = -<a, b> (build_aknn_source.cpp:125), rows
    ascending, self excluded, recall@100 against the exact -<a, b> table."""
    z = dict(np.load(tc.GOLDEN / "sample_ip_d32.npz"))
    base = tmp_path / "b.bin"
    formats.write_fbin(base, z["base"])
    pfx = tmp_path / "p"
    rc, out, err = tc.run("build_aknn_source", base, pfx, 100, 64, 8, 64, 4, 10, "ip")
    assert rc == 0, err
    assert "metric=ip" in out
    ids, keys = formats.read_rec(f"{pfx}_baseknn_aknn.rec", 256, 100)
    n = 256
    assert (ids < n).all() and (ids != np.arange(n)[:, None]).all()
    assert (np.diff(keys, axis=1) >= 0).all() and (keys < 0).any()
    x = z["base"].astype(np.float64)
    # the keys are the negated inner products of the listed pairs (FP32, sequential sum)
    assert np.allclose(keys, -np.einsum("id,ikd->ik", x, x[ids]), atol=1e-3)
    hit = np.mean([len(set(ids[i]) & set(z["exact_ids"][i])) / 100 for i in range(n)])
    assert hit > 0.95, hit
    rc, _, err = tc.run("build_aknn_source", base, pfx, 100, 64, 8, 64, 4, 10, "ip", env={"ANQI_NNITERS": "2"})
    assert rc == 2 and "ANQI_NNITERS" in err


def test_rknn_query_cli_ip_matches_reference_lines(tmp_path):
    """rknn_query on a metric=ip prefix: cold (graph built on the device from the
    reference's warm start) within 0.02 recall of the reference's lines; on the
    reference's own graph, the reference's result lines exactly."""
    pfx, env, z = ip_prefix(tmp_path)
    ref_lines = {(int(k), int(L)): list(v) for (k, L), v in zip(z["ref_lines_k_L"], z["ref_lines"])}
    for k in (10, 50, 100):
        rc, out, err = tc.run("rknn_query", "16,32,64,128", pfx, 48, 500, 64, 600, k, env=env)
        assert rc == 0, err
        assert "[rknn] metric=ip" in out
        for L, v in lines(out).items():
            r = ref_lines[k, L]
            assert abs(v[0] - r[0]) < 0.02 and v[1] >= 0.99, (k, L, v, r)
    gfiles = list(Path(env["ANQI_GRAPH_CACHE_DIR"]).glob("fd_metric_*"))
    assert len(gfiles) == 1
    gfiles[0].write_bytes(z["graph_file"].tobytes())
    for k in (10, 50, 100):
        rc, out, err = tc.run("rknn_query", "16,32,64,128", pfx, 48, 500, 64, 600, k, env=env)
        assert rc == 0, err
        assert "[rknn] loaded cached index" in out
        got = lines(out)
        assert sorted(got) == [16, 32, 64, 128]
        for L, v in got.items():
            assert v == ref_lines[k, L], (k, L, v, ref_lines[k, L])


def test_rknn_query_u8_base_equals_float_base(tmp_path):
    """ANQI_BASE_U8BIN: an integer-valued base given as uint8 gives the result
    lines of the same base given as float32 (the values widen exactly), with
    the uint8 file named in the cache identity."""
    from anqi import pipeline
    from anqi._lib import Context
    base, query = pipeline.mixture(3000, 16, 200, centers=20, sigma=20.0, seed=5)
    with Context(0) as ctx:
        ix = pipeline.build_index(ctx, base, aknn=dict(k=100, leaf=200, trees=8, ef=200), log=lambda *a: None)
        _, keys = pipeline.exact_thresholds(ctx, base, 100)
        gt = {k: pipeline.rknn_ground_truth(ctx, base, query, keys[:, k - 1]) for k in (10, 50, 100)}
    pfx = tmp_path / "mix"
    pipeline.write_prefix(str(pfx), base, query, ix, gt)
    u8 = tmp_path / "mix_base.u8bin"
    u8.write_bytes(np.array(base.shape, np.uint32).tobytes() + base.astype(np.uint8).tobytes())
    assert np.array_equal(base.astype(np.uint8).astype(np.float32), base)
    outs = []
    for name, extra in (("f32", {}), ("u8", {"ANQI_BASE_U8BIN": str(u8)})):
        env = dict(tc.RUN_FINAL_ENV, ANQI_PREBUILT_TOPK_REC=f"{pfx}_baseknn_aknn.rec",
                   ANQI_GRAPH_CACHE_DIR=str(tmp_path / name / "graph"),
                   ANQI_VERIFIER_CACHE_DIR=str(tmp_path / name / "verifier"), **extra)
        rc, out, err = tc.run("rknn_query", "16,64", pfx, 48, 500, 64, 600, 10, env=env)
        assert rc == 0, err
        assert ("loaded uint8 base directly as float" in out) == (name == "u8")
        outs.append(lines(out))
    assert outs[0] == outs[1] and sorted(outs[0]) == [16, 64]


@pytest.mark.parametrize("mode", ["command", "compact", "release"])
def test_rknn_query_streamed_warm_start(tmp_path, mode):
    """The streamed G48 warm start (index.h:1127-1203) gives the graph and the
    result lines of the in-memory one: from a command's stdout
    (ANQI_PREBUILT_WARM_START_COMMAND), from the table compacted to ids in
    place and then removed (ANQI_COMPACT_PREBUILT_TOPK_IDS_INPLACE), or with
    the table released after preparation (ANQI_RELEASE_PREBUILT_TOPK_AFTER_PREP)."""
    import shutil
    pfx, env, z = tc.sample_prefix(tmp_path, 32)
    rc, ref_out, err = tc.run("rknn_query", "16,32,64", pfx, 48, 500, 64, 600, 50, env=env)
    assert rc == 0, err
    rec = Path(f"{pfx}_baseknn_aknn.rec")
    copy = tmp_path / "warm.rec"
    shutil.copy(rec, copy)
    env2 = dict(env, ANQI_GRAPH_CACHE_DIR=str(tmp_path / "g2"), ANQI_VERIFIER_CACHE_DIR=str(tmp_path / "v2"))
    if mode == "command":
        env2["ANQI_PREBUILT_WARM_START_COMMAND"] = f"cat {copy}"
    elif mode == "compact":
        env2["ANQI_COMPACT_PREBUILT_TOPK_IDS_INPLACE"] = "1"
        env2["ANQI_PREBUILT_TOPK_REC"] = str(copy)
    else:
        env2["ANQI_RELEASE_PREBUILT_TOPK_AFTER_PREP"] = "1"
        env2["ANQI_PREBUILT_TOPK_REC"] = str(copy)
    rc, out, err = tc.run("rknn_query", "16,32,64", pfx, 48, 500, 64, 600, 50, env=env2)
    assert rc == 0, err
    assert lines(out) == lines(ref_out)
    g1 = list(Path(env["ANQI_GRAPH_CACHE_DIR"]).glob("fd_metric_*"))
    g2 = list((tmp_path / "g2").glob("fd_metric_*"))
    assert len(g1) == 1 and len(g2) == 1
    # the same adjacency and entry tree: all but the build-time field
    # ([u64 n, dim, M][f32 seconds], then the rows and the tree)
    a, b = g1[0].read_bytes(), g2[0].read_bytes()
    assert len(a) == len(b) and a[:24] == b[:24] and a[28:] == b[28:]
    if mode == "command":
        assert "source=prebuilt-stream" in out and copy.exists()
    else:
        assert not copy.exists()


@pytest.mark.skipif(not tc.REF_BIN.exists(), reason="reference binaries not built")
def test_rknn_query_scale_profile_degree20_kpivot10(tmp_path):
    """The scale path's graph profile (degree 20, K_pivot = ANQI_GRAPH_NK = 10):
    this driver builds and queries it; on the reference's own degree-20 graph
    (built by the reference binary here) it prints the reference's result
    lines exactly."""
    pfx, env, z = tc.sample_prefix(tmp_path, 32)
    env = dict(env, ANQI_GRAPH_NK="10")
    ref_env = {k: v for k, v in os.environ.items() if not k.startswith("ANQI_")}
    ref_env.update(env, OMP_NUM_THREADS="1", ANQI_GRAPH_CACHE_DIR=str(tmp_path / "ref" / "graph"),
                   ANQI_VERIFIER_CACHE_DIR=str(tmp_path / "ref" / "verifier"))
    for sub in ("graph", "verifier"):
        (tmp_path / "ref" / sub).mkdir(parents=True)
    ref = subprocess.run([str(tc.REF_BIN), "16,32,64", str(pfx), "20", "500", "64", "600", "10"], env=ref_env,
                         capture_output=True, text=True, timeout=300)
    assert ref.returncode == 0, ref.stderr
    rc, ours, err = tc.run("rknn_query", "16,32,64", pfx, 20, 500, 64, 600, 10, env=env)
    assert rc == 0, err
    assert "graph degree M=20" in ours
    for L, v in lines(ours).items():
        r = lines(ref.stdout)[L]
        assert abs(v[0] - r[0]) < 0.05, (L, v, r)
    gref = list((tmp_path / "ref" / "graph").glob("fd_metric_*"))
    gours = list(Path(env["ANQI_GRAPH_CACHE_DIR"]).glob("fd_metric_*"))
    assert len(gref) == 1 and len(gours) == 1 and gref[0].name == gours[0].name
    gours[0].write_bytes(gref[0].read_bytes())
    for suffix in ("_approxlift_graph_", "_anqi_meta_graph_"):
        for p in (tmp_path / "ref" / "graph").glob(suffix + "*"):
            (Path(env["ANQI_GRAPH_CACHE_DIR"]) / p.name).write_bytes(p.read_bytes())
    rc, ours, err = tc.run("rknn_query", "16,32,64", pfx, 20, 500, 64, 600, 10, env=env)
    assert rc == 0, err
    assert "[rknn] loaded cached index" in ours
    assert lines(ours) == lines(ref.stdout)


@pytest.mark.skipif(not tc.REF_BIN.exists(), reason="reference binaries not built")
@pytest.mark.parametrize("style", ["global", "batch"])
def test_rknn_query_vamana(tmp_path, style):
    """ANQI_VAMANA=1 (the global passes, or the batched style; 2 passes of
    L = 128): the graph cache is named as the reference names it, recall is
    within 0.05 of the reference's own Vamana-refined build, and on the
    reference's refined graph the result lines are the reference's."""
    pfx, env, z = tc.sample_prefix(tmp_path, 32)
    env = dict(env, ANQI_VAMANA="1", ANQI_VAMANA_STYLE=style)
    ref_env = {k: v for k, v in os.environ.items() if not k.startswith("ANQI_")}
    ref_env.update(env, OMP_NUM_THREADS="1", ANQI_GRAPH_CACHE_DIR=str(tmp_path / "ref" / "graph"),
                   ANQI_VERIFIER_CACHE_DIR=str(tmp_path / "ref" / "verifier"))
    for sub in ("graph", "verifier"):
        (tmp_path / "ref" / sub).mkdir(parents=True)
    ref = subprocess.run([str(tc.REF_BIN), "16,32,64", str(pfx), "48", "500", "64", "600", "10"], env=ref_env,
                         capture_output=True, text=True, timeout=300)
    assert ref.returncode == 0, ref.stderr
    rc, ours, err = tc.run("rknn_query", "16,32,64", pfx, 48, 500, 64, 600, 10, env=env)
    assert rc == 0, err
    rl = lines(ref.stdout)
    for L, v in lines(ours).items():
        assert abs(v[0] - rl[L][0]) < 0.05, (L, v, rl[L])
    gref = list((tmp_path / "ref" / "graph").glob("fd_metric_*"))
    gours = list(Path(env["ANQI_GRAPH_CACHE_DIR"]).glob("fd_metric_*"))
    assert len(gref) == 1 and len(gours) == 1 and gref[0].name == gours[0].name
    gours[0].write_bytes(gref[0].read_bytes())
    for suffix in ("_approxlift_graph_", "_anqi_meta_graph_"):
        for p in (tmp_path / "ref" / "graph").glob(suffix + "*"):
            (Path(env["ANQI_GRAPH_CACHE_DIR"]) / p.name).write_bytes(p.read_bytes())
    rc, ours, err = tc.run("rknn_query", "16,32,64", pfx, 48, 500, 64, 600, 10, env=env)
    assert rc == 0, err
    assert lines(ours) == lines(ref.stdout)


@pytest.mark.skipif(not tc.REF_BIN.exists(), reason="reference binaries not built")
@pytest.mark.parametrize("policy", ["ball_rng", "residual_cover", "lsg_bubble_hybrid", "bubble_auto"])
def test_rknn_query_edge_policy(tmp_path, policy):
    """ANQI_EDGE_POLICY with a residual table (ANQI_EDGE_RESID_FILE) and an LSG
    mu table: the graph cache is named as the reference names it (the _edge
    key), the build's recall is within 0.05 of the reference's own build under
    the policy, and on the reference's graph the result lines are the
    reference's."""
    pfx, env, z = tc.sample_prefix(tmp_path, 32)
    n = z["base"].shape[0]
    rng = np.random.default_rng(4)
    rf = tmp_path / "resid.bin"
    mf = tmp_path / "mu.bin"
    rng.normal(0.0, 2.0, size=(n, 100)).astype(np.float32).tofile(rf)
    np.exp(rng.normal(0.0, 0.3, size=n)).astype(np.float32).tofile(mf)
    env = dict(env, ANQI_EDGE_POLICY=policy, ANQI_EDGE_RESID_FILE=str(rf), ANQI_LSG_MU_FILE=str(mf))
    ref_env = {k: v for k, v in os.environ.items() if not k.startswith("ANQI_")}
    ref_env.update(env, OMP_NUM_THREADS="1", ANQI_GRAPH_CACHE_DIR=str(tmp_path / "ref" / "graph"),
                   ANQI_VERIFIER_CACHE_DIR=str(tmp_path / "ref" / "verifier"))
    for sub in ("graph", "verifier"):
        (tmp_path / "ref" / sub).mkdir(parents=True)
    ref = subprocess.run([str(tc.REF_BIN), "16,32,64", str(pfx), "48", "500", "64", "600", "10"], env=ref_env,
                         capture_output=True, text=True, timeout=300)
    assert ref.returncode == 0, ref.stderr
    rc, ours, err = tc.run("rknn_query", "16,32,64", pfx, 48, 500, 64, 600, 10, env=env)
    assert rc == 0, err
    assert "[edge-policy]" in err
    rl = lines(ref.stdout)
    for L, v in lines(ours).items():
        assert abs(v[0] - rl[L][0]) < 0.05, (L, v, rl[L])
    gref = list((tmp_path / "ref" / "graph").glob("fd_metric_*"))
    gours = list(Path(env["ANQI_GRAPH_CACHE_DIR"]).glob("fd_metric_*"))
    assert len(gref) == 1 and len(gours) == 1 and gref[0].name == gours[0].name
    gours[0].write_bytes(gref[0].read_bytes())
    for suffix in ("_approxlift_graph_", "_anqi_meta_graph_"):
        for p in (tmp_path / "ref" / "graph").glob(suffix + "*"):
            (Path(env["ANQI_GRAPH_CACHE_DIR"]) / p.name).write_bytes(p.read_bytes())
    rc, ours, err = tc.run("rknn_query", "16,32,64", pfx, 48, 500, 64, 600, 10, env=env)
    assert rc == 0, err
    assert lines(ours) == lines(ref.stdout)


def test_rknn_query_edge_policy_errors(tmp_path):
    """The reference's exit-2 errors of the policy configuration, at graph
    build time: LSG without its mu table, a missing residual table."""
    pfx, env, _ = tc.sample_prefix(tmp_path, 32)
    rc, _, err = tc.run("rknn_query", "16", pfx, 48, 500, 64, 600, 10, env=dict(env, ANQI_EDGE_POLICY="lsg_rng"))
    assert rc == 2 and "requires ANQI_LSG_MU_FILE" in err
    rc, _, err = tc.run("rknn_query", "16", pfx, 48, 500, 64, 600, 10,
                        env=dict(env, ANQI_EDGE_POLICY="ball_rng", ANQI_EDGE_RESID_FILE=str(tmp_path / "none.bin")))
    assert rc == 2 and "residual_cover requested but missing" in err
