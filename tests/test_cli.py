"""Command-line drivers: argv handling and exit codes of the reference's CLIs
(tools/build_aknn_source.cpp:39-66, tools/dataset_gt.cpp:147-190,
src/rknn_query.cpp:1547-1720) -- every case here is rejected before the device
is touched, so this runs on CPU."""
import os
import struct
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from anqi import formats

REPO = Path(__file__).resolve().parent.parent
BIN = REPO / "anqi-implementation_b200" / "bin"
GOLDEN = REPO / "tests" / "golden"


@pytest.fixture(scope="module", autouse=True)
def built():
    if not all((BIN / b).exists() for b in ("build_aknn_source", "dataset_gt", "rknn_query")):
        subprocess.run([sys.executable, str(REPO / "anqi-implementation_b200" / "build.py")], check=True)


def run(name, *args, env=None):
    e = {k: v for k, v in os.environ.items() if not k.startswith("ANQI_")}
    e.update(env or {})
    p = subprocess.run([str(BIN / name), *map(str, args)], capture_output=True, text=True, env=e, timeout=120)
    return p.returncode, p.stdout, p.stderr


def write_fbin(path, x):
    formats.write_fbin(path, np.asarray(x, np.float32))


# ------------------------------------------------------------ build_aknn_source

def test_aknn_usage_and_arguments(tmp_path):
    assert run("build_aknn_source")[0] == 2
    assert run("build_aknn_source", *["x"] * 10)[0] == 2
    base = tmp_path / "b.bin"
    write_fbin(base, np.zeros((300, 4)))
    rc, _, err = run("build_aknn_source", base, tmp_path / "p", 100, 64, 8, 64, 4, 10, "cosine")
    assert rc == 2 and "metric must be l2 or ip" in err
    assert run("build_aknn_source", base, tmp_path / "p", "abc")[0] == 2


def test_aknn_bad_input_exits_3(tmp_path):
    rc, _, err = run("build_aknn_source", tmp_path / "missing.bin", tmp_path / "p")
    assert rc == 3 and "invalid base file or K" in err
    small = tmp_path / "small.bin"
    write_fbin(small, np.zeros((100, 4)))          # n <= K
    assert run("build_aknn_source", small, tmp_path / "p", 100)[0] == 3
    trunc = tmp_path / "trunc.bin"
    trunc.write_bytes(struct.pack("<II", 500, 4) + b"\0" * 16)
    assert run("build_aknn_source", trunc, tmp_path / "p")[0] == 3


# ------------------------------------------------------------------- dataset_gt

def test_dgt_usage_and_options(tmp_path):
    assert run("dataset_gt")[0] == 2
    assert run("dataset_gt", "--bogus", "1")[0] == 2
    rc, _, err = run("dataset_gt", "--base", "b", "--out_prefix", "p", "--mode", "all")
    assert rc == 2 and "mode must be" in err
    assert run("dataset_gt", "--base", "b", "--out_prefix", "p", "--K", "0", "--mode", "thresholds")[0] == 2
    assert run("dataset_gt", "--base", "b", "--out_prefix", "p", "--K")[0] == 2       # missing value
    assert run("dataset_gt", "--base", "b", "--out_prefix", "p")[0] == 2              # both needs --query
    assert run("dataset_gt", "--base", "b", "--out_prefix", "p", "--mode", "thresholds", "--metric", "cos")[0] == 2


def test_dgt_bad_input(tmp_path):
    rc, _, err = run("dataset_gt", "--base", tmp_path / "none.bin", "--out_prefix", tmp_path / "p",
                     "--mode", "thresholds")
    assert rc == 3 and "cannot open" in err
    base = tmp_path / "b.bin"
    write_fbin(base, np.zeros((50, 4)))
    rc, out, err = run("dataset_gt", "--base", base, "--out_prefix", tmp_path / "p", "--mode", "thresholds",
                       "--K", "100")
    assert rc == 2 and "rk_k <= K < base vector count" in err
    # ground-truth mode with a threshold table of the wrong n
    tbl = tmp_path / "t_baseknn_gt.bin"
    tbl.write_bytes(struct.pack("<II", 49, 10) + b"\0" * (49 * 10 * 8))
    q = tmp_path / "q.bin"
    write_fbin(q, np.zeros((3, 4)))
    rc, _, err = run("dataset_gt", "--base", base, "--query", q, "--out_prefix", tmp_path / "p", "--K", "10",
                     "--rk_k", "5", "--mode", "ground-truth", "--threshold-table", tbl)
    assert rc == 3 and "invalid threshold table" in err


# ------------------------------------------------------------------- rknn_query

RUN_FINAL_ENV = {
    "ANQI_GRAPH_GEOMETRY": "anyk_lift", "ANQI_RADIUS_MODE": "rankm_resid_u8_lrq_floor",
    "ANQI_VERIFIER_PLACEMENT": "postfilter", "ANQI_RANKM": "8", "ANQI_NK": "100", "ANQI_GRAPH_NK": "100",
    "ANQI_RANKM_SLACK": "0", "ANQI_RECHECK": "0", "ANQI_RQ_OBJECTIVE": "radius_reconstruction", "ANQI_ALPHA": "1.2",
    "ANQI_LIFTNNK": "50", "ANQI_GRAPHNND": "6", "ANQI_BUILD_BREAKDOWN": "1", "ANQI_PREBUILT_TOPK_K": "100",
    "ANQI_BENCH_CALIBRATED_TIMING": "0",
}


def sample_prefix(tmp_path, d=8):
    """The reference sample's prefix files (scripts/run_sample.sh) from the golden fixture."""
    z = dict(np.load(GOLDEN / f"sample_d{d}.npz"))
    pfx = tmp_path / "sample"
    formats.write_fbin(f"{pfx}_base.bin", z["base"])
    formats.write_fbin(f"{pfx}_query.bin", z["query"])
    Path(f"{pfx}_lifted.meta").write_text(f"0 {d} 100 l2 1.0\n")
    formats.write_rec(f"{pfx}_baseknn_aknn.rec", z["rec_ids"], z["rec_keys"])
    formats.write_basis(f"{pfx}_radbasis_M8.bin", z["mu"], z["basis"])
    formats.write_codebook(f"{pfx}_learned_rq_codebook_M8_u8.bin", z["codebook"])
    for k in (10, 50, 100):
        formats.write_rknn_csr(f"{pfx}_rknn_gt_k{k}.bin", z[f"gt_off_{k}"], z[f"gt_ids_{k}"], z[f"gt_keys_{k}"])
    env = dict(RUN_FINAL_ENV)
    env["ANQI_PREBUILT_TOPK_REC"] = f"{pfx}_baseknn_aknn.rec"
    env["ANQI_GRAPH_CACHE_DIR"] = str(tmp_path / "cache" / "graph")
    env["ANQI_VERIFIER_CACHE_DIR"] = str(tmp_path / "cache" / "verifier")
    return pfx, env, z


def test_rknn_usage_and_arguments(tmp_path):
    pfx, env, _ = sample_prefix(tmp_path)
    assert run("rknn_query")[0] == 2
    assert run("rknn_query", "16", pfx, 48, 500, 64, 600, 10, 7)[0] == 2
    rc, _, err = run("rknn_query", "16,x", pfx, env=env)
    assert rc == 2 and "invalid L_DESCENT=x" in err
    assert run("rknn_query", "16,,32", pfx, env=env)[0] == 2
    assert run("rknn_query", "16", pfx, 0, env=env)[0] == 2
    assert run("rknn_query", "16", pfx, 48, 500, 64, 600, 200, env=env)[0] == 2     # Kq > NK
    assert run("rknn_query", "16", pfx, env={**env, "ANQI_NK": "0"})[0] == 2
    assert run("rknn_query", "16", pfx, env={**env, "ANQI_RANKM": "x"})[0] == 2


def test_rknn_bad_inputs_exit_3(tmp_path):
    pfx, env, _ = sample_prefix(tmp_path)
    rc, _, err = run("rknn_query", "16", tmp_path / "nothing", env=env)
    assert rc == 3 and "lift metadata" in err
    # no k-specific GT for Kq=20 (metadata k=100)
    rc, _, err = run("rknn_query", "16", pfx, 48, 500, 64, 600, 20, env=env)
    assert rc == 3 and "missing k-specific reverse-kNN GT" in err
    # GT header naming the wrong query count
    bad = Path(f"{pfx}_rknn_gt_k10.bin")
    raw = bad.read_bytes()
    bad.write_bytes(struct.pack("<I", 31) + raw[4:])
    rc, _, err = run("rknn_query", "16", pfx, 48, 500, 64, 600, 10, env=env)
    assert rc == 3 and "invalid reverse-kNN GT header" in err
    bad.write_bytes(raw[:-4])
    rc, _, err = run("rknn_query", "16", pfx, 48, 500, 64, 600, 10, env=env)
    assert rc == 3 and "invalid reverse-kNN GT size" in err
    bad.write_bytes(raw)
    # metadata dimension disagreeing with the vectors
    Path(f"{pfx}_lifted.meta").write_text("0 9 100 l2 1.0\n")
    rc, _, err = run("rknn_query", "16", pfx, 48, 500, 64, 600, 10, env=env)
    assert rc == 3 and "dimension does not match" in err
    Path(f"{pfx}_lifted.meta").write_text("0 8 100 l2 1.0\n")
    # missing rank-M basis / corrupt codebook
    basis = Path(f"{pfx}_radbasis_M8.bin")
    braw = basis.read_bytes()
    basis.unlink()
    rc, _, err = run("rknn_query", "16", pfx, 48, 500, 64, 600, 10, env=env)
    assert rc == 3 and "rank-M basis" in err
    basis.write_bytes(braw)
    cb = Path(f"{pfx}_learned_rq_codebook_M8_u8.bin")
    cb.write_bytes(b"XXXXXXXX" + cb.read_bytes()[8:])
    rc, _, err = run("rknn_query", "16", pfx, 48, 500, 64, 600, 10, env=env)
    assert rc == 3 and "bad learned RQ codebook magic" in err


@pytest.mark.parametrize("var,val", [
    ("ANQI_GRAPH_GEOMETRY", "original"), ("ANQI_GRAPH_GEOMETRY", "bogus"), ("ANQI_RADIUS_MODE", "knots"),
    ("ANQI_RADIUS_MODE", "rankm_resid_u8_floor"), ("ANQI_RADIUS_MODE", "analytic_rankm"),
    ("ANQI_VERIFIER_PLACEMENT", "integrated"), ("ANQI_VERIFIER_PLACEMENT", "x"), ("ANQI_RECHECK", "1"),
    ("ANQI_SPECIFIC", "1"),
    ("ANQI_RQ_OBJECTIVE", "predicate_boundary"), ("ANQI_CANDIDATE_ENVELOPE", "verifier"),
    ("ANQI_RANKM_SLACK", "-1"), ("ANQI_RADIUS_RELAX", "0.1"),
])
def test_rknn_configurations_outside_the_path_exit_2(tmp_path, var, val):
    pfx, env, _ = sample_prefix(tmp_path)
    extra = {"ANQI_VAMANA": "1"} if var == "ANQI_VAMANA_STYLE" else {}
    rc, out, err = run("rknn_query", "16", pfx, 48, 500, 64, 600, 10, env={**env, **extra, var: val})
    assert rc == 2, (out, err)


def test_rknn_exact_f32_rejects_slack(tmp_path):
    pfx, env, _ = sample_prefix(tmp_path)
    rc, _, err = run("rknn_query", "16", pfx, 48, 500, 64, 600, 10,
                     env={**env, "ANQI_RADIUS_MODE": "exact_f32", "ANQI_RANKM_SLACK": "0.1"})
    assert rc == 2 and "exact_f32 postfilter does not accept ANQI_RANKM_SLACK" in err


def test_rknn_verifier_mode_files_are_validated(tmp_path):
    """A learned codebook of the wrong width and a malformed analytic model
    exit 3 before any device work, as the reference does."""
    pfx, env, _ = sample_prefix(tmp_path)
    import lrq_forms as lf
    f, _ = lf.load()
    formats.write_codebook(f"{pfx}_learned_rq_codebook_M8_u4.bin", lf.codebook(f, 2), 8, 4)
    rc, _, err = run("rknn_query", "16", pfx, 48, 500, 64, 600, 10,
                     env={**env, "ANQI_RADIUS_MODE": "rankm_resid_u4_lrq_floor"})
    assert rc == 3, err
    Path(f"{pfx}_analytic_rankm_M8.bin").write_bytes(b"ANQIPW1\0" + b"\0" * 40)
    rc, _, err = run("rknn_query", "16", pfx, 48, 500, 64, 600, 10,
                     env={**env, "ANQI_RADIUS_MODE": "analytic_rankm", "ANQI_CANDIDATE_ENVELOPE": "graph_horizon"})
    assert rc == 3 and "analytic Rank-M header mismatch" in err


def test_rknn_ip_metric_refusals(tmp_path):
    """Under metric=ip the reference refuses the analytic verifier (an L2 power
    law) and a non-zero slack on the compact verifier (signed thresholds):
    rknn_query.cpp:1812-1816, 2417-2422."""
    pfx, env, _ = sample_prefix(tmp_path)
    Path(f"{pfx}_lifted.meta").write_text("0 8 100 ip 1.0\n")
    rc, _, err = run("rknn_query", "16", pfx, 48, 500, 64, 600, 10,
                     env={**env, "ANQI_RADIUS_MODE": "analytic_rankm", "ANQI_CANDIDATE_ENVELOPE": "graph_horizon"})
    assert rc == 2 and "does not support IP" in err
    rc, _, err = run("rknn_query", "16", pfx, 48, 500, 64, 600, 10, env={**env, "ANQI_RANKM_SLACK": "0.1"})
    assert rc == 2 and "ANQI_RANKM_SLACK=0" in err


REF_BIN = REPO / "oracle" / "_ref" / "rknn_query"


@pytest.mark.skipif(not REF_BIN.exists(), reason="reference binaries not built (make -C oracle ref)")
def test_rknn_finds_and_validates_the_reference_caches(tmp_path):
    """The reference's rknn_query (CPU) builds its graph / lift / verifier
    caches; this driver computes the same identity keys, finds every cache,
    and parses the reference's graph file, before it needs the device."""
    pfx, env, _ = sample_prefix(tmp_path)
    for d in (env["ANQI_GRAPH_CACHE_DIR"], env["ANQI_VERIFIER_CACHE_DIR"]):
        Path(d).mkdir(parents=True, exist_ok=True)
    e = {k: v for k, v in os.environ.items() if not k.startswith("ANQI_")}
    e.update(env)
    e["OMP_NUM_THREADS"] = "2"
    ref = subprocess.run([str(REF_BIN), "16", str(pfx), "48", "500", "64", "600", "10"], env=e, capture_output=True,
                         text=True, timeout=300)
    assert ref.returncode == 0, ref.stderr
    rc, out, err = run("rknn_query", "16", pfx, 48, 500, 64, 600, 10, env=env)
    key = [ln for ln in ref.stdout.splitlines() if ln.startswith("[rknn] graph cache key=")]
    assert key and key[0] in out
    cfg = [ln for ln in ref.stdout.splitlines() if ln.startswith("Index config:")]
    assert cfg and cfg[0] in out
    assert "[rknn] loaded independent compact verifier" in out
    assert "[rknn] loaded cached index" in out
    degree = [ln for ln in ref.stdout.splitlines() if ln.startswith("Degree:")]
    assert degree and degree[0] in out
    if rc != 0:  # no device here: everything up to the device stage ran
        assert rc == 7 and "no usable CUDA device" in err


def test_rknn_u8_base_validation(tmp_path):
    """ANQI_BASE_U8BIN (rknn_query.cpp:55-107): a missing or mis-sized uint8
    base exits 3 with the reference's messages, before any device work."""
    pfx, env, _ = sample_prefix(tmp_path)
    rc, _, err = run("rknn_query", "16", pfx, 48, 500, 64, 600, 10,
                     env={**env, "ANQI_BASE_U8BIN": str(tmp_path / "missing.u8bin")})
    assert rc == 3 and "cannot open uint8 base" in err
    bad = tmp_path / "bad.u8bin"
    bad.write_bytes(np.array([256, 8], np.uint32).tobytes() + bytes(256 * 8 - 1))
    rc, _, err = run("rknn_query", "16", pfx, 48, 500, 64, 600, 10, env={**env, "ANQI_BASE_U8BIN": str(bad)})
    assert rc == 3 and "bad uint8 base" in err


def test_rknn_streamed_warm_start_options(tmp_path):
    """The streamed warm start takes one source: a command or the compacted
    id file, not both (rknn_query.cpp:2106-2111)."""
    pfx, env, _ = sample_prefix(tmp_path)
    rc, _, err = run("rknn_query", "16", pfx, 48, 500, 64, 600, 10,
                     env={**env, "ANQI_PREBUILT_WARM_START_COMMAND": "cat /dev/null",
                          "ANQI_COMPACT_PREBUILT_TOPK_IDS_INPLACE": "1"})
    assert rc == 2 and "cannot be combined" in err
