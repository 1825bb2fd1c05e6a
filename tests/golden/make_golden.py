#!/usr/bin/env python3
"""Generate the golden fixtures from the reference implementation itself.

Runs only where the reference tree and the binaries built by ``make -C oracle ref``
exist.  Every number stored in the fixtures comes from the reference's own code:
its CLIs (build_aknn_source, dataset_gt, rknn_query), its NumPy trainer, and
oracle/ref_harness (the reference's functions driven stage by stage, one thread).

Fixtures:
  dist.npz        distance kernels of include/distance.h on random pairs
  sample_d8.npz   the reference's own sample (scripts/make_sample_dataset.py:24-26,
                  256 x 8 base, 32 queries, N(0,1), seed 20260819)
  sample_d32.npz  the same recipe at d = 32 (the small configuration of the build plan)
  sample_ip_d32.npz  the d = 32 sample under the ip metric (every stage, as sample_d32.npz)
  lrq_forms.npz   CompactLrqVerifier in every form (bits 0/2/4/8/16/32, three policies,
                  signed IP keys) and the analytic Rank-M model, on the d = 32 sample
  vamana.npz      the Vamana refine of build_index (global passes, the batched style
                  with its options, each with and without an edge policy) after the
                  G48 commit, on the d = 32 sample's lifted rows
  edge_policies.npz  the G48 select and commit stages (gather_candidates +
                  prune_pool_to_ids, commit_edges) under every edge policy of
                  include/index.h:283-829, on the d = 32 sample's lifted rows, with a
                  seeded residual table and LSG mu table

Usage: python tests/golden/make_golden.py --ref REFERENCE_TREE
       (or set ANQI_REFERENCE to the reference source tree)
"""
from __future__ import annotations

import argparse
import os
import re
import shutil
import struct
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
REFBIN = REPO / "oracle" / "_ref"


def write_fbin(path: Path, x: np.ndarray) -> None:
    x = np.ascontiguousarray(x, dtype=np.float32)
    with path.open("wb") as f:
        f.write(struct.pack("<II", x.shape[0], x.shape[1]))
        x.tofile(f)


def read_fbin(path: Path) -> np.ndarray:
    raw = path.read_bytes()
    n, d = struct.unpack("<II", raw[:8])
    return np.frombuffer(raw[8:], dtype=np.float32).reshape(n, d).copy()


def read_csr64(path: Path):
    raw = path.read_bytes()
    n = struct.unpack("<Q", raw[:8])[0]
    off = np.frombuffer(raw[8 : 8 + 8 * (n + 1)], dtype=np.uint64).copy()
    ids = np.frombuffer(raw[8 + 8 * (n + 1) :], dtype=np.uint32).copy()
    return off, ids


def read_heaps(path: Path, n: int, k: int):
    raw = np.fromfile(path, dtype=np.uint32)
    ids = raw[: n * k].reshape(n, k).copy()
    vals = raw[n * k :].view(np.float32).reshape(n, k).copy()
    return ids, vals


def run(cmd, env=None, cwd=None) -> str:
    full_env = dict(os.environ)
    if env:
        full_env.update(env)
    p = subprocess.run([str(c) for c in cmd], env=full_env, cwd=cwd, capture_output=True, text=True)
    if p.returncode != 0:
        sys.stderr.write(p.stdout[-4000:] + p.stderr[-4000:])
        raise SystemExit(f"command failed ({p.returncode}): {' '.join(map(str, cmd))}")
    return p.stdout


def dist_fixture(out: Path) -> None:
    rng = np.random.default_rng(7)
    data = {}
    for dim, m in [(8, 32), (10, 32), (16, 32), (32, 32), (34, 32), (128, 32), (130, 32), (962, 8)]:
        a = rng.normal(size=(m, dim)).astype(np.float32)
        b = rng.normal(size=(m, dim)).astype(np.float32)
        if dim in (128, 130):  # integer-valued rows as in the 1M x 128 mixture
            a[: m // 2] = np.round(rng.uniform(0, 255, size=(m // 2, dim))).astype(np.float32)
            b[: m // 2] = np.round(rng.uniform(0, 255, size=(m // 2, dim))).astype(np.float32)
        with tempfile.TemporaryDirectory() as td:
            inp = Path(td) / "in.bin"
            with inp.open("wb") as f:
                f.write(struct.pack("<II", m, dim))
                for i in range(m):
                    a[i].tofile(f)
                    b[i].tofile(f)
            run([REFBIN / "ref_harness", "dist", inp, Path(td) / "out.bin"])
            res = np.fromfile(Path(td) / "out.bin", dtype=np.float32).reshape(m, 4)
        data[f"a_{dim}"] = a
        data[f"b_{dim}"] = b
        data[f"l2_{dim}"] = res[:, 0]
        data[f"ip_{dim}"] = res[:, 1]
        data[f"norm_{dim}"] = res[:, 2]
        data[f"d2_{dim}"] = res[:, 3]
    np.savez_compressed(out, **data)


RESULT_RE = re.compile(
    r"\[rknn\] L_descent=(\d+)\s*\| recall=([\d.]+) precision=([\d.]+) F1=([\d.]+) \| "
    r"avg cand=(\d+) pred=(\d+) #dist=(\d+)"
)


def sample_fixture(ref: Path, d: int, out: Path, metric: str = "l2") -> None:
    work = Path(tempfile.mkdtemp(prefix=f"anqi_golden_d{d}_"))
    ip = metric == "ip"
    henv = {"ANQI_HARNESS_METRIC": metric}
    pfx = work / "sample"
    try:
        rng = np.random.default_rng(20260819)
        base = rng.normal(0.0, 1.0, size=(256, d)).astype(np.float32)
        query = rng.normal(0.0, 1.0, size=(32, d)).astype(np.float32)
        write_fbin(Path(f"{pfx}_base.bin"), base)
        write_fbin(Path(f"{pfx}_query.bin"), query)
        Path(f"{pfx}_lifted.meta").write_text(f"0 {d} 100 {metric} 1.0\n")
        one = {"OMP_NUM_THREADS": "1"}
        # AKNN source: run_sample.sh:16-17 parameters, one thread for a reproducible file.
        run([REFBIN / "build_aknn_source", f"{pfx}_base.bin", pfx, 100, 64, 8, 64, 1, 10, metric], env=one)
        thr = work / "thr"
        run([REFBIN / "dataset_gt", "--base", f"{pfx}_base.bin", "--K", 100, "--rk_k", 100, "--threads", 1,
             "--tile", 64, "--mode", "thresholds", "--metric", metric, "--out_prefix", thr], env=one)
        for k in (10, 50, 100):
            t = work / f"gt{k}"
            run([REFBIN / "dataset_gt", "--base", f"{pfx}_base.bin", "--query", f"{pfx}_query.bin", "--K", 100,
                 "--rk_k", k, "--threads", 1, "--tile", 64, "--mode", "ground-truth", "--metric", metric,
                 "--threshold-table", f"{thr}_baseknn_gt.bin", "--out_prefix", t], env=one)
            shutil.copy(f"{t}_rknn_gt.bin", f"{pfx}_rknn_gt_k{k}.bin")
        run([sys.executable, ref / "tools" / "train_final_m8_u8.py", "--pfx", pfx, "--threshold-source",
             f"{pfx}_baseknn_aknn.rec"], env=one)
        # rknn_query with the pinned environment of scripts/run_final.sh:55-95.
        env = {
            "OMP_NUM_THREADS": "1", "ANQI_GRAPH_GEOMETRY": "anyk_lift",
            "ANQI_RADIUS_MODE": "rankm_resid_u8_lrq_floor", "ANQI_VERIFIER_PLACEMENT": "postfilter",
            "ANQI_RANKM": "8", "ANQI_NK": "100", "ANQI_GRAPH_NK": "100", "ANQI_RANKM_SLACK": "0",
            "ANQI_RECHECK": "0", "ANQI_RQ_OBJECTIVE": "radius_reconstruction", "ANQI_ALPHA": "1.2",
            "ANQI_LIFTNNK": "50", "ANQI_GRAPHNND": "6", "ANQI_BUILD_BREAKDOWN": "1",
            "ANQI_PREBUILT_TOPK_REC": f"{pfx}_baseknn_aknn.rec", "ANQI_PREBUILT_TOPK_K": "100",
            "ANQI_GRAPH_CACHE_DIR": str(work / "cache" / "graph"),
            "ANQI_VERIFIER_CACHE_DIR": str(work / "cache" / "verifier"),
            "ANQI_BENCH_CALIBRATED_TIMING": "0", "ANQI_AKNN_BUILD_SECONDS": "0",
            "ANQI_VERIFIER_TRAIN_SECONDS": "0",
        }
        for key in list(os.environ):
            if key.startswith("ANQI_") and key not in env:
                env[key] = ""
        (work / "cache" / "graph").mkdir(parents=True)
        (work / "cache" / "verifier").mkdir(parents=True)
        ref_lines = {}
        for k in (10, 50, 100):
            stdout = run([REFBIN / "rknn_query", "16,32,64,128", pfx, 48, 500, 64, 600, k], env=env)
            for m in RESULT_RE.finditer(stdout):
                ref_lines[(k, int(m.group(1)))] = [float(m.group(i)) for i in range(2, 8)]
        lifted_files = sorted((work / "cache" / "graph").glob("_approxlift_graph_*.bin"))
        meta_files = sorted((work / "cache" / "graph").glob("_anqi_meta_graph_*.txt"))
        assert len(lifted_files) == 1 and len(meta_files) == 1
        lifted = read_fbin(lifted_files[0])
        mstar2, scale = (float(v) for v in meta_files[0].read_text().split())

        h = work / "h"
        run([REFBIN / "ref_harness", "verifier", pfx, h, 8, "floor", int(ip)])
        run([REFBIN / "ref_harness", "graph", lifted_files[0], f"{pfx}_baseknn_aknn.rec", 50, 48, h])
        thr_all = np.fromfile(f"{h}_thresholds.bin", dtype=np.float32).reshape(4, 256)
        query_out = {}
        meta_path = work / "meta.txt"
        meta_path.write_text(f"{mstar2!r} {scale!r}\n")
        for ki, k in enumerate((1, 10, 50, 100)):
            if k == 1:
                continue
            tp = work / f"thr{k}.bin"
            thr_all[ki].tofile(tp)
            for L in (16, 32, 64, 128):
                q = work / f"q{k}_{L}"
                run([REFBIN / "ref_harness", "query", lifted_files[0], f"{h}_graph.bin", f"{pfx}_base.bin",
                     f"{pfx}_query.bin", meta_path, tp, L, q], env=henv)
                off, ids = read_csr64(Path(f"{q}_cand.bin"))
                poff, pids = read_csr64(Path(f"{q}_pred.bin"))
                query_out[f"q_cand_off_{k}_{L}"] = off
                query_out[f"q_cand_{k}_{L}"] = ids
                query_out[f"q_pred_off_{k}_{L}"] = poff
                query_out[f"q_pred_{k}_{L}"] = pids
                query_out[f"q_ndist_{k}_{L}"] = np.fromfile(f"{q}_ndist.bin", dtype=np.uint32)
        a = work / "a"
        run([REFBIN / "ref_harness", "aknn", f"{pfx}_base.bin", a, 100, 64, 8, 64, 10, metric])

        rec = np.fromfile(f"{pfx}_baseknn_aknn.rec", dtype=np.uint32).reshape(256, 100, 2)
        data = dict(query_out)
        data["base"] = base
        data["query"] = query
        data["rec_ids"] = rec[:, :, 0].copy()
        data["rec_keys"] = rec[:, :, 1].view(np.float32).copy()
        for k in (10, 50, 100):
            raw = Path(f"{pfx}_rknn_gt_k{k}.bin").read_bytes()
            nq = struct.unpack("<I", raw[:4])[0]
            off = np.frombuffer(raw[4 : 4 + 4 * (nq + 1)], dtype=np.uint32)
            tot = int(off[-1])
            body = raw[4 + 4 * (nq + 1) :]
            data[f"gt_off_{k}"] = off.copy()
            data[f"gt_ids_{k}"] = np.frombuffer(body[: 4 * tot], dtype=np.uint32).copy()
            data[f"gt_keys_{k}"] = np.frombuffer(body[4 * tot :], dtype=np.float32).copy()
        raw = Path(f"{thr}_baseknn_gt.bin").read_bytes()
        data["exact_ids"] = np.frombuffer(raw[8 : 8 + 256 * 100 * 4], dtype=np.uint32).reshape(256, 100).copy()
        data["exact_keys"] = np.frombuffer(raw[8 + 256 * 100 * 4 :], dtype=np.float32).reshape(256, 100).copy()
        braw = Path(f"{pfx}_radbasis_M8.bin").read_bytes()
        data["mu"] = np.frombuffer(braw[8 : 8 + 400], dtype=np.float32).copy()
        data["basis"] = np.frombuffer(braw[408:], dtype=np.float32).reshape(8, 100).copy()
        craw = Path(f"{pfx}_learned_rq_codebook_M8_u8.bin").read_bytes()
        data["codebook"] = np.frombuffer(craw[24:], dtype=np.float32).reshape(100, 256).copy()
        vraw = Path(f"{h}_verifier.bin").read_bytes()
        data["verifier_bytes"] = np.frombuffer(vraw, dtype=np.uint8).copy()
        data["coeff"] = np.frombuffer(vraw[36 : 36 + 256 * 8 * 4], dtype=np.float32).reshape(256, 8).copy()
        data["codes"] = np.frombuffer(vraw[36 + 256 * 8 * 4 :], dtype=np.uint8).reshape(256, 100).copy()
        data["thresholds"] = thr_all  # k = 1, 10, 50, 100
        data["lifted"] = lifted
        data["mstar2"] = np.float64(mstar2)
        data["scale"] = np.float64(scale)
        for stage in ("warm", "join"):
            ids, vals = read_heaps(Path(f"{h}_g0_{stage}.bin"), 256, 50)
            data[f"g_{stage}_ids"] = ids
            data[f"g_{stage}_vals"] = vals
        for name in ("g0_rev", "O", "adj"):
            off, ids = read_csr64(Path(f"{h}_{name}.bin"))
            data[f"g_{name}_off"] = off
            data[f"g_{name}"] = ids
        data["g_pool_sizes"] = np.fromfile(f"{h}_pool_sizes.bin", dtype=np.uint32)
        data["graph_file"] = np.frombuffer(Path(f"{h}_graph.bin").read_bytes(), dtype=np.uint8).copy()
        off, ids = read_csr64(Path(f"{a}_leaves.bin"))
        data["a_leaf_off"] = off
        data["a_leaves"] = ids
        ids, vals = read_heaps(Path(f"{a}_g0_init.bin"), 256, 100)
        data["a_init_ids"] = ids
        data["a_init_vals"] = vals
        off, ids = read_csr64(Path(f"{a}_g0_rev.bin"))
        data["a_rev_off"] = off
        data["a_rev"] = ids
        fin = np.fromfile(f"{a}_final.bin", dtype=np.uint32)
        data["a_final_ids"] = fin[: 256 * 100].reshape(256, 100).copy()
        data["a_final_d"] = fin[256 * 100 :].view(np.float32).reshape(256, 100).copy()
        data["a_pool_sizes"] = np.fromfile(f"{a}_pool_sizes.bin", dtype=np.uint32)
        keys = sorted(ref_lines)
        data["ref_lines_k_L"] = np.array(keys, dtype=np.int32)
        data["ref_lines"] = np.array([ref_lines[x] for x in keys], dtype=np.float64)
        if ip:
            # the ip metric's scalar distance on random pairs (include/distance.h:170-174)
            prng = np.random.default_rng(9)
            for dim in (3, 8, 13, 32, 130):
                pa = prng.normal(size=(24, dim)).astype(np.float32)
                pb = prng.normal(size=(24, dim)).astype(np.float32)
                inp = work / f"ipd{dim}.bin"
                with inp.open("wb") as f:
                    f.write(struct.pack("<II", 24, dim))
                    for i in range(24):
                        pa[i].tofile(f)
                        pb[i].tofile(f)
                run([REFBIN / "ref_harness", "ipdist", inp, work / f"ipd{dim}.out"])
                data[f"ipd_a_{dim}"] = pa
                data[f"ipd_b_{dim}"] = pb
                data[f"ipd_{dim}"] = np.fromfile(work / f"ipd{dim}.out", dtype=np.float32)
        np.savez_compressed(out, **data)
    finally:
        shutil.rmtree(work, ignore_errors=True)


# (bits, policy, signed keys): every CompactLrqVerifier form and both key signs
LRQ_FORMS = [(0, "floor", 0), (2, "floor", 0), (2, "nearest", 0), (4, "ceil", 0), (8, "nearest", 0),
             (8, "ceil", 0), (16, "floor", 0), (32, "floor", 0), (8, "floor", 1), (32, "floor", 1)]


def form_codebook(lo: np.ndarray, hi: np.ndarray, bits: int) -> np.ndarray:
    """Sorted codebook rows: 2^bits evenly spaced centres from lo[k] to hi[k]
    (any sorted codebook exercises the codec; the tests rebuild it from lo/hi)."""
    cs = 1 << bits
    t = np.arange(cs, dtype=np.float64) / (cs - 1)
    return (lo[:, None].astype(np.float64) + t[None, :] * (hi - lo)[:, None].astype(np.float64)).astype(np.float32)


def lrq_forms_fixture(sample: Path, out: Path) -> None:
    """The reference's CompactLrqVerifier (build, save, materialize_k) in every
    form, on the d = 32 sample's AKNN cutoffs and basis; signed forms shift the
    keys and mu below zero as IP keys are."""
    z = dict(np.load(sample))
    data = {"lo": None, "hi": None}
    keys, mu, basis = z["rec_keys"].astype(np.float32), z["mu"].astype(np.float32), z["basis"].astype(np.float32)
    # residual range of the sample, widened a little (the codebook spans it)
    c = (keys.astype(np.float64) - mu) @ basis.astype(np.float64).T
    res = keys - (mu + c @ basis)
    lo = (res.min(0) - 0.25).astype(np.float32)
    hi = (res.max(0) + 0.25).astype(np.float32)
    data["lo"], data["hi"] = lo, hi
    shift = np.float32(keys.max() + 7.0)
    work = Path(tempfile.mkdtemp(prefix="anqi_golden_lrq_"))
    try:
        for bits, policy, signed in LRQ_FORMS:
            pfx = work / f"f{bits}{policy}{signed}"
            k_src = keys - shift if signed else keys
            m_src = mu - shift if signed else mu
            write_fbin(Path(f"{pfx}_base.bin"), z["base"])
            rec = np.empty(keys.shape + (2,), np.uint32)
            rec[:, :, 0] = z["rec_ids"]
            rec[:, :, 1] = k_src.view(np.uint32)
            rec.tofile(f"{pfx}_baseknn_aknn.rec")
            with open(f"{pfx}_radbasis_M8.bin", "wb") as f:
                f.write(struct.pack("<ii", 100, 8))
                m_src.astype(np.float32).tofile(f)
                basis.tofile(f)
            if bits in (2, 4, 8, 16):
                with open(f"{pfx}_learned_rq_codebook_M8_u{bits}.bin", "wb") as f:
                    f.write(b"ANQIRQ1\0" + struct.pack("<iiii", 100, 8, bits, 1 << bits))
                    form_codebook(lo, hi, bits).tofile(f)
            run([REFBIN / "ref_harness", "verifier", pfx, pfx, bits, policy, signed])
            tag = f"{bits}_{policy}_{signed}"
            data[f"vf_{tag}"] = np.frombuffer(Path(f"{pfx}_verifier.bin").read_bytes(), np.uint8)
            data[f"thr_{tag}"] = np.fromfile(f"{pfx}_thresholds.bin", np.float32).reshape(4, -1)
        data["shift"] = np.array([shift], np.float32)
        # analytic Rank-M models (ANQIPW1), flags 3 and 7 (centred log ratio)
        rng = np.random.default_rng(23)
        for flags in (3, 7):
            coeff = rng.normal(0.0, 1.0, size=(256, 8)).astype(np.float32)
            coeff[:, 0] = np.abs(coeff[:, 0]) * 5.0
            b0 = 0.37 if flags == 3 else -0.21
            path = work / f"pw{flags}.bin"
            with open(path, "wb") as f:
                f.write(b"ANQIPW1\0" + struct.pack("<QIIII", 256, 100, 8, 10, flags) + struct.pack("<d", b0))
                coeff.tofile(f)
            run([REFBIN / "ref_harness", "analytic", path, 256, 8, work / f"pw{flags}"])
            data[f"pw_coeff_{flags}"] = coeff
            data[f"pw_b0_{flags}"] = np.array([b0])
            data[f"pw_thr_{flags}"] = np.fromfile(work / f"pw{flags}_thresholds.bin", np.float32).reshape(2, 4, -1)
        np.savez_compressed(out, **data)
    finally:
        shutil.rmtree(work, ignore_errors=True)


# (name, environment): ANQI_EDGE_POLICY and its options (include/index.h:305-440)
EDGE_POLICIES = [
    ("residual_cover", {"ANQI_EDGE_POLICY": "residual_cover"}),
    ("residual_cover_scaled", {"ANQI_EDGE_POLICY": "residual_cover", "ANQI_EDGE_RESID_LAMBDA": "0.5",
                               "_scale": "1.7"}),
    ("residual_cover_ks", {"ANQI_EDGE_POLICY": "residual_cover", "ANQI_EDGE_KS": "0,5,200,7",
                           "ANQI_EDGE_RESID_BUDGET": "9"}),
    ("ball_rng", {"ANQI_EDGE_POLICY": "ball_rng"}),
    ("ball_rng_any", {"ANQI_EDGE_POLICY": "ball_rng", "ANQI_EDGE_BALL_OCCLUSION": "any", "_scale": "0.8"}),
    ("ball_rng_budget0", {"ANQI_EDGE_POLICY": "ball_rng", "ANQI_EDGE_RESID_BUDGET": "0"}),
    ("bubble_rng", {"ANQI_EDGE_POLICY": "bubble_rng", "ANQI_EDGE_RESID_LAMBDA": "2.0"}),
    ("ball_hybrid", {"ANQI_EDGE_POLICY": "ball_hybrid"}),
    ("ball_hybrid_budget0", {"ANQI_EDGE_POLICY": "ball_hybrid", "ANQI_EDGE_RESID_BUDGET": "0"}),
    ("ball_multik", {"ANQI_EDGE_POLICY": "ball_multik", "ANQI_EDGE_KS": "10,50,100"}),
    ("bubble_hybrid", {"ANQI_EDGE_POLICY": "bubble_hybrid", "ANQI_EDGE_KS": "10,50",
                       "ANQI_EDGE_RESID_BUDGET": "24"}),
    ("bubble_multik", {"ANQI_EDGE_POLICY": "bubble_multik", "ANQI_EDGE_BALL_OCCLUSION": "any"}),
    ("lsg_rng", {"ANQI_EDGE_POLICY": "lsg_rng"}),
    ("lsg_rng_half", {"ANQI_EDGE_POLICY": "lsg_rng", "ANQI_LSG_ALPHA": "0.5"}),
    ("lsg_rng_zero", {"ANQI_EDGE_POLICY": "lsg_rng", "ANQI_LSG_ALPHA": "0"}),
    ("lsg_bubble_hybrid", {"ANQI_EDGE_POLICY": "lsg_bubble_hybrid"}),
    ("bubble_auto", {"ANQI_EDGE_POLICY": "bubble_auto"}),
    ("bubble_auto_small", {"ANQI_EDGE_POLICY": "bubble_auto", "ANQI_EDGE_AUTO_CANDIDATES": "8",
                           "ANQI_EDGE_AUTO_MAX_SWAPS": "3", "ANQI_EDGE_BALL_OCCLUSION": "any"}),
    ("bubble_auto_full", {"ANQI_EDGE_POLICY": "bubble_auto_full", "ANQI_EDGE_KS": "10,100"}),
    ("unknown", {"ANQI_EDGE_POLICY": "no_such_policy"}),
]


def edge_policy_fixture(sample: Path, out: Path) -> None:
    """The reference's select (gather_candidates + prune_pool_to_ids) and
    commit_edges under every edge policy, driven by oracle/ref_harness graph
    on the d = 32 sample's lifted rows and AKNN records.  The residual table
    (n x 100) and the LSG mu table are seeded draws scaled to the sample's
    lifted distances; "_scale" writes the lift meta file the policy reads its
    scale from (otherwise absent: scale^2 = 1)."""
    z = dict(np.load(sample))
    lifted, rec_ids, rec_keys = z["lifted"], z["rec_ids"], z["rec_keys"]
    n = lifted.shape[0]
    rng = np.random.default_rng(31)
    med = float(np.median(z["g_join_vals"][z["g_join_vals"] < np.float32(3e38)]))
    resid = rng.normal(0.0, 0.3 * med, size=(n, 100)).astype(np.float32)
    mu = np.exp(rng.normal(0.0, 0.35, size=n)).astype(np.float32)
    data = {"resid": resid, "mu": mu, "names": np.array([p[0] for p in EDGE_POLICIES])}
    work = Path(tempfile.mkdtemp(prefix="anqi_golden_edge_"))
    try:
        lf = work / "lifted.bin"
        write_fbin(lf, lifted)
        rec = np.empty((n, 100, 2), np.uint32)
        rec[:, :, 0] = rec_ids
        rec[:, :, 1] = rec_keys.view(np.uint32)
        rf = work / "warm.rec"
        rec.tofile(rf)
        resid_f = work / "resid.bin"
        resid.tofile(resid_f)
        mu_f = work / "mu.bin"
        mu.tofile(mu_f)
        for name, env in EDGE_POLICIES:
            h = work / name
            (work / f"{name}_scratch").mkdir()
            env = dict(env)
            scale = env.pop("_scale", None)
            if scale is not None:
                (work / f"{name}_scratch" / "_anqi_meta.txt").write_text(f"1.5 {scale}\n")
            env.setdefault("ANQI_EDGE_RESID_FILE", str(resid_f))
            env.setdefault("ANQI_LSG_MU_FILE", str(mu_f))
            run([REFBIN / "ref_harness", "graph", lf, rf, 50, 48, h], env=env)
            for stage in ("O", "adj"):
                off, ids = read_csr64(Path(f"{h}_{stage}.bin"))
                data[f"{name}_{stage}_off"] = off
                data[f"{name}_{stage}"] = ids
            data[f"{name}_env"] = np.array([f"{k}={v}" for k, v in sorted(env.items())
                                            if k not in ("ANQI_EDGE_RESID_FILE", "ANQI_LSG_MU_FILE")])
            data[f"{name}_scale"] = np.float64(float(scale) if scale is not None else 1.0)
        np.savez_compressed(out, **data)
    finally:
        shutil.rmtree(work, ignore_errors=True)


# (name, environment) of the Vamana refine (include/index.h:936-1065, 1262-1285)
VAMANA_CONFIGS = [
    ("global", {"ANQI_VAMANA": "1", "ANQI_VAMANA_L": "32", "ANQI_VAMANA_PASS": "2"}),
    ("batch", {"ANQI_VAMANA": "1", "ANQI_VAMANA_STYLE": "batch", "ANQI_VAMANA_L": "32", "ANQI_VAMANA_PASS": "2"}),
    ("batch_opts", {"ANQI_VAMANA": "1", "ANQI_VAMANA_STYLE": "batch", "ANQI_VAMANA_L": "24", "ANQI_VAMANA_PASS": "3",
                    "ANQI_VAMANA_BATCH_FRAC": "0.1", "ANQI_VAMANA_BATCH_BASE": "3", "ANQI_VAMANA_MAX_BATCH": "20",
                    "ANQI_VAMANA_ENTRY": "17", "ANQI_VAMANA_EARLY_ALPHA": "1.1", "ANQI_VAMANA_EARLY_ALPHA_ONE": "1"}),
    ("batch_one_alpha", {"ANQI_VAMANA": "1", "ANQI_VAMANA_STYLE": "batch", "ANQI_VAMANA_L": "40",
                         "ANQI_VAMANA_PASS": "1", "ANQI_VAMANA_EARLY_ALPHA_ONE": "0", "ANQI_VAMANA_BATCH_BASE": "1.5"}),
    ("batch_ball", {"ANQI_VAMANA": "1", "ANQI_VAMANA_STYLE": "batch", "ANQI_VAMANA_L": "32", "ANQI_VAMANA_PASS": "2",
                    "ANQI_EDGE_POLICY": "ball_rng"}),
    ("global_cover", {"ANQI_VAMANA": "1", "ANQI_VAMANA_L": "32", "ANQI_VAMANA_PASS": "1",
                      "ANQI_EDGE_POLICY": "residual_cover"}),
]


def vamana_fixture(sample: Path, edge: Path, out: Path) -> None:
    """The reference's build_index Vamana refine after the G48 commit, driven
    by oracle/ref_harness graph with ANQI_VAMANA set, on the d = 32 sample
    (the edge policies' residual table where a policy is set)."""
    z = dict(np.load(sample))
    e = dict(np.load(edge))
    lifted, rec_ids, rec_keys = z["lifted"], z["rec_ids"], z["rec_keys"]
    n = lifted.shape[0]
    data = {"names": np.array([c[0] for c in VAMANA_CONFIGS])}
    work = Path(tempfile.mkdtemp(prefix="anqi_golden_vam_"))
    try:
        lf = work / "lifted.bin"
        write_fbin(lf, lifted)
        rec = np.empty((n, 100, 2), np.uint32)
        rec[:, :, 0] = rec_ids
        rec[:, :, 1] = rec_keys.view(np.uint32)
        rf = work / "warm.rec"
        rec.tofile(rf)
        resid_f = work / "resid.bin"
        e["resid"].tofile(resid_f)
        for name, env in VAMANA_CONFIGS:
            h = work / name
            (work / f"{name}_scratch").mkdir()
            env = dict(env, ANQI_EDGE_RESID_FILE=str(resid_f))
            run([REFBIN / "ref_harness", "graph", lf, rf, 50, 48, h], env=env)
            off, ids = read_csr64(Path(f"{h}_vam_adj.bin"))
            data[f"{name}_off"] = off
            data[f"{name}_adj"] = ids
            data[f"{name}_env"] = np.array([f"{k}={v}" for k, v in sorted(env.items()) if k != "ANQI_EDGE_RESID_FILE"])
        np.savez_compressed(out, **data)
    finally:
        shutil.rmtree(work, ignore_errors=True)


def main() -> int:
    ap = argparse.ArgumentParser()
    env = os.environ.get("ANQI_REFERENCE")
    ap.add_argument("--ref", type=Path, default=Path(env) if env else None,
                    help="reference source tree (default: $ANQI_REFERENCE)")
    ap.add_argument("--only", choices=("lrq_forms", "sample_ip", "edge_policies", "vamana"),
                    help="regenerate one fixture")
    args = ap.parse_args()
    if args.ref is None or not (args.ref / "include" / "index.h").exists():
        raise SystemExit("give the reference source tree with --ref or ANQI_REFERENCE")
    if not (REFBIN / "ref_harness").exists():
        raise SystemExit("build the reference first: make -C oracle ref")
    if args.only == "lrq_forms":
        lrq_forms_fixture(HERE / "sample_d32.npz", HERE / "lrq_forms.npz")
        return 0
    if args.only == "sample_ip":
        sample_fixture(args.ref, 32, HERE / "sample_ip_d32.npz", metric="ip")
        return 0
    if args.only == "edge_policies":
        edge_policy_fixture(HERE / "sample_d32.npz", HERE / "edge_policies.npz")
        return 0
    if args.only == "vamana":
        vamana_fixture(HERE / "sample_d32.npz", HERE / "edge_policies.npz", HERE / "vamana.npz")
        return 0
    dist_fixture(HERE / "dist.npz")
    sample_fixture(args.ref, 8, HERE / "sample_d8.npz")
    sample_fixture(args.ref, 32, HERE / "sample_d32.npz")
    lrq_forms_fixture(HERE / "sample_d32.npz", HERE / "lrq_forms.npz")
    sample_fixture(args.ref, 32, HERE / "sample_ip_d32.npz", metric="ip")
    edge_policy_fixture(HERE / "sample_d32.npz", HERE / "edge_policies.npz")
    vamana_fixture(HERE / "sample_d32.npz", HERE / "edge_policies.npz", HERE / "vamana.npz")
    for p in sorted(HERE.glob("*.npz")):
        print(f"{p.name}: {p.stat().st_size} bytes")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
