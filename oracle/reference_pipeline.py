"""Test infrastructure only: the reference's own pipeline, end to end, on the
host CPU -- the benchmark's reference arm.

Every process this starts runs the reference's code or a CPU checker; none
loads the B200 library:

1. ``build_aknn_source`` (the reference binary, oracle/_ref) writes the AKNN
   source records and its own build seconds (tools/build_aknn_source.cpp:141-155);
2. the LRQ trainer: ``anqi.lrq_train`` is a NumPy restatement of
   tools/train_final_m8_u8.py that writes byte-identical files (pinned by
   tests/test_cpu_host.py);
3. exact reverse-kNN ground truth: ``oracle/gt_cpu`` (host CPU, bit-identical to
   tools/dataset_gt.cpp on small-integer data, pinned by tests/test_gt_cpu.py);
4. ``rknn_query`` (the reference binary) under scripts/run_final.sh's pinned
   environment, calibrated timing off: it builds the lifted G48 graph and the
   verifier once (cached for the next k), then runs the query loop -- lift,
   range_search, postfilter and evaluation -- once per entry of its L list and
   prints one result line per entry (src/rknn_query.cpp:2846-2877).
"""
from __future__ import annotations

import os
import re
import subprocess
import sys
import time
from pathlib import Path

REPO = Path(__file__).resolve().parent.parent
REF_BIN = REPO / "oracle" / "_ref"
GT_CPU = REPO / "oracle" / "gt_cpu"

# scripts/run_final.sh:68-95 (the pinned configuration), calibrated timing off
RUN_FINAL_ENV = {
    "ANQI_GRAPH_GEOMETRY": "anyk_lift", "ANQI_RADIUS_MODE": "rankm_resid_u8_lrq_floor",
    "ANQI_VERIFIER_PLACEMENT": "postfilter", "ANQI_RANKM": "8", "ANQI_NK": "100", "ANQI_GRAPH_NK": "100",
    "ANQI_RANKM_SLACK": "0", "ANQI_RECHECK": "0", "ANQI_RQ_OBJECTIVE": "radius_reconstruction", "ANQI_ALPHA": "1.2",
    "ANQI_LIFTNNK": "50", "ANQI_GRAPHNND": "6", "ANQI_BUILD_BREAKDOWN": "1", "ANQI_PREBUILT_TOPK_K": "100",
    "ANQI_BENCH_CALIBRATED_TIMING": "0",
}
UNSET = ("ANQI_GRAPH_RANKM", "ANQI_SPECIFIC", "ANQI_CANDIDATE_ENVELOPE", "ANQI_RADIUS_RELAX", "ANQI_RQ_CODEBOOK",
         "ANQI_RQ_CODEBOOK_ID", "ANQI_RQ_BASIS_ID", "ANQI_RADIUS_SOURCE_ID", "ANQI_GRAPH_RADIUS_SOURCE_PFX",
         "ANQI_GRAPH_RADIUS_ID", "ANQI_VAMANA", "ANQI_EDGE_POLICY", "ANQI_QUERY_VISITED", "ANQI_TIME_BREAKDOWN",
         "ANQI_BENCH_REPEATS", "ANQI_QUERY_SINGLE_ENTRY", "ANQI_VAMANA_QUERY_ENTRY")

POINT = re.compile(r"\[rknn\] L_descent=(\d+)\s*\| recall=([\d.]+) precision=([\d.]+) F1=([\d.]+) \| avg cand=([\d.]+) "
                   r"pred=([\d.]+) #dist=([\d.]+) \| QPS=([\d.]+)")
GDIST = re.compile(r"DIST_BREAKDOWN L_descent=(\d+) #graph_dist=([\d.]+) #verify_dist=([\d.]+)")
BUILD = re.compile(r"\[rknn\] BUILD_TIME=([\d.]+)s .*index=([\d.]+)s")
BREAKDOWN = re.compile(r"BUILD_BREAKDOWN .*graph_index_s=([\d.]+) index_total_s=([\d.]+)")


def unavailable_reason() -> str | None:
    for exe in ("build_aknn_source", "rknn_query"):
        if not (REF_BIN / exe).exists():
            return f"oracle/_ref/{exe} is not built (make -C oracle ref REF=<reference tree>)"
    if not GT_CPU.exists():
        return "oracle/gt_cpu is not built (make -C oracle oracle)"
    flags = Path("/proc/cpuinfo").read_text() if Path("/proc/cpuinfo").exists() else ""
    if "avx512f" not in flags:
        return "host CPU lacks AVX-512 (the reference's binaries require it)"
    return None


def _run(cmd, env, log, timeout):
    t0 = time.perf_counter()
    p = subprocess.run([str(c) for c in cmd], capture_output=True, text=True, env=env, timeout=timeout)
    dt = time.perf_counter() - t0
    if p.returncode != 0:
        raise RuntimeError(f"{Path(str(cmd[0])).name} exited {p.returncode}: {(p.stderr or p.stdout)[-400:]}")
    log(f"{Path(str(cmd[0])).name} {dt:.1f}s")
    return p.stdout, dt


def read_seconds(path: Path) -> float:
    for line in Path(path).read_text().splitlines():
        f = line.split()
        if len(f) == 2 and f[0] == "seconds":
            return float(f[1])
    raise ValueError(f"no seconds line in {path}")


def build(pfx: Path, threads: int, log=print, timeout: float = 3600.0) -> dict:
    """Steps 1-3 on prefix files PFX_base.bin / PFX_query.bin (and PFX_lifted.meta)."""
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    out = {}
    _, out["aknn_wall_s"] = _run([REF_BIN / "build_aknn_source", f"{pfx}_base.bin", pfx, 100, 500, 64, 600, threads, 10,
                                  "l2"], env, log, timeout)
    out["aknn_build_s"] = read_seconds(Path(f"{pfx}_aknn_build_time.meta"))
    tenv = dict(env, PYTHONPATH=str(REPO / "anqi-implementation_b200"))
    _, out["verifier_train_wall_s"] = _run([sys.executable, "-m", "anqi.lrq_train", "--pfx", pfx, "--threshold-source",
                                            f"{pfx}_baseknn_aknn.rec"], tenv, log, timeout)
    out["verifier_train_s"] = read_seconds(Path(f"{pfx}_verifier_train_time.meta"))
    gt_out, out["ground_truth_s"] = _run([GT_CPU, f"{pfx}_base.bin", f"{pfx}_query.bin", f"{pfx}_baseknn_aknn.rec",
                                          pfx, 100, "10,50,100", threads], env, log, timeout)
    out["ground_truth_path"] = gt_out.strip().splitlines()[-1]
    return out


def query(pfx: Path, k: int, Ls, threads: int, cache: Path, build_info: dict, log=print,
          timeout: float = 3600.0) -> dict:
    """Step 4 for one k: rknn_query over the L list; returns the result points
    in list order and the build / load line."""
    env = {key: v for key, v in os.environ.items() if key not in UNSET}
    env.update(RUN_FINAL_ENV)
    env.update({"OMP_NUM_THREADS": str(threads), "ANQI_PREBUILT_TOPK_REC": f"{pfx}_baseknn_aknn.rec",
                "ANQI_GRAPH_CACHE_DIR": str(cache / "graph"), "ANQI_VERIFIER_CACHE_DIR": str(cache / "verifier"),
                "ANQI_AKNN_BUILD_SECONDS": f"{build_info['aknn_build_s']:.6f}",
                "ANQI_VERIFIER_TRAIN_SECONDS": f"{build_info['verifier_train_s']:.6f}"})
    (cache / "graph").mkdir(parents=True, exist_ok=True)
    (cache / "verifier").mkdir(parents=True, exist_ok=True)
    stdout, wall = _run([REF_BIN / "rknn_query", ",".join(str(L) for L in Ls), pfx, 48, 500, 64, 600, k], env, log,
                        timeout)
    points = []
    gd = [m for m in GDIST.finditer(stdout)]
    for i, m in enumerate(POINT.finditer(stdout)):
        p = {"L": int(m.group(1)), "recall": float(m.group(2)), "precision": float(m.group(3)),
             "f1": float(m.group(4)), "cand": float(m.group(5)), "pred": float(m.group(6)),
             "dist": float(m.group(7)), "qps": float(m.group(8))}
        if i < len(gd):
            p["graph_dist"] = float(gd[i].group(2))
        points.append(p)
    if len(points) != len(Ls):
        raise RuntimeError(f"rknn_query printed {len(points)} result lines for {len(Ls)} beam widths")
    res = {"points": points, "wall_s": wall}
    b = BUILD.search(stdout)
    if b:
        res["build_time_s"] = float(b.group(1))
        res["index_s"] = float(b.group(2))
    bd = BREAKDOWN.search(stdout)
    if bd:
        res["graph_index_s"] = float(bd.group(1))
    return res
