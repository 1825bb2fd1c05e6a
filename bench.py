#!/usr/bin/env python3
"""RkNN query throughput of the B200 implementation on the 1M x 128 mixture.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the reference's full-size configuration): 1,000,000 x 128 base
vectors, integers in [0, 255] from a 1,000-centre Gaussian mixture, 10,000
queries from the same mixture.  The index (AKNN top-100 source, M8/u8 LRQ
verifier, d+2 lift, G48 graph) is built on the GPU first (not timed as
queries); the exact RkNN ground truth is computed on the GPU for recall.

One step = one batch of 30,000 queries: the 10,000 queries once each for
k = 10, 50 and 100 (per-query k in a single launch), beam width L for all.
``value`` is queries/s over K steps with the batch resident in HBM (CUDA events
on the library's stream; each step one replay of the batch's CUDA graph);
``e2e`` is the same through the host-buffer C ABI
call (query upload from pinned memory and result download into pinned
buffers reused across calls, both inside the timed region).  The timed working set (lifted + base vectors, graph) is ~1.3 GB,
larger than the 126 MB L2.

Beside the timed steps: recall / precision / QPS over the reference's beam
width list (``per_L``), and, in the CPU-baseline leg, the reference's query
code on this index (timed on a bounded sample) and compared with the CUDA
results query by query (``parity``).

``--impl reference`` runs the reference's own pipeline on this host's cores
(its build_aknn_source, its trainer's NumPy restatement, CPU ground truth,
its rknn_query; oracle/reference_pipeline.py) on the same data, no GPU library
in any of its processes, and times the same steps with rknn_query's own clock.
Under torchrun every rank holds an index replica and runs its own batch
(weak scaling); rank 0 prints the line.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO / "anqi-implementation_b200"))

METRIC = "RkNN queries/s (1M x 128, k in {10,50,100}, FP32 bit-exact path)"
# the reference's own beam-width list (scripts/run_final.sh protocol)
SWEEP_L = [20, 52, 85, 128, 256, 512, 1024]


def bench_config(a, ks, world):
    """The workload both arms measure (identical in both lines)."""
    return {"workload": f"rknn_query {a.n}x{a.d}, {a.nq} queries x k{{{a.ks}}}, L={a.L}, "
                        "G48 graph, M8/u8 LRQ postfilter", "n": a.n, "d": a.d, "nq": a.nq,
            "queries_per_step": a.nq * len(ks), "ks": ks, "L": a.L, "parallelism": f"replicas x{world}",
            "l2": "working set > L2 (lifted+base+graph ~1.3 GB)"}


def log(*a):
    print("[bench]", *a, file=sys.stderr, flush=True)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--n", type=int, default=1_000_000)
    ap.add_argument("--d", type=int, default=128)
    ap.add_argument("--nq", type=int, default=10_000)
    ap.add_argument("--L", type=int, default=128)
    ap.add_argument("--ks", default="10,50,100")
    ap.add_argument("--data", choices=("mixture", "gaussian"), default="mixture",
                    help="mixture: the 1,000-centre integer mixture; gaussian: L2-normalised N(0,1) rows "
                         "(the 1M x 960 shape); exact ground truth needs d <= 256 (tensor path)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-gt", action="store_true", help="skip the exact ground truth (profiling runs; no recall)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU seconds of the cpu_baseline sample")
    ap.add_argument("--keep", type=Path, default=None, help="write the index prefix files here")
    ap.add_argument("--batched-queries", type=int, default=100_000,
                    help="queries of the batching form (per-query k and L, CUDA graph); 0 skips it")
    ap.add_argument("--batch", type=int, default=10_000)
    ap.add_argument("--batched-reps", type=int, default=2, help="timed passes over the batching-form queries")
    ap.add_argument("--graph-options", type=int, default=200_000,
                    help="rows of the mixture on which the graph options (both Vamana styles, an edge "
                         "policy) are built and queried beside the default graph; 0 skips it")
    ap.add_argument("--ip-metric", type=int, default=200_000,
                    help="rows of an L2-normalised N(0,1) index built and queried under the ip metric "
                         "(AKNN source, LRQ, lift, graph, exact ground truth); 0 skips it")
    ap.add_argument("--shape960", type=int, default=1_000_000,
                    help="rows of the batching form's second shape (L2-normalised N(0,1), d = 960) run after the "
                         "main line, with QPS and recall; 0 skips it")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class Clocks:
    """Samples nvidia-smi clocks/throttle reasons while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # the timed region starts once the sampler reports
            t0 = time.time()
            while not self.rows and time.time() - t0 < 10 and self.proc.poll() is None:
                time.sleep(0.02)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def mark(self):
        """Samples from here on are the ones taken during the timed region."""
        self.first = len(self.rows)

    def summary(self):
        rows = self.rows[getattr(self, "first", 0):] or self.rows[-1:]
        self.rows = rows
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) > 8 for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def measured_peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def build_workload(ctx, a, rank, log):
    from anqi import pipeline
    t0 = time.perf_counter()
    if a.data == "gaussian":
        base, query = pipeline.gaussian(a.n, a.d, a.nq, seed=20260819 + rank, normalize=True)
    else:
        base, query = pipeline.mixture(a.n, a.d, a.nq, seed=20260819 + rank)
    log(f"data {base.shape} + {query.shape} in {time.perf_counter() - t0:.1f}s")
    ix = pipeline.build_index(ctx, base, train_workers=os.cpu_count() or 8, log=log)
    # the same AKNN source build with init_knn on FP32 CUDA cores (the plain
    # path): its lists must equal the tensor-core build's
    t0 = time.perf_counter()
    # (above 256 dimensions both builds run init_knn on the CUDA cores)
    ids32, keys32, st32 = (pipeline.aknn_build(ctx, base, precision="fp32") if a.d <= 256
                           else (ix.aknn_ids, ix.aknn_keys, ix.timings["aknn_stats"]))
    ix.timings["aknn_build_fp32_s"] = time.perf_counter() - t0
    # the index's build ran first, in a fresh context (it also mapped the
    # build scratch); one more tensor-core build compares like with like
    t0 = time.perf_counter()
    _, _, st16 = pipeline.aknn_build(ctx, base) if a.d <= 256 else (None, None, ix.timings["aknn_stats"])
    ix.timings["aknn_build_warm_s"] = time.perf_counter() - t0
    ix.timings["aknn_fp32_identical"] = bool(np.array_equal(ids32, ix.aknn_ids) and
                                             np.array_equal(keys32.view(np.uint32), ix.aknn_keys.view(np.uint32)))
    st = st16
    ix.timings["aknn_init_ms"] = {"bf16": round(st["init_ms"], 1), "fp32": round(st32["init_ms"], 1)}
    # the library's own clock around the build (excludes the Python-side host copies)
    ix.timings["aknn_total_ms"] = {"bf16": round(st["total_ms"], 1), "fp32": round(st32["total_ms"], 1),
                                   "bf16_first_build": round(ix.timings["aknn_stats"]["total_ms"], 1)}
    ix.timings["aknn_gather_kernel_ms"] = round(st["gather_kernel_ms"], 1)
    # the G48 build's LocalJoin in both forms from the same warm start: BF16
    # tensor-core filter + FP32 recheck (the index's) and FP32 CUDA cores
    wi, wv = pipeline.graph_warm_start(ctx, ix.lifted, ix.aknn_ids)
    j16 = pipeline.graph_localjoin(ctx, ix.lifted, wi, wv, "bf16")
    j32 = pipeline.graph_localjoin(ctx, ix.lifted, wi, wv, "fp32")
    ix.timings["localjoin"] = {
        "bf16_ms": round(j16[3], 1), "fp32_ms": round(j32[3], 1), "updates_per_round": j32[2],
        "identical": bool(j16[2] == j32[2] and np.array_equal(j16[0], j32[0])
                          and np.array_equal(j16[1].view(np.uint32), j32[1].view(np.uint32)))}
    del wi, wv, j16, j32
    log(f"LocalJoin {ix.timings['localjoin']}")
    # the LRQ fit in both forms on the same cutoff matrix: the index's (GPU
    # kernels, anqi.lrq_fit) and the NumPy trainer's; codebooks compared per
    # column range, thresholds per object at every k
    from anqi import lrq_train
    t0 = time.perf_counter()
    fit_np = lrq_train.train(ix.aknn_keys, len(ix.aknn_keys), workers=os.cpu_count() or 8, log=lambda s: None)
    t_np = time.perf_counter() - t0
    mu_c, g_c, b_c = (np.asarray(v, np.float32) for v in fit_np)
    coeff_c, codes_c = ctx.lrq_encode(ix.aknn_keys, mu_c, g_c, b_c)
    span = (b_c[:, -1].astype(np.float64) - b_c[:, 0])[:, None]
    agree = {}
    for k in (10, 50, 100):
        t_g = ctx.lrq_materialize(ix.coeff, ix.codes, ix.mu, ix.basis, ix.codebook, k)
        t_c = ctx.lrq_materialize(coeff_c, codes_c, mu_c, g_c, b_c, k)
        agree[k] = round(float(np.mean(np.isclose(t_g, t_c, rtol=1e-6, atol=1e-6))), 6)
    ix.numpy_fit = (coeff_c, codes_c, mu_c, g_c, b_c)
    ix.timings["lrq_fit"] = {"gpu_s": round(ix.timings["lrq_train_s"], 3), "numpy_s": round(t_np, 3),
                             "codebook_max_rel": float(np.max(np.abs(ix.codebook.astype(np.float64) - b_c) / span)),
                             "threshold_agree": agree}
    log(f"LRQ fit {ix.timings['lrq_fit']}")
    log(f"AKNN fp32 build {ix.timings['aknn_build_fp32_s']:.2f}s identical={ix.timings['aknn_fp32_identical']}")
    ks = [int(k) for k in a.ks.split(",")]
    if a.no_gt or a.d > 1024:
        return base, query, ix, ks, None
    # exact ground truth on the BF16 tensor path (bit-identical to FP32; the
    # AKNN lists bound each row's 100th key)
    t0 = time.perf_counter()
    _, ex_keys = pipeline.exact_thresholds(ctx, base, 100, method="tc", hints=ix.aknn_ids)
    t_thr = time.perf_counter() - t0
    ix.exact_keys = ex_keys
    gt = {}
    t0 = time.perf_counter()
    for k in ks:
        gt[k] = pipeline.rknn_ground_truth(ctx, base, query, ex_keys[:, k - 1], method="tc")
    log(f"exact thresholds {t_thr:.1f}s, RkNN ground truth {time.perf_counter() - t0:.1f}s, "
        f"mean |R| = {[round(float(np.diff(gt[k][0]).mean()), 2) for k in ks]}")
    ix.timings["exact_thresholds_s"] = t_thr
    ix.timings["rknn_ground_truth_s"] = time.perf_counter() - t0
    return base, query, ix, ks, gt


def write_index_files(d: Path, base, query, ix, ks, gt, ctx):
    """Index + workload files the reference harness reads (reference formats)."""
    from anqi import formats
    d.mkdir(parents=True, exist_ok=True)
    formats.write_fbin(d / "lifted.bin", ix.lifted)
    formats.write_fbin(d / "base.bin", base)
    formats.write_fbin(d / "query.bin", query)
    g = formats.Graph(len(base), ix.lifted.shape[1], ix.links.shape[1], ix.deg, ix.links, ix.tree)
    formats.write_graph(d / "graph.bin", g)
    formats.write_graph_meta(d / "meta.txt", ix.mstar2, ix.scale)
    for k in ks:
        thr = ctx.lrq_materialize(ix.coeff, ix.codes, ix.mu, ix.basis, ix.codebook, k)
        thr.tofile(d / f"thr{k}.bin")
        off, ids, keys = gt[k]
        formats.write_rknn_csr(d / f"gt{k}.bin", off, ids, keys)


def reference_qbench(d: Path, ks, L, threads, warmup, steps, nq):
    exe = REPO / "oracle" / "_ref" / "ref_harness"
    if not exe.exists():
        return None, "oracle/_ref/ref_harness is not built (needs the reference sources)"
    flags = Path("/proc/cpuinfo").read_text() if Path("/proc/cpuinfo").exists() else ""
    if "avx512f" not in flags:
        return None, "host CPU lacks AVX-512 (the reference requires it)"
    cmd = [str(exe), "qbench", str(d / "lifted.bin"), str(d / "graph.bin"), str(d / "base.bin"), str(d / "query.bin"),
           str(d / "meta.txt"), str(L), str(threads), str(warmup), str(steps), str(nq)]
    for k in ks:
        cmd += [str(d / f"thr{k}.bin"), str(d / f"gt{k}.bin")]
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        return None, f"reference harness failed ({p.returncode}): {p.stderr[-300:]}"
    line = [l for l in p.stdout.splitlines() if l.startswith("{")][-1]
    return json.loads(line), None


def run_batched(ctx, a, base, ix, rank):
    """Batching form: batched_queries more queries from the mixture, per-query
    k uniform in {10, 50, 100} and beam width uniform in [64, 600], run as
    batches of `batch` queries, each one replay of the captured CUDA graph
    (lift + entry, leaf ordering, search with the LRQ postfilter, CSR
    compaction).  Per-batch device latency (CUDA events) p50 / p99 and QPS over
    the whole run; recall against the exact RkNN of every query's own k."""
    from anqi import pipeline
    nqb, bs = a.batched_queries, a.batch
    q = pipeline.mixture_queries(nqb, a.d, qseed=7 + rank)
    rng = np.random.default_rng(11 + rank)
    ks = rng.choice(np.array([10, 50, 100], np.uint32), nqb).astype(np.uint32)
    Ls = rng.integers(64, 601, nqb).astype(np.uint32)
    nb = nqb // bs
    lat, preds = [], []
    for rep in range(1 + a.batched_reps):
        for i in range(nb):
            sl = slice(i * bs, (i + 1) * bs)
            Lb = Ls[sl].copy()
            Lb[0] = 600  # one beam-width bound for every batch: one captured graph
            ctx.query_upload(q[sl], ks[sl], Lb)
            if rep == 0 and i == 0:
                ctx.query_run_graph()  # plain run + capture
            ctx.timer_start()
            st = ctx.query_run_graph()
            lat.append(ctx.timer_stop())
            if rep == 0:
                preds.append(ctx.query_download())
    lat = np.array(lat[nb:] if a.batched_reps else lat)
    out = {"queries": nqb, "batch": bs, "k": "uniform {10,50,100}", "L": "uniform [64,600] (bound 600)",
           "qps": round(bs * len(lat) / (lat.sum() / 1e3), 1), "p50_ms": round(float(np.percentile(lat, 50)), 3),
           "p99_ms": round(float(np.percentile(lat, 99)), 3), "batches_timed": int(len(lat)), "cuda_graph": True,
           "visited_table": [st["visited_table"], st["visited_l2_table"]],
           "shape": {"warps_per_block": st["warps_per_block"], "candidate_tile": st["candidate_tile"]}}
    ex_keys = getattr(ix, "exact_keys", None)
    if ex_keys is not None:
        # exact RkNN of each query at its own k (tensor path), recall / precision
        rec = prec = 0.0
        ne = 0
        for k in (10, 50, 100):
            sel = np.nonzero(ks[:nb * bs] == k)[0]
            off, ids, _ = pipeline.rknn_ground_truth(ctx, base, q[sel], ex_keys[:, k - 1], method="tc")
            for j, qi in enumerate(sel):
                truth = ids[off[j]:off[j + 1]]
                if len(truth) == 0:
                    continue
                r = preds[qi // bs]
                p = r.pred(qi % bs)
                hit = len(np.intersect1d(p, truth))
                rec += hit / len(truth)
                prec += 1.0 if len(p) == 0 else hit / len(p)
                ne += 1
        out["recall"] = round(rec / max(ne, 1), 6)
        out["precision"] = round(prec / max(ne, 1), 6)
    return out


class _Env:
    """Sets environment variables for a block (the library reads its
    switches at call time) and restores them after."""

    def __init__(self, **kv):
        self.kv = kv

    def __enter__(self):
        self.old = {k: os.environ.get(k) for k in self.kv}
        os.environ.update(self.kv)

    def __exit__(self, *exc):
        for k, v in self.old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def run_plain(a, dev, ix, query, ks, steps, warmup):
    """The plain FP32 GPU path the batched form is compared with: the same
    bit-exact search kernel on the given object numbering (no breadth-first
    renumbering), work in query order (no leaf ordering), one plain launch per
    k (no CUDA graph, no per-query k), fixed launch shape and visited set (no
    autotuning).  Queries/s over `steps` passes of the three launches, each
    timed on the device around the launch (entry, search, compaction)."""
    from anqi import pipeline
    from anqi._lib import Context
    with _Env(ANQI_B200_RENUMBER="0", ANQI_B200_ORDER="0", ANQI_B200_HASH="0,4096", ANQI_B200_SHAPE="4,8"):
        with Context(dev) as c2:
            pipeline.load_index(c2, ix, ks)
            ms = 0.0
            for rep in range(warmup + steps):
                for k in ks:
                    c2.query_upload(query, k, a.L)
                    c2.timer_start()
                    c2.query_run()
                    t = c2.timer_stop()
                    if rep >= warmup:
                        ms += t
    nq = len(query)
    return {"qps": round(steps * nq * len(ks) / (ms / 1e3), 1), "ms_per_pass": round(ms / steps, 4),
            "launches_per_pass": len(ks), "renumbered": False, "leaf_ordered": False, "cuda_graph": False,
            "visited_table": [0, 4096], "shape": {"warps_per_block": 4, "candidate_tile": 8}}


def run_graph_options(ctx, a):
    """The G48 build's options on an n-row mixture index: the default graph,
    the global Vamana refine, the batched Vamana refine and the ball_rng edge
    policy (its residual table: each object's decoded LRQ residual at k = 10,
    50, 100, the table the reference's integrated verifier writes).  Per
    graph: device build seconds, then recall / precision and QPS of one
    launch over the queries at k = 10, 50, 100 (L = 128), against the exact
    RkNN."""
    import dataclasses
    from anqi import pipeline, vamana, edge_policy
    n, nq = a.graph_options, 2000
    base, query = pipeline.mixture(n, a.d, nq, seed=20260819)
    ix = pipeline.build_index(ctx, base, log=lambda *m: None)
    ks = [10, 50, 100]
    _, ex = pipeline.exact_thresholds(ctx, base, 100, method="tc", hints=ix.aknn_ids)
    gt = {k: pipeline.rknn_ground_truth(ctx, base, query, ex[:, k - 1], method="tc") for k in ks}
    # the residual table of the policy: materialized threshold minus the rank-M reconstruction
    recon = ix.mu[None, :].astype(np.float64) + ix.coeff.astype(np.float64) @ ix.basis.astype(np.float64)
    resid = np.zeros((n, 100), np.float32)
    for k in ks:
        resid[:, k - 1] = (ctx.lrq_materialize(ix.coeff, ix.codes, ix.mu, ix.basis, ix.codebook, k)
                           - recon[:, k - 1]).astype(np.float32)
    pol = edge_policy.EdgePolicy("ball_rng", flags=edge_policy.BALL | edge_policy.PURE, ks=ks, nk=100, budget=16,
                                 occlude_all=True, auto_candidates=48, auto_max_swaps=48, lam=1.0,
                                 scale2=float(ix.scale) ** 2, resid=resid)
    variants = {
        "default": {},
        "vamana_global": {"vamana": vamana.from_env({"ANQI_VAMANA": "1"})},
        "vamana_batch": {"vamana": vamana.from_env({"ANQI_VAMANA": "1", "ANQI_VAMANA_STYLE": "batch"}, ix.lifted)},
        "edge_ball_rng": {"edge": pol},
    }
    out = {"n": n, "nq": nq, "L": a.L}
    qb = np.ascontiguousarray(np.tile(query, (len(ks), 1)))
    kb = np.repeat(np.array(ks, np.uint32), nq)
    for name, kw in variants.items():
        t0 = time.perf_counter()
        deg, links, tree, st = pipeline.graph_build(ctx, ix.lifted, ix.aknn_ids, **kw)
        build_s = time.perf_counter() - t0
        gix = dataclasses.replace(ix, deg=deg, links=links, tree=tree)
        pipeline.load_index(ctx, gix, ks)
        res = {"graph_build_s": round(build_s, 3), "graph_library_ms": round(st["total_ms"], 1),
               "mean_degree": round(float(deg.mean()), 2), "per_k": {}}
        for k in ks:
            ctx.query_upload(query, k, a.L)
            ctx.query_run()
            e = ctx.query_evaluate(gt[k][0], gt[k][1])
            res["per_k"][k] = {"recall": round(e["recall"], 6), "precision": round(e["precision"], 6)}
        ctx.query_upload(qb, kb, np.full(len(kb), a.L, np.uint32))
        for _ in range(3):
            ctx.query_run_graph()
        ctx.timer_start()
        for _ in range(10):
            ctx.query_run_graph()
        ms = ctx.timer_stop()
        res["qps"] = round(10 * len(kb) / (ms / 1e3), 1)
        out[name] = res
    return out


def run_ip_metric(ctx, a):
    """The ip metric on an n-row L2-normalised N(0,1) index (d = a.d): the
    AKNN source under ip (angular forest, record keys -<a, b>), the LRQ fit on
    those signed keys (u8, floor), the ip lift (s^2 r), the G48 graph, the
    exact ip ground truth (keys -<a, b>, FP32 CUDA cores), then recall /
    precision per k and the QPS of one CUDA-graph replay over the queries at
    every k (L = a.L).  The same stages as build_aknn_source / lrq_train /
    dataset_gt / rknn_query with metric ip."""
    from anqi import pipeline, lrq_fit
    n, nq, ks = a.ip_metric, 2000, [10, 50, 100]
    base, query = pipeline.gaussian(n, a.d, nq, seed=20260819, normalize=True)
    t = {}
    t0 = time.perf_counter()
    ids, keys, st = pipeline.aknn_build(ctx, base, metric="ip")
    t["aknn_build"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    mu, basis, cb = (np.asarray(v, np.float32) for v in
                     lrq_fit.train_gpu(keys, len(keys), device=ctx.device, log=lambda s: None))
    t["lrq_train"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    coeff, codes, _ = ctx.lrq_encode_bits(keys, mu, basis, cb, 8)
    lifted, m2, sc = ctx.lift(base, keys[:, -1], metric="ip")
    t["encode_lift"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    deg, links, tree, _ = pipeline.graph_build(ctx, lifted, ids)
    t["graph"] = time.perf_counter() - t0
    # the exact ground truth on the BF16 tensor path (the AKNN lists bound each
    # row's 100th key) and on FP32 CUDA cores: identical outputs
    t0 = time.perf_counter()
    ex_ids, ex = pipeline.exact_thresholds(ctx, base, 100, method="tc", hints=ids, metric="ip")
    t["exact_thresholds"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    gt = {k: pipeline.rknn_ground_truth(ctx, base, query, ex[:, k - 1], method="tc", metric="ip") for k in ks}
    t["rknn_ground_truth"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    f_ids, f_keys = pipeline.exact_thresholds(ctx, base, 100, metric="ip")
    t["exact_thresholds_fp32"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    f_gt = {k: pipeline.rknn_ground_truth(ctx, base, query, f_keys[:, k - 1], metric="ip") for k in ks}
    t["rknn_ground_truth_fp32"] = time.perf_counter() - t0
    gt_identical = bool(np.array_equal(f_ids, ex_ids) and np.array_equal(f_keys.view(np.uint32), ex.view(np.uint32))
                        and all(np.array_equal(f_gt[k][0], gt[k][0]) and np.array_equal(f_gt[k][1], gt[k][1])
                                for k in ks))
    del f_ids, f_keys, f_gt
    # the AKNN lists against the exact top-100 on every 100th row
    rows = range(0, n, 100)
    aknn_recall = float(np.mean([len(np.intersect1d(ids[i], ex_ids[i])) for i in rows])) / 100.0
    del ex_ids
    ctx.index_load(base, lifted, deg, links, tree, sc, m2, metric="ip")
    ctx.verifier_load_bits(coeff, codes, None, keys.shape[1], mu, basis, cb, 8, signed_keys=True)
    for k in ks:
        ctx.verifier_materialize(k)
    per_k = {}
    for k in ks:
        ctx.query_upload(query, k, a.L)
        ctx.query_run()
        e = ctx.query_evaluate(gt[k][0], gt[k][1])
        per_k[k] = {"recall": round(e["recall"], 6), "precision": round(e["precision"], 6),
                    "mean_gt": round(float(np.diff(gt[k][0]).mean()), 3)}
    qb = np.ascontiguousarray(np.tile(query, (len(ks), 1)))
    kb = np.repeat(np.array(ks, np.uint32), nq)
    ctx.query_upload(qb, kb, np.full(len(kb), a.L, np.uint32))
    for _ in range(3):
        ctx.query_run_graph()
    ctx.timer_start()
    for _ in range(10):
        ctx.query_run_graph()
    ms = ctx.timer_stop()
    return {"n": n, "d": a.d, "nq": nq, "L": a.L, "data": "L2-normalised N(0,1) rows, metric ip",
            "seconds": {k: round(v, 3) for k, v in t.items()},
            "aknn_init_ms": round(st["init_ms"], 1), "aknn_gather_kernel_ms": round(st["gather_kernel_ms"], 1),
            "exact_gt_tc_equals_fp32": gt_identical, "aknn_recall_at_100": round(aknn_recall, 5), "mean_degree": round(float(deg.mean()), 2),
            "per_k": per_k, "qps": round(10 * len(kb) / (ms / 1e3), 1)}


def run_shape960(ctx, a, steps, warmup):
    """The batching form's second shape: n x 960 L2-normalised N(0,1) rows and
    10,000 queries, the whole index built here (AKNN source with the K-chunked
    tensor-core init_knn, LRQ fit, lift, G48 graph), the exact ground truth on
    the K-chunked tensor path, then the resident step of the main line (one
    graph replay over 10,000 queries x k = 10, 50, 100 at L) timed with CUDA
    events, and recall / precision per k against the exact RkNN."""
    from anqi import pipeline
    n, d, nq = a.shape960, 960, a.nq
    t0 = time.perf_counter()
    base, query = pipeline.gaussian(n, d, nq, seed=20260819, normalize=True)
    ix = pipeline.build_index(ctx, base, log=lambda *m: None)
    build_s = time.perf_counter() - t0
    ks = [10, 50, 100]
    t0 = time.perf_counter()
    _, ex = pipeline.exact_thresholds(ctx, base, 100, method="tc", hints=ix.aknn_ids)
    gt = {k: pipeline.rknn_ground_truth(ctx, base, query, ex[:, k - 1], method="tc") for k in ks}
    gt_s = time.perf_counter() - t0
    pipeline.load_index(ctx, ix, ks)
    per_k = {}
    for k in ks:
        off, ids, _ = gt[k]
        ctx.query_upload(query, k, a.L)
        ctx.query_run()
        e = ctx.query_evaluate(off, ids)
        per_k[k] = {"recall": round(e["recall"], 6), "precision": round(e["precision"], 6)}
    qb = np.ascontiguousarray(np.tile(query, (len(ks), 1)))
    kb = np.repeat(np.array(ks, np.uint32), nq)
    ctx.query_upload(qb, kb, np.full(len(kb), a.L, np.uint32))
    for _ in range(warmup):
        ctx.query_run_graph()
    ctx.timer_start()
    for _ in range(steps):
        st = ctx.query_run_graph()
    ms = ctx.timer_stop()
    t = ix.timings
    return {"n": n, "d": d, "nq": nq, "L": a.L, "queries_per_step": len(kb),
            "qps": round(steps * len(kb) / (ms / 1e3), 1), "ms_per_step": round(ms / steps, 4),
            "per_k": per_k, "search_ms": round(st["search_ms"], 4),
            "build_s": {"total": round(build_s, 3), "aknn": round(t["aknn_build_s"], 3),
                        "lrq_train": round(t["lrq_train_s"], 3), "lift": round(t["lift_s"], 3),
                        "graph": round(t["graph_build_s"], 3),
                        "aknn_init_ms": round(t["aknn_stats"]["init_ms"], 1),
                        "aknn_gather_kernel_ms": round(t["aknn_stats"]["gather_kernel_ms"], 1)},
            "exact_ground_truth_s": round(gt_s, 3),
            "shape": {"warps_per_block": st["warps_per_block"], "candidate_tile": st["candidate_tile"]}}


def run_ours(a, rank, world, local):
    from anqi._lib import Context
    import torch
    dev = local if world > 1 else 0
    ctx = Context(dev)
    base, query, ix, ks, gt = build_workload(ctx, a, rank, lambda *m: log(f"rank{rank}", *m) if rank == 0 else None)
    from anqi import pipeline
    pipeline.load_index(ctx, ix, ks)
    nq = len(query)
    nb = nq * len(ks)
    qb = np.ascontiguousarray(np.tile(query, (len(ks), 1)))
    kb = np.repeat(np.array(ks, np.uint32), nq)
    Lb = np.full(nb, a.L, np.uint32)
    # recall of the batch (device evaluation against the exact CSR)
    ev = {"recall": None, "precision": None}
    per_k = {}
    if gt is not None:
        ctx.query_upload(qb, kb, Lb)
        ctx.query_run(keep_candidates=True)
        gt_off = np.zeros(nb + 1, np.uint32)
        parts = []
        for j, k in enumerate(ks):
            off, ids, _ = gt[k]
            gt_off[j * nq + 1:(j + 1) * nq + 1] = off[1:] + gt_off[j * nq]
            parts.append(ids)
        gt_ids = np.concatenate(parts).astype(np.uint32)
        ev = ctx.query_evaluate(gt_off, gt_ids)
        for j, k in enumerate(ks):
            ctx.query_upload(query, k, a.L)
            ctx.query_run(keep_candidates=True)
            off, ids, _ = gt[k]
            e = ctx.query_evaluate(off, ids)
            per_k[k] = {"recall": round(e["recall"], 6), "precision": round(e["precision"], 6),
                        "candidate_recall": round(e["candidate_recall"], 6)}
        # the same queries with the NumPy-fit verifier: the recall the fit costs or gains
        coeff_c, codes_c, mu_c, g_c, b_c = ix.numpy_fit
        ctx.verifier_load(coeff_c, codes_c, mu_c, g_c, b_c)
        for j, k in enumerate(ks):
            ctx.verifier_materialize(k)
            ctx.query_upload(query, k, a.L)
            ctx.query_run()
            off, ids, _ = gt[k]
            e = ctx.query_evaluate(off, ids)
            ix.timings["lrq_fit"].setdefault("recall_numpy_fit", {})[k] = round(e["recall"], 6)
            ix.timings["lrq_fit"].setdefault("recall_gpu_fit", {})[k] = per_k[k]["recall"]
        ctx.verifier_load(ix.coeff, ix.codes, ix.mu, ix.basis, ix.codebook)
        for k in ks:
            ctx.verifier_materialize(k)
    # ---- the reference's beam-width sweep, one launch of nq queries per (k, L):
    # recall / precision and QPS with the device evaluation inside the timing,
    # as the reference's query loop has it
    per_L = []
    if gt is not None:
        for k in ks:
            off, ids, _ = gt[k]
            for L in SWEEP_L:
                ctx.query_upload(query, k, L)
                ctx.gt_load(off, ids)
                ctx.query_run()
                ctx.timer_start()
                ctx.query_run()
                s = ctx.query_evaluate_sums()
                ms_L = ctx.timer_stop()
                ne = max(1, s["nonempty"])
                per_L.append({"k": k, "L": L, "recall": round(s["recall"] / ne, 6),
                              "precision": round(s["precision"] / ne, 6), "qps": round(nq / (ms_L / 1e3), 1),
                              "graph_dist": round(s["graph_dist"] / ne, 1)})
    # per-query results at the bench's beam width, for the comparison with the
    # reference's query code in the CPU-baseline leg
    ours_k = {k: ctx.rknn_query(query, k, a.L, keep_candidates=True) for k in ks} if gt is not None else {}
    # ---- resident batch: warm-up, then K timed steps, each one replay of the
    # batch's captured CUDA graph (entry, leaf order, search, compaction)
    ctx.query_upload(qb, kb, Lb)
    for _ in range(a.warmup):
        ctx.query_run_graph()
    stats = []
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    with Clocks(dev) as clk:
        clk.mark()
        ctx.timer_start()
        for _ in range(a.steps):
            stats.append(ctx.query_run_graph())
        ms = ctx.timer_stop()
    clocks = clk.summary()
    # ---- end to end through the host-buffer C ABI from pinned memory
    pin_q = torch.empty(qb.shape, dtype=torch.float32, pin_memory=True).numpy()
    pin_q[:] = qb
    pin_k = torch.empty(kb.shape, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    pin_k[:] = kb
    pin_L = torch.empty(Lb.shape, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    pin_L[:] = Lb
    r = ctx.rknn_query(pin_q, pin_k, pin_L)
    # results land in pinned buffers reused by every call, as a serving loop does
    def pinned_u32(n):
        return torch.empty(n, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    out = (pinned_u32(nb + 1), pinned_u32(int(r.pred_off[-1]) + 4096), pinned_u32(nb))
    for _ in range(a.warmup):
        r = ctx.rknn_query(pin_q, pin_k, pin_L, out=out)
    e2e_stats = []
    ctx.timer_start()
    for _ in range(a.steps):
        r = ctx.rknn_query(pin_q, pin_k, pin_L, out=out)
        e2e_stats.append(r.stats)
    e2e_ms = ctx.timer_stop()
    from anqi.dist import max_over_ranks
    ms, e2e_ms = max_over_ranks([ms, e2e_ms], device=f"cuda:{dev}" if world > 1 else None)
    value = world * a.steps * nb / (ms / 1e3)
    e2e_value = world * a.steps * nb / (e2e_ms / 1e3)
    # ---- roofline of the search kernel: algorithmic bytes per launch
    s0 = ctx.query_run(counters=True)
    D = a.d + 2
    X = s0["n_expand"] + s0["n_flood"]
    alg_bytes = s0["n_dist"] * 4 * D + X * 4 * (1 + ix.links.shape[1]) + s0["n_cand"] * (4 * a.d + 4)
    kernel_ms = statistics.median([s["search_ms"] for s in stats])
    achieved = alg_bytes / (kernel_ms / 1e3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = None
    tf = REPO / "profiles" / "search_kernel_traffic.json"
    if tf.exists():
        try:
            tj = json.loads(tf.read_text())
            traffic = int(tj["bytes_per_graph_dist"] * s0["n_dist"])
        except (ValueError, KeyError):
            traffic = None
    batched = run_batched(ctx, a, base, ix, rank) if a.batched_queries else None
    # error of every distance form against FP64 on 20,000 random pairs: base
    # rows against queries (the verifier / ground-truth key) and lifted rows
    # against lifted rows (the graph build's LocalJoin key)
    from anqi import precision as prec
    fp64_error = {"base_query": prec.report(ctx, base, query),
                  "lifted": prec.report(ctx, ix.lifted, ix.lifted, seed=5)}
    # the plain FP32 GPU path on the same index and queries, for the batched form's speed-up
    plain = run_plain(a, dev, ix, query, ks, max(3, min(a.steps, 10)), 2) if a.batched_queries else None
    if batched is not None and plain is not None:
        batched["plain_fp32"] = plain
        batched["speedup_vs_plain"] = {"resident_step": round(value / world / plain["qps"], 3)}
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": "queries/s", "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": round(ms / a.steps, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": ("synthetic (seeded 1,000-centre mixture, integers in [0,255])" if a.data == "mixture"
                 else "synthetic (seeded N(0,1), L2-normalised rows)"),
        "config": bench_config(a, ks, world),
        "e2e": {"value": round(e2e_value, 1), "unit": "queries/s",
                "h2d_bytes_per_step": int(e2e_stats[-1]["h2d_bytes"]),
                "d2h_bytes_per_step": int(e2e_stats[-1]["d2h_bytes"])},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic, "peak_source": peak_kind,
                     "kernel": "rknn_search_kernel", "kernel_ms": round(kernel_ms, 4),
                     "alg_bytes_per_launch": int(alg_bytes),
                     "visited_table": int(stats[-1]["visited_table"]),
                     "visited_l2_table": int(stats[-1]["visited_l2_table"])},
        # per step one graph replay: entry, leaf count, leaf scan, leaf scatter,
        # search, CSR scan, CSR gather
        "gpu_launches": 7 * a.steps,
        "clocks": clocks,
        "recall": None if ev["recall"] is None else round(ev["recall"], 6),
        "precision": None if ev["precision"] is None else round(ev["precision"], 6), "per_k": per_k,
        "per_L": per_L,
        "counters_per_query": {"graph_dist": round(s0["n_dist"] / nb, 1), "expansions": round(X / nb, 1),
                               "candidates": round(s0["n_cand"] / nb, 1), "verified": round(s0["n_pred"] / nb, 2)},
        "batched_form": batched,
        "build_s": {k: round(v, 3) for k, v in ix.timings.items() if isinstance(v, float)},
        "localjoin": ix.timings["localjoin"],
        "lrq_fit": ix.timings.get("lrq_fit"),
        "fp64_error": fp64_error,
        "aknn_build": {"bf16_tensor_init_s": round(ix.timings["aknn_build_warm_s"], 3),
                       "fp32_init_s": round(ix.timings["aknn_build_fp32_s"], 3),
                       "bf16_first_build_s": round(ix.timings["aknn_build_s"], 3),
                       "identical": ix.timings["aknn_fp32_identical"], "init_ms": ix.timings["aknn_init_ms"],
                       "library_total_ms": ix.timings["aknn_total_ms"],
                       "gather_kernel_ms": ix.timings["aknn_gather_kernel_ms"]},
    }
    if rank == 0 and world == 1 and not a.no_cpu_baseline and gt is not None:
        tmp = Path(a.keep) if a.keep else Path(tempfile.mkdtemp(prefix="anqi_bench_"))
        try:
            write_index_files(tmp, base, query, ix, ks, gt, ctx)
            threads = os.cpu_count() or 1
            # bounded sample: enough queries for about cpu_seconds of CPU work
            probe, err = reference_qbench(tmp, ks, a.L, threads, 0, 1, 1000)
            if probe is None:
                line["cpu_baseline"] = {"unavailable": err}
            else:
                per_q = probe["seconds"] / probe["queries_per_step"]
                nqs = int(min(nq, max(200, a.cpu_seconds / max(per_q, 1e-9) / len(ks))))
                res, err = reference_qbench(tmp, ks, a.L, threads, 0, 1, nqs)
                if res is None:
                    line["cpu_baseline"] = {"unavailable": err}
                else:
                    line["cpu_baseline"] = {"value": round(res["qps"], 1), "unit": "queries/s", "cores": threads,
                                            "kind": "reference",
                                            "sample": f"first {nqs} queries x k{{{a.ks}}}, L={a.L}, same index; "
                                                      "reference range_search + postfilter + evaluation",
                                            "per_k": res["per_k"]}
            # query-by-query parity on this index: the reference's range_search
            # + postfilter (one thread) with its entry descent's ties sent
            # left, and with its own random tie side
            if probe is not None:
                sys.path.insert(0, str(REPO / "oracle"))
                import harness_io as hio
                par = {"L": a.L}
                for mode in ("left", "tree"):
                    t0 = time.perf_counter()
                    ref = hio.run_qparity(tmp, a.L, mode, nq, ks)
                    par[f"{mode}_entry"] = hio.compare(ref, ours_k, nq)
                    log(f"parity ({mode} entry) {par[f'{mode}_entry']} in {time.perf_counter() - t0:.1f}s")
                line["parity"] = par
        finally:
            if not a.keep:
                shutil.rmtree(tmp, ignore_errors=True)
    if a.graph_options and world == 1 and a.data == "mixture":
        # after the main line's measurements: another index replaces it
        try:
            line["graph_options"] = run_graph_options(ctx, a)
        except Exception as e:  # reported, not fatal: the main line stands
            line["graph_options"] = {"error": f"{type(e).__name__}: {e}"}
    if a.ip_metric and world == 1:
        # after the main line's measurements: another index replaces it
        try:
            line["ip_metric"] = run_ip_metric(ctx, a)
        except Exception as e:  # reported, not fatal: the main line stands
            line["ip_metric"] = {"error": f"{type(e).__name__}: {e}"}
    if a.shape960 and world == 1 and a.d == 128:
        # after the main line's measurements: the second shape replaces the index
        try:
            line["batched_form_960"] = run_shape960(ctx, a, max(3, min(a.steps, 10)), max(3, a.warmup))
        except Exception as e:  # reported, not fatal: the main line stands
            line["batched_form_960"] = {"error": f"{type(e).__name__}: {e}"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()


def run_reference(a, rank, world, local):
    """The reference's own pipeline on this host's CPU cores, no GPU library in
    any of its processes (oracle/reference_pipeline.py): its build_aknn_source,
    the NumPy trainer (byte-identical restatement of its trainer), exact ground
    truth on the CPU, then its rknn_query.  rknn_query runs once per k over an
    L list holding W + K copies of the bench's beam width (one step each) and
    then the sweep; a step's time is the sum over k of nq / QPS, the reference's
    own clock around its query loop (lift, range_search, postfilter,
    evaluation)."""
    if rank != 0:
        return
    sys.path.insert(0, str(REPO / "oracle"))
    import reference_pipeline as rp
    from anqi import formats, pipeline

    def unavailable(why):
        print(json.dumps({"impl": "reference", "unavailable": why}), flush=True)

    why = rp.unavailable_reason()
    if why:
        return unavailable(why)
    if a.data != "mixture":
        return unavailable("the reference arm runs the integer mixture (its CPU ground truth needs small integers)")
    threads = os.cpu_count() or 1
    ks = [int(k) for k in a.ks.split(",")]
    tmp = Path(a.keep) if a.keep else Path(tempfile.mkdtemp(prefix="anqi_ref_"))
    try:
        tmp.mkdir(parents=True, exist_ok=True)
        t0 = time.perf_counter()
        base, query = pipeline.mixture(a.n, a.d, a.nq, seed=20260819 + rank)
        pfx = tmp / "m"
        formats.write_fbin(f"{pfx}_base.bin", base)
        formats.write_fbin(f"{pfx}_query.bin", query)
        Path(f"{pfx}_lifted.meta").write_text(f"0 {a.d} 100 l2 1.0\n")
        del base
        log(f"reference-arm data in {time.perf_counter() - t0:.1f}s; {threads} host threads")
        rlog = lambda m: log("reference-arm", m)  # noqa: E731
        info = rp.build(pfx, threads, log=rlog)
        Ls = [a.L] * (a.warmup + a.steps) + SWEEP_L
        runs = {k: rp.query(pfx, k, Ls, threads, tmp / "cache", info, log=rlog) for k in ks}
        nq = len(query)
        step_s = [sum(nq / runs[k]["points"][s]["qps"] for k in ks) for s in range(a.warmup, a.warmup + a.steps)]
        value = a.steps * nq * len(ks) / sum(step_s)
        first = runs[ks[0]]
        per_k = {k: {x: runs[k]["points"][a.warmup][x] for x in ("recall", "precision", "cand", "pred", "dist",
                                                                  "graph_dist") if x in runs[k]["points"][a.warmup]}
                 for k in ks}
        per_L = [{"k": k, **{x: p[x] for x in ("L", "recall", "precision", "qps", "graph_dist") if x in p}}
                 for k in ks for p in runs[k]["points"][a.warmup + a.steps:]]
        line = {
            "metric": METRIC, "value": round(value, 1), "unit": "queries/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": round(1e3 * sum(step_s) / a.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded 1,000-centre mixture, integers in [0,255])",
            "config": bench_config(a, ks, world),
            "impl": "reference",
            "cpu_baseline": {"value": round(value, 1), "unit": "queries/s", "cores": threads, "kind": "reference",
                             "sample": f"the whole step ({nq} queries x k{{{a.ks}}}, L={a.L}) on the reference's "
                                       "own index; its rknn_query timing (query lift, range_search, postfilter, "
                                       "evaluation), one L-list entry per step"},
            "e2e": {"value": round(value, 1), "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "per_k": per_k,
            "per_L": per_L,
            "build_s": {"aknn_source": round(info["aknn_build_s"], 3),
                        "verifier_train": round(info["verifier_train_s"], 3),
                        "graph_index": first.get("graph_index_s"), "index_total": first.get("index_s"),
                        "ground_truth_cpu": round(info["ground_truth_s"], 3)},
            "ground_truth": json.loads(info["ground_truth_path"]),
        }
        print(json.dumps(line), flush=True)
    except (RuntimeError, OSError, ValueError, subprocess.TimeoutExpired) as e:
        unavailable(f"reference pipeline failed: {str(e)[:300]}")
    finally:
        if not a.keep:
            shutil.rmtree(tmp, ignore_errors=True)


def main():
    a = parse()
    rank, world, local = dist_env()
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=900))
    try:
        if a.impl == "reference":
            run_reference(a, rank, world, local)
        else:
            run_ours(a, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
