"""End-to-end flows over the C ABI: synthetic data, GPU index build, exact
ground truth, and the reference's prefix files.

The order of stages is the reference's pinned pipeline (scripts/run_final.sh:55-97):
build_aknn_source -> train_final_m8_u8.py -> rknn_query (LRQ encode, lift,
graph build, queries).  Every stage except the NumPy trainer runs on the GPU.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import formats, lrq_train
from ._lib import edge_policy_c, METRICS, AknnParams, BuildStats, Context, GraphParams

EMPTY = 0xFFFFFFFF


def mixture(n: int, d: int = 128, nq: int = 10_000, centers: int = 1000, sigma: float = 20.0, seed: int = 20260819):
    """The 1M x 128 workload: integer values in [0, 255] from a Gaussian mixture
    with centres uniform in [0, 128], per-dimension sigma 20, clipped and
    rounded; queries from the same mixture (same centres)."""
    rng = np.random.default_rng(seed)
    c = rng.uniform(0.0, 128.0, size=(centers, d))
    out = np.empty((n + nq, d), np.float32)
    step = 131072
    for s in range(0, n + nq, step):
        e = min(n + nq, s + step)
        lab = rng.integers(0, centers, size=e - s)
        v = c[lab] + rng.normal(0.0, sigma, size=(e - s, d))
        out[s:e] = np.rint(np.clip(v, 0.0, 255.0))
    return out[:n], out[n:]


def mixture_queries(nq: int, d: int = 128, centers: int = 1000, sigma: float = 20.0, seed: int = 20260819,
                    qseed: int = 1):
    """More queries from the mixture of `mixture(..., seed)` (same centres),
    drawn from their own stream so the base rows stay as they are."""
    c = np.random.default_rng(seed).uniform(0.0, 128.0, size=(centers, d))
    rng = np.random.default_rng([seed, qseed])
    lab = rng.integers(0, centers, size=nq)
    return np.rint(np.clip(c[lab] + rng.normal(0.0, sigma, size=(nq, d)), 0.0, 255.0)).astype(np.float32)


def gaussian(n: int, d: int, nq: int, seed: int = 20260819, normalize: bool = False):
    rng = np.random.default_rng(seed)
    b = rng.standard_normal((n, d), dtype=np.float32)
    q = rng.standard_normal((nq, d), dtype=np.float32)
    if normalize:
        b /= np.linalg.norm(b, axis=1, keepdims=True)
        q /= np.linalg.norm(q, axis=1, keepdims=True)
    return b, q


@dataclass
class Index:
    base: np.ndarray
    aknn_ids: np.ndarray
    aknn_keys: np.ndarray
    mu: np.ndarray
    basis: np.ndarray
    codebook: np.ndarray
    coeff: np.ndarray
    codes: np.ndarray
    lifted: np.ndarray
    mstar2: float
    scale: float
    deg: np.ndarray
    links: np.ndarray
    tree: formats.RPTree
    timings: dict = field(default_factory=dict)


def aknn_build(ctx: Context, base: np.ndarray, k=100, leaf=500, trees=64, ef=600, seed=10, nn_iters=0, nn_sample=20,
               precision="bf16", metric="l2"):
    """build_aknn_source: returns ids (n x k) and the record keys: max(0, d) for
    l2, d - 1 = -<a, b> for ip (build_aknn_source.cpp:125-126).
    precision "bf16": init_knn leaf distances on BF16 tensor-core tiles with FP32
    recheck (both metrics); "fp32": CUDA cores.  Both give identical output."""
    base = np.ascontiguousarray(base, np.float32)
    n, d = base.shape
    p = AknnParams(k, leaf, trees, ef, 8, seed, nn_iters, nn_sample, {"fp32": 0, "bf16": 1}[precision],
                   METRICS[metric])
    ids = np.empty((n, k), np.uint32)
    dist = np.empty((n, k), np.float32)
    st = BuildStats()
    ctx._check(ctx.lib.anqi_aknn_build(ctx.h, base, n, d, C.byref(p), ids, dist, C.byref(st)), "aknn_build")
    # the record keys in place (a second n x k array costs a pass over memory)
    if metric == "ip":
        np.subtract(dist, np.float32(1.0), out=dist)
    else:
        np.maximum(dist, np.float32(0.0), out=dist)
    return ids, dist, st.as_dict()


def vamana_params(gp: GraphParams, vp) -> GraphParams:
    """anqi_graph_params' Vamana fields from an anqi.vamana.VamanaParams."""
    gp.vamana_passes = max(0, vp.passes)
    gp.vamana_L = vp.L
    gp.vamana_batch = int(vp.style not in ("global", "old"))
    gp.vamana_entry = vp.entry
    gp.vamana_batch_frac = vp.batch_frac
    gp.vamana_max_batch = vp.max_batch % 2**64
    gp.vamana_batch_base = vp.batch_base
    gp.vamana_early_alpha = vp.early_alpha
    gp.vamana_early_alpha_one = int(vp.early_alpha_one)
    return gp


def graph_build(ctx: Context, lifted: np.ndarray, warm_ids: np.ndarray, degree=48, nn_k=50, explore=100,
                ef_alpha=8, join_iters=6, join_sample=20, leaf=100, seed=10, alpha=1.2, warm_width=100,
                precision="bf16", vamana_passes=0, vamana_L=128, edge=None, vamana=None):
    """build_index with the flat AKNN warm start; returns deg, links, post-order tree, stats.
    precision "bf16": LocalJoin pairs filtered on BF16 tensor-core tiles, kept
    pairs recomputed in FP32 (identical graph); "fp32": CUDA cores only.
    vamana_passes: global Vamana refine passes; edge: an anqi.edge_policy
    EdgePolicy for the prunes (None: the default prune)."""
    lifted = np.ascontiguousarray(lifted, np.float32)
    warm_ids = np.ascontiguousarray(warm_ids, np.uint32)
    n, dim = lifted.shape
    gp = GraphParams(degree, nn_k, explore, ef_alpha, join_iters, join_sample, leaf, 100, seed, alpha, warm_width,
                     {"fp32": 0, "bf16": 1}[precision], vamana_passes, vamana_L)
    edge_c = edge_policy_c(edge)
    if edge_c is not None:
        gp.edge = C.addressof(edge_c)
    if vamana is not None:  # an anqi.vamana.VamanaParams (its passes and width win)
        vamana_params(gp, vamana)
    deg = np.empty(n, np.uint32)
    links = np.empty((n, degree), np.uint32)
    st = BuildStats()
    ctx._check(ctx.lib.anqi_graph_build(ctx.h, lifted, n, dim, warm_ids, warm_ids.shape[1], C.byref(gp), deg, links,
                                        C.byref(st)), "graph_build")
    nn = C.c_uint32()
    npt = C.c_uint64()
    ctx._check(ctx.lib.anqi_graph_tree_size(ctx.h, C.byref(nn), C.byref(npt)), "tree_size")
    m = nn.value
    left = np.empty(m, np.uint32)
    right = np.empty(m, np.uint32)
    lo = np.empty(m, np.uint32)
    lc = np.empty(m, np.uint32)
    off = np.empty(m, np.float32)
    hyp = np.empty((m, dim), np.float32)
    perm = np.empty(npt.value, np.uint32)
    ctx._check(ctx.lib.anqi_graph_tree_copy(ctx.h, left, right, off, hyp, lo, lc, perm), "tree_copy")
    tree = formats.bfs_tree_to_postorder(left, right, off, hyp, lo, lc, perm, leaf, dim)
    return deg, links, tree, st.as_dict()


def graph_warm_start(ctx: Context, lifted: np.ndarray, warm_ids: np.ndarray, width=100, K=50):
    """Warm-start heaps of the G48 build (index.h:1204-1218): ids, vals (n x K)."""
    lifted = np.ascontiguousarray(lifted, np.float32)
    warm_ids = np.ascontiguousarray(warm_ids, np.uint32)
    n, dim = lifted.shape
    ids = np.empty((n, K), np.uint32)
    vals = np.empty((n, K), np.float32)
    ctx._check(ctx.lib.anqi_graph_warm_start(ctx.h, lifted, n, dim, warm_ids, warm_ids.shape[1], width, K, ids, vals),
               "graph_warm_start")
    return ids, vals


def graph_localjoin(ctx: Context, lifted: np.ndarray, ids, vals, precision="bf16", sample=20, rounds=6):
    """LocalJoin rounds on given heaps (index.h:1468-1487, snapshot form):
    returns ids, vals, per-round updates, device milliseconds of the rounds."""
    lifted = np.ascontiguousarray(lifted, np.float32)
    ids = np.ascontiguousarray(ids, np.uint32).copy()
    vals = np.ascontiguousarray(vals, np.float32).copy()
    n, dim = lifted.shape
    up = np.zeros(rounds, np.uint64)
    done = C.c_uint32()
    ms = C.c_float()
    ctx._check(ctx.lib.anqi_graph_localjoin_precision(ctx.h, lifted, n, dim, ids.shape[1], sample, rounds,
                                                      {"fp32": 0, "bf16": 1}[precision], ids, vals, up,
                                                      C.byref(done), C.byref(ms)), "graph_localjoin")
    return ids, vals, [int(u) for u in up[:done.value]], ms.value


def build_index(ctx: Context, base: np.ndarray, aknn=None, graph=None, train_workers: int = 8, log=print,
                train: str = "gpu") -> Index:
    """The whole index: AKNN source, LRQ fit (train "gpu": anqi.lrq_fit's
    kernels; "numpy": the reference trainer's NumPy fit, byte-identical
    files), LRQ encode, lift and the G48 graph."""
    aknn = aknn or {}
    graph = graph or {}
    t = {}
    t0 = time.perf_counter()
    ids, keys, st = aknn_build(ctx, base, **aknn)
    t["aknn_build_s"] = time.perf_counter() - t0
    t["aknn_stats"] = st
    log(f"[anqi] AKNN source built in {t['aknn_build_s']:.2f}s {st}")
    t0 = time.perf_counter()
    if train == "gpu":
        from . import lrq_fit
        mu, basis, cb = lrq_fit.train_gpu(keys, len(keys), device=ctx.device, log=lambda s: None)
    else:
        mu, basis, cb = lrq_train.train(keys, len(keys), workers=train_workers, log=lambda s: None)
    mu, basis, cb = (np.asarray(a, np.float32) for a in (mu, basis, cb))
    t["lrq_train_s"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    coeff, codes = ctx.lrq_encode(keys, mu, basis, cb)
    t["lrq_encode_s"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    lifted, m2, sc = ctx.lift(base, keys[:, -1])
    t["lift_s"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    deg, links, tree, gst = graph_build(ctx, lifted, ids, **graph)
    t["graph_build_s"] = time.perf_counter() - t0
    t["graph_stats"] = gst
    log(f"[anqi] LRQ train {t['lrq_train_s']:.2f}s encode {t['lrq_encode_s']:.2f}s lift {t['lift_s']:.2f}s "
        f"graph {t['graph_build_s']:.2f}s {gst}")
    return Index(base, ids, keys, mu, basis, cb, coeff, codes, lifted, m2, sc, deg, links, tree, t)


def load_index(ctx: Context, ix: Index, ks=(10, 50, 100)) -> None:
    ctx.index_load(ix.base, ix.lifted, ix.deg, ix.links, ix.tree, ix.scale, ix.mstar2)
    ctx.verifier_load(ix.coeff, ix.codes, ix.mu, ix.basis, ix.codebook)
    for k in ks:
        ctx.verifier_materialize(k)


def exact_thresholds(ctx: Context, base: np.ndarray, K: int = 100, method: str = "fp32", hints=None,
                     metric: str = "l2"):
    """Exact top-K (dataset_gt --mode thresholds).  method "tc": BF16 tensor-core
    tiles with FP32 recheck (bit-identical output); hints = AKNN lists bound each
    row's K-th key (an AKNN build runs when they are absent).  metric "ip": keys
    -<a, b>."""
    base = np.ascontiguousarray(base, np.float32)
    n, d = base.shape
    if method == "tc" and d <= 1024:
        return ctx.exact_topk_tc(base, K, hints, metric)
    ids = np.empty((n, K), np.uint32)
    keys = np.empty((n, K), np.float32)
    ctx._check(ctx.lib.anqi_exact_topk_metric(ctx.h, base, n, d, K, METRICS[metric], ids, keys), "exact_topk")
    return ids, keys


def rknn_ground_truth(ctx: Context, base: np.ndarray, query: np.ndarray, rk2: np.ndarray, method: str = "fp32",
                      metric: str = "l2"):
    """Exact RkNN CSR (dataset_gt --mode ground-truth); method "tc" as above."""
    if method == "tc" and base.shape[1] <= 1024:
        return ctx.rknn_ground_truth_tc(base, query, rk2, metric)
    base = np.ascontiguousarray(base, np.float32)
    query = np.ascontiguousarray(query, np.float32)
    n, d = base.shape
    nq = query.shape[0]
    off = np.empty(nq + 1, np.uint32)
    tot = C.c_uint64()
    cap = max(1024, 256 * nq)
    while True:
        ids = np.empty(cap, np.uint32)
        keys = np.empty(cap, np.float32)
        rc = ctx.lib.anqi_rknn_ground_truth_metric(ctx.h, base, n, query, nq, d, np.ascontiguousarray(rk2, np.float32),
                                                   METRICS[metric], off, ids, keys, cap, C.byref(tot))
        if rc == 9 and tot.value > cap:
            cap = int(tot.value)
            continue
        ctx._check(rc, "rknn_ground_truth")
        return off.copy(), ids[:tot.value].copy(), keys[:tot.value].copy()


def write_prefix(pfx: str, base, query, ix: Index | None = None, gt: dict | None = None, lifted_meta_k: int = 100):
    """The reference's prefix files (scripts/run_final.sh:19-28)."""
    formats.write_fbin(f"{pfx}_base.bin", base)
    formats.write_fbin(f"{pfx}_query.bin", query)
    Path(f"{pfx}_lifted.meta").write_text(f"0 {base.shape[1]} {lifted_meta_k} l2 1.0\n")
    if ix is not None:
        formats.write_rec(f"{pfx}_baseknn_aknn.rec", ix.aknn_ids, ix.aknn_keys)
        formats.write_basis(f"{pfx}_radbasis_M8.bin", ix.mu, ix.basis)
        formats.write_codebook(f"{pfx}_learned_rq_codebook_M8_u8.bin", ix.codebook)
    for k, (off, ids, keys) in (gt or {}).items():
        formats.write_rknn_csr(f"{pfx}_rknn_gt_k{k}.bin", off, ids, keys)
