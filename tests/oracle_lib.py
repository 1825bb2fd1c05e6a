"""ctypes bindings of oracle/liboracle.so -- the test-only C restatement.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use this.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent.parent
LIB_PATH = REPO / "oracle" / "liboracle.so"

u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
EMPTY = 0xFFFFFFFF


def _load() -> C.CDLL:
    if not LIB_PATH.exists():
        subprocess.run(["make", "-s", "-C", str(REPO / "oracle"), "oracle"], check=True)
    lib = C.CDLL(str(LIB_PATH))
    sig = {
        "ao_l2sqr": (C.c_float, [f32p, f32p, C.c_uint32]),
        "ao_ip": (C.c_float, [f32p, f32p, C.c_uint32]),
        "ao_norm": (C.c_float, [f32p, C.c_uint32]),
        "ao_d2": (C.c_float, [f32p, f32p, C.c_float, C.c_float, C.c_uint32]),
        "ao_norms": (None, [f32p, C.c_uint64, C.c_uint32, f32p]),
        "ao_lrq_encode": (None, [f32p, C.c_uint64, C.c_uint32, C.c_uint32, f32p, f32p, f32p, C.c_uint32, f32p, u8p]),
        "ao_lrq_materialize": (None, [f32p, u8p, C.c_uint64, C.c_uint32, C.c_uint32, f32p, f32p, f32p,
                                      C.c_uint32, C.c_uint32, C.c_double, f32p]),
        "ao_lrq_encode_bits": (None, [f32p, C.c_uint64, C.c_uint32, C.c_uint32, f32p, f32p, C.c_void_p, C.c_uint32,
                                      C.c_uint32, C.c_uint32, f32p, C.c_void_p, C.c_void_p]),
        "ao_lrq_materialize_bits": (None, [f32p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint32,
                                           C.c_uint32, f32p, f32p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_double,
                                           C.c_int, f32p]),
        "ao_analytic_rankm_materialize": (None, [f32p, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_double,
                                                 C.c_uint32, C.c_double, f32p]),
        "ao_lift": (None, [f32p, C.c_uint64, C.c_uint32, f32p, f32p, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
        "ao_lift_query": (None, [f32p, C.c_uint32, C.c_double, f32p]),
        "ao_lift_metric": (None, [f32p, C.c_uint64, C.c_uint32, f32p, C.c_uint32, f32p, C.POINTER(C.c_double),
                                  C.POINTER(C.c_double)]),
        "ao_ip_dist": (C.c_float, [f32p, f32p, C.c_uint32]),
        "ao_init_knn_metric": (None, [f32p, f32p, C.c_uint32, C.c_uint64, C.c_uint32, u64p, u32p, C.c_uint64,
                                      C.c_uint32, u32p, f32p]),
        "ao_exact_topk_metric": (None, [f32p, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, u32p, f32p]),
        "ao_rknn_gt_metric": (C.c_int64, [f32p, C.c_uint64, f32p, C.c_uint64, C.c_uint32, f32p, C.c_uint32, u32p,
                                          u32p, f32p, C.c_uint64]),
        "ao_heap_push": (C.c_int, [u32p, f32p, C.c_uint32, C.c_uint32, C.c_float]),
        "ao_warm_start": (None, [f32p, f32p, C.c_uint32, C.c_uint64, u32p, C.c_uint32, C.c_uint32, C.c_uint32,
                                 u32p, f32p]),
        "ao_localjoin_round": (C.c_uint64, [f32p, f32p, C.c_uint32, C.c_uint64, C.c_uint32, C.c_uint32, u32p, f32p]),
        "ao_reverse": (None, [u32p, C.c_uint64, C.c_uint32, u64p, u32p]),
        "ao_init_knn": (None, [f32p, f32p, C.c_uint32, C.c_uint64, C.c_uint32, u64p, u32p, C.c_uint64, u32p, f32p]),
        "ao_graph_commit": (None, [f32p, f32p, C.c_uint32, C.c_uint64, u32p, u32p, C.c_uint32, C.c_float, u32p, u32p]),
        "ao_vamana_select": (None, [f32p, f32p, C.c_uint32, C.c_uint64, u32p, u32p, C.c_uint32, u32p, C.c_uint32,
                                    u32p, C.c_uint32, C.c_float, u32p, u32p]),
        "ao_exact_topk": (None, [f32p, C.c_uint64, C.c_uint32, C.c_uint32, u32p, f32p]),
        "ao_rknn_gt": (C.c_int64, [f32p, C.c_uint64, f32p, C.c_uint64, C.c_uint32, f32p, u32p, u32p, f32p, C.c_uint64]),
        "ao_hash64": (C.c_uint64, [C.c_uint64]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


LIB = _load()


class AoIndex(C.Structure):
    _fields_ = [
        ("n", C.c_uint64), ("dim", C.c_uint32), ("d", C.c_uint32), ("degree", C.c_uint32),
        ("lifted", C.c_void_p), ("deg", C.c_void_p), ("links", C.c_void_p), ("base", C.c_void_p),
        ("tree_nodes", C.c_uint32), ("tree_left", C.c_void_p), ("tree_right", C.c_void_p),
        ("tree_offset", C.c_void_p), ("tree_hyperplane", C.c_void_p), ("tree_leaf_first", C.c_void_p),
        ("scale", C.c_double), ("mstar2", C.c_double), ("metric", C.c_uint32),
    ]


class AoKnnGraph(C.Structure):
    _fields_ = [
        ("n", C.c_uint64), ("dim", C.c_uint32), ("x", C.c_void_p), ("norms", C.c_void_p), ("K", C.c_uint32),
        ("g_ids", C.c_void_p), ("g_vals", C.c_void_p), ("rev_off", C.c_void_p), ("rev_ids", C.c_void_p),
        ("metric", C.c_uint32),
    ]


class AoTreeOut(C.Structure):
    _fields_ = [
        ("left", C.c_void_p), ("right", C.c_void_p), ("offset", C.c_void_p), ("hyperplane", C.c_void_p),
        ("leaf_off", C.c_void_p), ("leaf_cnt", C.c_void_p), ("perm", C.c_void_p), ("cap_nodes", C.c_uint32),
    ]


LIB.ao_range_search.restype = C.c_int
LIB.ao_range_search.argtypes = [C.POINTER(AoIndex), f32p, C.c_uint32, f32p, u32p, C.c_uint32, C.POINTER(C.c_uint32),
                                u32p, C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
LIB.ao_gather.restype = C.c_int64
LIB.ao_gather.argtypes = [C.POINTER(AoKnnGraph), C.c_uint64, C.c_uint32, C.c_uint32, f32p, u32p, C.c_uint64]
LIB.ao_aknn_rows.restype = None
LIB.ao_aknn_rows.argtypes = [C.POINTER(AoKnnGraph), C.c_uint32, C.c_uint32, C.c_uint32, u32p, f32p]
LIB.ao_graph_select_policy.restype = None
LIB.ao_graph_select_policy.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_float, C.c_void_p, u32p,
                                       u32p]
LIB.ao_graph_commit_policy.restype = None
LIB.ao_graph_commit_policy.argtypes = [f32p, f32p, C.c_uint32, C.c_uint64, u32p, u32p, C.c_uint32, C.c_float,
                                       C.c_void_p, u32p, u32p]
LIB.ao_vamana_select_policy.restype = None
LIB.ao_vamana_select_policy.argtypes = [f32p, f32p, C.c_uint32, C.c_uint64, u32p, u32p, C.c_uint32, u32p, C.c_uint32,
                                        u32p, C.c_uint32, C.c_float, C.c_void_p, u32p, u32p]
LIB.ao_vamana_batch_refine.restype = None
LIB.ao_vamana_batch_refine.argtypes = [f32p, f32p, C.c_uint32, C.c_uint64, u32p, u32p, C.c_uint32, u32p, C.c_uint32,
                                       C.c_uint32, C.c_uint32, C.c_int, C.c_float, C.c_float, C.c_int, C.c_double,
                                       C.c_uint64, C.c_double, C.c_uint64, C.c_void_p]
LIB.ao_vamana_batch_order.restype = None
LIB.ao_vamana_batch_order.argtypes = [u32p, C.c_uint64, C.c_uint64, C.c_int]
LIB.ao_graph_select.restype = None
LIB.ao_graph_select.argtypes = [C.POINTER(AoKnnGraph), C.c_uint32, C.c_uint32, C.c_uint32, C.c_float, u32p, u32p]
LIB.ao_rp_tree.restype = C.c_int64
LIB.ao_rp_tree.argtypes = [f32p, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint32,
                           C.POINTER(AoTreeOut)]
LIB.ao_rp_tree_metric.restype = C.c_int64
LIB.ao_rp_tree_metric.argtypes = [f32p, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint32,
                                  C.c_uint32, C.POINTER(AoTreeOut)]


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


# ---------------------------------------------------------------- helpers


def norms(x: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(x, np.float32)
    out = np.empty(x.shape[0], np.float32)
    LIB.ao_norms(x, x.shape[0], x.shape[1], out)
    return out


def lrq_encode(keys, mu, basis, codebook):
    keys = np.ascontiguousarray(keys, np.float32)
    n, nk = keys.shape
    rankm = basis.shape[0]
    coeff = np.empty((n, rankm), np.float32)
    codes = np.empty((n, nk), np.uint8)
    LIB.ao_lrq_encode(keys, n, nk, rankm, np.ascontiguousarray(mu, np.float32),
                      np.ascontiguousarray(basis, np.float32), np.ascontiguousarray(codebook, np.float32),
                      codebook.shape[1], coeff, codes)
    return coeff, codes


def lrq_materialize(coeff, codes, mu, basis, codebook, k, scale=1.0):
    n, nk = codes.shape
    thr = np.empty(n, np.float32)
    LIB.ao_lrq_materialize(np.ascontiguousarray(coeff, np.float32), np.ascontiguousarray(codes, np.uint8), n, nk,
                           basis.shape[0], np.ascontiguousarray(mu, np.float32),
                           np.ascontiguousarray(basis, np.float32), np.ascontiguousarray(codebook, np.float32),
                           codebook.shape[1], k, scale, thr)
    return thr


def _vp(a):
    return None if a is None else a.ctypes.data


def lrq_encode_bits(keys, mu, basis, codebook, bits, policy):
    """Every codec form: returns coeff, packed codes (bytes, object-major) or
    None, float residuals or None."""
    keys = np.ascontiguousarray(keys, np.float32)
    n, nk = keys.shape
    rankm = basis.shape[0]
    coeff = np.empty((n, rankm), np.float32)
    codes = np.zeros((n * nk * bits + 7) // 8, np.uint8) if bits in (2, 4, 8, 16) else None
    resid = np.empty((n, nk), np.float32) if bits == 32 else None
    cb = None if codebook is None else np.ascontiguousarray(codebook, np.float32)
    LIB.ao_lrq_encode_bits(keys, n, nk, rankm, np.ascontiguousarray(mu, np.float32),
                           np.ascontiguousarray(basis, np.float32), _vp(cb), 0 if cb is None else cb.shape[1], bits,
                           policy, coeff, _vp(codes), _vp(resid))
    return coeff, codes, resid


def lrq_materialize_bits(coeff, codes, resid, n, nk, mu, basis, codebook, bits, k, scale=1.0, signed_keys=False):
    thr = np.empty(n, np.float32)
    cb = None if codebook is None else np.ascontiguousarray(codebook, np.float32)
    LIB.ao_lrq_materialize_bits(np.ascontiguousarray(coeff, np.float32), _vp(codes), _vp(resid), n, nk,
                                basis.shape[0], bits, np.ascontiguousarray(mu, np.float32),
                                np.ascontiguousarray(basis, np.float32), _vp(cb), 0 if cb is None else cb.shape[1], k,
                                scale, int(signed_keys), thr)
    return thr


def analytic_rankm_materialize(coeff, train_kmax, flags, b0, k, scale=1.0):
    coeff = np.ascontiguousarray(coeff, np.float32)
    thr = np.empty(coeff.shape[0], np.float32)
    LIB.ao_analytic_rankm_materialize(coeff, coeff.shape[0], coeff.shape[1], train_kmax, flags, b0, k, scale, thr)
    return thr


def lift(base, radius, metric=0):
    base = np.ascontiguousarray(base, np.float32)
    n, d = base.shape
    out = np.empty((n, d + 2), np.float32)
    m2 = C.c_double()
    sc = C.c_double()
    LIB.ao_lift_metric(base, n, d, np.ascontiguousarray(radius, np.float32), metric, out, C.byref(m2), C.byref(sc))
    return out, m2.value, sc.value


def warm_start(x, nrm, cand, width, K):
    n, dim = x.shape
    ids = np.empty((n, K), np.uint32)
    vals = np.empty((n, K), np.float32)
    cand = np.ascontiguousarray(cand, np.uint32)
    LIB.ao_warm_start(x, nrm, dim, n, cand, cand.shape[1], width, K, ids, vals)
    return ids, vals


def localjoin(x, nrm, ids, vals, sample=20, rounds=6):
    """nndescent_refine (index.h:1468-1487) with the early exit upd < n/200."""
    n, dim = x.shape
    K = ids.shape[1]
    ids = ids.copy()
    vals = vals.copy()
    ups = []
    for _ in range(rounds):
        upd = LIB.ao_localjoin_round(x, nrm, dim, n, K, sample, ids, vals)
        ups.append(int(upd))
        if upd < n // 200:
            break
    return ids, vals, ups


def reverse(ids):
    n, K = ids.shape
    off = np.zeros(n + 1, np.uint64)
    tot = int(np.sum((ids != EMPTY) & (ids < n)))
    rev = np.zeros(max(tot, 1), np.uint32)
    LIB.ao_reverse(np.ascontiguousarray(ids, np.uint32), n, K, off, rev)
    return off, rev[:tot]


def knn_graph(x, nrm, ids, vals, rev_off, rev, metric=0):
    keep = (x, nrm, ids, vals, rev_off, rev)
    g = AoKnnGraph(x.shape[0], x.shape[1], _p(x), _p(nrm), ids.shape[1], _p(ids), _p(vals), _p(rev_off),
                   _p(rev) if rev.size else _p(np.zeros(1, np.uint32)), metric)
    g._keep = keep
    return g


def graph_select(x, nrm, ids, vals, M=48, ef=100, cap=800, alpha=1.2):
    x = np.ascontiguousarray(x, np.float32)
    ids = np.ascontiguousarray(ids, np.uint32)
    vals = np.ascontiguousarray(vals, np.float32)
    off, rev = reverse(ids)
    rev = rev if rev.size else np.zeros(1, np.uint32)
    g = knn_graph(x, nrm, ids, vals, off, rev)
    n = x.shape[0]
    O = np.empty((n, M), np.uint32)
    Od = np.empty(n, np.uint32)
    LIB.ao_graph_select(C.byref(g), ef, cap, M, alpha, O, Od)
    return O, Od


def vamana_select(x, nrm, links, deg, g0, entry, Lb=128, alpha=1.2):
    x = np.ascontiguousarray(x, np.float32)
    n, M = links.shape
    O = np.empty((n, M), np.uint32)
    Od = np.empty(n, np.uint32)
    LIB.ao_vamana_select(x, nrm, x.shape[1], n, np.ascontiguousarray(links, np.uint32),
                         np.ascontiguousarray(deg, np.uint32), M, np.ascontiguousarray(g0, np.uint32), g0.shape[1],
                         np.ascontiguousarray(entry, np.uint32), Lb, alpha, O, Od)
    return O, Od


class AoEdgePolicy(C.Structure):
    _fields_ = [
        ("flags", C.c_uint32), ("nks", C.c_uint32), ("ks", C.c_uint32 * 8), ("nk", C.c_uint32),
        ("budget", C.c_uint32), ("occlude_all", C.c_uint32), ("auto_candidates", C.c_uint32),
        ("auto_max_swaps", C.c_uint32), ("lam", C.c_double), ("scale2", C.c_double), ("lsg_alpha", C.c_double),
        ("resid", C.c_void_p), ("mu", C.c_void_p),
    ]


def edge_policy(pol):
    """ao_edge_policy of an anqi.edge_policy.EdgePolicy (None: the default prune)."""
    if pol is None or not pol.active:
        return None
    resid = np.ascontiguousarray(pol.resid, np.float32) if pol.resid is not None else np.zeros(1, np.float32)
    mu = np.ascontiguousarray(pol.mu, np.float32) if pol.mu is not None else np.zeros(1, np.float32)
    ks = (C.c_uint32 * 8)(*(list(pol.ks) + [0] * (8 - len(pol.ks))))
    s = AoEdgePolicy(pol.flags, len(pol.ks), ks, pol.nk, pol.budget, int(pol.occlude_all), pol.auto_candidates,
                     pol.auto_max_swaps, pol.lam, pol.scale2, pol.lsg_alpha, _p(resid), _p(mu))
    s._keep = (resid, mu)
    return s


def graph_select_policy(x, nrm, ids, vals, pol, M=48, ef=100, cap=800, alpha=1.2):
    x = np.ascontiguousarray(x, np.float32)
    ids = np.ascontiguousarray(ids, np.uint32)
    vals = np.ascontiguousarray(vals, np.float32)
    off, rev = reverse(ids)
    rev = rev if rev.size else np.zeros(1, np.uint32)
    g = knn_graph(x, nrm, ids, vals, off, rev)
    n = x.shape[0]
    O = np.empty((n, M), np.uint32)
    Od = np.empty(n, np.uint32)
    ep = edge_policy(pol)
    LIB.ao_graph_select_policy(C.byref(g), ef, cap, M, alpha, C.byref(ep) if ep is not None else None, O, Od)
    return O, Od


def graph_commit_policy(x, nrm, O, Od, pol, alpha=1.2):
    n, M = O.shape
    links = np.empty((n, M), np.uint32)
    deg = np.empty(n, np.uint32)
    ep = edge_policy(pol)
    LIB.ao_graph_commit_policy(x, nrm, x.shape[1], n, np.ascontiguousarray(O, np.uint32),
                               np.ascontiguousarray(Od, np.uint32), M, alpha,
                               C.byref(ep) if ep is not None else None, links, deg)
    return links, deg


def vamana_select_policy(x, nrm, links, deg, g0, entry, pol, Lb=128, alpha=1.2):
    x = np.ascontiguousarray(x, np.float32)
    n, M = links.shape
    O = np.empty((n, M), np.uint32)
    Od = np.empty(n, np.uint32)
    ep = edge_policy(pol)
    LIB.ao_vamana_select_policy(x, nrm, x.shape[1], n, np.ascontiguousarray(links, np.uint32),
                                np.ascontiguousarray(deg, np.uint32), M, np.ascontiguousarray(g0, np.uint32),
                                g0.shape[1], np.ascontiguousarray(entry, np.uint32), Lb, alpha,
                                C.byref(ep) if ep is not None else None, O, Od)
    return O, Od


def vamana_batch_refine(x, nrm, links, deg, g0, vp, pol=None, alpha=1.2, seed=10):
    """vamana_batch_refine on copies of links / deg; vp: anqi.vamana.VamanaParams."""
    x = np.ascontiguousarray(x, np.float32)
    links = np.ascontiguousarray(links, np.uint32).copy()
    deg = np.ascontiguousarray(deg, np.uint32).copy()
    n, M = links.shape
    ep = edge_policy(pol)
    LIB.ao_vamana_batch_refine(x, nrm, x.shape[1], n, links, deg, M, np.ascontiguousarray(g0, np.uint32), g0.shape[1],
                               vp.entry, vp.L, vp.passes, alpha, vp.early_alpha, int(vp.early_alpha_one),
                               vp.batch_frac, vp.max_batch, vp.batch_base, seed,
                               C.byref(ep) if ep is not None else None)
    return links, deg


def vamana_batch_order(n, seed, passes):
    o = np.arange(n, dtype=np.uint32)
    for p in range(passes):
        LIB.ao_vamana_batch_order(o, n, seed, p)
    return o


def graph_commit(x, nrm, O, Od, alpha=1.2):
    n, M = O.shape
    links = np.empty((n, M), np.uint32)
    deg = np.empty(n, np.uint32)
    LIB.ao_graph_commit(x, nrm, x.shape[1], n, np.ascontiguousarray(O, np.uint32), np.ascontiguousarray(Od, np.uint32),
                        M, alpha, links, deg)
    return links, deg


def aknn_rows(x, nrm, ids, vals, K=100, ef=600, ef_alpha=8, metric=0):
    x = np.ascontiguousarray(x, np.float32)
    ids = np.ascontiguousarray(ids, np.uint32)
    vals = np.ascontiguousarray(vals, np.float32)
    off, rev = reverse(ids)
    rev = rev if rev.size else np.zeros(1, np.uint32)
    g = knn_graph(x, nrm, ids, vals, off, rev, metric)
    n = x.shape[0]
    out_i = np.empty((n, K), np.uint32)
    out_d = np.empty((n, K), np.float32)
    LIB.ao_aknn_rows(C.byref(g), ef, max(K, ef_alpha * ef), K, out_i, out_d)
    return out_i, out_d


def init_knn(x, nrm, leaf_off, leaves, K, metric=0):
    n, dim = x.shape
    out_i = np.empty((n, K), np.uint32)
    out_d = np.empty((n, K), np.float32)
    LIB.ao_init_knn_metric(x, nrm, dim, n, K, np.ascontiguousarray(leaf_off, np.uint64),
                           np.ascontiguousarray(leaves, np.uint32), len(leaf_off) - 1, metric, out_i, out_d)
    return out_i, out_d


def rp_tree(x, leaf_size, max_depth=100, seed=10, tree=0, angular=0):
    """Deterministic RP tree; returns dict of BFS-ordered node arrays + perm."""
    x = np.ascontiguousarray(x, np.float32)
    n, dim = x.shape
    cap = 4 * n + 8
    arr = {
        "left": np.empty(cap, np.uint32), "right": np.empty(cap, np.uint32), "offset": np.empty(cap, np.float32),
        "hyperplane": np.zeros((cap, dim), np.float32), "leaf_off": np.empty(cap, np.uint32),
        "leaf_cnt": np.empty(cap, np.uint32), "perm": np.empty(n, np.uint32),
    }
    t = AoTreeOut(_p(arr["left"]), _p(arr["right"]), _p(arr["offset"]), _p(arr["hyperplane"]), _p(arr["leaf_off"]),
                  _p(arr["leaf_cnt"]), _p(arr["perm"]), cap)
    nn = LIB.ao_rp_tree_metric(x, n, dim, leaf_size, max_depth, seed, tree, angular, C.byref(t))
    assert nn > 0
    for k in ("left", "right", "offset", "hyperplane", "leaf_off", "leaf_cnt"):
        arr[k] = arr[k][:nn].copy()
    arr["n_nodes"] = int(nn)
    return arr


def exact_topk(base, K, metric=0):
    base = np.ascontiguousarray(base, np.float32)
    n, d = base.shape
    ids = np.empty((n, K), np.uint32)
    keys = np.empty((n, K), np.float32)
    LIB.ao_exact_topk_metric(base, n, d, K, metric, ids, keys)
    return ids, keys


def rknn_gt(base, query, rk2, metric=0):
    base = np.ascontiguousarray(base, np.float32)
    query = np.ascontiguousarray(query, np.float32)
    n, d = base.shape
    nq = query.shape[0]
    cap = max(1, n * nq)
    off = np.empty(nq + 1, np.uint32)
    ids = np.empty(cap, np.uint32)
    keys = np.empty(cap, np.float32)
    tot = LIB.ao_rknn_gt_metric(base, n, query, nq, d, np.ascontiguousarray(rk2, np.float32), metric, off, ids, keys,
                                cap)
    assert tot >= 0
    return off, ids[:tot], keys[:tot]


class TreeArrays:
    """Post-order tree arrays as the reference persists them (root last)."""

    def __init__(self, left, right, offset, hyperplane, leaf_first):
        self.left = np.ascontiguousarray(left, np.uint32)
        self.right = np.ascontiguousarray(right, np.uint32)
        self.offset = np.ascontiguousarray(offset, np.float32)
        self.hyperplane = np.ascontiguousarray(hyperplane, np.float32)
        self.leaf_first = np.ascontiguousarray(leaf_first, np.uint32)


def range_search_all(lifted, links, deg, base, tree: TreeArrays, scale, mstar2, queries, thr, L, metric=0):
    """Runs ao_range_search for each query; returns lists of candidate arrays,
    predicted arrays and distance counts."""
    lifted = np.ascontiguousarray(lifted, np.float32)
    links = np.ascontiguousarray(links, np.uint32)
    deg = np.ascontiguousarray(deg, np.uint32)
    base = np.ascontiguousarray(base, np.float32)
    n, dim = lifted.shape
    ix = AoIndex(n, dim, base.shape[1], links.shape[1], _p(lifted), _p(deg), _p(links), _p(base),
                 len(tree.left), _p(tree.left), _p(tree.right), _p(tree.offset), _p(tree.hyperplane),
                 _p(tree.leaf_first), scale, mstar2, metric)
    cap = n
    cand = np.empty(cap, np.uint32)
    pred = np.empty(cap, np.uint32)
    nc, npd, nd = C.c_uint32(), C.c_uint32(), C.c_uint32()
    cands, preds, nds = [], [], []
    thr = np.ascontiguousarray(thr, np.float32)
    for q in np.ascontiguousarray(queries, np.float32):
        rc = LIB.ao_range_search(C.byref(ix), q, L, thr, cand, cap, C.byref(nc), pred, cap, C.byref(npd), C.byref(nd))
        assert rc == 0
        cands.append(cand[: nc.value].copy())
        preds.append(pred[: npd.value].copy())
        nds.append(nd.value)
    return cands, preds, np.array(nds, np.uint32)
