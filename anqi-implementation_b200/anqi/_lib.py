"""ctypes bindings of libanqi.so (include/anqi.h).

The shared library is the product: every call here goes to CUDA kernels built
for sm_100a.  There is no CPU fallback -- if the library or a GPU is missing,
``Context()`` raises.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import formats

PKG = Path(__file__).resolve().parent.parent
LIB_PATH = Path(os.environ.get("ANQI_LIBRARY", PKG / "lib" / "libanqi.so"))
EMPTY = 0xFFFFFFFF

ANQI_OK = 0
ANQI_ERR_ARGS = 2
ANQI_ERR_FORMAT = 3
ANQI_ERR_INVARIANT = 5
ANQI_ERR_DEVICE = 7
ANQI_ERR_TIMEOUT = 8
ANQI_ERR_CAPACITY = 9


class AnqiError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[anqi status {status}] {msg}")
        self.status = status


_f32 = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64 = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u32 = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u64 = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_u8 = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_vp = C.c_void_p


class IndexDesc(C.Structure):
    _fields_ = [
        ("n", C.c_uint64), ("d", C.c_uint32), ("degree", C.c_uint32), ("base", _vp), ("lifted", _vp),
        ("deg", _vp), ("links", _vp), ("tree_nodes", C.c_uint32), ("tree_left", _vp), ("tree_right", _vp),
        ("tree_offset", _vp), ("tree_hyperplane", _vp), ("tree_leaf_first", _vp), ("scale", C.c_double),
        ("mstar2", C.c_double), ("metric", C.c_uint32),
    ]


class EvalSums(C.Structure):
    _fields_ = [("recall", C.c_double), ("precision", C.c_double), ("f1", C.c_double), ("cand_recall", C.c_double),
                ("cand", C.c_double), ("pred", C.c_double), ("graph_dist", C.c_double), ("nonempty", C.c_uint32)]


class QueryStats(C.Structure):
    _fields_ = [
        ("n_dist", C.c_uint64), ("n_expand", C.c_uint64), ("n_cand", C.c_uint64), ("n_pred", C.c_uint64),
        ("n_flood", C.c_uint64), ("search_ms", C.c_float), ("total_ms", C.c_float), ("h2d_bytes", C.c_uint64),
        ("d2h_bytes", C.c_uint64), ("visited_table", C.c_uint32),
        ("visited_l2_table", C.c_uint32), ("warps_per_block", C.c_uint32), ("candidate_tile", C.c_uint32),
    ]


class AknnParams(C.Structure):
    _fields_ = [("k", C.c_uint32), ("leaf", C.c_uint32), ("trees", C.c_uint32), ("ef", C.c_uint32),
                ("ef_alpha", C.c_uint32), ("seed", C.c_uint64), ("nn_iters", C.c_uint32), ("nn_sample", C.c_uint32),
                ("precision", C.c_uint32), ("metric", C.c_uint32)]


class GraphParams(C.Structure):
    _fields_ = [("degree", C.c_uint32), ("nn_k", C.c_uint32), ("explore", C.c_uint32), ("ef_alpha", C.c_uint32),
                ("join_iters", C.c_uint32), ("join_sample", C.c_uint32), ("leaf", C.c_uint32),
                ("max_depth", C.c_uint32), ("seed", C.c_uint64), ("alpha", C.c_float), ("warm_width", C.c_uint32),
                ("precision", C.c_uint32), ("vamana_passes", C.c_uint32), ("vamana_L", C.c_uint32),
                ("edge", C.c_void_p), ("vamana_batch", C.c_uint32), ("vamana_entry", C.c_uint32),
                ("vamana_batch_frac", C.c_double), ("vamana_max_batch", C.c_uint64),
                ("vamana_batch_base", C.c_double), ("vamana_early_alpha", C.c_float),
                ("vamana_early_alpha_one", C.c_uint32)]


class EdgePolicyC(C.Structure):
    """anqi_edge_policy (include/anqi.h)."""
    _fields_ = [("flags", C.c_uint32), ("nks", C.c_uint32), ("ks", C.c_uint32 * 8), ("nk", C.c_uint32),
                ("budget", C.c_uint32), ("occlude_all", C.c_uint32), ("auto_candidates", C.c_uint32),
                ("auto_max_swaps", C.c_uint32), ("lam", C.c_double), ("scale2", C.c_double),
                ("lsg_alpha", C.c_double), ("resid", C.c_void_p), ("mu", C.c_void_p)]


def edge_policy_c(pol):
    """anqi_edge_policy of an anqi.edge_policy.EdgePolicy, or None for the
    default prune; the returned struct keeps its tables alive."""
    if pol is None or not pol.active:
        return None
    resid = np.ascontiguousarray(pol.resid, np.float32) if pol.resid is not None else None
    mu = np.ascontiguousarray(pol.mu, np.float32) if pol.mu is not None else None
    ks = (C.c_uint32 * 8)(*(list(pol.ks) + [0] * (8 - len(pol.ks))))
    s = EdgePolicyC(pol.flags, len(pol.ks), ks, pol.nk, pol.budget, int(pol.occlude_all), pol.auto_candidates,
                    pol.auto_max_swaps, pol.lam, pol.scale2, pol.lsg_alpha,
                    resid.ctypes.data if resid is not None else None, mu.ctypes.data if mu is not None else None)
    s._keep = (resid, mu)
    return s


class BuildStats(C.Structure):
    _fields_ = [("total_ms", C.c_double), ("forest_ms", C.c_double), ("init_ms", C.c_double),
                ("join_ms", C.c_double), ("reverse_ms", C.c_double), ("gather_ms", C.c_double),
                ("join_updates", C.c_uint64), ("pool_total", C.c_uint64), ("gather_kernel_ms", C.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


_SIGS = {
    "anqi_ctx_create": [C.c_int, C.POINTER(_vp)],
    "anqi_ctx_destroy": [_vp],
    "anqi_last_error": [_vp],
    "anqi_version": [],
    "anqi_inject_fault": [_vp, C.c_uint32],
    "anqi_device_bytes": [_vp],
    "anqi_timer_start": [_vp],
    "anqi_timer_stop": [_vp, C.POINTER(C.c_float)],
    "anqi_pair_distances": [_vp, _f32, _f32, C.c_uint64, C.c_uint32, _f32, _f32],
    "anqi_pair_distances_group": [_vp, _f32, _f32, C.c_uint64, C.c_uint32, C.c_uint32, _f32, _f32],
    "anqi_lrq_encode": [_vp, _f32, C.c_uint64, C.c_uint32, C.c_uint32, _f32, _f32, _f32, C.c_uint32, _f32, _u8],
    "anqi_lrq_materialize": [_vp, _f32, _u8, C.c_uint64, C.c_uint32, C.c_uint32, _f32, _f32, _f32, C.c_uint32,
                             C.c_uint32, C.c_double, _f32],
    "anqi_lrq_encode_bits": [_vp, _f32, C.c_uint64, C.c_uint32, C.c_uint32, _f32, _f32, _vp, C.c_uint32,
                             C.c_uint32, C.c_uint32, _f32, _vp, _vp],
    "anqi_lrq_materialize_bits": [_vp, _f32, _vp, _vp, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, _f32, _f32,
                                  _vp, C.c_uint32, C.c_uint32, C.c_double, C.c_int, _f32],
    "anqi_analytic_rankm_materialize": [_vp, _f32, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                        C.c_double, C.c_uint32, C.c_double, _f32],
    "anqi_lift": [_vp, _f32, C.c_uint64, C.c_uint32, _f32, _f32, C.POINTER(C.c_double), C.POINTER(C.c_double)],
    "anqi_lift_metric": [_vp, _f32, C.c_uint64, C.c_uint32, _f32, C.c_uint32, _f32, C.POINTER(C.c_double),
                         C.POINTER(C.c_double)],
    "anqi_rp_forest": [_vp, _f32, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64,
                       C.c_uint32, _u32, _u32, _u32, _f32, _f32, _u32, _u32, _u32],
    "anqi_rp_forest_metric": [_vp, _f32, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64,
                              C.c_uint32, C.c_uint32, _u32, _u32, _u32, _f32, _f32, _u32, _u32, _u32],
    "anqi_aknn_build": [_vp, _f32, C.c_uint64, C.c_uint32, C.POINTER(AknnParams), _u32, _f32,
                        C.POINTER(BuildStats)],
    "anqi_aknn_init": [_vp, _f32, C.c_uint64, C.c_uint32, _u64, _u32, C.c_uint64, C.c_uint32, _u32, _f32],
    "anqi_aknn_gather": [_vp, _f32, C.c_uint64, C.c_uint32, _u32, _f32, C.c_uint32, C.c_uint32, C.c_uint32,
                         C.c_uint32, _u32, _f32],
    "anqi_aknn_init_metric": [_vp, _f32, C.c_uint64, C.c_uint32, _u64, _u32, C.c_uint64, C.c_uint32, C.c_uint32, _u32,
                              _f32],
    "anqi_aknn_gather_metric": [_vp, _f32, C.c_uint64, C.c_uint32, _u32, _f32, C.c_uint32, C.c_uint32, C.c_uint32,
                                C.c_uint32, C.c_uint32, _u32, _f32],
    "anqi_graph_build": [_vp, _f32, C.c_uint64, C.c_uint32, _u32, C.c_uint32, C.POINTER(GraphParams), _u32, _u32,
                         C.POINTER(BuildStats)],
    "anqi_graph_build_begin": [_vp, _f32, C.c_uint64, C.c_uint32, C.POINTER(GraphParams)],
    "anqi_graph_build_warm_rows": [_vp, C.c_uint64, C.c_uint64, _u32, C.c_uint32],
    "anqi_graph_build_finish": [_vp, _u32, _u32, C.POINTER(BuildStats)],
    "anqi_graph_tree_size": [_vp, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)],
    "anqi_graph_tree_copy": [_vp, _u32, _u32, _f32, _f32, _u32, _u32, _u32],
    "anqi_graph_warm_start": [_vp, _f32, C.c_uint64, C.c_uint32, _u32, C.c_uint32, C.c_uint32, C.c_uint32, _u32,
                              _f32],
    "anqi_graph_localjoin": [_vp, _f32, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, _u32, _f32,
                             _u64, C.POINTER(C.c_uint32)],
    "anqi_graph_localjoin_precision": [_vp, _f32, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                       C.c_uint32, _u32, _f32, _u64, C.POINTER(C.c_uint32), C.POINTER(C.c_float)],
    "anqi_graph_select": [_vp, _f32, C.c_uint64, C.c_uint32, _u32, _f32, C.c_uint32, C.c_uint32, C.c_uint32,
                          C.c_uint32, C.c_float, _u32, _u32],
    "anqi_graph_commit": [_vp, _f32, C.c_uint64, C.c_uint32, _u32, _u32, C.c_uint32, C.c_float, _u32, _u32],
    "anqi_graph_select_policy": [_vp, _f32, C.c_uint64, C.c_uint32, _u32, _f32, C.c_uint32, C.c_uint32, C.c_uint32,
                                 C.c_uint32, C.c_float, _vp, _u32, _u32],
    "anqi_graph_commit_policy": [_vp, _f32, C.c_uint64, C.c_uint32, _u32, _u32, C.c_uint32, C.c_float, _vp, _u32,
                                 _u32],
    "anqi_graph_vamana_batch_refine": [_vp, _f32, C.c_uint64, C.c_uint32, _u32, _u32, _u32, C.c_uint32, _vp],
    "anqi_graph_vamana_select": [_vp, _f32, C.c_uint64, C.c_uint32, _u32, _u32, C.c_uint32, _u32, C.c_uint32, _u32,
                                 C.c_uint32, C.c_float, _u32, _u32],
    "anqi_index_load": [_vp, C.POINTER(IndexDesc)],
    "anqi_verifier_load": [_vp, _f32, _u8, C.c_uint64, C.c_uint32, C.c_uint32, _f32, _f32, _f32, C.c_uint32],
    "anqi_verifier_load_bits": [_vp, _f32, _vp, _vp, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, _f32, _f32,
                                _vp, C.c_uint32, C.c_int],
    "anqi_verifier_load_analytic": [_vp, _f32, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                    C.c_double],
    "anqi_verifier_materialize": [_vp, C.c_uint32, C.c_double],
    "anqi_set_thresholds": [_vp, C.c_uint32, _f32],
    "anqi_rknn_query": [_vp, _f32, C.c_uint32, _vp, C.c_uint32, _vp, C.c_uint32, _u32, _u32, C.c_uint64, _vp, _vp,
                        C.c_uint64, _vp, C.POINTER(QueryStats)],
    "anqi_query_upload": [_vp, _f32, C.c_uint32, _vp, C.c_uint32, _vp, C.c_uint32],
    "anqi_query_run": [_vp, C.c_int, C.POINTER(QueryStats)],
    "anqi_query_run_graph": [_vp, C.c_int, C.POINTER(QueryStats)],
    "anqi_query_counters": [_vp, C.POINTER(QueryStats)],
    "anqi_query_download": [_vp, _u32, _vp, C.c_uint64, _vp, _vp, C.c_uint64, _vp],
    "anqi_query_evaluate": [_vp, _u32, _u32, C.c_uint64, C.POINTER(C.c_double), C.POINTER(C.c_double),
                            C.POINTER(C.c_double), C.POINTER(C.c_uint32)],
    "anqi_gt_load": [_vp, _u32, _u32, C.c_uint64],
    "anqi_query_evaluate_sums": [_vp, C.POINTER(EvalSums)],
    "anqi_rknn_query_noalloc": [_vp, _vp, C.c_uint32, _vp, C.c_uint32, C.c_uint32, _vp, _vp, _vp, _vp],
    "anqi_lrq_objective_forward": [_vp, C.c_uint64, C.c_uint32, C.c_uint32, _vp, _vp, _vp, C.c_uint32, _vp, _vp,
                                   _vp, _vp, _vp, _vp],
    "anqi_lrq_objective_backward": [_vp, C.c_uint64, C.c_uint32, C.c_uint32, _vp, _vp, _vp, _vp, _vp,
                                    C.c_uint32, C.c_double, _vp, _vp, _vp, _vp],
    "anqi_lrq_fit_stats": [_vp, _vp, C.c_uint64, C.c_uint32, _vp, _vp, C.c_uint64, _vp, _vp, _vp],
    "anqi_lrq_fit_residual": [_vp, _vp, C.c_uint64, C.c_uint32, _vp, _vp, C.c_uint32, _vp, _vp, _vp],
    "anqi_lrq_fit_range": [_vp, C.c_uint64, C.c_uint32, _vp, _vp, C.c_uint32, _vp, _vp, _vp],
    "anqi_lrq_fit_codebooks_scratch": [C.c_uint64, C.c_uint32],
    "anqi_lrq_fit_codebooks": [_vp, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, _vp, C.c_uint64, _vp, _vp],
    "anqi_lrq_fit_decode": [_vp, C.c_uint64, C.c_uint32, _vp, C.c_uint32, _vp, _vp, C.c_uint32,
                            C.POINTER(C.c_uint32), _vp],
    "anqi_exact_topk_tc": [_vp, _f32, C.c_uint64, C.c_uint32, C.c_uint32, _vp, C.c_uint32, _u32, _f32],
    "anqi_exact_topk_tc_metric": [_vp, _f32, C.c_uint64, C.c_uint32, C.c_uint32, _vp, C.c_uint32, C.c_uint32, _u32,
                                  _f32],
    "anqi_rknn_ground_truth_tc": [_vp, _f32, C.c_uint64, _f32, C.c_uint64, C.c_uint32, _f32, _u32, _u32, _f32,
                                  C.c_uint64, C.POINTER(C.c_uint64)],
    "anqi_rknn_ground_truth_tc_metric": [_vp, _f32, C.c_uint64, _f32, C.c_uint64, C.c_uint32, _f32, C.c_uint32, _u32,
                                         _u32, _f32, C.c_uint64, C.POINTER(C.c_uint64)],
    "anqi_bf16_gram": [_vp, _f32, C.c_uint64, _f32, C.c_uint64, C.c_uint32, _f32],
    "anqi_exact_topk": [_vp, _f32, C.c_uint64, C.c_uint32, C.c_uint32, _u32, _f32],
    "anqi_rknn_ground_truth": [_vp, _f32, C.c_uint64, _f32, C.c_uint64, C.c_uint32, _f32, _u32, _u32, _f32,
                               C.c_uint64, C.POINTER(C.c_uint64)],
    "anqi_exact_topk_metric": [_vp, _f32, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, _u32, _f32],
    "anqi_rknn_ground_truth_metric": [_vp, _f32, C.c_uint64, _f32, C.c_uint64, C.c_uint32, _f32, C.c_uint32, _u32,
                                      _u32, _f32, C.c_uint64, C.POINTER(C.c_uint64)],
}

#: metric codes of the C ABI (ANQI_METRIC_L2 / ANQI_METRIC_IP)
METRICS = {"l2": 0, "ip": 1}

#: every symbol include/anqi.h declares (checked by the CPU tests)
EXPORTED = tuple(_SIGS)

_lib = None


def load_library() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise AnqiError(ANQI_ERR_DEVICE, f"libanqi.so not built ({LIB_PATH}); run anqi-implementation_b200/build.py")
    lib = C.CDLL(str(LIB_PATH))
    missing = [name for name in _SIGS if not hasattr(lib, name)]
    if missing:
        raise AnqiError(ANQI_ERR_DEVICE, f"{LIB_PATH} lacks exported symbols: {missing}")
    for name, args in _SIGS.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = C.c_int
    lib.anqi_ctx_destroy.restype = None
    lib.anqi_last_error.restype = C.c_char_p
    lib.anqi_device_bytes.restype = C.c_uint64
    lib.anqi_lrq_fit_codebooks_scratch.restype = C.c_uint64
    _lib = lib
    return lib


def _c(a, dtype) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=dtype)


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


@dataclass
class QueryResult:
    pred_off: np.ndarray
    pred_ids: np.ndarray
    cand_off: np.ndarray | None
    cand_ids: np.ndarray | None
    n_dist: np.ndarray | None
    stats: dict

    def pred(self, i: int) -> np.ndarray:
        return self.pred_ids[self.pred_off[i]:self.pred_off[i + 1]]

    def cand(self, i: int) -> np.ndarray:
        return self.cand_ids[self.cand_off[i]:self.cand_off[i + 1]]


class Context:
    """One CUDA context: device memory, one stream, an optional resident index."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        h = C.c_void_p()
        self.device = device
        rc = self.lib.anqi_ctx_create(device, C.byref(h))
        if rc != ANQI_OK:
            raise AnqiError(rc, f"cannot create a context on CUDA device {device}")
        self.h = h
        self._keep = []

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.anqi_ctx_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int, what: str) -> None:
        if rc != ANQI_OK:
            msg = self.lib.anqi_last_error(self.h)
            raise AnqiError(rc, f"{what}: {msg.decode() if msg else ''}")

    def inject_fault(self, flags: int) -> None:
        """Test hook (anqi_inject_fault): 1 = the search issues no row copies, so
        its bounded waits run out and queries fail with ANQI_ERR_TIMEOUT; 0 = off."""
        self._check(self.lib.anqi_inject_fault(self.h, flags), "inject_fault")

    def timer_start(self) -> None:
        self._check(self.lib.anqi_timer_start(self.h), "timer_start")

    def timer_stop(self) -> float:
        ms = C.c_float()
        self._check(self.lib.anqi_timer_stop(self.h, C.byref(ms)), "timer_stop")
        return ms.value

    @property
    def device_bytes(self) -> int:
        return int(self.lib.anqi_device_bytes(self.h))

    # ------------------------------------------------------------ kernels

    def pair_distances(self, a, b, group=4):
        a = _c(a, np.float32)
        b = _c(b, np.float32)
        m, dim = a.shape
        l2 = np.empty(m, np.float32)
        ip = np.empty(m, np.float32)
        self._check(self.lib.anqi_pair_distances_group(self.h, a, b, m, dim, group, l2, ip), "pair_distances")
        return l2, ip

    def lrq_encode(self, keys, mu, basis, codebook):
        keys = _c(keys, np.float32)
        n, nk = keys.shape
        rankm = basis.shape[0]
        coeff = np.empty((n, rankm), np.float32)
        codes = np.empty((n, nk), np.uint8)
        self._check(self.lib.anqi_lrq_encode(self.h, keys, n, nk, rankm, _c(mu, np.float32), _c(basis, np.float32),
                                             _c(codebook, np.float32), codebook.shape[1], coeff, codes), "lrq_encode")
        return coeff, codes

    def lrq_materialize(self, coeff, codes, mu, basis, codebook, k, radius_scale=1.0):
        codes = _c(codes, np.uint8)
        n, nk = codes.shape
        thr = np.empty(n, np.float32)
        self._check(self.lib.anqi_lrq_materialize(self.h, _c(coeff, np.float32), codes, n, nk, basis.shape[0],
                                                  _c(mu, np.float32), _c(basis, np.float32),
                                                  _c(codebook, np.float32), codebook.shape[1], k, radius_scale, thr),
                    "lrq_materialize")
        return thr

    def lrq_encode_bits(self, keys, mu, basis, codebook, bits: int, policy: str = "floor"):
        """Every CompactLrqVerifier form: returns coeff, packed code bytes (or
        None), float residuals (bits 32, else None)."""
        keys = _c(keys, np.float32)
        n, nk = keys.shape
        rankm = basis.shape[0]
        coeff = np.empty((n, rankm), np.float32)
        codes = np.zeros(formats.packed_code_bytes(n * nk, bits), np.uint8) if bits in formats.PACKED_BITS else None
        resid = np.empty((n, nk), np.float32) if bits == 32 else None
        cb = None if codebook is None else _c(codebook, np.float32)
        self._check(self.lib.anqi_lrq_encode_bits(self.h, keys, n, nk, rankm, _c(mu, np.float32), _c(basis, np.float32),
                                                  _ptr(cb), 0 if cb is None else cb.shape[1], bits,
                                                  formats.POLICY_CODE[policy], coeff, _ptr(codes), _ptr(resid)),
                    "lrq_encode_bits")
        return coeff, codes, resid

    def lrq_materialize_bits(self, coeff, codes, resid, nk: int, mu, basis, codebook, bits: int, k: int,
                             radius_scale=1.0, signed_keys=False):
        coeff = _c(coeff, np.float32)
        n = coeff.shape[0]
        thr = np.empty(n, np.float32)
        cb = None if codebook is None else _c(codebook, np.float32)
        self._check(self.lib.anqi_lrq_materialize_bits(
            self.h, coeff, _ptr(None if codes is None else _c(codes, np.uint8)),
            _ptr(None if resid is None else _c(resid, np.float32)), n, nk, basis.shape[0], bits, _c(mu, np.float32),
            _c(basis, np.float32), _ptr(cb), 0 if cb is None else cb.shape[1], k, radius_scale, int(signed_keys), thr),
            "lrq_materialize_bits")
        return thr

    def analytic_materialize(self, model, k: int, radius_scale=1.0):
        """AnalyticRankMVerifier::materialize_k for a formats.AnalyticModel."""
        coeff = _c(model.coeff, np.float32)
        thr = np.empty(coeff.shape[0], np.float32)
        self._check(self.lib.anqi_analytic_rankm_materialize(self.h, coeff, coeff.shape[0], coeff.shape[1],
                                                             model.train_kmax, model.fit_kmin, model.flags,
                                                             model.b0, k, radius_scale, thr),
                    "analytic_rankm_materialize")
        return thr

    def lift(self, base, radius, metric: str = "l2"):
        base = _c(base, np.float32)
        n, d = base.shape
        out = np.empty((n, d + 2), np.float32)
        m2, sc = C.c_double(), C.c_double()
        self._check(self.lib.anqi_lift_metric(self.h, base, n, d, _c(radius, np.float32), METRICS[metric], out,
                                              C.byref(m2), C.byref(sc)), "lift")
        return out, m2.value, sc.value

    # ------------------------------------------------------------- index

    def index_load(self, base, lifted, deg, links, tree, scale: float, mstar2: float, metric: str = "l2") -> None:
        """tree: post-order arrays with attributes left/right/offset/hyperplane and leaf_first()."""
        base = _c(base, np.float32)
        lifted = _c(lifted, np.float32)
        deg = _c(deg, np.uint32)
        links = _c(links, np.uint32)
        tl = _c(tree.left, np.uint32)
        tr = _c(tree.right, np.uint32)
        to = _c(tree.offset, np.float32)
        th = _c(tree.hyperplane, np.float32)
        tf = _c(tree.leaf_first(), np.uint32)
        n, d = base.shape
        desc = IndexDesc(n, d, links.shape[1], _ptr(base), _ptr(lifted), _ptr(deg), _ptr(links), len(tl), _ptr(tl),
                         _ptr(tr), _ptr(to), _ptr(th), _ptr(tf), float(scale), float(mstar2), METRICS[metric])
        self._check(self.lib.anqi_index_load(self.h, C.byref(desc)), "index_load")
        self.n = n
        self.d = d

    def verifier_load(self, coeff, codes, mu, basis, codebook) -> None:
        codes = _c(codes, np.uint8)
        n, nk = codes.shape
        self._check(self.lib.anqi_verifier_load(self.h, _c(coeff, np.float32), codes, n, nk, basis.shape[0],
                                                _c(mu, np.float32), _c(basis, np.float32), _c(codebook, np.float32),
                                                codebook.shape[1]), "verifier_load")

    def verifier_load_bits(self, coeff, codes, resid, nk: int, mu, basis, codebook, bits: int,
                           signed_keys=False) -> None:
        coeff = _c(coeff, np.float32)
        cb = None if codebook is None else _c(codebook, np.float32)
        self._check(self.lib.anqi_verifier_load_bits(
            self.h, coeff, _ptr(None if codes is None else _c(codes, np.uint8)),
            _ptr(None if resid is None else _c(resid, np.float32)), coeff.shape[0], nk, basis.shape[0], bits,
            _c(mu, np.float32), _c(basis, np.float32), _ptr(cb), 0 if cb is None else cb.shape[1],
            int(signed_keys)), "verifier_load_bits")

    def verifier_load_analytic(self, model) -> None:
        coeff = _c(model.coeff, np.float32)
        self._check(self.lib.anqi_verifier_load_analytic(self.h, coeff, coeff.shape[0], coeff.shape[1],
                                                         model.train_kmax, model.fit_kmin, model.flags, model.b0),
                    "verifier_load_analytic")

    def verifier_materialize(self, k: int, radius_scale: float = 1.0) -> None:
        self._check(self.lib.anqi_verifier_materialize(self.h, k, radius_scale), "verifier_materialize")

    def set_thresholds(self, k: int, thr) -> None:
        self._check(self.lib.anqi_set_thresholds(self.h, k, _c(thr, np.float32)), "set_thresholds")

    # ----------------------------------------------------------- queries

    @staticmethod
    def _per_query(v, nq):
        if v is None or np.isscalar(v):
            return None, int(v or 0)
        a = _c(v, np.uint32)
        assert a.shape == (nq,)
        return a, 0

    def rknn_query(self, queries, k, L, keep_candidates=False, pred_cap=None, out=None) -> QueryResult:
        """Host-buffer end-to-end call (queries H2D, results D2H inside).

        out: optional (pred_off, pred_ids, n_dist) uint32 arrays of nq + 1,
        any capacity and nq entries -- e.g. pinned buffers reused across
        calls; the results are then copied straight into them (a larger
        pred_ids is allocated if the results outgrow it)."""
        queries = _c(queries, np.float32)
        nq = queries.shape[0]
        ka, kall = self._per_query(k, nq)
        La, Lall = self._per_query(L, nq)
        st = QueryStats()
        cap = pred_cap or max(1024, nq * 256)
        if out is not None:
            o_off, o_ids, o_nd = out
            if (o_off.dtype != np.uint32 or o_ids.dtype != np.uint32 or o_nd.dtype != np.uint32
                    or o_off.shape != (nq + 1,) or o_nd.shape != (nq,) or o_ids.ndim != 1
                    or not (o_off.flags.c_contiguous and o_ids.flags.c_contiguous and o_nd.flags.c_contiguous)):
                raise ValueError("out: uint32 C-contiguous arrays of nq + 1, any and nq entries")
            cap = len(o_ids)
        while True:
            if out is not None and cap == len(out[1]):
                pred_off, pred_ids, nd = out
            else:
                pred_off = np.empty(nq + 1, np.uint32)
                pred_ids = np.empty(cap, np.uint32)
            cand_off = np.empty(nq + 1, np.uint32) if keep_candidates else None
            ccap = cap * 4 if keep_candidates else 0
            cand_ids = np.empty(ccap, np.uint32) if keep_candidates else None
            if out is None or cap != len(out[1]):
                nd = np.empty(nq, np.uint32)
            rc = self.lib.anqi_rknn_query(self.h, queries, nq, _ptr(ka), kall, _ptr(La), Lall, pred_off, pred_ids, cap,
                                          _ptr(cand_off), _ptr(cand_ids), ccap, _ptr(nd), C.byref(st))
            if rc == ANQI_ERR_CAPACITY:
                cap *= 4
                continue
            self._check(rc, "rknn_query")
            break
        stats = {k2: getattr(st, k2) for k2, _ in QueryStats._fields_}
        if out is not None and pred_ids is out[1]:
            # the caller's buffers hold the results: views, no copies
            return QueryResult(pred_off, pred_ids[:pred_off[-1]], cand_off,
                               None if cand_ids is None else cand_ids[:cand_off[-1]].copy(), nd, stats)
        return QueryResult(pred_off, pred_ids[:pred_off[-1]].copy(), cand_off,
                           None if cand_ids is None else cand_ids[:cand_off[-1]].copy(), nd, stats)

    def query_upload(self, queries, k, L) -> None:
        queries = _c(queries, np.float32)
        nq = queries.shape[0]
        ka, kall = self._per_query(k, nq)
        La, Lall = self._per_query(L, nq)
        self._keep = [ka, La]
        self.nq = nq
        self._check(self.lib.anqi_query_upload(self.h, queries, nq, _ptr(ka), kall, _ptr(La), Lall), "query_upload")

    def query_run(self, keep_candidates=False, counters=False) -> dict:
        st = QueryStats()
        self._check(self.lib.anqi_query_run(self.h, int(keep_candidates), C.byref(st)), "query_run")
        if counters:
            self._check(self.lib.anqi_query_counters(self.h, C.byref(st)), "query_counters")
        return {k2: getattr(st, k2) for k2, _ in QueryStats._fields_}

    def query_run_graph(self, keep_candidates=False) -> dict:
        """anqi_query_run through a captured CUDA graph (same results)."""
        st = QueryStats()
        self._check(self.lib.anqi_query_run_graph(self.h, int(keep_candidates), C.byref(st)), "query_run_graph")
        return {k2: getattr(st, k2) for k2, _ in QueryStats._fields_}

    def query_download(self, with_candidates=False) -> QueryResult:
        nq = self.nq
        pred_off = np.empty(nq + 1, np.uint32)
        self._check(self.lib.anqi_query_download(self.h, pred_off, None, 0, None, None, 0, None), "query_download")
        pred_ids = np.empty(max(1, int(pred_off[-1])), np.uint32)
        cand_off = np.empty(nq + 1, np.uint32) if with_candidates else None
        nd = np.empty(nq, np.uint32)
        if with_candidates:
            self._check(self.lib.anqi_query_download(self.h, pred_off, _ptr(pred_ids), len(pred_ids),
                                                     _ptr(cand_off), None, 0, None), "query_download")
            cand_ids = np.empty(max(1, int(cand_off[-1])), np.uint32)
        else:
            cand_ids = None
        self._check(self.lib.anqi_query_download(self.h, pred_off, _ptr(pred_ids), len(pred_ids), _ptr(cand_off),
                                                 _ptr(cand_ids), 0 if cand_ids is None else len(cand_ids),
                                                 _ptr(nd)), "query_download")
        return QueryResult(pred_off, pred_ids[:pred_off[-1]], cand_off,
                           None if cand_ids is None else cand_ids[:cand_off[-1]], nd, {})

    def gt_load(self, gt_off, gt_ids) -> None:
        """Keeps a ground-truth CSR on the device for the current batch."""
        gt_off = _c(gt_off, np.uint32)
        gt_ids = _c(gt_ids, np.uint32) if len(gt_ids) else np.zeros(1, np.uint32)
        self._check(self.lib.anqi_gt_load(self.h, gt_off, gt_ids, int(gt_off[-1])), "gt_load")

    def query_evaluate_sums(self) -> dict:
        """Sums over queries with non-empty truth of the last run's metrics."""
        e = EvalSums()
        self._check(self.lib.anqi_query_evaluate_sums(self.h, C.byref(e)), "query_evaluate_sums")
        return {k: getattr(e, k) for k, _ in EvalSums._fields_}

    def exact_topk_tc(self, base: np.ndarray, K: int, hints: np.ndarray | None = None, metric: str = "l2"):
        """Exact top-K (ids, keys) on the BF16 tensor path; equals anqi_exact_topk_metric."""
        base = _c(base, np.float32)
        n, d = base.shape
        ids = np.empty((n, K), np.uint32)
        keys = np.empty((n, K), np.float32)
        h = None if hints is None else _c(hints, np.uint32)
        self._check(self.lib.anqi_exact_topk_tc_metric(self.h, base, n, d, K, _ptr(h), 0 if h is None else h.shape[1],
                                                       METRICS[metric], ids, keys), "exact_topk_tc")
        return ids, keys

    def rknn_ground_truth_tc(self, base: np.ndarray, query: np.ndarray, rk2: np.ndarray, metric: str = "l2"):
        """Reverse-kNN CSR (off, ids, keys) on the BF16 tensor path; equals anqi_rknn_ground_truth_metric."""
        base = _c(base, np.float32)
        query = _c(query, np.float32)
        rk2 = _c(rk2, np.float32)
        n, d = base.shape
        nq = query.shape[0]
        off = np.empty(nq + 1, np.uint32)
        tot = C.c_uint64()
        cap = max(1024, 64 * nq)
        while True:
            ids = np.empty(cap, np.uint32)
            keys = np.empty(cap, np.float32)
            rc = self.lib.anqi_rknn_ground_truth_tc_metric(self.h, base, n, query, nq, d, rk2, METRICS[metric], off,
                                                           ids, keys, cap, C.byref(tot))
            if rc == ANQI_ERR_CAPACITY and tot.value > cap:
                cap = int(tot.value)
                continue
            self._check(rc, "rknn_ground_truth_tc")
            return off.copy(), ids[:tot.value].copy(), keys[:tot.value].copy()

    def bf16_gram(self, a: np.ndarray, b: np.ndarray) -> np.ndarray:
        """<bf16(a_i), bf16(b_j)> accumulated in FP32 on the tensor cores."""
        a = _c(a, np.float32)
        b = _c(b, np.float32)
        out = np.empty((a.shape[0], b.shape[0]), np.float32)
        self._check(self.lib.anqi_bf16_gram(self.h, a, a.shape[0], b, b.shape[0], a.shape[1], out), "bf16_gram")
        return out

    def query_evaluate(self, gt_off, gt_ids) -> dict:
        gt_off = _c(gt_off, np.uint32)
        gt_ids = _c(gt_ids, np.uint32) if len(gt_ids) else np.zeros(1, np.uint32)
        r, p, cr = C.c_double(), C.c_double(), C.c_double()
        ne = C.c_uint32()
        self._check(self.lib.anqi_query_evaluate(self.h, gt_off, gt_ids, int(gt_off[-1]), C.byref(r), C.byref(p),
                                                 C.byref(cr), C.byref(ne)), "query_evaluate")
        d = max(1, ne.value)
        return {"recall": r.value / d, "precision": p.value / d, "candidate_recall": cr.value / d,
                "nonempty": ne.value}
