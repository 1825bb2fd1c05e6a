"""The Vamana refine's settings as the reference reads them from its
environment (include/index.h:1262-1285 for the style, the beam width and the
passes; :936-955 for the batched style's batch sizes, early alpha and entry,
choose_vamana_entry :190-222), for anqi_graph_params."""
from __future__ import annotations

import re
from dataclasses import dataclass
from typing import Mapping

import numpy as np

from .edge_policy import c_atof, c_atoi


@dataclass
class VamanaParams:
    style: str = "global"        # "global" / "old" (per-row RP-tree entries) or "batch"
    L: int = 128
    passes: int = 2
    batch_frac: float = 0.02
    max_batch: int = 1000000
    batch_base: float = 2.0
    early_alpha: float = 1.0
    early_alpha_one: bool = True
    entry: int = 0


def choose_entry(env: Mapping[str, str], x: np.ndarray | None) -> int:
    """choose_vamana_entry (index.h:190-222): an id (mod n), or the sampled
    point closest to the sample mean for "medoid" / "centroid"; 0 by default."""
    ev = env.get("ANQI_VAMANA_ENTRY", "")
    if not ev:
        return 0
    n = 0 if x is None else len(x)
    if ev in ("medoid", "centroid"):
        if x is None:
            raise ValueError("the medoid entry needs the rows")
        sample = c_atoi(env["ANQI_VAMANA_ENTRY_SAMPLE"]) if "ANQI_VAMANA_ENTRY_SAMPLE" in env else min(n, 100000)
        sample = max(1, min(sample, n))
        step = max(1, n // sample)
        ids = (np.arange(sample, dtype=np.uint64) * step) % n
        xs = np.asarray(x, np.float64)[ids]
        mean = np.zeros(x.shape[1])
        for r in xs:  # the sums in sample order, as the reference adds them
            mean += r
        mean /= sample
        best, bestd = 0, np.inf
        for t, i in enumerate(ids):
            z = xs[t] - mean
            dd = 0.0
            for v in z:
                dd += v * v
            if dd < bestd:
                best, bestd = int(i), dd
        return best
    # strtoull: blanks, an optional sign (a minus wraps modulo 2^64), digits
    m = re.match(r"\s*([+-]?)(\d+)", ev)
    if not m or n == 0:
        return 0
    v = min(int(m.group(2)), 2**64 - 1)
    if m.group(1) == "-":
        v = (2**64 - v) % 2**64
    return v % n


def from_env(env: Mapping[str, str], x: np.ndarray | None = None) -> VamanaParams | None:
    """None when ANQI_VAMANA is unset."""
    if "ANQI_VAMANA" not in env:
        return None
    p = VamanaParams()
    p.style = env.get("ANQI_VAMANA_STYLE", "global")
    p.L = c_atoi(env["ANQI_VAMANA_L"]) if "ANQI_VAMANA_L" in env else 128
    p.passes = c_atoi(env["ANQI_VAMANA_PASS"]) if "ANQI_VAMANA_PASS" in env else 2
    if p.style not in ("global", "old"):
        p.batch_frac = c_atof(env["ANQI_VAMANA_BATCH_FRAC"]) if "ANQI_VAMANA_BATCH_FRAC" in env else 0.02
        p.max_batch = c_atoi(env["ANQI_VAMANA_MAX_BATCH"]) if "ANQI_VAMANA_MAX_BATCH" in env else 1000000
        p.batch_base = c_atof(env["ANQI_VAMANA_BATCH_BASE"]) if "ANQI_VAMANA_BATCH_BASE" in env else 2.0
        p.early_alpha = c_atof(env["ANQI_VAMANA_EARLY_ALPHA"]) if "ANQI_VAMANA_EARLY_ALPHA" in env else 1.0
        p.early_alpha_one = (c_atoi(env["ANQI_VAMANA_EARLY_ALPHA_ONE"]) if "ANQI_VAMANA_EARLY_ALPHA_ONE" in env
                             else 1) != 0
        p.entry = choose_entry(env, x)
    return p
