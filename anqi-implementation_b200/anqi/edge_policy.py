"""Edge policies of the G48 prune: what the reference derives from its
environment in configure_edge_residual_cover (include/index.h:305-440),
resolved to the flags and parameters the prune kernels take
(prune_pool_to_ids, :772-829).

  residual_cover                     rng_extend to M - budget, residual-cover
                                     edges, rng_extend to M
  ball_rng, bubble_rng               ball-occlusion RNG over the pool ordered by
                                     dist - lambda * max_k radj, then rng_extend
  ball_hybrid, ball_multik,          rng_extend to M - budget, ball RNG,
  bubble_hybrid, bubble_multik       rng_extend
  lsg_rng                            RNG in the LSG metric d2 / (mu_a mu_b)^alpha
  lsg_bubble_hybrid                  LSG to M - budget, ball RNG, LSG
  bubble_auto, bubble_auto_full      RNG, then the verification-constrained
                                     swap optimizer over the top
                                     ANQI_EDGE_AUTO_CANDIDATES ball alternatives
                                     (all of the pool for _full)

Anything else names no policy (the default prune), as in the reference.
Errors the reference reports with exit status 2 raise PolicyError with its
message.
"""
from __future__ import annotations

import math
import os
import re
from dataclasses import dataclass, field
from pathlib import Path
from typing import Mapping

import numpy as np

COVER, BALL, PURE, LSG, AUTO, AUTO_FULL = 1, 2, 4, 8, 16, 32
NEEDS_RESIDUAL = ("residual_cover", "ball_rng", "ball_hybrid", "ball_multik", "bubble_rng", "bubble_hybrid",
                  "bubble_multik", "bubble_auto", "bubble_auto_full", "lsg_bubble_hybrid")
MAX_KS = 8


class PolicyError(ValueError):
    pass


def c_atoi(s: str) -> int:
    """atoi: optional leading blanks and sign, then digits; 0 when none."""
    m = re.match(r"\s*([+-]?\d+)", s)
    return int(m.group(1)) if m else 0


def c_atof(s: str) -> float:
    """atof (strtod's decimal and special forms): the longest numeric prefix; 0 when none."""
    m = re.match(r"\s*([+-]?(?:(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?|inf(?:inity)?|nan))", s, re.IGNORECASE)
    return float(m.group(1)) if m else 0.0


def parse_int_list(s: str) -> list[int]:
    """parse_int_list (index.h:249-258): comma-separated, positive values kept."""
    out = []
    for tok in s.split(","):
        if not tok:
            continue
        v = c_atoi(tok)
        if v > 0:
            out.append(v)
    return out


@dataclass
class EdgePolicy:
    name: str
    flags: int = 0
    ks: list[int] = field(default_factory=list)
    nk: int = 100
    budget: int = 0
    occlude_all: bool = True
    auto_candidates: int = 1
    auto_max_swaps: int = 1
    lam: float = 1.0
    scale2: float = 1.0
    lsg_alpha: float = 1.0
    resid: np.ndarray | None = None  # n x nk float32
    mu: np.ndarray | None = None     # n float32

    @property
    def active(self) -> bool:
        return self.flags != 0


def read_meta_scale2(path: Path) -> float:
    """The scale^2 the policy reads from <folder>_anqi_meta.txt ("M*^2 scale"),
    1 when the file is absent or unreadable (index.h:389-393)."""
    try:
        parts = Path(path).read_text().split()
        return float(parts[1]) * float(parts[1])
    except (OSError, IndexError, ValueError):
        return 1.0


def from_env(env: Mapping[str, str], n: int, M: int, folder: str = "", scale2: float | None = None) -> EdgePolicy | None:
    """The policy of env (None when ANQI_EDGE_POLICY is unset or empty).
    folder: the graph's folder prefix, where the default residual table
    (<folder>_anqi_rankm_residual.bin) and the lift meta
    (<folder>_anqi_meta.txt) live; scale2 overrides the meta file."""
    pol = env.get("ANQI_EDGE_POLICY", "")
    if not pol:
        return None
    p = EdgePolicy(pol)
    if pol in ("lsg_rng", "lsg_bubble_hybrid"):
        p.lsg_alpha = c_atof(env["ANQI_LSG_ALPHA"]) if "ANQI_LSG_ALPHA" in env else 1.0
        if not math.isfinite(p.lsg_alpha) or p.lsg_alpha < 0.0:
            raise PolicyError(f"[edge-policy] invalid ANQI_LSG_ALPHA={p.lsg_alpha!r}")
        mu_path = env.get("ANQI_LSG_MU_FILE", "")
        if not mu_path:
            raise PolicyError("[edge-policy] lsg_rng requires ANQI_LSG_MU_FILE")
        try:
            size = os.path.getsize(mu_path)
        except OSError:
            raise PolicyError(f"[edge-policy] lsg_rng cannot open mu table {mu_path}") from None
        if size != n * 4:
            raise PolicyError(f"[edge-policy] lsg mu size mismatch {mu_path}: expected {n * 4} bytes, got {size}")
        mu = np.fromfile(mu_path, dtype=np.float32, count=n)
        bad = np.flatnonzero(~np.isfinite(mu) | (mu <= 0))
        if bad.size:
            raise PolicyError(f"[edge-policy] invalid lsg mu[{bad[0]}]={mu[bad[0]]:.9g}")
        p.mu = mu
        p.flags |= LSG
        if pol == "lsg_rng":
            return p
    if pol not in NEEDS_RESIDUAL:
        return p
    nk = c_atoi(env["ANQI_EDGE_NK"]) if "ANQI_EDGE_NK" in env else 100
    if nk == 0:
        nk = 100
    if nk < 0:
        raise PolicyError(f"[edge-policy] invalid ANQI_EDGE_NK={nk}")
    p.nk = nk
    budget = c_atoi(env["ANQI_EDGE_RESID_BUDGET"]) if "ANQI_EDGE_RESID_BUDGET" in env else 16
    p.budget = min(max(0, budget), M)
    p.auto_candidates = max(1, c_atoi(env["ANQI_EDGE_AUTO_CANDIDATES"]) if "ANQI_EDGE_AUTO_CANDIDATES" in env else M)
    p.auto_max_swaps = max(1, c_atoi(env["ANQI_EDGE_AUTO_MAX_SWAPS"]) if "ANQI_EDGE_AUTO_MAX_SWAPS" in env else M)
    p.lam = c_atof(env["ANQI_EDGE_RESID_LAMBDA"]) if "ANQI_EDGE_RESID_LAMBDA" in env else 1.0
    ks = parse_int_list(env["ANQI_EDGE_KS"] if "ANQI_EDGE_KS" in env else "10,50,100")
    p.ks = [k for k in ks if 1 <= k <= nk]
    if not p.ks:
        return p
    if len(p.ks) > MAX_KS:
        raise PolicyError(f"[edge-policy] at most {MAX_KS} values in ANQI_EDGE_KS are supported here")
    auto = pol in ("bubble_auto", "bubble_auto_full")
    if p.budget == 0 and pol != "ball_rng" and not auto:
        return p
    p.scale2 = read_meta_scale2(Path(f"{folder}_anqi_meta.txt")) if scale2 is None else scale2
    resid_path = env["ANQI_EDGE_RESID_FILE"] if "ANQI_EDGE_RESID_FILE" in env else f"{folder}_anqi_rankm_residual.bin"
    try:
        size = os.path.getsize(resid_path)
    except OSError:
        raise PolicyError(f"[edge-policy] residual_cover requested but missing {resid_path}") from None
    if size != n * nk * 4:
        raise PolicyError(f"[edge-policy] residual table stride/size mismatch {resid_path}: expected {n * nk * 4} "
                          f"bytes (n={n} edge_nk={nk}), got {size} bytes; set ANQI_EDGE_NK to the table stride")
    p.resid = np.fromfile(resid_path, dtype=np.float32, count=n * nk).reshape(n, nk)
    if pol == "residual_cover":
        p.flags |= COVER
    else:
        p.flags |= BALL
        if pol in ("ball_rng", "bubble_rng"):
            p.flags |= PURE
        p.occlude_all = env.get("ANQI_EDGE_BALL_OCCLUSION", "all") != "any"
    if auto:
        p.flags |= AUTO | (AUTO_FULL if pol == "bubble_auto_full" else 0)
    return p
