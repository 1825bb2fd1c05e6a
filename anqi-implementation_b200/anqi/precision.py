"""Error of every distance form against FP64, on random base/query pairs.

    python -m anqi.precision [--n 1000000] [--nq 10000] [--pairs 20000]

Forms (all through libanqi.so on the GPU):
* ``l2_fp32``: squared L2 in the reference's FP32 lane order
  (include/distance.h:58-86; the graph and lift distances);
* ``key_fp32``: |q|^2 + |x|^2 - 2 <q, x> in FP32 (dataset_gt.cpp:294, the
  verifier and ground-truth key);
* ``key_bf16``: the same key from BF16 tensor-core tiles with FP32
  accumulation (the precision form's filter), with the bound eps the filter
  uses checked on every pair: |key_bf16 - key_fp32| <= eps.
Printed as one JSON line.
"""
from __future__ import annotations

import argparse
import json

import numpy as np


def bound(q, x, d):
    """eps of the tensor filter (csrc/tc.cu), per pair, from FP64 row data."""
    u, g = 2.0 ** -24, 2.0 * (d + (-d) % 16) * 2.0 ** -24
    def bf(v):
        w = np.ascontiguousarray(v, np.float32).view(np.uint32).astype(np.uint64)
        w = (w + 0x7FFF + ((w >> 16) & 1)) >> 16 << 16
        return w.astype(np.uint32).view(np.float32).astype(np.float64)
    qn, xn = np.linalg.norm(q, axis=1), np.linalg.norm(x, axis=1)
    qe, xe = np.linalg.norm(q - bf(q), axis=1), np.linalg.norm(x - bf(x), axis=1)
    exact = (np.all((q == np.rint(q)) & (np.abs(q) <= 256), axis=1) & np.all((x == np.rint(x)) & (np.abs(x) <= 256),
                                                                             axis=1) & (d <= 128))
    eps = (2 * (qe * xn + qn * xe + qe * xe) + 4 * g * ((qn + qe) * (xn + xe) + qn * xn)
           + 4 * u * (qn ** 2 + xn ** 2 + 2 * qn * xn))
    return np.where(exact, 0.0, eps)


def stats(err, ref):
    a = np.abs(err)
    r = a / np.maximum(np.abs(ref), 1e-30)
    return {"max_abs": float(a.max()), "mean_abs": float(a.mean()), "max_rel": float(r.max()),
            "mean_rel": float(r.mean())}


def report(ctx, base, query, pairs=20000, seed=3):
    rng = np.random.default_rng(seed)
    qi = rng.integers(0, len(query), pairs)
    xi = rng.integers(0, len(base), pairs)
    q = np.ascontiguousarray(query[qi], np.float32)
    x = np.ascontiguousarray(base[xi], np.float32)
    q64, x64 = q.astype(np.float64), x.astype(np.float64)
    l2_64 = np.sum((q64 - x64) ** 2, axis=1)
    l2_32, ip_32 = ctx.pair_distances(q, x)
    _, qn32 = ctx.pair_distances(q, q)
    _, xn32 = ctx.pair_distances(x, x)
    f = np.float32
    key_32 = (qn32.astype(f) + xn32.astype(f)).astype(f) - (f(2) * ip_32).astype(f)
    # BF16 tensor tiles: diagonal of 128 x 128 Gram blocks
    ip_bf = np.empty(pairs, np.float32)
    for s in range(0, pairs, 128):
        g = ctx.bf16_gram(q[s:s + 128], x[s:s + 128])
        ip_bf[s:s + 128] = np.diagonal(g)
    key_bf = (qn32.astype(f) + xn32.astype(f)).astype(f) - (f(2) * ip_bf).astype(f)
    eps = bound(q64, x64, q.shape[1])
    gap = np.abs(key_bf.astype(np.float64) - key_32.astype(np.float64))
    return {
        "pairs": pairs, "d": int(q.shape[1]),
        "l2_fp32": stats(l2_32.astype(np.float64) - l2_64, l2_64),
        "key_fp32": stats(key_32.astype(np.float64) - l2_64, l2_64),
        "key_bf16": stats(key_bf.astype(np.float64) - l2_64, l2_64),
        "bound": {"holds": bool(np.all(gap <= eps)), "max_gap_over_eps": float(np.max(gap / np.maximum(eps, 1e-300)))
                  if np.any(eps > 0) else 0.0, "pairs_exact_path": int(np.sum(eps == 0)),
                  "max_gap": float(gap.max())},
    }


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=1_000_000)
    ap.add_argument("--nq", type=int, default=10_000)
    ap.add_argument("--pairs", type=int, default=20_000)
    a = ap.parse_args(argv)
    from . import pipeline
    from ._lib import Context
    ctx = Context(0)
    base, query = pipeline.mixture(a.n, 128, a.nq)
    out = {"mixture_1m_x128": report(ctx, base, query, a.pairs)}
    rng = np.random.default_rng(4)
    g = rng.normal(size=(50_000, 96)).astype(np.float32)   # non-integer rows exercise the rounding terms
    out["gaussian_50k_x96"] = report(ctx, g[:40_000], g[40_000:], a.pairs)
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
