"""LRQ gradient fit against the NumPy trainer's fit, end to end.

    python -m anqi.lrq_eval [--n 1000000] [--nq 10000] [--steps 300] [--lr 1e-3]

On the 1M x 128 mixture: the GPU builds the AKNN source; the NumPy trainer
fits (mu, G, B) on 120,000 sampled cutoff rows (tools/train_final_m8_u8.py).
The CUDA objective (anqi.lrq_torch) then continues from that solution with
Adam.  Both codebooks get the trainer's endpoint widening to the residual
range of all rows (:159-174, 221-226).  All n rows are encoded with each, and
the query path runs with each verifier.  Printed as one JSON line: the
objective per variant, the codebook difference, and RkNN recall / precision
at k = 10, 50, 100 against the exact ground truth.
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np


def widen(keys, n, mu, G, B):
    from . import lrq_train
    lo, hi = lrq_train.residual_range(keys, n, mu.astype(np.float64), G.astype(np.float64))
    B = B.astype(np.float64).copy()
    B[:, 0] = np.minimum(B[:, 0], lo)
    B[:, -1] = np.maximum(B[:, -1], hi)
    return np.maximum.accumulate(B, axis=1)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=1_000_000)
    ap.add_argument("--nq", type=int, default=10_000)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--L", type=int, default=128)
    a = ap.parse_args(argv)
    import torch
    from . import lrq_torch, lrq_train, pipeline
    from ._lib import Context

    log = lambda *m: print("[lrq-eval]", *m, file=sys.stderr, flush=True)  # noqa: E731
    ctx = Context(0)
    base, query = pipeline.mixture(a.n, 128, a.nq)
    ix = pipeline.build_index(ctx, base, train_workers=16, log=log)
    keys = ix.aknn_keys
    _, ex = pipeline.exact_thresholds(ctx, base, 100)
    gt = {k: pipeline.rknn_ground_truth(ctx, base, query, ex[:, k - 1]) for k in (10, 50, 100)}

    rng = np.random.default_rng(lrq_train.SEED)
    ids = np.sort(rng.choice(a.n, size=min(lrq_train.TRAIN_ROWS, a.n), replace=False))
    dev = torch.device("cuda:0")
    T = torch.tensor(np.asarray(keys[ids], np.float64), device=dev)
    mu0, G0, B0 = (torch.tensor(np.asarray(x, np.float64), device=dev) for x in (ix.mu, ix.basis, ix.codebook))
    loss_np, _ = lrq_torch.lrq_loss(T, mu0, G0, B0)
    t0 = time.perf_counter()
    mu1, G1, B1, hist = lrq_torch.fit(T, mu0, G0, B0, steps=a.steps, lr=a.lr)
    torch.cuda.synchronize()
    fit_s = time.perf_counter() - t0
    variants = {
        "numpy": (ix.mu, ix.basis, ix.codebook),
        "cuda_fit": (mu1.cpu().numpy().astype(np.float32), G1.cpu().numpy().astype(np.float32),
                     widen(keys, a.n, mu1.cpu().numpy(), G1.cpu().numpy(), B1.cpu().numpy()).astype(np.float32)),
    }
    out = {"n": a.n, "train_rows": int(len(ids)), "steps": a.steps, "lr": a.lr, "fit_s": round(fit_s, 3),
           "objective": {"numpy": float(loss_np), "cuda_fit": hist[-1]},
           "codebook_max_abs_diff": float(np.abs(variants["cuda_fit"][2] - ix.codebook).max()),
           "codebook_rms_diff": float(np.sqrt(np.mean((variants["cuda_fit"][2] - ix.codebook) ** 2))),
           "recall": {}}
    for name, (mu, G, B) in variants.items():
        coeff, codes = ctx.lrq_encode(keys, mu, G, B)
        ctx.index_load(base, ix.lifted, ix.deg, ix.links, ix.tree, ix.scale, ix.mstar2)
        ctx.verifier_load(coeff, codes, mu, G, B)
        res = {}
        for k in (10, 50, 100):
            ctx.verifier_materialize(k)
            ctx.query_upload(query, k, a.L)
            ctx.query_run(keep_candidates=True)
            off, gids, _ = gt[k]
            e = ctx.query_evaluate(off, gids)
            res[k] = {"recall": round(e["recall"], 6), "precision": round(e["precision"], 6)}
        out["recall"][name] = res
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
