#!/usr/bin/env python3
"""Rank-M radial basis + u8 residual codebook (LRQ) trainer.

Same command line, algorithm, outputs and NumPy operation order as the
reference trainer (tools/train_final_m8_u8.py:81-258), so the written basis and
codebook files are byte-identical for the same NumPy build:

* basis: top-M eigenvectors of the covariance of the first min(120000, n)
  cutoff rows (train_final_m8_u8.py:81-89, 198-199);
* a seeded sorted sample of rows (:201-203);
* three rounds of {rank-M reconstruction, 256-centre 1-D Lloyd per rank
  column from quantile initial centres with prefix-sum updates and a monotone
  repair, nearest decode, basis refit on rows - decoded} (:97-157, 206-218);
* codebook endpoints widened to the residual range of all rows, then made
  monotone (:159-174, 221-226).

The CUDA forward/backward of the same objective lives in anqi.lrq_torch.
"""
from __future__ import annotations

import argparse
import os
import struct
import sys
import time
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

import numpy as np

RANK_M = 8
K_MAX = 100
BITS = 8
CODE_SIZE = 1 << BITS
TRAIN_ROWS = 120_000
RECURSIVE_ITERS = 3
LLOYD_ITERS = 8
SEED = 10
CHUNK = 65_536


def fit_basis(rows: np.ndarray, rank_m: int = RANK_M):
    mean = rows.mean(axis=0)
    centered = rows - mean
    cov = centered.T @ centered / max(1, rows.shape[0])
    w, v = np.linalg.eigh(cov)
    order = np.argsort(w)[::-1]
    basis = np.ascontiguousarray(v[:, order[:rank_m]].T)
    explained = float(w[order[:rank_m]].sum() / max(w.sum(), 1e-30))
    return mean, basis, explained


def reconstruct(rows: np.ndarray, mean: np.ndarray, basis: np.ndarray) -> np.ndarray:
    return mean + ((rows - mean) @ basis.T) @ basis


def lloyd_1d(values: np.ndarray, iterations: int, code_size: int = CODE_SIZE) -> np.ndarray:
    """1-D k-means on sorted values; prefix sums give every cell mean in O(k)."""
    s = np.sort(np.asarray(values, dtype=np.float64))
    if not np.isfinite(s).all():
        raise RuntimeError("threshold residuals contain non-finite values")
    if s[0] == s[-1]:
        return np.full(code_size, s[0], dtype=np.float64)
    centers = np.quantile(s, (np.arange(code_size, dtype=np.float64) + 0.5) / code_size).astype(np.float64)
    prefix = np.concatenate(([0.0], np.cumsum(s)))
    for _ in range(iterations):
        cuts = np.searchsorted(s, (centers[:-1] + centers[1:]) * 0.5, side="right")
        lo = np.concatenate(([0], cuts))
        hi = np.concatenate((cuts, [s.size]))
        cnt = hi - lo
        upd = centers.copy()
        live = cnt > 0
        upd[live] = (prefix[hi] - prefix[lo])[live] / cnt[live]
        upd = np.maximum.accumulate(upd)
        done = np.max(np.abs(upd - centers)) < 1e-12
        centers = upd
        if done:
            break
    return centers


def train_codebooks(residual: np.ndarray, iterations: int, workers: int) -> np.ndarray:
    nk = residual.shape[1]
    out = np.empty((nk, CODE_SIZE), dtype=np.float64)
    if workers <= 1:
        for c in range(nk):
            out[c] = lloyd_1d(residual[:, c], iterations)
    else:
        with ThreadPoolExecutor(max_workers=min(workers, nk), thread_name_prefix="lrq") as ex:
            for c, cb in zip(range(nk), ex.map(lambda col: lloyd_1d(residual[:, col], iterations), range(nk))):
                out[c] = cb
    return out


def decode_nearest(residual: np.ndarray, codebooks: np.ndarray) -> np.ndarray:
    out = np.empty_like(residual, dtype=np.float64)
    for c in range(residual.shape[1]):
        cb = codebooks[c]
        v = residual[:, c]
        ins = np.searchsorted(cb, v, side="left")
        hi = np.clip(ins, 0, CODE_SIZE - 1)
        lo = np.clip(ins - 1, 0, CODE_SIZE - 1)
        out[:, c] = np.where(np.abs(cb[hi] - v) < np.abs(v - cb[lo]), cb[hi], cb[lo])
    return out


def residual_range(keys, n: int, mean, basis, chunk: int = CHUNK):
    lo = np.full(mean.shape[0], np.inf)
    hi = np.full(mean.shape[0], -np.inf)
    for s in range(0, n, chunk):
        block = np.asarray(keys[s:s + chunk], dtype=np.float64)
        r = block - reconstruct(block, mean, basis)
        lo = np.minimum(lo, r.min(axis=0))
        hi = np.maximum(hi, r.max(axis=0))
    return lo, hi


def train(keys, n: int, train_sample: int = TRAIN_ROWS, seed: int = SEED, recursive_iters: int = RECURSIVE_ITERS,
          lloyd_iters: int = LLOYD_ITERS, workers: int = 1, chunk: int = CHUNK, log=print):
    """keys: n x 100 cutoff matrix (array or memmap).  Returns (mu, basis, codebooks) as float32."""
    if n < CODE_SIZE:
        raise RuntimeError(f"at least {CODE_SIZE} rows are required for u8 training, got {n}")
    sample_n = min(train_sample, n)
    mean, basis, explained = fit_basis(np.asarray(keys[:sample_n], dtype=np.float64))
    rng = np.random.default_rng(seed)
    ids = np.sort(rng.choice(n, size=sample_n, replace=False))
    rows = np.asarray(keys[ids], dtype=np.float64)
    codebooks = None
    for it in range(recursive_iters):
        rec = reconstruct(rows, mean, basis)
        res = rows - rec
        codebooks = train_codebooks(res, lloyd_iters, workers)
        dec = decode_nearest(res, codebooks)
        rmse = float(np.sqrt(np.mean((rec + dec - rows) ** 2)))
        log(f"[verifier-train] round={it + 1}/{recursive_iters} sample_rmse={rmse:.6g} explained={explained:.6f}")
        if it + 1 < recursive_iters:
            mean, basis, explained = fit_basis(rows - dec)
    lo, hi = residual_range(keys, n, mean, basis, chunk)
    codebooks[:, 0] = np.minimum(codebooks[:, 0], lo)
    codebooks[:, -1] = np.maximum(codebooks[:, -1], hi)
    codebooks = np.maximum.accumulate(codebooks, axis=1)
    if not (np.isfinite(mean).all() and np.isfinite(basis).all() and np.isfinite(codebooks).all()):
        raise RuntimeError("trained verifier contains non-finite values")
    if np.any(np.diff(codebooks, axis=1) < 0):
        raise RuntimeError("trained codebook is not sorted")
    return mean, basis, codebooks


def write_outputs(pfx: str, mean, basis, codebooks) -> tuple[Path, Path]:
    bp = Path(f"{pfx}_radbasis_M{RANK_M}.bin")
    cp = Path(f"{pfx}_learned_rq_codebook_M{RANK_M}_u{BITS}.bin")
    with bp.open("wb") as f:
        f.write(struct.pack("<ii", K_MAX, RANK_M))
        f.write(np.asarray(mean, dtype="<f4").tobytes(order="C"))
        f.write(np.asarray(basis, dtype="<f4").tobytes(order="C"))
    with cp.open("wb") as f:
        f.write(b"ANQIRQ1\0")
        f.write(struct.pack("<iiii", K_MAX, RANK_M, BITS, CODE_SIZE))
        f.write(np.asarray(codebooks, dtype="<f4").tobytes(order="C"))
    if bp.stat().st_size != 8 + (K_MAX + RANK_M * K_MAX) * 4:
        raise RuntimeError(f"bad basis output size: {bp}")
    if cp.stat().st_size != 8 + 16 + K_MAX * CODE_SIZE * 4:
        raise RuntimeError(f"bad codebook output size: {cp}")
    return bp, cp


def main(argv=None) -> int:
    started = time.perf_counter()
    ap = argparse.ArgumentParser(description="Train the recursive M8+u8 LRQ verifier from the AKNN cutoff matrix.")
    ap.add_argument("--pfx", required=True, type=Path)
    ap.add_argument("--threshold-source", type=Path)
    ap.add_argument("--train-sample", type=int, default=TRAIN_ROWS)
    ap.add_argument("--seed", type=int, default=SEED)
    ap.add_argument("--recursive-iters", type=int, default=RECURSIVE_ITERS)
    ap.add_argument("--lloyd-iters", type=int, default=LLOYD_ITERS)
    ap.add_argument("--chunk", type=int, default=CHUNK)
    ap.add_argument("--codebook-workers", type=int,
                    default=int(os.environ.get("ANQI_CODEBOOK_WORKERS", os.environ.get("OMP_NUM_THREADS", "1"))))
    ap.add_argument("--device", choices=("cpu", "gpu"), default="cpu",
                    help="cpu: the NumPy fit (byte-identical files); gpu: anqi.lrq_fit's kernels (the same rounds, "
                         "equal to rounding)")
    a = ap.parse_args(argv)
    for name in ("train_sample", "recursive_iters", "lloyd_iters", "chunk", "codebook_workers"):
        if getattr(a, name) < 1:
            ap.error(f"--{name.replace('_', '-')} must be positive")
    from . import formats
    src = a.threshold_source or Path(f"{a.pfx}_baseknn_aknn.rec")
    n, _ = formats.fbin_shape(f"{a.pfx}_base.bin")
    if n == 0:
        raise RuntimeError("invalid base header")
    _, keys = formats.read_rec(src, n, K_MAX, mmap=True)
    if a.device == "gpu":
        from . import lrq_fit
        mean, basis, cb = lrq_fit.train_gpu(keys, n, a.train_sample, a.seed, a.recursive_iters, a.lloyd_iters,
                                            log=lambda s: print(s, flush=True))
    else:
        mean, basis, cb = train(keys, n, a.train_sample, a.seed, a.recursive_iters, a.lloyd_iters,
                                a.codebook_workers, a.chunk, log=lambda s: print(s, flush=True))
    bp, cp = write_outputs(str(a.pfx), mean, basis, cb)
    elapsed = time.perf_counter() - started
    Path(f"{a.pfx}_verifier_train_time.meta").write_text(
        "ANQI_VERIFIER_TRAIN_V1\n" f"seconds {elapsed:.17g}\n" f"n {n}\n" f"k {K_MAX}\n" f"rank_m {RANK_M}\n"
        f"bits {BITS}\n", encoding="utf-8")
    print(f"[verifier-train] n={n} sample={min(a.train_sample, n)} seed={a.seed} rank_m={RANK_M} bits={BITS} "
          f"rounds={a.recursive_iters} source={src} basis={bp} codebook={cp} VERIFIER_TRAIN_TIME={elapsed:.6f}s",
          flush=True)
    return 0


if __name__ == "__main__":
    sys.path.insert(0, str(Path(__file__).resolve().parent.parent))
    raise SystemExit(main())
