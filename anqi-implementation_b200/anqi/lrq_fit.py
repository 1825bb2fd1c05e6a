"""LRQ verifier fit on the GPU: the trainer's rounds (anqi.lrq_train, after
tools/train_final_m8_u8.py:81-258) with every pass over the rows in the
anqi_lrq_fit_* kernels (FP64); only the nk x nk eigen-decomposition and the
seeded row sample stay on the host.

Same inputs, outputs and round structure as lrq_train.train.  Sums run in
other orders than NumPy's (covariance, reconstruction), so basis and codebooks
agree with the NumPy fit to rounding, not bit for bit; the byte-identical
NumPy trainer stays the default of the command line (lrq_train.main).
PyTorch only holds the device memory and names the stream.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import lrq_train
from ._lib import AnqiError, load_library


def _ok(rc: int, what: str) -> None:
    if rc != 0:
        raise AnqiError(rc, f"{what} failed (status {rc})")


def train_gpu(keys, n: int, train_sample: int = lrq_train.TRAIN_ROWS, seed: int = lrq_train.SEED,
              recursive_iters: int = lrq_train.RECURSIVE_ITERS, lloyd_iters: int = lrq_train.LLOYD_ITERS,
              rank_m: int = lrq_train.RANK_M, code_size: int = lrq_train.CODE_SIZE, device: int = 0, log=print):
    """keys: n x nk cutoff matrix (array or memmap).  Returns (mu, basis,
    codebooks) as float64 arrays, like lrq_train.train."""
    import torch

    lib = load_library()
    if n < code_size:
        raise RuntimeError(f"at least {code_size} rows are required for u8 training, got {n}")
    dev = torch.device("cuda", device)
    st = torch.cuda.current_stream(dev).cuda_stream
    keys_h = np.ascontiguousarray(np.asarray(keys[:n]), np.float32)
    nk = keys_h.shape[1]
    K = torch.from_numpy(keys_h).to(dev)
    sample_n = min(train_sample, n)
    f64 = dict(dtype=torch.float64, device=dev)
    nblk = (sample_n + 1023) // 1024
    stat_scr = torch.empty(nblk * nk * nk, **f64)
    mean_d = torch.empty(nk, **f64)
    cov_d = torch.empty(nk * nk, **f64)
    status = torch.zeros(1, dtype=torch.int32, device=dev)

    def fit_basis(ids_d, sub_d):
        _ok(lib.anqi_lrq_fit_stats(K.data_ptr(), ids_d.data_ptr() if ids_d is not None else None, sample_n, nk,
                                   sub_d.data_ptr() if sub_d is not None else None, stat_scr.data_ptr(),
                                   stat_scr.numel(), mean_d.data_ptr(), cov_d.data_ptr(), st), "lrq_fit_stats")
        mean = mean_d.cpu().numpy().copy()
        cov = cov_d.cpu().numpy().reshape(nk, nk)
        if not (np.isfinite(mean).all() and np.isfinite(cov).all()):
            raise RuntimeError("threshold rows contain non-finite values")
        w, v = np.linalg.eigh(cov)
        order = np.argsort(w)[::-1]
        basis = np.ascontiguousarray(v[:, order[:rank_m]].T)
        explained = float(w[order[:rank_m]].sum() / max(w.sum(), 1e-30))
        return mean, basis, explained

    # the basis of the first sample_n rows (train_final_m8_u8.py:198-199)
    mean, basis, explained = fit_basis(None, None)
    rng = np.random.default_rng(seed)
    ids = np.sort(rng.choice(n, size=sample_n, replace=False)).astype(np.int32)
    ids_d = torch.from_numpy(ids).to(dev)
    res = torch.empty(nk * sample_n, **f64)
    dec = torch.empty(nk * sample_n, **f64)
    cb_d = torch.empty(nk * code_size, **f64)
    scr = torch.empty(int(lib.anqi_lrq_fit_codebooks_scratch(sample_n, nk)), **f64)
    part = torch.empty(1024, **f64)
    npart = C.c_uint32()
    mu_d = torch.empty(nk, **f64)
    g_d = torch.empty(rank_m * nk, **f64)
    codebooks = None
    for it in range(recursive_iters):
        mu_d.copy_(torch.from_numpy(mean))
        g_d.copy_(torch.from_numpy(basis.reshape(-1)))
        _ok(lib.anqi_lrq_fit_residual(K.data_ptr(), ids_d.data_ptr(), sample_n, nk, mu_d.data_ptr(), g_d.data_ptr(),
                                      rank_m, res.data_ptr(), status.data_ptr(), st), "lrq_fit_residual")
        _ok(lib.anqi_lrq_fit_codebooks(res.data_ptr(), sample_n, nk, code_size, lloyd_iters, scr.data_ptr(),
                                       scr.numel(), cb_d.data_ptr(), st), "lrq_fit_codebooks")
        _ok(lib.anqi_lrq_fit_decode(res.data_ptr(), sample_n, nk, cb_d.data_ptr(), code_size, dec.data_ptr(),
                                    part.data_ptr(), part.numel(), C.byref(npart), st), "lrq_fit_decode")
        if int(status.item()) != 0:
            raise RuntimeError("threshold residuals contain non-finite values")
        codebooks = cb_d.cpu().numpy().reshape(nk, code_size).copy()
        rmse = float(np.sqrt(part[:npart.value].sum().item() / (sample_n * nk)))
        log(f"[verifier-train] round={it + 1}/{recursive_iters} sample_rmse={rmse:.6g} explained={explained:.6f}")
        if it + 1 < recursive_iters:
            mean, basis, explained = fit_basis(ids_d, dec)
    # codebook endpoints widened to the residual range of all rows (:221-226)
    mu_d.copy_(torch.from_numpy(mean))
    g_d.copy_(torch.from_numpy(basis.reshape(-1)))
    lohi = torch.empty(2 * nk, **f64)
    _ok(lib.anqi_lrq_fit_range(K.data_ptr(), n, nk, mu_d.data_ptr(), g_d.data_ptr(), rank_m, lohi.data_ptr(),
                               status.data_ptr(), st), "lrq_fit_range")
    lh = lohi.cpu().numpy().reshape(nk, 2)
    if int(status.item()) != 0:
        raise RuntimeError("threshold residuals contain non-finite values")
    codebooks[:, 0] = np.minimum(codebooks[:, 0], lh[:, 0])
    codebooks[:, -1] = np.maximum(codebooks[:, -1], lh[:, 1])
    codebooks = np.maximum.accumulate(codebooks, axis=1)
    if not (np.isfinite(mean).all() and np.isfinite(basis).all() and np.isfinite(codebooks).all()):
        raise RuntimeError("trained verifier contains non-finite values")
    if np.any(np.diff(codebooks, axis=1) < 0):
        raise RuntimeError("trained codebook is not sorted")
    return mean, basis, codebooks
