"""CUDA forward/backward of the LRQ radius-reconstruction objective behind
``torch.autograd.Function``, and a gradient fit of (mu, G, B) that starts
from the NumPy trainer's solution.

The objective is the one the reference trainer's rounds minimise
(tools/train_final_m8_u8.py:90-157, 206-218): rank-M reconstruction
``mu + ((T - mu) G^T) G`` plus the nearest codebook entry of the residual per
rank column (``decode_nearest``, :146-156), squared error averaged over all
entries.  The codes are recomputed at every forward and held fixed in the
backward (they are piecewise constant in the parameters).  The kernels are
``anqi_lrq_objective_forward`` / ``_backward`` in libanqi.so (FP64); there is
no PyTorch fallback: a missing library or device raises.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib


def _p(t: torch.Tensor | None):
    return None if t is None else C.c_void_p(t.data_ptr())


def _stream(device) -> C.c_void_p:
    return C.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _check(rc: int, what: str) -> None:
    if rc != _lib.ANQI_OK:
        raise _lib.AnqiError(rc, f"{what} failed (status {rc})")


def _prep(t: torch.Tensor, name: str) -> torch.Tensor:
    if not t.is_cuda or t.dtype != torch.float64:
        raise TypeError(f"{name} must be a float64 CUDA tensor")
    return t.contiguous()


def objective_forward(T, mu, G, B, codes=None):
    """(sum r^2, r, c, a) with codes a from decode_nearest unless ``codes`` is given."""
    lib = _lib.load_library()
    T, mu, G, B = (_prep(x, n) for x, n in ((T, "T"), (mu, "mu"), (G, "G"), (B, "B")))
    n, nk = T.shape
    m, cs = G.shape[0], B.shape[1]
    r = torch.empty_like(T)
    c = torch.empty((n, m), dtype=torch.float64, device=T.device)
    a = torch.empty((n, nk), dtype=torch.uint8, device=T.device)
    loss = torch.empty(1, dtype=torch.float64, device=T.device)
    if codes is not None:
        codes = codes.to(device=T.device, dtype=torch.uint8).contiguous()
    _check(lib.anqi_lrq_objective_forward(_p(T), n, nk, m, _p(mu), _p(G), _p(B), cs, _p(codes), _p(r), _p(c),
                                          _p(a), _p(loss), _stream(T.device)), "LRQ objective forward")
    return loss[0], r, c, a


def objective_backward(T, mu, G, r, c, a, cs: int, scale: float):
    lib = _lib.load_library()
    n, nk = T.shape
    m = G.shape[0]
    g_mu = torch.empty_like(mu)
    g_G = torch.empty_like(G)
    g_B = torch.empty((nk, cs), dtype=torch.float64, device=T.device)
    _check(lib.anqi_lrq_objective_backward(_p(T), n, nk, m, _p(mu), _p(G), _p(r), _p(c), _p(a), cs, float(scale),
                                           _p(g_mu), _p(g_G), _p(g_B), _stream(T.device)), "LRQ objective backward")
    return g_mu, g_G, g_B


class LrqObjective(torch.autograd.Function):
    """mean over all entries of (mu + c G + B[k, a] - T)^2; gradients for mu, G, B."""

    @staticmethod
    def forward(ctx, T, mu, G, B, codes=None):
        T, mu, G, B = (_prep(x, n) for x, n in ((T, "T"), (mu, "mu"), (G, "G"), (B, "B")))
        total, r, c, a = objective_forward(T, mu, G, B, codes)
        ctx.save_for_backward(T, mu, G, r, c, a)
        ctx.cs = B.shape[1]
        ctx.mark_non_differentiable(a)
        return total / T.numel(), a

    @staticmethod
    def backward(ctx, g_loss, g_codes):
        T, mu, G, r, c, a = ctx.saved_tensors
        g_mu, g_G, g_B = objective_backward(T, mu, G, r, c, a, ctx.cs, 2.0 / T.numel())
        return None, g_mu * g_loss, g_G * g_loss, g_B * g_loss, None


def lrq_loss(T, mu, G, B, codes=None):
    """Mean squared reconstruction error and the codes it used."""
    return LrqObjective.apply(T, mu, G, B, codes)


def fit(T, mu, G, B, steps: int = 200, lr: float = 1e-3, lr_basis: float | None = None, log=None):
    """Adam on (mu, G, B) from a starting point (the NumPy trainer's output);
    codebook rows are kept ascending after every step, as the trainer keeps
    them (:224-226).  mu and B are in radius units, the basis rows have unit
    norm, so the basis gets its own (smaller, lr/100 by default) step.
    Returns the fitted tensors and the loss history."""
    mu = mu.detach().clone().requires_grad_(True)
    G = G.detach().clone().requires_grad_(True)
    B = B.detach().clone().requires_grad_(True)
    opt = torch.optim.Adam([{"params": [mu, B], "lr": lr},
                            {"params": [G], "lr": lr * 1e-2 if lr_basis is None else lr_basis}])
    hist = []
    for step in range(steps):
        opt.zero_grad(set_to_none=True)
        loss, _ = lrq_loss(T, mu, G, B)
        loss.backward()
        opt.step()
        with torch.no_grad():
            B.copy_(torch.cummax(B, dim=1).values)
        hist.append(float(loss.detach()))
        if log and (step % 50 == 0 or step == steps - 1):
            log(f"[lrq-fit] step {step} loss {hist[-1]:.6g}")
    with torch.no_grad():
        final, _ = lrq_loss(T, mu, G, B)
    hist.append(float(final))
    return mu.detach(), G.detach(), B.detach(), hist
