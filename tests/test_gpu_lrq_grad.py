"""CUDA forward/backward of the LRQ radius-reconstruction objective
(anqi.lrq_torch): the forward against the NumPy trainer's own reconstruction
and nearest decode, the backward against a plain PyTorch FP64 gradient of the
same expression, central finite differences (FP64, step 1e-4), and a short
gradient fit started from the NumPy trainer's solution."""
import numpy as np
import pytest
import torch

from anqi import lrq_train

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def numpy_codes(residual, codebooks):
    """decode_nearest (tools/train_final_m8_u8.py:146-156) returning indices."""
    cs = codebooks.shape[1]
    idx = np.empty(residual.shape, np.int64)
    for k in range(residual.shape[1]):
        cen, v = codebooks[k], residual[:, k]
        ins = np.searchsorted(cen, v, side="left")
        hi = np.clip(ins, 0, cs - 1)
        lo = np.clip(ins - 1, 0, cs - 1)
        idx[:, k] = np.where(np.abs(cen[hi] - v) < np.abs(v - cen[lo]), hi, lo)
    return idx


@pytest.fixture(scope="module")
def problem():
    rng = np.random.default_rng(7)
    n, nk = 3000, 100
    # increasing cutoff curves with a low-rank structure, like AKNN key rows
    base = np.cumsum(rng.gamma(2.0, 1.0, size=(n, nk)), axis=1)
    T = base * rng.uniform(0.5, 2.0, size=(n, 1))
    mu, G, _ = lrq_train.fit_basis(T)
    resid = T - lrq_train.reconstruct(T, mu, G)
    B = np.stack([lrq_train.lloyd_1d(resid[:, k], 8) for k in range(nk)])
    return T, mu, G, B


def tt(x):
    return torch.tensor(np.asarray(x, np.float64), device=DEV)


def test_forward_matches_numpy_trainer(problem):
    from anqi import lrq_torch
    T, mu, G, B = problem
    loss, codes = lrq_torch.lrq_loss(tt(T), tt(mu), tt(G), tt(B))
    rec = lrq_train.reconstruct(T, mu, G)
    idx = numpy_codes(T - rec, B)
    assert np.array_equal(codes.cpu().numpy(), idx)
    decoded = B[np.arange(B.shape[0])[None, :], idx]
    ref = np.mean((rec + decoded - T) ** 2)
    assert abs(float(loss) - ref) <= 1e-12 * ref


def torch_reference_loss(T, mu, G, B, codes):
    c = (T - mu) @ G.T
    base = mu + c @ G
    dec = torch.gather(B, 1, codes.long().T).T
    return torch.mean((base + dec - T) ** 2)


def test_backward_matches_reference_gradient(problem):
    from anqi import lrq_torch
    T, mu, G, B = (tt(x) for x in problem)
    p = [x.clone().requires_grad_(True) for x in (mu, G, B)]
    loss, codes = lrq_torch.lrq_loss(T, *p)
    loss.backward()
    q = [x.clone().requires_grad_(True) for x in (mu, G, B)]
    ref = torch_reference_loss(T, *q, codes)
    ref.backward()
    assert abs(float(loss.detach()) - float(ref.detach())) <= 1e-12 * float(ref.detach())
    for a, b, name in zip(p, q, ("mu", "G", "B")):
        err = (a.grad - b.grad).abs().max() / b.grad.abs().max()
        assert float(err) < 1e-10, (name, float(err))


def test_finite_differences(problem):
    """Central differences in FP64 at step h = 1e-4 and h/2, combined by
    Richardson extrapolation ((4 D(h/2) - D(h)) / 3) so that the h^2 term of
    the quartic dependence on G cancels; codes of the unperturbed point held
    fixed (the objective the backward differentiates)."""
    from anqi import lrq_torch
    T, mu, G, B = (tt(x) for x in problem)
    p = [x.clone().requires_grad_(True) for x in (mu, G, B)]
    loss, codes = lrq_torch.lrq_loss(T, *p)
    loss.backward()
    rng = np.random.default_rng(3)
    h = 1e-4

    def central(which, flat, d, step):
        args = [x.detach() for x in p]
        args[which] = (flat + step * d).view_as(p[which])
        lp, _ = lrq_torch.lrq_loss(T, *args, codes)
        args[which] = (flat - step * d).view_as(p[which])
        lm, _ = lrq_torch.lrq_loss(T, *args, codes)
        return (float(lp) - float(lm)) / (2 * step)

    def richardson(which, flat, d):
        return (4 * central(which, flat, d, h / 2) - central(which, flat, d, h)) / 3

    for which in range(3):
        flat = p[which].detach().flatten()
        grad = p[which].grad.flatten()
        if which == 2:  # codebook entries that some code uses
            used = torch.unique(codes.long() + 256 * torch.arange(codes.shape[1], device=DEV)[None, :])
            picks = used[torch.randperm(len(used), device=DEV)[:12]].tolist()
        else:
            picks = rng.choice(flat.numel(), size=12, replace=False).tolist()
        for i in picks:
            e = torch.zeros_like(flat)
            e[i] = 1.0
            fd, g = richardson(which, flat, e), float(grad[i])
            assert abs(fd - g) <= 1e-6 * max(1.0, abs(g)), (which, i, fd, g)
        d = torch.randn_like(flat)
        fd, g = richardson(which, flat, d), float(torch.dot(grad, d))
        assert abs(fd - g) <= 1e-6 * max(1.0, abs(g)), (which, fd, g)


def test_fit_from_numpy_solution_does_not_degrade(problem):
    """Adam from the NumPy trainer's (mu, G, B): the loss never rises above the
    start by more than 1e-6 relative at the end, the codebook rows stay
    ascending, and the fitted codebook agrees with the NumPy one within the
    Adam step bound (steps x lr x (1 - beta1) / sqrt(1 - beta2) per entry;
    the ascending projection moves no entry further than the largest step)."""
    from anqi import lrq_torch
    T, mu, G, B = (tt(x) for x in problem)
    steps, lr = 60, 1e-3
    mu2, G2, B2, hist = lrq_torch.fit(T, mu, G, B, steps=steps, lr=lr)
    assert hist[-1] <= hist[0] * (1 + 1e-6), (hist[0], hist[-1])
    assert bool((B2[:, 1:] >= B2[:, :-1]).all())
    assert float((B2 - B).abs().max()) <= steps * lr * 0.1 / (0.001 ** 0.5) * 1.01
