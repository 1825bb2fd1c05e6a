"""The LRQ fit on the GPU (anqi.lrq_fit, anqi_lrq_fit_* kernels) against the
NumPy trainer (anqi.lrq_train, the reference's trainer restated): same rounds,
sums in other orders, so the tolerance is stated here.  What the verifier
uses: the thresholds the two fits materialise agree (relative 1e-6) for at
least 99% of the objects at k = 10, 50, 100 (99.6% measured on this sample).  The parameters: the mean to a
relative 1e-6, the basis directions to 1e-6, 97% of the codebook centres to
1e-5 of their column's range and every centre to 1e-3 (a value on a cell
boundary may fall on the other side of it, move a cell mean, and the Lloyd
passes of that column then drift apart a little: on this 12,000-row sample
about 1.3% of the centres, all within 3e-4).  At 1M x 100 the bench measures
a largest difference of 2e-8 of the range and identical thresholds."""
import numpy as np
import pytest

from anqi import lrq_fit, lrq_train
from anqi._lib import Context

pytestmark = pytest.mark.gpu


def cutoff_matrix(n, nk=100, seed=3):
    """Ascending rows shaped like AKNN cutoff keys: a per-row scale times a
    power law in the rank, plus noise, sorted."""
    rng = np.random.default_rng(seed)
    a = rng.gamma(2.0, 50.0, size=(n, 1))
    b = rng.uniform(0.2, 0.8, size=(n, 1))
    r = np.arange(1, nk + 1, dtype=np.float64)[None, :]
    x = a * r ** b + rng.normal(scale=2.0, size=(n, nk))
    return np.sort(x, axis=1).astype(np.float32)


@pytest.mark.parametrize("n,sample", [(30000, 12000), (5000, 5000)])
def test_gpu_fit_matches_numpy_fit(n, sample):
    keys = cutoff_matrix(n)
    mu_c, g_c, b_c = lrq_train.train(keys, n, train_sample=sample, log=lambda s: None)
    mu_g, g_g, b_g = lrq_fit.train_gpu(keys, n, train_sample=sample, log=lambda s: None)
    # the verifier both fits give: materialised thresholds per object
    with Context(0) as ctx:
        mats = []
        for mu, g, b in ((mu_c, g_c, b_c), (mu_g, g_g, b_g)):
            mu32, g32, b32 = (np.asarray(v, np.float32) for v in (mu, g, b))
            coeff, codes = ctx.lrq_encode(keys, mu32, g32, b32)
            mats.append([ctx.lrq_materialize(coeff, codes, mu32, g32, b32, k) for k in (10, 50, 100)])
    for tc, tg in zip(*mats):
        same = np.mean(np.isclose(tc, tg, rtol=1e-6, atol=1e-6))
        assert same >= 0.99, same
    rel = np.max(np.abs(mu_g - mu_c) / np.maximum(np.abs(mu_c), 1.0))
    assert rel < 1e-6, rel
    # basis rows: the same directions up to sign
    dots = np.abs(np.sum(g_g * g_c, axis=1))
    assert np.all(np.abs(dots - 1.0) < 1e-6), dots
    span = (b_c[:, -1] - b_c[:, 0])[:, None]
    err = np.abs(b_g - b_c) / span
    assert np.mean(err < 1e-5) >= 0.97 and err.max() < 1e-3, (np.mean(err < 1e-5), err.max())


def test_gpu_fit_rejects_non_finite_rows():
    keys = cutoff_matrix(2000)
    keys[17, 40] = np.nan
    with pytest.raises(RuntimeError, match="non-finite"):
        lrq_fit.train_gpu(keys, 2000, train_sample=2000, log=lambda s: None)
