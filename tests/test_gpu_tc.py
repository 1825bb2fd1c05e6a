"""BF16 tensor-core tiles (tcgen05, csrc/tc.cu): the Gram tile primitive
against NumPy on bf16-rounded inputs, and the precision-form ground truth
against the FP32 path (bit-exact outputs)."""
import numpy as np
import pytest

from anqi._lib import Context

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    with Context(0) as c:
        yield c


def bf16(x):
    """Round-to-nearest-even to bfloat16, returned as float64."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16 << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


@pytest.mark.parametrize("na,nb,d", [(128, 128, 128), (300, 200, 128), (37, 260, 8), (129, 5, 32), (64, 64, 256)])
def test_gram_integer_inputs_exact(ctx, na, nb, d):
    rng = np.random.default_rng(na + nb + d)
    a = rng.integers(0, 256, size=(na, d)).astype(np.float32)
    b = rng.integers(0, 256, size=(nb, d)).astype(np.float32)
    got = ctx.bf16_gram(a, b)
    ref = a.astype(np.float64) @ b.astype(np.float64).T
    if d * 255 * 255 < 2 ** 24:
        assert np.array_equal(got.astype(np.float64), ref)
    else:
        assert np.max(np.abs(got - ref) / np.maximum(ref, 1)) < 1e-6


def test_gram_float_inputs_within_fp32_accumulation(ctx):
    rng = np.random.default_rng(5)
    a = rng.normal(size=(256, 96)).astype(np.float32)
    b = rng.normal(size=(192, 96)).astype(np.float32)
    got = ctx.bf16_gram(a, b).astype(np.float64)
    ref = bf16(a) @ bf16(b).T
    bound = 2 * 96 * 2.0 ** -24 * (np.abs(bf16(a)) @ np.abs(bf16(b)).T)
    assert np.all(np.abs(got - ref) <= bound + 1e-30)


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def mixture(n, d, seed, integer=True):
    rng = np.random.default_rng(seed)
    cen = rng.uniform(0, 128, size=(40, d))
    x = cen[rng.integers(0, 40, size=n)] + rng.normal(scale=20, size=(n, d))
    if integer:
        return np.clip(np.rint(x), 0, 255).astype(np.float32)
    return (x / 50.0).astype(np.float32)


@pytest.mark.parametrize("integer", [True, False])
def test_exact_topk_tc_equals_fp32(ctx, integer):
    from anqi import pipeline
    base = mixture(3000, 128 if integer else 40, 3 + integer, integer)
    base[17] = base[5]            # duplicates: exact ties at key 0 and elsewhere
    base[2999] = base[5]
    ids32, keys32 = pipeline.exact_thresholds(ctx, base, 100)
    ids, keys = ctx.exact_topk_tc(base, 100, hints=ids32[:, ::-1].copy())   # perfect hints, any order
    assert np.array_equal(ids, ids32) and np.array_equal(bits(keys), bits(keys32))
    ids2, keys2 = ctx.exact_topk_tc(base, 100)                               # hints from an AKNN build
    assert np.array_equal(ids2, ids32) and np.array_equal(bits(keys2), bits(keys32))


def test_exact_topk_tc_reference_sample(ctx, sample):
    ids, keys = ctx.exact_topk_tc(sample["base"], 100)
    assert np.array_equal(ids, sample["exact_ids"]) and np.array_equal(bits(keys), bits(sample["exact_keys"]))


@pytest.mark.parametrize("integer", [True, False])
def test_rknn_gt_tc_equals_fp32(ctx, integer):
    from anqi import pipeline
    d = 128 if integer else 72
    both = mixture(5300, d, 11, integer)       # queries from the same centres as the base
    base, query = both[:5000], both[5000:]
    _, ex = pipeline.exact_thresholds(ctx, base, 50)
    for k in (10, 50):
        off, ids, keys = pipeline.rknn_ground_truth(ctx, base, query, ex[:, k - 1])
        off2, ids2, keys2 = ctx.rknn_ground_truth_tc(base, query, ex[:, k - 1])
        assert np.array_equal(off, off2) and np.array_equal(ids, ids2) and np.array_equal(bits(keys), bits(keys2))
        assert off[-1] > 0


def test_rknn_gt_tc_reference_sample(ctx, sample):
    for ki, k in enumerate((10, 50, 100)):
        off, ids, keys = ctx.rknn_ground_truth_tc(sample["base"], sample["query"], sample["exact_keys"][:, k - 1])
        assert np.array_equal(off, sample[f"gt_off_{k}"]) and np.array_equal(ids, sample[f"gt_ids_{k}"])
        assert np.array_equal(bits(keys), bits(sample[f"gt_keys_{k}"]))


def unit_gaussian(n, d, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(n, d))
    return (x / np.linalg.norm(x, axis=1, keepdims=True)).astype(np.float32)


@pytest.mark.parametrize("d", [300, 960])
def test_wide_tensor_path_equals_fp32(ctx, d):
    """Rows above 256 dimensions: both operands stream through the K-chunk
    ring (64 elements per chunk, MMAs accumulating in TMEM).  Exact top-K,
    RkNN CSR and the AKNN build with the tensor-core init_knn equal the FP32
    path bit for bit (L2-normalised N(0,1) rows, the batching form's second
    shape, and an integer mixture)."""
    from anqi import pipeline
    both = unit_gaussian(3300, d, d) if d == 960 else mixture(3300, d, 7, True)  # queries from the same law
    base, query = both[:3000].copy(), both[3000:]
    base[11] = base[3]
    ids32, keys32 = pipeline.exact_thresholds(ctx, base, 100)
    ids, keys = ctx.exact_topk_tc(base, 100, hints=ids32)
    assert np.array_equal(ids, ids32) and np.array_equal(bits(keys), bits(keys32))
    ids2, keys2 = ctx.exact_topk_tc(base, 100)
    assert np.array_equal(ids2, ids32) and np.array_equal(bits(keys2), bits(keys32))
    for k in (10, 100):
        off, gid, gkey = pipeline.rknn_ground_truth(ctx, base, query, keys32[:, k - 1])
        off2, gid2, gkey2 = ctx.rknn_ground_truth_tc(base, query, keys32[:, k - 1])
        assert np.array_equal(off, off2) and np.array_equal(gid, gid2) and np.array_equal(bits(gkey), bits(gkey2))
        assert off[-1] > 0
    a_ids, a_keys, _ = pipeline.aknn_build(ctx, base, k=50, leaf=300, trees=8, ef=150, precision="bf16")
    f_ids, f_keys, _ = pipeline.aknn_build(ctx, base, k=50, leaf=300, trees=8, ef=150, precision="fp32")
    assert np.array_equal(a_ids, f_ids) and np.array_equal(bits(a_keys), bits(f_keys))


@pytest.mark.parametrize("data,d", [("normalized", 96), ("integers", 64), ("sparse_integers", 40), ("wide", 300)])
def test_ip_tensor_ground_truth_equals_fp32(ctx, data, d):
    """The ip metric on the tensor path (key -<a, b>: half the product terms of
    the l2 bound, FP32 recheck in the lane order): exact top-K, with the AKNN
    lists as hints and without, and the RkNN CSR equal the FP32 path bit for
    bit.  Sparse integer rows make exactly-zero products of either sign."""
    from anqi import pipeline
    rng = np.random.default_rng(d)
    n, nq, K = 3000, 300, 50
    if data == "normalized" or data == "wide":
        x = rng.normal(size=(n + nq, d))
        x /= np.linalg.norm(x, axis=1, keepdims=True)
    elif data == "integers":
        x = rng.integers(-8, 9, size=(n + nq, d))
    else:
        x = rng.integers(-2, 3, size=(n + nq, d)) * (rng.random((n + nq, d)) < 0.1)
    x = x.astype(np.float32)
    base, query = x[:n], x[n:]
    fi, fk = pipeline.exact_thresholds(ctx, base, K, metric="ip")
    hints, _, _ = pipeline.aknn_build(ctx, base, k=K, leaf=200, trees=6, ef=100, metric="ip")
    for h in (hints, None):
        ti, tk = pipeline.exact_thresholds(ctx, base, K, method="tc", hints=h, metric="ip")
        assert np.array_equal(ti, fi)
        assert np.array_equal(tk.view(np.uint32), fk.view(np.uint32))
    for k in (1, 10, K):
        fo, fid, fkey = pipeline.rknn_ground_truth(ctx, base, query, fk[:, k - 1], metric="ip")
        to, tid, tkey = pipeline.rknn_ground_truth(ctx, base, query, fk[:, k - 1], method="tc", metric="ip")
        assert np.array_equal(fo, to)
        assert np.array_equal(fid, tid)
        assert np.array_equal(fkey.view(np.uint32), tkey.view(np.uint32))
