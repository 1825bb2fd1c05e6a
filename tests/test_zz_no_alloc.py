"""The allocation-free query entry point (anqi_rknn_query_noalloc).

It serves callers that cannot allocate device memory (their device memory all
comes from a host framework's pool, or their budget is fixed up front), so
they hand in device arrays they already own and the library uses a fixed
static scratch array instead of cudaMalloc.  This checks, through the C ABI,
that two calls in a row return exactly what the allocating entry point
(anqi_rknn_query) returns on the same index and queries, and that an index
too large for the fixed scratch is rejected.  Cases: d = 32 and d = 128 (the
product's stride), and an index of 34 million objects (the small index held in
the first rows of larger arrays), where only three query slots fit in the
scratch and the blocks run three warps.  Collected last on purpose: it runs
after every other test, and it also passes on its own."""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as ol
from anqi import formats
from anqi._lib import ANQI_ERR_CAPACITY, ANQI_OK, Context, load_library

pytestmark = pytest.mark.gpu


class DeviceIndex(C.Structure):
    _fields_ = [
        ("n", C.c_uint64), ("d", C.c_uint32), ("degree", C.c_uint32), ("base", C.c_void_p),
        ("base_stride", C.c_uint32), ("lifted", C.c_void_p), ("lifted_stride", C.c_uint32), ("deg", C.c_void_p),
        ("links", C.c_void_p), ("tree_nodes", C.c_uint32), ("tree_left", C.c_void_p), ("tree_right", C.c_void_p),
        ("tree_offset", C.c_void_p), ("tree_hyperplane", C.c_void_p), ("tree_leaf_first", C.c_void_p),
        ("scale", C.c_double), ("mstar2", C.c_double), ("metric", C.c_uint32),
    ]


def small_index(n=5000, d=32, nq=400, seed=17):
    rng = np.random.default_rng(seed)
    centers = rng.normal(scale=3.0, size=(30, d))
    x = (centers[rng.integers(0, 30, size=n + nq)] + rng.normal(size=(n + nq, d))).astype(np.float32)
    base, query = x[:n], x[n:]
    nrm = ol.norms(base)
    d2 = nrm[:, None] + nrm[None, :] - 2.0 * (base.astype(np.float64) @ base.T)
    np.fill_diagonal(d2, np.inf)
    order = np.argsort(d2, axis=1)
    knn = order[:, :100].astype(np.uint32)
    radius = np.take_along_axis(d2, order[:, 99:100], 1)[:, 0].astype(np.float32)
    lifted, m2, sc = ol.lift(base, radius)
    ln = ol.norms(lifted)
    ids, vals = ol.warm_start(lifted, ln, knn, 100, 50)
    ids, vals, _ = ol.localjoin(lifted, ln, ids, vals)
    O, Od = ol.graph_select(lifted, ln, ids, vals)
    links, deg = ol.graph_commit(lifted, ln, O, Od)
    t = ol.rp_tree(lifted, 100)
    tree = formats.bfs_tree_to_postorder(t["left"], t["right"], t["offset"], t["hyperplane"], t["leaf_off"],
                                        t["leaf_cnt"], t["perm"], 100, d + 2)
    thr = np.take_along_axis(d2, order[:, 9:10], 1)[:, 0].astype(np.float32)
    return base, query, lifted, links, deg, tree, sc, m2, thr


def padded(torch, a, stride):
    a = np.ascontiguousarray(a, np.float32)
    out = np.zeros((a.shape[0], stride), np.float32)
    out[:, :a.shape[1]] = a
    return torch.from_numpy(out).cuda()


def bind(lib):
    lib.anqi_rknn_query_noalloc.argtypes = [C.POINTER(DeviceIndex), C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32,
                                            C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.anqi_rknn_query_noalloc.restype = C.c_int
    return lib


def device_rows(torch, a, stride, rows=None):
    """a (m x w) in the first m rows of a device array of `rows` x stride
    floats (rows beyond m are allocated but never written)."""
    a = np.ascontiguousarray(a, np.float32)
    rows = rows or a.shape[0]
    t = torch.empty((rows, stride), dtype=torch.float32, device="cuda")
    t[:a.shape[0]] = padded(torch, a, stride)
    return t


def device_u32(torch, a, rows=None):
    a = np.ascontiguousarray(a).astype(np.uint32)
    rows = rows or a.shape[0]
    t = torch.empty((rows,) + a.shape[1:], dtype=torch.int32, device="cuda")
    t[:a.shape[0]] = torch.from_numpy(a.view(np.int32))
    return t


def check_noalloc(torch, d, n_alloc=None, L=64):
    """Two calls in a row through the C ABI equal anqi_rknn_query's results.
    n_alloc: the object count the index arrays (and the call) declare; the
    index's own objects are the first rows."""
    base, query, lifted, links, deg, tree, sc, m2, thr = small_index(d=d)
    n = len(base)
    with Context(0) as ctx:
        ctx.index_load(base, lifted, deg, links, tree, sc, m2)
        ctx.set_thresholds(10, thr)
        ref = ctx.rknn_query(query, 10, L)
    lib = bind(load_library())
    bs = (d + 3) // 4 * 4
    ls = (d + 2 + 3) // 4 * 4
    rows = n_alloc or n
    t_base = device_rows(torch, base, bs, rows)
    t_lift = device_rows(torch, lifted, ls, rows)
    t_deg = device_u32(torch, deg, rows)
    t_links = device_u32(torch, links, rows)
    t_thr = device_rows(torch, thr[:, None], 1, rows)
    t_left = device_u32(torch, tree.left)
    t_right = device_u32(torch, tree.right)
    t_off = torch.from_numpy(tree.offset.copy()).cuda()
    t_hyp = padded(torch, tree.hyperplane, ls)
    t_leaf = device_u32(torch, tree.leaf_first())
    t_q = padded(torch, query, bs)
    ix = DeviceIndex(rows, d, links.shape[1], t_base.data_ptr(), bs, t_lift.data_ptr(), ls, t_deg.data_ptr(),
                     t_links.data_ptr(), tree.n_nodes, t_left.data_ptr(), t_right.data_ptr(), t_off.data_ptr(),
                     t_hyp.data_ptr(), t_leaf.data_ptr(), sc, m2)
    nq = len(query)
    max_pred = 512
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call in range(2):
        cnt = torch.zeros(nq, dtype=torch.int32, device="cuda")
        ids = torch.full((nq, max_pred), -1, dtype=torch.int32, device="cuda")
        nd = torch.zeros(nq, dtype=torch.int32, device="cuda")
        rc = lib.anqi_rknn_query_noalloc(C.byref(ix), t_q.data_ptr(), nq, t_thr.data_ptr(), L, max_pred,
                                         cnt.data_ptr(), ids.data_ptr(), nd.data_ptr(), stream)
        assert rc == ANQI_OK, rc
        torch.cuda.synchronize()
        cnt_h = cnt.cpu().numpy().astype(np.uint32)
        ids_h = ids.cpu().numpy().view(np.uint32)
        assert np.array_equal(cnt_h, np.diff(ref.pred_off)), call
        assert np.array_equal(nd.cpu().numpy().astype(np.uint32), ref.n_dist), call
        for q in range(nq):
            assert np.array_equal(ids_h[q, :cnt_h[q]], ref.pred(q)), (call, q)
        assert int(cnt_h.sum()) > 0


@pytest.mark.parametrize("d", [32, 128])
def test_noalloc_matches_allocating_query_twice(d):
    torch = pytest.importorskip("torch")
    check_noalloc(torch, d)


def test_noalloc_three_slots_at_34m_objects():
    """n = 34M: a slot is 1,062,500 bitmap words + 10,240, so three fit in the
    scratch and each block runs three warps (the largest n with four slots is
    about 33.5M)."""
    torch = pytest.importorskip("torch")
    n_big = 34_000_000
    slot_words = (n_big + 31) // 32 + 2048 + 8192
    assert ((16 << 20) // 4 - 64) // slot_words == 3
    check_noalloc(torch, 32, n_alloc=n_big)
    torch.cuda.empty_cache()


def test_noalloc_rejects_an_index_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    lib = bind(load_library())
    buf = torch.zeros(4096, dtype=torch.float32, device="cuda")
    p = buf.data_ptr()
    huge = DeviceIndex(1 << 30, 8, 48, p, 8, p, 16, p, p, 1, p, p, p, p, p, 1.0, 1.0)
    rc = lib.anqi_rknn_query_noalloc(C.byref(huge), p, 1, p, 16, 8, p, p, None, None)
    assert rc == ANQI_ERR_CAPACITY
