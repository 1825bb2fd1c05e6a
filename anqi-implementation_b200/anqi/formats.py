"""Prefix-file formats of the reference, read and written byte-for-byte.

Each reader/writer cites the reference code that defines the layout:

* fbin base/query: ``[u32 n][u32 d][f32 n*d]`` (include/utils.h:129-152,
  src/rknn_query.cpp:23-53)
* ``_baseknn_aknn.rec``: ``n*K x {u32 id, f32 key}`` (tools/build_aknn_source.cpp:119-137)
* ``_radbasis_M8.bin``: ``[i32 K][i32 M][f32 mu(K)][f32 G(M*K)]`` (tools/train_final_m8_u8.py:176-180)
* ``_learned_rq_codebook_M8_u8.bin``: ``"ANQIRQ1\\0"[i32 K, M, bits, code_size][f32 K*code_size]``
  (tools/train_final_m8_u8.py:183-187, src/rknn_query.cpp:407-454)
* ``_lifted.meta``: text ``M*^2 d k metric scale`` (src/rknn_query.cpp:1602-1616)
* RkNN CSR: ``[u32 nq][u32 off(nq+1)][u32 ids][f32 keys]`` (tools/dataset_gt.cpp:302-313)
* exact thresholds: ``[u32 n][u32 K][u32 ids n*K][f32 keys n*K]`` (tools/dataset_gt.cpp:249-253)
* verifier artifact ``"ANQIVF2\\0"`` (src/rknn_query.cpp:755-838)
* graph cache: ``[size_t n, dim, M][f32 ctime]{u32 deg, deg*u32}`` + RP tree
  (include/index.h:1810-1875)
* timing sidecars ``ANQI_AKNN_BUILD_V1`` / ``ANQI_VERIFIER_TRAIN_V1`` /
  ``ANQI_THRESHOLD_BUILD_V1`` (tools/build_aknn_source.cpp:141-155,
  tools/train_final_m8_u8.py:247-255, tools/dataset_gt.cpp:116-135)
"""
from __future__ import annotations

import os
import struct
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

EMPTY = 0xFFFFFFFF
REC_DTYPE = np.dtype([("id", "<u4"), ("key", "<f4")])


class FormatError(ValueError):
    """A prefix file is missing, truncated or has an inconsistent header."""


def _publish(path: Path, data: bytes) -> None:
    """Write via ``<path>.part`` + rename, as the reference publishes outputs."""
    tmp = Path(str(path) + ".part")
    tmp.write_bytes(data)
    os.replace(tmp, path)


# ----------------------------------------------------------------- fbin


def read_fbin(path, mmap: bool = False) -> np.ndarray:
    path = Path(path)
    try:
        size = path.stat().st_size
    except OSError as e:
        raise FormatError(f"cannot open fbin: {path}") from e
    with path.open("rb") as f:
        hdr = f.read(8)
    if len(hdr) != 8:
        raise FormatError(f"invalid fbin header: {path}")
    n, d = struct.unpack("<II", hdr)
    if n == 0 or d == 0 or size != 8 + 4 * n * d:
        raise FormatError(f"invalid fbin size: {path}")
    if mmap:
        return np.memmap(path, dtype="<f4", mode="r", offset=8, shape=(n, d))
    return np.fromfile(path, dtype="<f4", offset=8).reshape(n, d)


def write_fbin(path, x: np.ndarray) -> None:
    x = np.ascontiguousarray(x, dtype="<f4")
    if x.ndim != 2:
        raise ValueError("fbin wants a 2-D array")
    _publish(Path(path), struct.pack("<II", x.shape[0], x.shape[1]) + x.tobytes())


def fbin_shape(path) -> tuple[int, int]:
    with Path(path).open("rb") as f:
        hdr = f.read(8)
    if len(hdr) != 8:
        raise FormatError(f"invalid fbin header: {path}")
    return struct.unpack("<II", hdr)


# ------------------------------------------------------------------ .rec


def read_rec(path, n: int, k: int = 100, mmap: bool = False):
    path = Path(path)
    if not path.exists() or path.stat().st_size != n * k * 8:
        raise FormatError(f"bad AKNN record size for {path}")
    if mmap:
        rec = np.memmap(path, dtype=REC_DTYPE, mode="r", shape=(n, k))
    else:
        rec = np.fromfile(path, dtype=REC_DTYPE).reshape(n, k)
    return rec["id"], rec["key"]


def write_rec(path, ids: np.ndarray, keys: np.ndarray) -> None:
    rec = np.empty(ids.shape, dtype=REC_DTYPE)
    rec["id"] = ids
    rec["key"] = keys
    _publish(Path(path), rec.tobytes())


# ---------------------------------------------------------- basis / codebook


def read_basis(path, nk: int = 100, rankm: int = 8):
    raw = Path(path).read_bytes()
    if len(raw) < 8:
        raise FormatError(f"missing or invalid rank-M basis {path}")
    kb, mb = struct.unpack("<ii", raw[:8])
    if kb != nk or mb != rankm or len(raw) != 8 + 4 * (kb + mb * kb):
        raise FormatError(f"invalid rank-M basis {path} (K={kb} M={mb})")
    mu = np.frombuffer(raw, "<f4", kb, 8).copy()
    g = np.frombuffer(raw, "<f4", mb * kb, 8 + 4 * kb).reshape(mb, kb).copy()
    return mu, g


def write_basis(path, mu: np.ndarray, basis: np.ndarray) -> None:
    rankm, nk = basis.shape
    data = struct.pack("<ii", nk, rankm) + np.asarray(mu, "<f4").tobytes() + np.asarray(basis, "<f4").tobytes()
    Path(path).write_bytes(data)


CODEBOOK_MAGIC = b"ANQIRQ1\0"


def read_codebook(path, nk: int = 100, rankm: int = 8, bits: int = 8) -> np.ndarray:
    raw = Path(path).read_bytes()
    if len(raw) < 24 or raw[:8] != CODEBOOK_MAGIC:
        raise FormatError(f"bad learned RQ codebook magic {path}")
    k, m, b, cs = struct.unpack("<iiii", raw[8:24])
    if k != nk or m != rankm or b != bits or cs <= 0:
        raise FormatError(f"bad learned RQ codebook header {path}")
    if len(raw) != 24 + 4 * k * cs:
        raise FormatError(f"truncated or oversized learned RQ codebook {path}")
    cb = np.frombuffer(raw, "<f4", k * cs, 24).reshape(k, cs).copy()
    if np.any(np.diff(cb, axis=1) < 0):
        raise FormatError(f"LRQ codebook row is not sorted: {path}")
    return cb


def write_codebook(path, codebook: np.ndarray, rankm: int = 8, bits: int = 8) -> None:
    nk, cs = codebook.shape
    data = CODEBOOK_MAGIC + struct.pack("<iiii", nk, rankm, bits, cs) + np.asarray(codebook, "<f4").tobytes()
    Path(path).write_bytes(data)


# ---------------------------------------------------------------- meta


@dataclass
class LiftedMeta:
    mstar2: float
    d: int
    k: int
    metric: str
    scale: float


def read_lifted_meta(path) -> LiftedMeta:
    try:
        parts = Path(path).read_text().split()
        meta = LiftedMeta(float(parts[0]), int(parts[1]), int(parts[2]), parts[3], float(parts[4]))
    except (OSError, IndexError, ValueError) as e:
        raise FormatError(f"invalid or missing lift metadata: {path}") from e
    if not np.isfinite(meta.mstar2) or meta.mstar2 < 0 or meta.d == 0 or meta.k == 0 or \
            meta.metric not in ("l2", "ip") or not np.isfinite(meta.scale) or meta.scale <= 0:
        raise FormatError(f"invalid or missing lift metadata: {path}")
    return meta


def write_graph_meta(path, mstar2: float, scale: float) -> None:
    """``_anqi_meta_graph_<h>.txt``: ``%.17g %.17g`` (src/rknn_query.cpp:2244)."""
    Path(path).write_text(f"{mstar2:.17g} {scale:.17g}\n")


def read_graph_meta(path) -> tuple[float, float]:
    a, b = Path(path).read_text().split()[:2]
    return float(a), float(b)


# ------------------------------------------------------------- RkNN CSR


def read_rknn_csr(path, n_base: int | None = None):
    raw = Path(path).read_bytes()
    if len(raw) < 4:
        raise FormatError(f"invalid reverse-kNN GT header: {path}")
    nq = struct.unpack("<I", raw[:4])[0]
    need = 4 + 4 * (nq + 1)
    if len(raw) < need:
        raise FormatError(f"invalid reverse-kNN GT offsets: {path}")
    off = np.frombuffer(raw, "<u4", nq + 1, 4).copy()
    if off[0] != 0 or np.any(np.diff(off.astype(np.int64)) < 0):
        raise FormatError(f"invalid reverse-kNN GT offsets: {path}")
    tot = int(off[-1])
    if len(raw) != need + 8 * tot:
        raise FormatError(f"invalid reverse-kNN GT size: {path}")
    ids = np.frombuffer(raw, "<u4", tot, need).copy()
    keys = np.frombuffer(raw, "<f4", tot, need + 4 * tot).copy()
    if n_base is not None and tot and int(ids.max()) >= n_base:
        raise FormatError(f"invalid reverse-kNN GT ids: {path}")
    return off, ids, keys


def write_rknn_csr(path, off: np.ndarray, ids: np.ndarray, keys: np.ndarray) -> None:
    nq = len(off) - 1
    data = struct.pack("<I", nq) + np.asarray(off, "<u4").tobytes() + np.asarray(ids, "<u4").tobytes() + \
        np.asarray(keys, "<f4").tobytes()
    Path(path).write_bytes(data)


def read_knn_table(path):
    raw = Path(path).read_bytes()
    n, k = struct.unpack("<II", raw[:8])
    if len(raw) != 8 + 8 * n * k:
        raise FormatError(f"invalid threshold-table size: {path}")
    ids = np.frombuffer(raw, "<u4", n * k, 8).reshape(n, k).copy()
    keys = np.frombuffer(raw, "<f4", n * k, 8 + 4 * n * k).reshape(n, k).copy()
    return ids, keys


def write_knn_table(path, ids: np.ndarray, keys: np.ndarray) -> None:
    n, k = ids.shape
    Path(path).write_bytes(struct.pack("<II", n, k) + np.asarray(ids, "<u4").tobytes() +
                           np.asarray(keys, "<f4").tobytes())


# ------------------------------------------------------------- verifier

VERIFIER_MAGIC = b"ANQIVF2\0"


PACKED_BITS = (2, 4, 8, 16)
POLICY_CODE = {"nearest": 0, "floor": 1, "ceil": 2}


def packed_code_bytes(count: int, bits: int) -> int:
    """include/packed_code_array.h:14-18."""
    return (count * bits + 7) // 8 if bits in PACKED_BITS else 0


def write_verifier(path, coeff: np.ndarray, codes: np.ndarray | None = None, bits: int = 8, policy: str = "floor",
                   residual: np.ndarray | None = None, nk: int | None = None) -> None:
    """``"ANQIVF2\\0"[u64 n][u32 nk, rankm, bits, code_size, policy]`` + coeff +
    packed codes + float residuals (src/rknn_query.cpp:755-789).  bits 0: no
    codes; 2/4/8/16: codes as packed bytes (or an n x nk array for u8); 32:
    residual n x nk.  code_size is 2^bits for packed codes, else 0."""
    n, rankm = coeff.shape
    if nk is None:
        nk = codes.shape[1] if codes is not None and codes.ndim == 2 else residual.shape[1]
    cs = 1 << bits if bits in PACKED_BITS else 0
    body = np.asarray(coeff, "<f4").tobytes()
    if bits in PACKED_BITS:
        cb = np.asarray(codes, np.uint8).tobytes()
        if len(cb) != packed_code_bytes(n * nk, bits):
            raise FormatError("packed code size does not match n x nk x bits")
        body += cb
    if bits == 32:
        body += np.asarray(residual, "<f4").tobytes()
    hdr = VERIFIER_MAGIC + struct.pack("<QIIIII", n, nk, rankm, bits, cs, POLICY_CODE.get(policy, 0))
    tmp = Path(str(path) + ".tmp")
    tmp.write_bytes(hdr + body)
    os.replace(tmp, path)


def read_verifier_any(path, n: int, nk: int = 100, rankm: int = 8, bits: int = 8, policy: str = "floor"):
    """Any ANQIVF2 form (CompactLrqVerifier::load, src/rknn_query.cpp:791-838):
    returns coeff (n x rankm), packed code bytes or None, residual (n x nk) or None."""
    raw = Path(path).read_bytes()
    if len(raw) < 36 or raw[:8] != VERIFIER_MAGIC:
        raise FormatError(f"LRQ verifier artifact header mismatch {path}")
    n64, nk32, m32, b32, cs32, pol = struct.unpack("<QIIIII", raw[8:36])
    cs = 1 << bits if bits in PACKED_BITS else 0
    if (n64 != n or nk32 != nk or m32 != rankm or b32 != bits or cs32 != cs
            or pol != POLICY_CODE.get(policy, 0)):
        raise FormatError(f"LRQ verifier artifact header mismatch {path}")
    cbytes = packed_code_bytes(n * nk, bits)
    rbytes = 4 * n * nk if bits == 32 else 0
    if len(raw) != 36 + 4 * n * rankm + cbytes + rbytes:
        raise FormatError(f"truncated or oversized LRQ verifier artifact {path}")
    coeff = np.frombuffer(raw, "<f4", n * rankm, 36).reshape(n, rankm).copy()
    at = 36 + 4 * n * rankm
    codes = np.frombuffer(raw, np.uint8, cbytes, at).copy() if cbytes else None
    resid = np.frombuffer(raw, "<f4", n * nk, at + cbytes).reshape(n, nk).copy() if rbytes else None
    return coeff, codes, resid


ANALYTIC_MAGIC = b"ANQIPW1\0"


@dataclass
class AnalyticModel:
    """``_analytic_rankm_M{M}.bin``: ``"ANQIPW1\\0"[u64 n][u32 train_kmax, rankm,
    fit_kmin, flags][f64 b0][f32 n x rankm]`` (src/rknn_query.cpp:528-573)."""

    train_kmax: int
    rankm: int
    fit_kmin: int
    flags: int
    b0: float
    coeff: np.ndarray


def read_analytic(path, n: int, rankm: int) -> AnalyticModel:
    raw = Path(path).read_bytes()
    if len(raw) < 40 or raw[:8] != ANALYTIC_MAGIC:
        raise FormatError(f"analytic Rank-M header mismatch {path}")
    n64, tk, m, fk, flags = struct.unpack("<QIIII", raw[8:32])
    (b0,) = struct.unpack("<d", raw[32:40])
    if (n64 != n or m != rankm or tk < 1 or fk < 1 or fk > tk or flags not in (3, 7) or not np.isfinite(b0)):
        raise FormatError(f"analytic Rank-M header mismatch {path}")
    if len(raw) != 40 + 4 * n * rankm:
        raise FormatError(f"truncated or oversized analytic Rank-M model {path}")
    return AnalyticModel(tk, m, fk, flags, b0, np.frombuffer(raw, "<f4", n * m, 40).reshape(n, m).copy())


def write_analytic(path, model: AnalyticModel) -> None:
    n, m = model.coeff.shape
    Path(path).write_bytes(ANALYTIC_MAGIC + struct.pack("<QIIII", n, model.train_kmax, m, model.fit_kmin, model.flags)
                           + struct.pack("<d", model.b0) + np.asarray(model.coeff, "<f4").tobytes())


def read_verifier(path, n: int, nk: int = 100, rankm: int = 8, bits: int = 8):
    raw = Path(path).read_bytes()
    if len(raw) < 36 or raw[:8] != VERIFIER_MAGIC:
        raise FormatError(f"LRQ verifier artifact header mismatch {path}")
    n64, nk32, m32, b32, cs32, pol = struct.unpack("<QIIIII", raw[8:36])
    if n64 != n or nk32 != nk or m32 != rankm or b32 != bits or cs32 != (1 << bits) or pol != 1:
        raise FormatError(f"LRQ verifier artifact header mismatch {path}")
    need = 36 + 4 * n * rankm + n * nk
    if len(raw) != need:
        raise FormatError(f"truncated or oversized LRQ verifier artifact {path}")
    coeff = np.frombuffer(raw, "<f4", n * rankm, 36).reshape(n, rankm).copy()
    codes = np.frombuffer(raw, np.uint8, n * nk, 36 + 4 * n * rankm).reshape(n, nk).copy()
    return coeff, codes


# ---------------------------------------------------------------- graph


@dataclass
class RPTree:
    """An RP tree in the reference's persisted post-order (root last).

    ``left``/``right`` hold child node numbers, ``EMPTY`` on leaves; leaves keep
    their full member list (``indices``), ``indices[0]`` is the query entry."""

    leaf_size: int
    left: np.ndarray
    right: np.ndarray
    offset: np.ndarray
    hyperplane: np.ndarray          # n_nodes x dim (zero rows on leaves)
    leaf_off: np.ndarray            # n_nodes + 1 into ``indices``
    indices: np.ndarray
    dim: int = 0

    @property
    def n_nodes(self) -> int:
        return len(self.left)

    @property
    def n_leaves(self) -> int:
        return int(np.sum(self.left == EMPTY))

    def leaf_first(self) -> np.ndarray:
        cnt = np.diff(self.leaf_off)
        first = np.full(self.n_nodes, EMPTY, np.uint32)
        has = cnt > 0
        first[has] = self.indices[self.leaf_off[:-1][has]]
        return first


@dataclass
class Graph:
    n: int
    dim: int
    M: int
    deg: np.ndarray
    links: np.ndarray               # n x M, EMPTY padded
    tree: RPTree
    construction_time: float = 0.0
    extra: dict = field(default_factory=dict)


def write_graph(path, g: Graph) -> None:
    """nndindex::save_index + save_tree (include/index.h:1810-1875)."""
    out = bytearray()
    out += struct.pack("<QQQf", g.n, g.dim, g.M, g.construction_time)
    deg = np.asarray(g.deg, np.uint32)
    links = np.asarray(g.links, np.uint32)
    # [u32 deg, deg x u32] per node, built vectorised
    total = int(deg.sum())
    body = np.empty(g.n + total, np.uint32)
    pos = np.arange(g.n, dtype=np.int64) + np.concatenate([[0], np.cumsum(deg[:-1], dtype=np.int64)])
    body[pos] = deg
    mask = np.arange(g.M)[None, :] < deg[:, None]
    rows, cols = np.nonzero(mask)
    body[pos[rows] + 1 + cols] = links[rows, cols]
    out += body.tobytes()
    t = g.tree
    out += struct.pack("<QQQ", t.leaf_size, t.n_leaves, t.n_nodes)
    for i in range(t.n_nodes):
        leaf = t.left[i] == EMPTY
        left = 0xFFFFFFFF if leaf else int(t.left[i])
        right = 0xFFFFFFFF if leaf else int(t.right[i])
        out += struct.pack("<QQf", left, right, float(t.offset[i]))
        if leaf:
            out += struct.pack("<Q", 0)
            idx = t.indices[t.leaf_off[i]:t.leaf_off[i + 1]]
            out += struct.pack("<Q", len(idx)) + np.asarray(idx, "<u4").tobytes()
        else:
            out += struct.pack("<Q", t.dim) + np.asarray(t.hyperplane[i], "<f4").tobytes()
            out += struct.pack("<Q", 0)
    Path(path).write_bytes(bytes(out))


def read_graph(path, n: int | None = None, dim: int | None = None, M: int | None = None) -> Graph:
    """nndindex::load_index + load_tree with the same validation (index.h:1827-1915)."""
    raw = Path(path).read_bytes()
    if len(raw) < 28:
        raise FormatError(f"incompatible or truncated cached index: {path}")
    fn, fdim, fM, ctime = struct.unpack("<QQQf", raw[:28])
    if (n is not None and fn != n) or (dim is not None and fdim != dim) or (M is not None and fM != M) \
            or not np.isfinite(ctime):
        raise FormatError(f"incompatible or truncated cached index: {path}")
    pos = 28
    u32 = np.frombuffer(raw, np.uint32, (len(raw) - 28) // 4, 28)
    deg = np.empty(fn, np.uint32)
    links = np.full((fn, fM), EMPTY, np.uint32)
    p = 0
    for i in range(fn):
        if p >= len(u32):
            raise FormatError(f"invalid adjacency data in cached index: {path}")
        d = int(u32[p])
        if d > fM or p + 1 + d > len(u32):
            raise FormatError(f"invalid adjacency data in cached index: {path}")
        deg[i] = d
        links[i, :d] = u32[p + 1:p + 1 + d]
        p += 1 + d
    if fn and deg.sum() and int(links[links != EMPTY].max()) >= fn:
        raise FormatError(f"invalid neighbor id in cached index: {path}")
    pos = 28 + 4 * p
    leaf_size, n_leaves, ns = struct.unpack("<QQQ", raw[pos:pos + 24])
    pos += 24
    if leaf_size == 0 or leaf_size > 1000000 or n_leaves == 0 or n_leaves > fn or ns == 0 or ns > 2 * fn:
        raise FormatError(f"invalid RP tree in cached index: {path}")
    left = np.empty(ns, np.uint32)
    right = np.empty(ns, np.uint32)
    offset = np.empty(ns, np.float32)
    hyper = np.zeros((ns, fdim), np.float32)
    leaf_off = np.zeros(ns + 1, np.int64)
    idx_parts = []
    for i in range(ns):
        l, r, off = struct.unpack("<QQf", raw[pos:pos + 20])
        pos += 20
        hs = struct.unpack("<Q", raw[pos:pos + 8])[0]
        pos += 8
        if hs > fdim or not np.isfinite(off):
            raise FormatError(f"invalid RP tree in cached index: {path}")
        if hs:
            hyper[i] = np.frombuffer(raw, "<f4", hs, pos)
        pos += 4 * hs
        isz = struct.unpack("<Q", raw[pos:pos + 8])[0]
        pos += 8
        if isz > fn:
            raise FormatError(f"invalid RP tree in cached index: {path}")
        idx = np.frombuffer(raw, "<u4", isz, pos)
        pos += 4 * isz
        leaf = l == 0xFFFFFFFF and r == 0xFFFFFFFF
        internal = l < i and r < i
        if (not leaf and not internal) or (leaf and isz == 0) or (internal and hs != fdim):
            raise FormatError(f"invalid RP tree in cached index: {path}")
        if isz and int(idx.max()) >= fn:
            raise FormatError(f"invalid RP tree in cached index: {path}")
        left[i] = EMPTY if leaf else l
        right[i] = EMPTY if leaf else r
        offset[i] = off
        idx_parts.append(idx)
        leaf_off[i + 1] = leaf_off[i] + isz
    indices = np.concatenate(idx_parts).astype(np.uint32) if idx_parts else np.zeros(0, np.uint32)
    tree = RPTree(int(leaf_size), left, right, offset, hyper, leaf_off, indices, int(fdim))
    return Graph(int(fn), int(fdim), int(fM), deg, links, tree, float(ctime))


def bfs_tree_to_postorder(left, right, offset, hyperplane, leaf_off, leaf_cnt, perm, leaf_size: int,
                          dim: int) -> RPTree:
    """Renumbers a breadth-first tree (children after parents) into the
    reference's post-order (left subtree, right subtree, node; rptrees.h:127-152)."""
    nn = len(left)
    order = []
    stack = [(0, False)]
    while stack:
        v, done = stack.pop()
        if left[v] == EMPTY or done:
            order.append(v)
            continue
        stack.append((v, True))
        stack.append((int(right[v]), False))
        stack.append((int(left[v]), False))
    newid = np.empty(nn, np.int64)
    newid[np.array(order)] = np.arange(len(order))
    m = len(order)
    o = np.array(order)
    L = np.asarray(left)[o].astype(np.int64)
    R = np.asarray(right)[o].astype(np.int64)
    leafmask = L == EMPTY
    nl = np.where(leafmask, EMPTY, newid[np.where(leafmask, 0, L)]).astype(np.uint32)
    nr = np.where(leafmask, EMPTY, newid[np.where(leafmask, 0, R)]).astype(np.uint32)
    cnt = np.where(leafmask, np.asarray(leaf_cnt)[o], 0).astype(np.int64)
    loff = np.zeros(m + 1, np.int64)
    loff[1:] = np.cumsum(cnt)
    indices = np.empty(int(loff[-1]), np.uint32)
    starts = np.asarray(leaf_off)[o]
    for j in np.nonzero(cnt)[0]:
        s = int(starts[j])
        indices[loff[j]:loff[j + 1]] = perm[s:s + cnt[j]]
    hyp = np.asarray(hyperplane)[o].copy()
    hyp[leafmask] = 0
    off = np.where(leafmask, np.float32(np.finfo(np.float32).max), np.asarray(offset)[o]).astype(np.float32)
    return RPTree(leaf_size, nl, nr, off, hyp, loff, indices, dim)


# --------------------------------------------------------------- timing


def write_timing(path, header: str, fields: list[tuple[str, object]]) -> None:
    lines = [header]
    for k, v in fields:
        lines.append(f"{k} {v!r}" if isinstance(v, float) else f"{k} {v}")
    Path(path).write_text("\n".join(lines) + "\n")


def read_timing_seconds(path, header: str) -> float:
    lines = Path(path).read_text().splitlines()
    if not lines or lines[0] != header:
        raise FormatError(f"invalid timing metadata header: {path}")
    for ln in lines[1:]:
        parts = ln.split()
        if len(parts) == 2 and parts[0] == "seconds":
            return float(parts[1])
    raise FormatError(f"invalid timing value in {path}")
