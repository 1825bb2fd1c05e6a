"""CPU-only checks: the C-ABI library and its exports, file formats, the LRQ
trainer against the reference's own outputs, tree renumbering, and the
multi-process (gloo, world size 2) plumbing."""
import ctypes
import os
import re
import struct
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from anqi import formats, lrq_train, pipeline
from anqi import dist as adist

REPO = Path(__file__).resolve().parent.parent
LIB = REPO / "anqi-implementation_b200" / "lib" / "libanqi.so"


def declared_symbols():
    text = (REPO / "include" / "anqi.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:int|void|uint64_t|const char\*)\s+(anqi_[a-z0-9_]+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    if not LIB.exists():
        subprocess.run([sys.executable, str(REPO / "anqi-implementation_b200" / "build.py")], check=True)
    lib = ctypes.CDLL(str(LIB))
    syms = declared_symbols()
    assert len(syms) >= 30
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    from anqi import _lib
    assert sorted(_lib.EXPORTED) == syms


def test_no_gpu_context_fails_loudly():
    from anqi._lib import AnqiError, Context
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(AnqiError):
        Context(0)


def test_format_roundtrips(tmp_path, sample):
    p = tmp_path / "x"
    formats.write_fbin(f"{p}_base.bin", sample["base"])
    assert np.array_equal(formats.read_fbin(f"{p}_base.bin"), sample["base"])
    formats.write_rec(f"{p}.rec", sample["rec_ids"], sample["rec_keys"])
    i, k = formats.read_rec(f"{p}.rec", 256)
    assert np.array_equal(i, sample["rec_ids"]) and np.array_equal(k, sample["rec_keys"])
    formats.write_basis(f"{p}_b.bin", sample["mu"], sample["basis"])
    mu, b = formats.read_basis(f"{p}_b.bin")
    assert np.array_equal(mu, sample["mu"]) and np.array_equal(b, sample["basis"])
    assert Path(f"{p}_b.bin").stat().st_size == 3608
    formats.write_codebook(f"{p}_c.bin", sample["codebook"])
    assert np.array_equal(formats.read_codebook(f"{p}_c.bin"), sample["codebook"])
    assert Path(f"{p}_c.bin").stat().st_size == 102424
    for k in (10, 50, 100):
        formats.write_rknn_csr(f"{p}_gt{k}.bin", sample[f"gt_off_{k}"], sample[f"gt_ids_{k}"], sample[f"gt_keys_{k}"])
        off, ids, keys = formats.read_rknn_csr(f"{p}_gt{k}.bin", 256)
        assert np.array_equal(off, sample[f"gt_off_{k}"]) and np.array_equal(ids, sample[f"gt_ids_{k}"])


def test_format_errors(tmp_path):
    bad = tmp_path / "bad.bin"
    bad.write_bytes(struct.pack("<II", 3, 4) + b"\0" * 10)
    with pytest.raises(formats.FormatError):
        formats.read_fbin(bad)
    (tmp_path / "cb.bin").write_bytes(b"ANQIRQ0\0" + b"\0" * 16)
    with pytest.raises(formats.FormatError):
        formats.read_codebook(tmp_path / "cb.bin")
    (tmp_path / "m.meta").write_text("0 8 100 cosine 1.0\n")
    with pytest.raises(formats.FormatError):
        formats.read_lifted_meta(tmp_path / "m.meta")
    g = tmp_path / "g.bin"
    g.write_bytes(struct.pack("<QQQf", 4, 10, 48, 0.0) + struct.pack("<I", 60))
    with pytest.raises(formats.FormatError):
        formats.read_graph(g)


def test_trainer_reproduces_reference_files(sample, tmp_path):
    mu, basis, cb = lrq_train.train(sample["rec_keys"], 256, log=lambda s: None)
    bp, cp = lrq_train.write_outputs(str(tmp_path / "s"), mu, basis, cb)
    raw_b = bp.read_bytes()
    assert raw_b[8:8 + 400] == sample["mu"].tobytes() and raw_b[408:] == sample["basis"].tobytes()
    assert cp.read_bytes()[24:] == sample["codebook"].tobytes()


def test_trainer_cli(tmp_path, sample):
    pfx = tmp_path / "t"
    formats.write_fbin(f"{pfx}_base.bin", sample["base"])
    formats.write_rec(f"{pfx}_baseknn_aknn.rec", sample["rec_ids"], sample["rec_keys"])
    env = dict(os.environ, PYTHONPATH=str(REPO / "anqi-implementation_b200"))
    p = subprocess.run([sys.executable, "-m", "anqi.lrq_train", "--pfx", str(pfx)], env=env, capture_output=True,
                       text=True)
    assert p.returncode == 0, p.stderr
    assert formats.read_timing_seconds(f"{pfx}_verifier_train_time.meta", "ANQI_VERIFIER_TRAIN_V1") >= 0
    assert np.array_equal(formats.read_codebook(f"{pfx}_learned_rq_codebook_M8_u8.bin"), sample["codebook"])


def test_postorder_tree_is_valid_reference_tree(tmp_path):
    import oracle_lib as ol
    x = pipeline.gaussian(3000, 12, 1, seed=3)[0]
    t = ol.rp_tree(x, 50)
    tree = formats.bfs_tree_to_postorder(t["left"], t["right"], t["offset"], t["hyperplane"], t["leaf_off"],
                                        t["leaf_cnt"], t["perm"], 50, 12)
    # load_tree's rules (index.h:1906-1911): children before parents, leaves non-empty, root last
    for i in range(tree.n_nodes):
        if tree.left[i] == formats.EMPTY:
            assert tree.leaf_off[i + 1] > tree.leaf_off[i]
        else:
            assert tree.left[i] < i and tree.right[i] < i
    assert sorted(tree.indices.tolist()) == list(range(3000))
    # the entry point of a point's own leaf: descend with the BFS arrays and the post-order arrays alike
    g = formats.Graph(3000, 12, 4, np.zeros(3000, np.uint32), np.full((3000, 4), formats.EMPTY, np.uint32), tree)
    formats.write_graph(tmp_path / "g.bin", g)
    g2 = formats.read_graph(tmp_path / "g.bin")
    assert np.array_equal(g2.tree.left, tree.left) and np.array_equal(g2.tree.indices, tree.indices)


def test_mixture_recipe():
    b, q = pipeline.mixture(20000, 128, 500, seed=1)
    assert b.dtype == np.float32 and b.shape == (20000, 128) and q.shape == (500, 128)
    assert b.min() >= 0 and b.max() <= 255 and np.all(b == np.rint(b))


def test_shard_range_partitions():
    for n in (0, 1, 7, 10000):
        for w in (1, 2, 3, 8):
            parts = [adist.shard_range(n, r, w) for r in range(w)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(parts[i][1] == parts[i + 1][0] for i in range(w - 1))


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, str(REPO / "anqi-implementation_b200"))
    from anqi import dist as ad
    dist.init_process_group("gloo", rank=rank, world_size=world)
    m = ad.max_over_ranks([1.0 + rank, 5.0 - rank])
    off = np.array([0, 1 + rank, 2 + 2 * rank], np.uint32)
    ids = np.arange(off[-1], dtype=np.uint32) + 100 * rank
    o, i = ad.gather_csr(off, ids)
    q.put((rank, m, o.tolist(), i.tolist()))
    dist.barrier()
    dist.destroy_process_group()


def test_gloo_world2_timing_and_gather():
    import multiprocessing as mp
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
    for rank, m, o, i in res:
        assert m == [2.0, 5.0]
        assert o == [0, 1, 2, 4, 6]
        assert i == [0, 1, 100, 101, 102, 103]
