"""The Vamana refine of the G48 build (include/index.h:856-1065, 1262-1285):
the batched style's insertion order against the C++ library's own
std::shuffle over std::mt19937_64, the settings read from the environment
(anqi.vamana), and the oracle's global passes and batched refine against the
reference's own refined graphs (tests/golden/vamana.npz, oracle/ref_harness
graph with ANQI_VAMANA set).  Bit-exact."""
import ctypes as C
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle_lib as ol
from anqi import edge_policy as ep
from anqi import formats, vamana

GOLDEN = Path(__file__).resolve().parent / "golden"
EMPTY = 0xFFFFFFFF

SHUFFLE_CPP = r"""
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <numeric>
#include <random>
#include <vector>
int main(int argc, char** argv) {
    const size_t n = std::strtoull(argv[1], nullptr, 10);
    const unsigned long long seed = std::strtoull(argv[2], nullptr, 10);
    const int passes = std::atoi(argv[3]);
    std::vector<unsigned> o(n);
    std::iota(o.begin(), o.end(), 0u);
    for (int p = 0; p < passes; p++) {
        std::mt19937_64 rng(seed + 0x9e3779b97f4a7c15ULL * (unsigned long long)(p + 1));
        std::shuffle(o.begin(), o.end(), rng);
    }
    for (size_t i = 0; i < n; i++) std::printf("%u\n", o[i]);
    return 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_batch_order_matches_std_shuffle(tmp_path):
    src = tmp_path / "s.cpp"
    src.write_text(SHUFFLE_CPP)
    exe = tmp_path / "s"
    subprocess.run(["g++", "-O2", "-std=c++17", str(src), "-o", str(exe)], check=True)
    for n in (1, 2, 3, 10, 257, 4096, 20001):
        for seed, passes in ((10, 1), (10, 3), (987654321, 2)):
            out = subprocess.run([str(exe), str(n), str(seed), str(passes)], capture_output=True, text=True,
                                 check=True).stdout.split()
            assert np.array_equal(ol.vamana_batch_order(n, seed, passes), np.array(out, dtype=np.uint32)), (n, seed)


def test_vamana_settings_from_env():
    assert vamana.from_env({}) is None
    p = vamana.from_env({"ANQI_VAMANA": "1"})
    assert (p.style, p.L, p.passes) == ("global", 128, 2)
    x = np.arange(40, dtype=np.float32).reshape(10, 4)
    p = vamana.from_env({"ANQI_VAMANA": "1", "ANQI_VAMANA_STYLE": "batch", "ANQI_VAMANA_ENTRY": "23",
                         "ANQI_VAMANA_BATCH_BASE": "1.5", "ANQI_VAMANA_EARLY_ALPHA_ONE": "0"}, x)
    assert p.entry == 3 and p.batch_base == 1.5 and not p.early_alpha_one
    assert vamana.from_env({"ANQI_VAMANA": "1", "ANQI_VAMANA_STYLE": "batch", "ANQI_VAMANA_ENTRY": "-1"}, x).entry == \
        (2**64 - 1) % 10
    # the sample point nearest the sample mean
    assert vamana.from_env({"ANQI_VAMANA": "1", "ANQI_VAMANA_STYLE": "batch", "ANQI_VAMANA_ENTRY": "medoid"},
                           x).entry in (4, 5)


@pytest.fixture(scope="module")
def fx():
    return (dict(np.load(GOLDEN / "vamana.npz")), dict(np.load(GOLDEN / "sample_d32.npz")),
            dict(np.load(GOLDEN / "edge_policies.npz")))


def rows(off, ids):
    return [list(ids[int(off[i]):int(off[i + 1])]) for i in range(len(off) - 1)]


def as_matrix(off, ids, M=48):
    r = rows(off, ids)
    L = np.full((len(r), M), EMPTY, np.uint32)
    for i, v in enumerate(r):
        L[i, :len(v)] = v
    return L, np.array([len(v) for v in r], np.uint32)


def config(fx, name, tmp_path):
    z, s, e = fx
    env = dict(kv.split("=", 1) for kv in z[f"{name}_env"])
    rf = tmp_path / "resid.bin"
    e["resid"].tofile(rf)
    env["ANQI_EDGE_RESID_FILE"] = str(rf)
    pol = ep.from_env(env, 256, 48, folder=str(tmp_path / "none"))
    return vamana.from_env(env, s["lifted"]), pol


def tree_entries(s):
    raw = s["graph_file"].tobytes()
    import tempfile
    with tempfile.NamedTemporaryFile(suffix=".bin") as f:
        f.write(raw)
        f.flush()
        g = formats.read_graph(f.name)
    t = g.tree
    nn = len(t.left)
    lf = np.full(nn, EMPTY, np.uint32)
    for v in range(nn):
        if t.left[v] == EMPTY and t.leaf_off[v] < t.leaf_off[v + 1]:
            lf[v] = t.indices[t.leaf_off[v]]
    x = np.ascontiguousarray(s["lifted"], np.float32)
    fn = ol.LIB.ao_tree_entry
    fn.restype = C.c_uint32
    hyp = np.ascontiguousarray(t.hyperplane, np.float32)
    args = [np.ascontiguousarray(a) for a in (t.left.astype(np.uint32), t.right.astype(np.uint32),
                                              t.offset.astype(np.float32))]
    return np.array([fn(nn, x.shape[1], args[0].ctypes.data_as(C.c_void_p), args[1].ctypes.data_as(C.c_void_p),
                        args[2].ctypes.data_as(C.c_void_p), hyp.ctypes.data_as(C.c_void_p),
                        lf.ctypes.data_as(C.c_void_p), x[i].ctypes.data_as(C.c_void_p)) for i in range(len(x))],
                    np.uint32)


NAMES = [str(n) for n in np.load(GOLDEN / "vamana.npz")["names"]]


@pytest.mark.parametrize("name", NAMES)
def test_oracle_vamana_vs_reference(fx, name, tmp_path):
    z, s, e = fx
    vp, pol = config(fx, name, tmp_path)
    x = np.ascontiguousarray(s["lifted"], np.float32)
    nrm = ol.norms(x)
    # the committed graph the refine starts from: the reference's, under the same policy
    if pol is None:
        links, deg = as_matrix(s["g_adj_off"], s["g_adj"])
    else:
        links, deg = as_matrix(e[f"{pol.name}_adj_off"], e[f"{pol.name}_adj"])
    g0 = s["g_join_ids"]
    if vp.style in ("global", "old"):
        entry = tree_entries(s)
        for _ in range(vp.passes):
            O, Od = ol.vamana_select_policy(x, nrm, links, deg, g0, entry, pol, Lb=vp.L)
            links, deg = ol.graph_commit_policy(x, nrm, O, Od, pol)
    else:
        links, deg = ol.vamana_batch_refine(x, nrm, links, deg, g0, vp, pol)
    ref = rows(z[f"{name}_off"], z[f"{name}_adj"])
    for i in range(256):
        assert list(links[i, :deg[i]]) == ref[i], (name, i)
