"""Test infrastructure only: files for, and runs of, the reference harness's
per-query parity mode (oracle/ref_harness.cpp ``qparity``), and the query-by-
query comparison of another implementation's results with its output.

Used by the GPU parity tests and by the benchmark's CPU-baseline leg; nothing
in the product imports it.

The harness runs the reference's own nndindex::range_search (include/index.h:
1535-1640) and FP32 postfilter (src/rknn_query.cpp:2555-2561) one query at a
time.  Its entry descent (include/rptrees.h:108-124) draws a random side when
a hyperplane margin is within EPS of zero; mode "left" sends those ties left
(the rule of the B200 entry kernel), mode "tree" keeps the reference's draw.
For every query the harness also reports whether the tie-left path met a tie.
"""
from __future__ import annotations

import subprocess
from dataclasses import dataclass
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent.parent
HARNESS = REPO / "oracle" / "_ref" / "ref_harness"


def write_query_files(d: Path, base, query, lifted, deg, links, tree, mstar2: float, scale: float,
                      thresholds: dict) -> None:
    """The inputs of ``qparity`` / ``qbench``: fbin vectors, the graph file in the
    reference's save_index layout, the lift meta, one raw f32 threshold file per k."""
    import sys

    sys.path.insert(0, str(REPO / "anqi-implementation_b200"))
    from anqi import formats

    d.mkdir(parents=True, exist_ok=True)
    formats.write_fbin(d / "lifted.bin", lifted)
    formats.write_fbin(d / "base.bin", base)
    formats.write_fbin(d / "query.bin", query)
    g = formats.Graph(len(base), lifted.shape[1], links.shape[1], deg, links, tree)
    formats.write_graph(d / "graph.bin", g)
    formats.write_graph_meta(d / "meta.txt", mstar2, scale)
    for k, thr in thresholds.items():
        np.ascontiguousarray(thr, np.float32).tofile(d / f"thr{k}.bin")


def read_dump_csr(path: Path):
    """[u64 rows][(rows+1) u64 offsets][u32 ids] (ref_harness.cpp dump_csr)."""
    raw = Path(path).read_bytes()
    n = int(np.frombuffer(raw, np.uint64, 1)[0])
    off = np.frombuffer(raw, np.uint64, n + 1, 8).astype(np.int64)
    ids = np.frombuffer(raw, np.uint32, int(off[-1]), 8 + 8 * (n + 1))
    return off, ids


@dataclass
class Parity:
    entry: np.ndarray  # tie-left entry object per query
    tie: np.ndarray  # the tie-left descent met |margin| <= EPS
    cand_off: np.ndarray
    cand: np.ndarray
    ndist: np.ndarray
    pred: dict  # k -> (off, ids)


def run_qparity(d: Path, L: int, mode: str, nq: int, ks, timeout: float = 3600.0) -> Parity:
    if not HARNESS.exists():
        raise FileNotFoundError("oracle/_ref/ref_harness is not built (make -C oracle ref REF=<reference tree>)")
    out = d / f"qp_{mode}"
    cmd = [str(HARNESS), "qparity", str(d / "lifted.bin"), str(d / "graph.bin"), str(d / "base.bin"),
           str(d / "query.bin"), str(d / "meta.txt"), str(L), mode, str(nq), str(out)]
    cmd += [str(d / f"thr{k}.bin") for k in ks]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    if p.returncode != 0:
        raise RuntimeError(f"ref_harness qparity failed ({p.returncode}): {p.stderr[-400:]}")
    ent = np.fromfile(f"{out}_entry.bin", np.uint32).reshape(-1, 2)
    coff, cand = read_dump_csr(Path(f"{out}_cand.bin"))
    nd = np.fromfile(f"{out}_ndist.bin", np.uint32)
    pred = {k: read_dump_csr(Path(f"{out}_pred{t}.bin")) for t, k in enumerate(ks)}
    return Parity(ent[:, 0].copy(), ent[:, 1].astype(bool), coff, cand, nd, pred)


def compare(ref: Parity, results: dict, nq: int) -> dict:
    """Query-by-query comparison with another implementation's results
    (k -> object with cand(i), pred(i), n_dist, as anqi._lib's query result):
    a query agrees when its candidates (in visit order), #dist and every k's
    verified set are identical.  Differing queries are split by whether the
    tie-left descent met a tie."""
    same = np.ones(nq, bool)
    for k, r in results.items():
        poff, pids = ref.pred[k]
        nd = np.asarray(r.n_dist[:nq]).astype(np.uint32)
        for i in range(nq):
            if not same[i]:
                continue
            if (nd[i] != ref.ndist[i] or not np.array_equal(r.cand(i), ref.cand[ref.cand_off[i]:ref.cand_off[i + 1]])
                    or not np.array_equal(r.pred(i), pids[poff[i]:poff[i + 1]])):
                same[i] = False
    tie = ref.tie[:nq]
    return {"queries": int(nq), "identical": int(same.sum()), "differ": int((~same).sum()),
            "differ_at_ties": int((~same & tie).sum()), "differ_without_tie": int((~same & ~tie).sum()),
            "tie_queries": int(tie.sum())}
