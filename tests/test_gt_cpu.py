"""oracle/gt_cpu (exact reverse-kNN ground truth on the host CPU, used by the
benchmark's reference arm) against the reference's own tools/dataset_gt on
small-integer data: thresholds (.rk) and CSR files byte for byte, through the
AMX BF16 tiles where this CPU has them and through the AVX-512 FP32 path."""
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

from anqi import formats, pipeline

REPO = Path(__file__).resolve().parent.parent
GT_CPU = REPO / "oracle" / "gt_cpu"
DATASET_GT = REPO / "oracle" / "_ref" / "dataset_gt"


def _hints(base, K=100, extra=0):
    x = base.astype(np.float64)
    nrm = (x * x).sum(1)
    d2 = nrm[:, None] + nrm[None, :] - 2 * x @ x.T
    np.fill_diagonal(d2, np.inf)
    # exact neighbours, optionally pushed out by `extra` ranks (looser, still valid bounds)
    o = np.argsort(d2, axis=1, kind="stable")[:, extra:extra + K].astype(np.uint32)
    rec = np.zeros(o.shape + (2,), np.uint32)
    rec[:, :, 0] = o
    return rec


@pytest.mark.skipif(not GT_CPU.exists() or not DATASET_GT.exists(), reason="needs oracle/gt_cpu and oracle/_ref")
@pytest.mark.parametrize("path", ["default", "avx512"])
@pytest.mark.parametrize("d,extra", [(128, 0), (40, 7)])
def test_gt_cpu_matches_dataset_gt(tmp_path, path, d, extra):
    base, _ = pipeline.mixture(3000, d, 0, centers=20, seed=99)
    query = pipeline.mixture_queries(150, d, centers=20, seed=99, qseed=3)
    # duplicate rows: ties at equal keys and zero distances
    base[17] = base[3]
    base[2000] = base[3]
    formats.write_fbin(tmp_path / "b.bin", base)
    formats.write_fbin(tmp_path / "q.bin", query)
    _hints(base, extra=extra).tofile(tmp_path / "h.rec")
    env = dict(os.environ)
    if path == "avx512":
        env["GT_CPU_NO_AMX"] = "1"
    p = subprocess.run([str(GT_CPU), tmp_path / "b.bin", tmp_path / "q.bin", tmp_path / "h.rec", tmp_path / "ours",
                        "100", "10,50,100", "4"], capture_output=True, text=True, env=env)
    assert p.returncode == 0, p.stderr
    for k in (10, 50, 100):
        subprocess.run([str(DATASET_GT), "--base", tmp_path / "b.bin", "--query", tmp_path / "q.bin", "--K", "100",
                        "--rk_k", str(k), "--out_prefix", tmp_path / f"ref{k}", "--threads", "4", "--mode", "both"],
                       capture_output=True, check=True)
        assert (tmp_path / f"ours_rknn_gt_k{k}.bin").read_bytes() == (tmp_path / f"ref{k}_rknn_gt.bin").read_bytes()
        assert (tmp_path / f"ours_k{k}.rk").read_bytes() == (tmp_path / f"ref{k}_rknn_gt.bin.rk").read_bytes()


@pytest.mark.skipif(not GT_CPU.exists(), reason="needs oracle/gt_cpu")
def test_gt_cpu_rejects_inexact_inputs(tmp_path):
    base = np.random.default_rng(1).normal(size=(300, 16)).astype(np.float32)
    formats.write_fbin(tmp_path / "b.bin", base)
    formats.write_fbin(tmp_path / "q.bin", base[:5])
    _hints(base, K=20).tofile(tmp_path / "h.rec")
    p = subprocess.run([str(GT_CPU), tmp_path / "b.bin", tmp_path / "q.bin", tmp_path / "h.rec", tmp_path / "o", "20",
                        "10", "2"], capture_output=True, text=True)
    assert p.returncode == 3 and "not small integers" in p.stderr
