"""Shared helpers for the tests of every CompactLrqVerifier form against the
reference's own outputs (tests/golden/lrq_forms.npz, made by make_golden.py)."""
from pathlib import Path

import numpy as np

from anqi import formats

GOLDEN = Path(__file__).resolve().parent / "golden"


def load():
    return dict(np.load(GOLDEN / "lrq_forms.npz")), dict(np.load(GOLDEN / "sample_d32.npz"))


def forms(z):
    out = []
    for key in sorted(z):
        if key.startswith("vf_"):
            bits, policy, signed = key[3:].split("_")
            out.append((int(bits), policy, int(signed)))
    return out


def codebook(z, bits):
    """The fixture's codebook for a bit width (evenly spaced between lo and hi)."""
    if bits not in formats.PACKED_BITS:
        return None
    lo, hi = z["lo"], z["hi"]
    cs = 1 << bits
    t = np.arange(cs, dtype=np.float64) / (cs - 1)
    return (lo[:, None].astype(np.float64) + t[None, :] * (hi - lo)[:, None].astype(np.float64)).astype(np.float32)


def inputs(z, s, signed):
    keys, mu, basis = s["rec_keys"].astype(np.float32), s["mu"].astype(np.float32), s["basis"].astype(np.float32)
    if signed:
        keys = keys - z["shift"][0]
        mu = mu - z["shift"][0]
    return keys, mu, basis


def reference_artifact(z, tmp_path, bits, policy, signed, nk=100, rankm=8):
    p = Path(tmp_path) / f"vf_{bits}_{policy}_{signed}.bin"
    p.write_bytes(z[f"vf_{bits}_{policy}_{signed}"].tobytes())
    return formats.read_verifier_any(p, 256, nk, rankm, bits, policy)
