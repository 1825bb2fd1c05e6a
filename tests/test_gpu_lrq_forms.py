"""The CUDA codec in every CompactLrqVerifier form against the reference's own
outputs (tests/golden/lrq_forms.npz): rank-M only, u2 / u4 / u8 / u16 codes
under each policy, float32 residuals, signed (IP) keys; and the analytic
Rank-M model.  Encode must reproduce the reference's artifact byte for byte,
materialize its thresholds bit for bit (host-buffer entry points and the
context's resident verifier)."""
import numpy as np
import pytest

import lrq_forms as lf
from anqi import formats
from anqi._lib import AnqiError, Context

pytestmark = pytest.mark.gpu


def test_lrq_encode_materialize_every_form(tmp_path):
    z, s = lf.load()
    with Context(0) as ctx:
        for bits, policy, signed in lf.forms(z):
            keys, mu, basis = lf.inputs(z, s, signed)
            cb = lf.codebook(z, bits)
            coeff, codes, resid = ctx.lrq_encode_bits(keys, mu, basis, cb, bits, policy)
            p = tmp_path / f"g_{bits}_{policy}_{signed}.bin"
            formats.write_verifier(p, coeff, codes, bits, policy, resid, nk=100)
            assert p.read_bytes() == z[f"vf_{bits}_{policy}_{signed}"].tobytes(), (bits, policy, signed)
            for i, k in enumerate((1, 10, 50, 100)):
                thr = ctx.lrq_materialize_bits(coeff, codes, resid, 100, mu, basis, cb, bits, k,
                                               signed_keys=bool(signed))
                ref = z[f"thr_{bits}_{policy}_{signed}"][i]
                assert np.array_equal(thr.view(np.uint32), ref.view(np.uint32)), (bits, policy, signed, k)


def test_analytic_rankm_materialize():
    z, _ = lf.load()
    with Context(0) as ctx:
        for flags in (3, 7):
            m = formats.AnalyticModel(100, 8, 10, flags, float(z[f"pw_b0_{flags}"][0]), z[f"pw_coeff_{flags}"])
            for si, scale in enumerate((1.0, 1.25)):
                for i, k in enumerate((1, 10, 50, 100)):
                    thr = ctx.analytic_materialize(m, k, scale)
                    assert np.array_equal(thr.view(np.uint32), z[f"pw_thr_{flags}"][si, i].view(np.uint32))


def test_resident_verifier_forms_drive_the_postfilter():
    """The context's verifier loaded in another form (u4 nearest, float32
    residuals, rank-M only, analytic): a query batch's verified sets equal the
    ones obtained with the same thresholds set explicitly."""
    z, s = lf.load()
    from anqi import formats as fm
    import tempfile
    from pathlib import Path
    with tempfile.TemporaryDirectory() as td:
        p = Path(td) / "g.bin"
        p.write_bytes(s["graph_file"].tobytes())
        g = fm.read_graph(p)
    with Context(0) as ctx:
        ctx.index_load(s["base"], s["lifted"], g.deg, g.links, g.tree, float(s["scale"]), float(s["mstar2"]))
        cases = [(4, "nearest"), (32, "floor"), (0, "floor")]
        for bits, policy in cases:
            keys, mu, basis = lf.inputs(z, s, 0)
            cb = lf.codebook(z, bits)
            coeff, codes, resid = ctx.lrq_encode_bits(keys, mu, basis, cb, bits, policy)
            ctx.verifier_load_bits(coeff, codes, resid, 100, mu, basis, cb, bits)
            ctx.verifier_materialize(10)
            a = ctx.rknn_query(s["query"], 10, 32)
            ctx.set_thresholds(10, ctx.lrq_materialize_bits(coeff, codes, resid, 100, mu, basis, cb, bits, 10))
            b = ctx.rknn_query(s["query"], 10, 32)
            assert np.array_equal(a.pred_off, b.pred_off) and np.array_equal(a.pred_ids, b.pred_ids), (bits, policy)
        m = fm.AnalyticModel(100, 8, 10, 7, float(z["pw_b0_7"][0]), z["pw_coeff_7"])
        ctx.verifier_load_analytic(m)
        ctx.verifier_materialize(50)
        a = ctx.rknn_query(s["query"], 50, 32)
        ctx.set_thresholds(50, ctx.analytic_materialize(m, 50))
        b = ctx.rknn_query(s["query"], 50, 32)
        assert np.array_equal(a.pred_off, b.pred_off) and np.array_equal(a.pred_ids, b.pred_ids)


def test_codec_argument_errors():
    z, s = lf.load()
    keys, mu, basis = lf.inputs(z, s, 0)
    with Context(0) as ctx:
        with pytest.raises(AnqiError) as e:  # u2 needs nk % 4 == 0
            ctx.lrq_encode_bits(keys[:, :98], mu[:98], basis[:, :98], lf.codebook(z, 2)[:98], 2, "floor")
        assert e.value.status == 3
        with pytest.raises(AnqiError) as e:  # bits 6 is no form
            ctx.lrq_encode_bits(keys, mu, basis, np.zeros((100, 64), np.float32), 6, "floor")
        assert e.value.status == 2
