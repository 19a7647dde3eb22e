"""The BSDF fixtures (tests/golden/bsdf_vectors.npz, made by
tests/golden/make_golden.py --bsdf) are the reference's own material code:
rebuilt from the compiled reference they come out identical. Hair materials
in Marschner mode go through the reference's private Marschner branches
(MarschnerHair.h:242-257, 284-375) reached from oracle/ref_harness.cpp. The
GPU side of these fixtures is tests/test_gpu_bsdf.py."""
import os

import numpy as np

from test_golden_features import golden_module

HERE = os.path.dirname(os.path.abspath(__file__))


def test_bsdf_fixtures_reproduce_from_the_reference(ref_built):
    G = golden_module()
    gold = np.load(os.path.join(HERE, "golden", "bsdf_vectors.npz"))
    for k, m in enumerate(G.bsdf_materials()):
        q = G.bsdf_queries(m, 512, 100 + k)
        assert np.array_equal(q, gold[f"m{k}_query"]), k
        r = ref_built.RefMaterial(m, variant="nocontract").query(q)
        assert np.array_equal(r, gold[f"m{k}_result"]), k
        assert (r["sample_pdf"] > 0).mean() > 0.3, k
    out = ref_built.mh_functions(gold["mh_grid"], float(gold["mh_eta"]), gold["mh_sigma_a"], variant="nocontract")
    assert np.array_equal(out, gold["mh_out"])


def test_marschner_fixture_is_not_kajiya_kay():
    """The Marschner-mode fixtures differ from the Kajiya-Kay ones on the same
    frames (the private branches were reached, not the public early return)."""
    G = golden_module()
    gold = np.load(os.path.join(HERE, "golden", "bsdf_vectors.npz"))
    mats = G.bsdf_materials()
    kk = [k for k, m in enumerate(mats) if m.type == 3 and m.hair_mode == 0]
    mh = [k for k, m in enumerate(mats) if m.type == 3 and m.hair_mode == 1]
    assert len(kk) == len(mh) == 4
    for a, b in zip(kk, mh):
        assert not np.allclose(gold[f"m{a}_result"]["f"], gold[f"m{b}_result"]["f"])


def test_marschner_lobe_functions_against_the_restatement(restate_built):
    """The restatement's lobe functions (oracle/restate, float) agree with the
    reference's mh_* on the fixture grid to a few float ulps."""
    gold = np.load(os.path.join(HERE, "golden", "bsdf_vectors.npz"))
    out = restate_built.mh_functions(gold["mh_grid"], float(gold["mh_eta"]), gold["mh_sigma_a"])
    ref = gold["mh_out"]
    scale = np.maximum(np.abs(ref), 1e-30)
    assert np.all(np.isfinite(out))
    assert (np.abs(out - ref) <= 1e-5 * scale + 1e-30).mean() >= 0.999
