"""The device BSDFs (ana_bsdf_batch: the functions k_shade calls) against the
reference's own material code on the committed fixtures
(tests/golden/bsdf_vectors.npz): Lambert, standard_surface, and hair in
Kajiya-Kay mode (what the reference executes) and in Marschner mode (the
reference's R/TT/TRT branches, MarschnerHair.h:242-257 for evaluate and
284-375 for sample).

Tolerance: the device rounds differently from glibc in its transcendental
functions (expf, logf, asinf, atan2f, sinhf, powf: a few ulps) and contracts
multiply-adds, so values agree to about 1e-5 relative and not bit for bit.
A query's error is the largest component error over the query's largest
component magnitude. Bars:
  - evaluate(): within 1e-4 for 98.5 % of frames and within 1e-2 for all
    (the Marschner lobes of beta_m 0.08 have variances near 4e-3, whose
    exponents of ~1/v amplify ulps);
  - sample(): the same lobe and direction (wi within 1e-4) for 99.5 %; the
    path weight f/pdf within 1e-3 for 98 %; f and pdf each within 1e-2 for
    90 % and within 1e-1 for all. A sampled direction carries the device's
    rounding into the lobe: at roughness 0.05 (GGX alpha^2 = 6e-6) a 1e-5
    change of the half-vector moves D by about 1e-2, while f/pdf, in which D
    cancels, stays within 1e-3."""
import os

import numpy as np
import pytest

from anacapa_b200 import api

from test_golden_features import golden_module

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def renderer(gpu):
    r = api.Renderer()
    yield r
    r.close()


def query_err(a, b):
    a = np.asarray(a, np.float64).reshape(len(a), -1)
    b = np.asarray(b, np.float64).reshape(len(b), -1)
    scale = np.maximum(np.abs(b).max(1), 1e-30)
    return np.abs(a - b).max(1) / scale


def compare(dev, ref):
    """Fractions of frames within the bars (see the module docstring)."""
    ev = np.maximum(query_err(dev["f"], ref["f"]), query_err(dev["pdf"], ref["pdf"]))
    vd, vr = dev["sample_pdf"] > 0, ref["sample_pdf"] > 0
    both = vd & vr
    wi = np.abs(dev["sample_wi"] - ref["sample_wi"]).max(1)
    same = (vd == vr) & (~both | (wi <= 1e-4))
    f = query_err(dev["sample_f"][both], ref["sample_f"][both])
    pdf = query_err(dev["sample_pdf"][both], ref["sample_pdf"][both])
    w = query_err(dev["sample_f"][both] / dev["sample_pdf"][both][:, None],
                  ref["sample_f"][both] / ref["sample_pdf"][both][:, None])
    fp = np.maximum(f, pdf)
    frac = (lambda x, t: float((x <= t).mean()) if len(x) else 1.0)
    return {"eval_1e-4": frac(ev, 1e-4), "eval_max": float(ev.max()), "sample_same": float(same.mean()),
            "weight_1e-3": frac(w, 1e-3), "f_pdf_1e-2": frac(fp, 1e-2),
            "f_pdf_max": float(fp.max()) if len(fp) else 0.0, "valid": float(vr.mean())}


MATS = golden_module().bsdf_materials()


@pytest.mark.parametrize("k", range(len(MATS)),
                         ids=[f"m{k}_{['lambert', 'emissive', 'standard', 'hair'][m.type]}"
                              f"{'_marschner' if m.type == 3 and m.hair_mode == 1 else ''}"
                              for k, m in enumerate(MATS)])
def test_bsdf_against_reference(renderer, k):
    gold = np.load(os.path.join(HERE, "golden", "bsdf_vectors.npz"))
    dev = renderer.bsdf(MATS[k], gold[f"m{k}_query"])
    ref = gold[f"m{k}_result"]
    st = compare(dev, ref)
    assert st["eval_1e-4"] >= 0.985 and st["eval_max"] <= 1e-2, st
    assert st["sample_same"] >= 0.995, st
    assert st["weight_1e-3"] >= 0.98, st
    assert st["f_pdf_1e-2"] >= 0.90 and st["f_pdf_max"] <= 1e-1, st
    # the sampled lobes' flags are the reference's where both sides sample
    both = (dev["sample_pdf"] > 0) & (ref["sample_pdf"] > 0)
    assert (dev["sample_flags"][both] == ref["sample_flags"][both]).mean() >= 0.99
