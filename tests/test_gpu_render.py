"""Image parity of the CUDA path tracer against the reference CPU
PathIntegrator (per sample, per pixel 3-sigma z-test at equal spp) and against
the FP64 restatement (RMSE)."""
import os

import numpy as np
import pytest

from anacapa_b200 import api
from anacapa_b200 import scenes as S

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = np.load(os.path.join(HERE, "golden", "reference_vectors.npz"))


@pytest.fixture(scope="module")
def renderer(gpu):
    r = api.Renderer()
    yield r
    r.close()


def lum(rgb):
    return 0.2722287 * rgb[..., 0] + 0.6740818 * rgb[..., 1] + 0.0536895 * rgb[..., 2]


def z_test(film_a, rgbw_b, lumsq_b):
    """Per-pixel 3-sigma z-test on luminance: |mean_a - mean_b| against the
    standard error of the difference, each side's variance from its sum of
    squared sample luminances (Film::varianceAt, src/film/Film.cpp:80-90).
    Returns the fraction of pixels that pass."""
    na, nb = film_a[..., 3], rgbw_b[..., 3]
    ma = lum(film_a[..., :3] / na[..., None])
    mb = lum(rgbw_b[..., :3] / nb[..., None])
    va = np.maximum(film_a[..., 4] / na - ma * ma, 0.0)
    vb = np.maximum(lumsq_b / nb - mb * mb, 0.0)
    se = np.sqrt(va / na + vb / nb)
    tol = 3.0 * se + 1e-6 * np.maximum(np.abs(ma), np.abs(mb)) + 1e-7
    return float((np.abs(ma - mb) <= tol).mean())


def test_per_sample_radiance_matches_reference(renderer):
    """One-spp renders at sample_start = s reproduce PathIntegrator::Li of the
    same (pixel, sample) — the Halton stream is restated exactly."""
    sc = S.cornell()
    renderer.upload(sc)
    q = GOLD["cornell_li_q"]
    got = np.zeros((len(q), 3), np.float32)
    for s in np.unique(q[:, 2]):
        renderer.render(sc.width, sc.height, 1, sc.max_depth, sample_start=int(s))
        img = renderer.image(sc.width, sc.height)
        sel = q[:, 2] == s
        got[sel] = img[q[sel, 1], q[sel, 0]]
    ref = GOLD["cornell_li"]
    close = np.all(np.abs(got - ref) <= 1e-4 * np.maximum(np.abs(ref), 1.0), axis=1)
    assert close.mean() >= 0.95, (got, ref)


def test_small_film_matches_reference(renderer):
    sc = S.cornell(32, 32, 4)
    renderer.upload(sc)
    renderer.render_scene(sc)
    f = renderer.film(32, 32)
    ref = GOLD["cornell32_rgbw"]
    assert np.array_equal(f[..., 3], ref[..., 3])
    rel = np.abs(f[..., :3] - ref[..., :3]) / np.maximum(np.abs(ref[..., :3]), 1e-3)
    assert (rel.max(-1) < 1e-3).mean() >= 0.99


ZCASES = {
    "cornell_256x256x16": lambda: S.cornell(),
    "throughput_480x270x8_full_geometry": lambda: S.throughput(480, 270, 8, 12),
    "hair_320x180x4_full_geometry": lambda: S.hair(320, 180, 4, 10),
}


@pytest.mark.parametrize("case", list(ZCASES))
def test_ztest_against_reference_cpu(renderer, ref_built, case):
    sc = ZCASES[case]()
    renderer.upload(sc)
    renderer.render_scene(sc)
    f = renderer.film(sc.width, sc.height)
    rs = ref_built.RefScene(sc, variant="record")
    rgbw, lsq, _ = rs.render()
    assert np.array_equal(f[..., 3], rgbw[..., 3])
    rate = z_test(f, rgbw, lsq)
    assert rate >= 0.997, rate
    # and the frame means agree tightly
    a = f[..., :3].sum((0, 1)) / f[..., 3].sum()
    b = rgbw[..., :3].sum((0, 1)) / rgbw[..., 3].sum()
    assert np.all(np.abs(a - b) <= 1e-3 * np.maximum(b, 1e-3)), (a, b)


def test_marschner_mode_against_restatement(renderer):
    """The Marschner R/TT/TRT lobes (dead code in the reference) against the
    CPU restatement of that code in float."""
    from oracle import restatebind as P
    sc = S.hair(96, 54, 4, 10, n_strands=20000, hair_mode=1)
    renderer.upload(sc)
    renderer.render_scene(sc)
    f = renderer.film(sc.width, sc.height)
    rgbw, lsq = P.PoScene(sc, 32).render()
    rate = z_test(f, rgbw, lsq)
    assert rate >= 0.99, rate


def test_progressive_accumulation(renderer):
    """sampleStart/sampleCount semantics (IIntegrator::renderFrame): two
    passes of 8 spp accumulate to one pass of 16."""
    sc = S.cornell(64, 64, 16)
    renderer.upload(sc)
    renderer.render(64, 64, 8, 8, sample_start=0, clear=True)
    renderer.render(64, 64, 8, 8, sample_start=8, clear=False)
    two = renderer.film(64, 64)
    renderer.render(64, 64, 16, 8, sample_start=0, clear=True)
    one = renderer.film(64, 64)
    assert np.array_equal(two[..., 3], one[..., 3])
    assert np.allclose(two[..., :3], one[..., :3], rtol=1e-4, atol=1e-5)
    assert np.allclose(two[..., 4], one[..., 4], rtol=1e-4, atol=1e-5)


def test_render_errors(gpu):
    r = api.Renderer()
    with pytest.raises(api.AnaError) as e:
        r.render(64, 64, 4, 8)
    assert e.value.code == api.ANA_ERR_STATE
    r.upload(S.cornell(16, 16, 1))
    with pytest.raises(api.AnaError) as e:
        r.render(16, 16, 0, 8)
    assert e.value.code == api.ANA_ERR_INVALID_ARG
    with pytest.raises(api.AnaError) as e:
        r.render(16, 16, 1, 999)
    assert e.value.code == api.ANA_ERR_INVALID_ARG
    r.render(16, 16, 1, 8)
    with pytest.raises(api.AnaError):
        r.film(8, 8)
    r.close()


def test_rmse_against_fp64_oracle(renderer):
    """RMSE of the GPU image against the FP64 converged image of the
    restatement (tests/golden/cornell128_fp64.npz) equals the reference CPU
    image's RMSE at the same spp, and falls as 1/sqrt(spp)."""
    g = np.load(os.path.join(HERE, "golden", "cornell128_fp64.npz"))
    conv = g["image"]
    sc = S.cornell(128, 128, 16)
    renderer.upload(sc)

    def rmse(img):
        return float(np.sqrt(np.mean((img - conv) ** 2)))

    renderer.render_scene(sc)
    e16 = rmse(renderer.image(128, 128))
    assert abs(e16 - float(g["ref_rmse_16spp"])) <= 0.02 * float(g["ref_rmse_16spp"])
    renderer.render(128, 128, 1024, 8)
    e1024 = rmse(renderer.image(128, 128))
    assert e1024 < e16 / 4.0, (e16, e1024)
