"""DirectionalLight (src/shading/lights/DirectionalLight.h) next to an area
light: per-sample radiance against PathIntegrator::Li of the same (pixel,
sample) — which also checks that the BSDF-sampling branch of estimateDirect,
and its sample dimensions, are skipped exactly when the delta light is picked
(PathIntegrator.cpp:210) — and the per-pixel z-test of whole frames, hard and
soft (cone) shadows."""
import numpy as np
import pytest

from anacapa_b200 import api
from anacapa_b200 import scenes as S

from test_gpu_render import z_test

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def renderer(gpu):
    r = api.Renderer()
    yield r
    r.close()


@pytest.mark.parametrize("half_angle", [0.0, 2.0], ids=["hard", "cone"])
def test_per_sample_radiance_matches_reference(renderer, ref_built, half_angle):
    sc = S.sunlit(96, 72, 1, 8, half_angle_deg=half_angle)
    renderer.upload(sc)
    rng = np.random.default_rng(7)
    q = np.stack([rng.integers(0, sc.width, 400), rng.integers(0, sc.height, 400),
                  rng.integers(0, 4, 400)], 1).astype(np.uint32)
    got = np.zeros((len(q), 3), np.float32)
    for s in np.unique(q[:, 2]):
        renderer.render(sc.width, sc.height, 1, sc.max_depth, sample_start=int(s))
        img = renderer.image(sc.width, sc.height)
        sel = q[:, 2] == s
        got[sel] = img[q[sel, 1], q[sel, 0]]
    ref = ref_built.RefScene(sc, variant="nocontract").li(q)
    close = np.all(np.abs(got - ref) <= 1e-4 * np.maximum(np.abs(ref), 1.0), axis=1)
    assert close.mean() >= 0.95, close.mean()


@pytest.mark.parametrize("half_angle", [0.0, 2.0], ids=["hard", "cone"])
def test_frame_z_test(renderer, ref_built, half_angle):
    sc = S.sunlit(128, 96, 16, 8, half_angle_deg=half_angle)
    renderer.upload(sc)
    renderer.render_scene(sc)
    film = renderer.film(sc.width, sc.height)
    rgbw, lsq, _ = ref_built.RefScene(sc, variant="nocontract").render()
    assert z_test(film, rgbw, lsq) >= 0.997
