"""Glass and alpha masks (src/shading/StandardSurface.h:197-438): smooth and
rough dielectric transmission, tinted shadow rays and MIS rays stepping
through transmissive surfaces (src/integrator/ShadowRay.h:26-61,
PathIntegrator.cpp:214-259), and stochastic alpha testing that draws a sample
dimension only for partial opacity (PathIntegrator.cpp:103-118). Per-sample
radiance against PathIntegrator::Li of the same (pixel, sample), whole frames
by the per-pixel z-test, the drop-in against the direct render."""
import dataclasses

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


def per_sample(renderer, sc, q):
    got = np.zeros((len(q), 3), np.float32)
    for s in np.unique(q[:, 2]):
        renderer.render(sc.width, sc.height, 1, sc.max_depth, sample_start=int(s))
        img = renderer.image(sc.width, sc.height)
        sel = q[:, 2] == s
        got[sel] = img[q[sel, 1], q[sel, 0]]
    return got


def test_per_sample_radiance_matches_reference(renderer, ref_built):
    sc = S.glass(96, 72, 1, 8)
    renderer.upload(sc)
    rng = np.random.default_rng(11)
    q = np.stack([rng.integers(0, sc.width, 600), rng.integers(0, sc.height, 600),
                  rng.integers(0, 4, 600)], 1).astype(np.uint32)
    got = per_sample(renderer, sc, q)
    ref = ref_built.RefScene(sc, variant="nocontract").li(q)
    close = np.all(np.abs(got - ref) <= 1e-4 * np.maximum(np.abs(ref), 1.0), axis=1)
    assert close.mean() >= 0.95, close.mean()


def test_alpha_cutout_draws_no_sample_dimension(renderer, ref_built):
    """Opacity 0 passes every ray without a sampler draw and opacity 1 tests
    none: with the partial card made fully cut out, or fully opaque, paths
    still match sample for sample (the dimension bookkeeping is exact)."""
    base = S.glass(64, 48, 1, 6)
    for opacity in (0.0, 1.0):
        mats = [dataclasses.replace(m, opacity=opacity) if m.alpha_mask and m.opacity > 0.0 else m
                for m in base.materials]
        sc = dataclasses.replace(base, materials=mats)
        renderer.upload(sc)
        rng = np.random.default_rng(3)
        q = np.stack([rng.integers(0, sc.width, 300), rng.integers(0, sc.height, 300),
                      rng.integers(0, 3, 300)], 1).astype(np.uint32)
        got = per_sample(renderer, sc, q)
        ref = ref_built.RefScene(sc, variant="nocontract").li(q)
        close = np.all(np.abs(got - ref) <= 1e-4 * np.maximum(np.abs(ref), 1.0), axis=1)
        assert close.mean() >= 0.95, (opacity, close.mean())


def test_frame_z_test(renderer, ref_built):
    sc = S.glass(128, 96, 16, 8)
    renderer.upload(sc)
    renderer.render_scene(sc)
    film = renderer.film(sc.width, sc.height)
    rgbw, lsq, _ = ref_built.RefScene(sc, variant="nocontract").render()
    assert z_test(film, rgbw, lsq) >= 0.997


def test_batch_with_an_opaque_scene(gpu):
    """A glass scene batched with an opaque one: the stepping shadow and MIS
    kernels serve the whole batch and give the opaque scene the film the
    any-hit kernels give it alone."""
    a, b = S.glass(64, 48, 4, 6), S.sunlit(64, 48, 4, 6)
    pa, pb = api.Prepared(a), api.Prepared(b)
    r = api.Renderer()
    try:
        r.upload(pb)
        r.render_scene(b)
        alone = r.film(b.width, b.height)
        r.upload_batch(api.Batch([pa, pb]))
        r.render_batch([api.scene_desc_tuple(a), api.scene_desc_tuple(b)])
        both = r.batch_film(1, b.width, b.height)
    finally:
        r.close()
    assert np.array_equal(both[..., 3], alone[..., 3])
    assert np.allclose(both, alone, rtol=1e-6, atol=1e-7)


def test_adjoint_rejects_glass(renderer):
    sc = S.glass(32, 24, 1, 4)
    renderer.upload(sc)
    with pytest.raises(api.AnaError, match="glass"):
        renderer.forward(sc.width, sc.height, 1, sc.max_depth)
