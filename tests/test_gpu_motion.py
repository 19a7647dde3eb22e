"""Motion blur (MeshDesc::motionKeys; BVHBackend.cpp:35-50, 86-95, 285-300,
356-367, 395-398, 420-435): object-space triangles bounded over their keys,
tested in object space against the world ray taken through the inverse of
the keys' interpolation at the ray's time, shaded through the forward
transform; every ray of a path carries the camera's shutter sample.
Hit identity at time 0 (traceBatch rays carry Ray::time's default), per-sample
radiance against PathIntegrator::Li, the per-pixel z-test of whole frames."""
import numpy as np
import pytest

from anacapa_b200 import api
from anacapa_b200 import scenes as S

from test_gpu_render import z_test
from test_gpu_trace import excluded_ties, gpu_ids, seeded_rays

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def renderer(gpu):
    r = api.Renderer()
    yield r
    r.close()


@pytest.mark.parametrize("occlusion", [False, True], ids=["closest", "any"])
def test_hits_at_time_zero_match_reference(renderer, ref_built, occlusion):
    sc = S.motion(64, 48, 1)
    rays = seeded_rays(5, 1 << 18, -2.5, 2.5)
    rays[:, 1] = np.abs(rays[:, 1])  # origins above the ground
    if occlusion:
        rays[:, 7] = np.random.default_rng(6).uniform(0.05, 4.0, len(rays)).astype(np.float32)
    renderer.upload(sc)
    g = renderer.trace(rays, occlusion=occlusion)
    rs = ref_built.RefScene(sc, variant="nocontract")
    if occlusion:
        assert np.array_equal(g["hit"] == 1, rs.occluded(rays))
        return
    ids, t = rs.trace(rays)
    same = (gpu_ids(g) == ids).all(1)
    bad = ~(same | excluded_ties(g, ids, t))
    assert not bad.any(), (bad.sum(), gpu_ids(g)[bad][:5], ids[bad][:5])
    hit = ids[:, 0] == 1
    assert np.array_equal(g["t"][hit & same], t[hit & same])
    moving = np.isin(ids[:, 1], [1, 2, 3, 4]) & hit
    assert moving.sum() > 1000


@pytest.mark.parametrize("occlusion", [False, True], ids=["closest", "any"])
def test_hits_at_ray_times_match_reference(renderer, ref_built, occlusion):
    """ana_trace_batch_timed: every ray at its own time in [-0.1, 1.1] (before
    the first key, between keys, after the last): hits bit for bit."""
    sc = S.motion(64, 48, 1)
    rays = seeded_rays(7, 1 << 18, -2.5, 2.5)
    rays[:, 1] = np.abs(rays[:, 1])
    times = np.random.default_rng(8).uniform(-0.1, 1.1, len(rays)).astype(np.float32)
    if occlusion:
        rays[:, 7] = np.random.default_rng(9).uniform(0.05, 4.0, len(rays)).astype(np.float32)
    renderer.upload(sc)
    g = renderer.trace(rays, occlusion=occlusion, times=times)
    rs = ref_built.RefScene(sc, variant="nocontract")
    if occlusion:
        assert np.array_equal(g["hit"] == 1, rs.occluded(rays, times=times))
        return
    ids, t = rs.trace(rays, times=times)
    same = (gpu_ids(g) == ids).all(1)
    bad = ~(same | excluded_ties(g, ids, t))
    assert not bad.any(), (bad.sum(), gpu_ids(g)[bad][:5], ids[bad][:5])
    hit = ids[:, 0] == 1
    assert np.array_equal(g["t"][hit & same], t[hit & same])
    # the times matter: at time 0 the moving meshes are hit elsewhere
    g0 = renderer.trace(rays)
    assert (gpu_ids(g0) != gpu_ids(g)).any(1).sum() > 100


@pytest.mark.parametrize("shutter", [(0.0, 1.0), (0.25, 0.75)], ids=["full", "half"])
def test_per_sample_radiance_matches_reference(renderer, ref_built, shutter):
    sc = S.motion(96, 72, 1, 6, shutter=shutter)
    renderer.upload(sc)
    rng = np.random.default_rng(13)
    q = np.stack([rng.integers(0, sc.width, 500), rng.integers(0, sc.height, 500),
                  rng.integers(0, 4, 500)], 1).astype(np.uint32)
    got = np.zeros((len(q), 3), np.float32)
    for s in np.unique(q[:, 2]):
        renderer.render(sc.width, sc.height, 1, sc.max_depth, sample_start=int(s))
        img = renderer.image(sc.width, sc.height)
        sel = q[:, 2] == s
        got[sel] = img[q[sel, 1], q[sel, 0]]
    ref = ref_built.RefScene(sc, variant="nocontract").li(q)
    close = np.all(np.abs(got - ref) <= 1e-4 * np.maximum(np.abs(ref), 1.0), axis=1)
    assert close.mean() >= 0.95, close.mean()


def test_frame_z_test(renderer, ref_built):
    sc = S.motion(128, 96, 16, 6)
    renderer.upload(sc)
    renderer.render_scene(sc)
    film = renderer.film(sc.width, sc.height)
    rgbw, lsq, _ = ref_built.RefScene(sc, variant="nocontract").render()
    assert z_test(film, rgbw, lsq) >= 0.997


def test_closed_shutter_and_adjoint_rejection(renderer):
    """A closed shutter (0, 0) renders every moving mesh at its first key;
    the differentiable pair rejects motion-blurred meshes."""
    sc = S.motion(64, 48, 4, 4, shutter=(0.0, 0.0))
    renderer.upload(sc)
    renderer.render_scene(sc)
    a = renderer.image(sc.width, sc.height)
    assert np.isfinite(a).all() and a.mean() > 0.01
    with pytest.raises(api.AnaError, match="motion"):
        renderer.forward(sc.width, sc.height, 1, sc.max_depth)
