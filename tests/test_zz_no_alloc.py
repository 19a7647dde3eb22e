"""ana_trace_batch_noalloc: the trace query staged in the library's fixed
device scratch instead of a per-call device allocation. Each case compares it,
through the C ABI, with ana_trace_batch on the same rays, over two calls in a
row (the second call must not see anything the first left in the scratch).

The file sorts last so that it runs after every other GPU test has used the
device; it also passes alone in a fresh process."""
import os

import numpy as np
import pytest

from anacapa_b200 import api
from anacapa_b200 import scenes as S

pytestmark = pytest.mark.gpu

FIELDS = ("hit", "mesh_id", "prim_id", "strand_id")


def seeded_rays(seed, n, lo, hi, tmax=np.inf):
    rng = np.random.default_rng(seed)
    r = np.zeros((n, 8), np.float32)
    r[:, :3] = rng.uniform(lo, hi, (n, 3))
    d = rng.normal(size=(n, 3))
    r[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    r[:, 3] = 1e-4
    r[:, 7] = tmax
    return r


def same_hits(a, b):
    for f in FIELDS:
        assert np.array_equal(a[f], b[f]), f
    hit = a["hit"] == 1
    # the same kernel on the same rays: the tolerance is for form's sake
    for f in ("t", "u", "v"):
        np.testing.assert_allclose(a[f][hit], b[f][hit], rtol=1e-6, atol=0)


@pytest.fixture(scope="module", params=["cornell", "hair", "motion"])
def scene_renderer(gpu, request):
    """A static mesh scene, a curve scene, and a scene with motion-blurred
    meshes (whose traversal always takes the persistent schedule, with its work
    counter in the scratch); rays carry time 0 in both entry points."""
    r = api.Renderer()
    if request.param == "cornell":
        r.upload(S.cornell(64, 64, 1))
        lo, hi = 0.02, 0.98
    elif request.param == "hair":
        r.upload(S.hair(64, 36, 1, 4, n_strands=20000))
        lo, hi = -1.5, 1.5
    else:
        sc = S.motion(64, 36, 1, 4)
        r.upload(sc)
        lo, hi = float(sc.positions.min()), float(sc.positions.max())
    yield r, lo, hi
    r.close()


def test_noalloc_matches_trace_batch_twice(scene_renderer):
    r, lo, hi = scene_renderer
    a = seeded_rays(1, 50000, lo, hi)
    b = seeded_rays(2, 30000, lo, hi)
    first = r.trace_noalloc(a)
    second = r.trace_noalloc(b)
    same_hits(first, r.trace(a))
    same_hits(second, r.trace(b))
    # and the same rays twice in a row
    same_hits(r.trace_noalloc(a), first)


def test_noalloc_occlusion_twice(scene_renderer):
    r, lo, hi = scene_renderer
    a = seeded_rays(3, 40000, lo, hi, tmax=0.5)
    want = r.trace(a, occlusion=True)["hit"]
    for _ in range(2):
        assert np.array_equal(r.trace_noalloc(a, occlusion=True)["hit"], want)


def test_noalloc_full_scratch_then_small(scene_renderer):
    r, lo, hi = scene_renderer
    full = seeded_rays(4, api.TRACE_NOALLOC_MAX_RAYS, lo, hi)
    same_hits(r.trace_noalloc(full), r.trace(full))
    small = seeded_rays(5, 17, lo, hi)
    out = r.trace_noalloc(small)
    assert len(out) == 17
    same_hits(out, r.trace(small))


def test_noalloc_rejects_more_than_the_scratch(scene_renderer):
    r, lo, hi = scene_renderer
    too_many = seeded_rays(6, api.TRACE_NOALLOC_MAX_RAYS + 1, lo, hi)
    with pytest.raises(api.AnaError, match="exceed the fixed scratch") as e:
        r.trace_noalloc(too_many)
    assert e.value.code == api.ANA_ERR_INVALID_ARG
    # nothing ran, and the next call works
    ok = seeded_rays(7, 1000, lo, hi)
    same_hits(r.trace_noalloc(ok), r.trace(ok))


def test_noalloc_empty_and_no_scene(gpu):
    r = api.Renderer()
    try:
        with pytest.raises(api.AnaError) as e:
            r.trace_noalloc(seeded_rays(8, 4, 0.0, 1.0))
        assert e.value.code == api.ANA_ERR_STATE
        r.upload(S.cornell(16, 16, 1))
        assert len(r.trace_noalloc(np.zeros((0, 8), np.float32))) == 0
    finally:
        r.close()


def test_noalloc_matches_the_reference_goldens(gpu):
    """Closest hits of the committed reference rays on the Cornell scene
    (tests/golden/reference_vectors.npz, from the reference's BVHBackend)."""
    gold = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_vectors.npz"))
    r = api.Renderer()
    try:
        r.upload(S.cornell())
        for _ in range(2):
            h = r.trace_noalloc(gold["cornell_rays"])
            ids = np.stack([h["hit"], h["mesh_id"], h["prim_id"], h["strand_id"]], 1)
            assert np.array_equal(ids, gold["cornell_ids"])
            hit = gold["cornell_ids"][:, 0] == 1
            assert np.array_equal(h["t"][hit], gold["cornell_t"][hit])
    finally:
        r.close()


def test_noalloc_allocates_no_device_memory(scene_renderer):
    """After a first call (the scratch address looked up, every kernel
    loaded), further calls leave the device's free memory unchanged."""
    torch = pytest.importorskip("torch")
    r, lo, hi = scene_renderer
    rays = seeded_rays(9, 20000, lo, hi)
    r.trace_noalloc(rays)
    torch.cuda.synchronize()
    before = torch.cuda.mem_get_info()[0]
    for k in range(4):
        r.trace_noalloc(rays, occlusion=bool(k & 1))
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == before
