"""Tiles and the adaptive two-pass schedule (ana_render_tiles,
ana_render_adaptive): RenderSession::render's tile-adaptive branch for a
tile-rendering integrator (src/render/RenderSession.cpp:548-653) with
PathIntegrator::renderTile (src/integrator/PathIntegrator.cpp:8-69).

Bars: tiles that cover a frame give the whole-frame film bit for bit; the
per-tile sample allocation equals a numpy restatement of the reference's
formula evaluated on the same base-pass film; the adaptive image passes the
per-pixel 3-sigma z-test against the reference CPU integrator rendering the
same tiles and sample ranges."""
import math

import numpy as np
import pytest

from anacapa_b200 import api
from anacapa_b200 import scenes as S

from test_gpu_render import z_test

pytestmark = pytest.mark.gpu


def tiles_of(W, H, ts, start, count):
    return [(x, y, min(ts, W - x), min(ts, H - y), start, count) for y in range(0, H, ts) for x in range(0, W, ts)]


def allocation(film, W, H, ts, extra):
    """The reference's allocation (RenderSession.cpp:590-634) in float32, in
    its order of operations: tile mean of Film::varianceAt, log(1 + v)
    weights, a uniform half and a variance-weighted half of the extra samples."""
    f = film.reshape(H, W, 5).astype(np.float32)
    one = np.float32(1.0)
    logw = []
    for (x, y, w, h, _, _) in tiles_of(W, H, ts, 0, 0):
        s = np.float32(0.0)
        for ty in range(h):
            for tx in range(w):
                r, g, b, wt, lsq = f[y + ty, x + tx]
                if wt <= 0:
                    v = np.float32(0.0)
                else:
                    inv = one / wt
                    mean = (r * np.float32(0.2126) + g * np.float32(0.7152) + b * np.float32(0.0722)) * inv
                    v = max(np.float32(0.0), lsq * inv - mean * mean)
                s = np.float32(s + v)
        logw.append(np.log(one + s / np.float32(w * h)))
    total = np.float32(0.0)
    for v in logw:
        total = np.float32(total + v)
    uniform, bonus_half = extra // 2, extra - extra // 2
    out = []
    for v in logw:
        # std::round: halves away from zero
        bonus = math.floor(float(np.float32(v / total) * np.float32(bonus_half * len(logw))) + 0.5) \
            if total > 1e-6 else 0
        out.append(min(uniform + bonus, extra))
    return np.array(out, np.uint32)


@pytest.fixture(scope="module")
def cornell(gpu):
    sc = S.cornell(96, 80, 8, 8)
    r = api.Renderer()
    r.upload(sc)
    yield r, sc
    r.close()


def test_tiles_covering_the_frame_equal_the_frame(cornell):
    r, sc = cornell
    r.render_scene(sc)
    whole = r.film(sc.width, sc.height)
    r.render_tiles(sc.width, sc.height, sc.max_depth, tiles_of(sc.width, sc.height, 32, 0, sc.spp), clear=True)
    assert np.array_equal(r.film(sc.width, sc.height), whole)


def test_tile_passes_accumulate(cornell):
    r, sc = cornell
    r.render_scene(sc)
    whole = r.film(sc.width, sc.height)
    half = sc.spp // 2
    r.render_tiles(sc.width, sc.height, sc.max_depth, tiles_of(sc.width, sc.height, 32, 0, half), clear=True)
    r.render_tiles(sc.width, sc.height, sc.max_depth, tiles_of(sc.width, sc.height, 32, half, sc.spp - half))
    np.testing.assert_allclose(r.film(sc.width, sc.height), whole, rtol=2e-5, atol=1e-6)


def test_tiles_are_validated(cornell):
    r, sc = cornell
    with pytest.raises(api.AnaError, match="overlap"):
        r.render_tiles(sc.width, sc.height, 4, [(0, 0, 16, 16, 0, 1), (8, 8, 16, 16, 0, 1)])
    with pytest.raises(api.AnaError, match="outside"):
        r.render_tiles(sc.width, sc.height, 4, [(90, 0, 16, 16, 0, 1)])


def test_adaptive_allocation_and_image(cornell, ref_built):
    r, sc = cornell
    W, H, spp, ts = 128, 128, 64, 32
    scene = S.cornell(W, H, spp, 8)
    r.upload(scene)
    try:
        extra = r.render_adaptive(W, H, spp, scene.max_depth, tile_size=ts)
        adaptive = r.film(W, H)
        base = min(32, max(16, spp // 16))
        # the allocation from the same base film
        r.render(W, H, base, scene.max_depth)
        want = allocation(r.film(W, H), W, H, ts, spp - base)
        assert np.array_equal(extra, want), (extra, want)
        assert extra.min() >= (spp - base) // 2 and extra.max() <= spp - base and len(set(extra.tolist())) > 1
        # the adaptive film is the base pass plus those tiles
        r.render_tiles(W, H, scene.max_depth, [t[:4] + (base, int(e)) for t, e in
                                               zip(tiles_of(W, H, ts, 0, 0), extra)])
        assert np.array_equal(r.film(W, H), adaptive)
        # the reference CPU integrator on the same tiles and sample ranges
        rs = ref_built.RefScene(scene, variant="nocontract")
        rgbw = np.zeros((H, W, 4), np.float64)
        lsq = np.zeros((H, W), np.float64)
        for (x, y, w, h, _, _), e in zip(tiles_of(W, H, ts, 0, 0), extra):
            for start, count in ((0, base), (base, int(e))):
                if count:
                    a, b, _ = rs.render(spp=count, sample_start=start, rect=(x, y, x + w, y + h))
                    rgbw += a
                    lsq += b
        assert z_test(adaptive, rgbw, lsq) >= 0.997
    finally:
        r.upload(sc)
