"""Denoising AOVs and film output on the device (PathIntegrator::renderTile's
first-hit albedo / normal, PathIntegrator.cpp:31-66, 120-124; Film::mergeTile
and Film::writeEXR / writePNG, Film.cpp:34-272): the AOV film against the
reference's tile loop, AOV accumulation across passes, the state rule, the
EXR / PNG written from the device film, and the drop-in writing through the
reference Film's own writers."""
import numpy as np
import pytest

from anacapa_b200 import api
from anacapa_b200 import scenes as S

from test_film_io import parse_exr

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def renderer(gpu):
    r = api.Renderer()
    yield r
    r.close()


def resolve(acc):
    w = acc[..., 3:4]
    return np.where(w > 0, acc[..., :3] * (1.0 / np.where(w > 0, w, 1.0)), 0.0).astype(np.float32)


CASES = {
    "cornell": lambda: S.cornell(64, 64, 8),
    "hair": lambda: S.hair(96, 54, 4, 10, n_strands=5000),
    "glass_alpha": lambda: S.glass(96, 72, 8),
    "motion": lambda: S.motion(96, 72, 8),
}


@pytest.mark.parametrize("case", list(CASES))
def test_aovs_match_reference(renderer, ref_built, case):
    sc = CASES[case]()
    renderer.upload(sc)
    renderer.render_scene(sc, aovs=True)
    al, nr = renderer.aovs(sc.width, sc.height)
    ral, rnr = ref_built.RefScene(sc, variant="nocontract").render_aov()
    ral, rnr = resolve(ral), resolve(rnr)
    # first hits are the reference's; the albedo is exact up to float rounding
    # of the material's reflectance, the normal up to the shading rounding
    close_a = np.all(np.abs(al - ral) <= 1e-5 * np.maximum(np.abs(ral), 1e-3), axis=-1)
    close_n = np.all(np.abs(nr - rnr) <= 1e-4, axis=-1)
    assert close_a.mean() >= 0.995, close_a.mean()
    assert close_n.mean() >= 0.99, close_n.mean()
    assert np.abs(ral).sum() > 0 and np.abs(rnr).sum() > 0


def test_aov_passes_accumulate_and_state_rule(renderer):
    sc = S.cornell(32, 32, 4)
    renderer.upload(sc)
    renderer.render(32, 32, 4, sc.max_depth, aovs=True)
    a1, n1 = renderer.aovs(32, 32)
    renderer.render(32, 32, 4, sc.max_depth, sample_start=4, clear=False, aovs=True)
    a2, n2 = renderer.aovs(32, 32)
    renderer.render(32, 32, 4, sc.max_depth, sample_start=4, aovs=True)
    b1, _ = renderer.aovs(32, 32)
    # two passes: the mean of the two per-pass averages (weight 1 each)
    assert np.allclose(a2, (a1 + b1) * 0.5, rtol=1e-6, atol=1e-7)
    # a pass without AOVs leaves the AOV film behind the beauty film
    renderer.render(32, 32, 4, sc.max_depth, sample_start=8, clear=False)
    with pytest.raises(api.AnaError, match="AOV"):
        renderer.aovs(32, 32)
    with pytest.raises(api.AnaError, match="AOV"):
        renderer.render(32, 32, 4, sc.max_depth, sample_start=12, clear=False, aovs=True)


def test_device_film_writers(renderer, tmp_path):
    Image = pytest.importorskip("PIL.Image")
    sc = S.sunlit(80, 60, 8)
    renderer.upload(sc)
    renderer.render_scene(sc, aovs=True)
    img = renderer.image(sc.width, sc.height)
    al, nr = renderer.aovs(sc.width, sc.height)
    renderer.write_exr(tmp_path / "f.exr", sc.width, sc.height, aovs=True)
    ch = parse_exr(tmp_path / "f.exr")
    rgb = np.stack([ch["R"], ch["G"], ch["B"]], -1)
    assert np.allclose(rgb, img, rtol=1e-6, atol=0)
    assert np.array_equal(np.stack([ch["albedo.R"], ch["albedo.G"], ch["albedo.B"]], -1), al)
    assert np.array_equal(np.stack([ch["normals.R"], ch["normals.G"], ch["normals.B"]], -1), nr)
    renderer.write_png(tmp_path / "f.png", sc.width, sc.height, exposure=1.0)
    png = np.asarray(Image.open(tmp_path / "f.png").convert("RGB"))
    assert png.shape == (sc.height, sc.width, 3) and png.max() > 0


def test_dropin_writes_through_reference_film(gpu, ref_built, tmp_path):
    if not ref_built.available("dropin"):
        pytest.skip("drop-in check library not built")
    import dataclasses
    sc = S.sunlit(80, 60, 8)
    rs = ref_built.RefScene(sc, variant="dropin")
    rs.dropin_write(tmp_path / "d.exr", tmp_path / "d.png", spp=4, passes=2, exposure=0.5)
    ch = parse_exr(tmp_path / "d.exr")
    sc = dataclasses.replace(sc, cam_basis=rs.camera_basis())
    r = api.Renderer()
    try:
        r.upload(sc)
        r.render(sc.width, sc.height, 4, sc.max_depth, aovs=True)
        r.render(sc.width, sc.height, 4, sc.max_depth, sample_start=4, clear=False, aovs=True)
        img = r.image(sc.width, sc.height)
        al, nr = r.aovs(sc.width, sc.height)
    finally:
        r.close()
    rgb = np.stack([ch["R"], ch["G"], ch["B"]], -1)
    assert np.allclose(rgb, img, rtol=1e-4, atol=1e-4)
    assert np.allclose(np.stack([ch["albedo.R"], ch["albedo.G"], ch["albedo.B"]], -1), al, rtol=1e-5, atol=1e-6)
    assert np.allclose(np.stack([ch["normals.R"], ch["normals.G"], ch["normals.B"]], -1), nr, rtol=1e-4,
                       atol=1e-5)
    assert (tmp_path / "d.png").exists()


def test_tiles_carry_aovs(renderer):
    """ana_render_tiles with ANA_RENDER_AOVS: tiles that cover the frame once
    give every pixel the AOVs of a whole-frame pass (each tile's average,
    weight 1, as renderTile and Film::mergeTile produce them)."""
    sc = S.cornell(96, 80, 4)
    renderer.upload(sc)
    renderer.render_scene(sc, aovs=True)
    a0, n0 = renderer.aovs(sc.width, sc.height)
    tiles = [(x, y, min(32, sc.width - x), min(32, sc.height - y), 0, sc.spp)
             for y in range(0, sc.height, 32) for x in range(0, sc.width, 32)]
    renderer.render_tiles(sc.width, sc.height, sc.max_depth, tiles, clear=True, aovs=True)
    a1, n1 = renderer.aovs(sc.width, sc.height)
    assert np.array_equal(a0, a1) and np.array_equal(n0, n1)
