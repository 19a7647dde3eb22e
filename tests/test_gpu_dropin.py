"""The drop-in: B200PathIntegrator (anacapa_b200/host) compiled against the
reference's own headers, driven through the reference's SceneView and Film
exactly as RenderSession::render's non-adaptive branch drives an IIntegrator
(prepare, then renderFrame with sampleStart/sampleCount)."""
import dataclasses

import numpy as np
import pytest

from anacapa_b200 import api
from anacapa_b200 import scenes as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dropin(gpu, ref_built):
    if not ref_built.available("dropin"):
        pytest.skip("drop-in check library not built (needs the reference tree at build time)")
    return ref_built


@pytest.mark.parametrize("make", [lambda: S.cornell(128, 128, 8),
                                  lambda: S.hair(96, 54, 4, 10, n_strands=5000),
                                  lambda: S.throughput(96, 54, 4, 12, n_spheres=64),
                                  lambda: S.sunlit(96, 72, 8),
                                  lambda: S.glass(96, 72, 8),
                                  lambda: S.motion(96, 72, 8)],
                         ids=["cornell", "hair", "throughput_small", "sunlit", "glass", "motion"])
def test_dropin_matches_direct_render(dropin, make):
    sc = make()
    rs = dropin.RefScene(sc, variant="dropin")
    # two progressive renderFrame passes of spp/2 samples each
    rgb, var = rs.dropin_render(spp=sc.spp // 2, passes=2)
    # the direct render gets the Camera the reference build computed (its
    # basis carries that build's rounding), which the drop-in passes on
    sc = dataclasses.replace(sc, cam_basis=rs.camera_basis())
    r = api.Renderer()
    r.upload(sc)
    r.render_scene(sc)
    direct = r.image(sc.width, sc.height)
    r.close()
    # DirectionalLight normalises its direction in float and prepare
    # normalises the probed direction again, one ulp away from the direct
    # scene's single normalisation: that case gets a 1e-4 band.
    tol = (1e-4, 1e-4) if sc.dir_lights else (1e-5, 1e-6)
    assert np.allclose(rgb, direct, rtol=tol[0], atol=tol[1]), np.abs(rgb - direct).max()
    assert np.isfinite(var).all() and (var >= 0).all()
