"""Host half of the drop-in (no device): B200PathIntegrator::prepareHost,
compiled against the reference's headers and fed the reference's own
SceneView, must build byte for byte the device layout that the C ABI builds
from the same scene description."""
import ctypes as C
import dataclasses

import pytest

from anacapa_b200 import api
from anacapa_b200 import scenes as S


def slot_ordered(sc: S.Scene) -> S.Scene:
    """The drop-in lists materials in order of first use by SceneView::materials
    (one entry per distinct material object); reorder the description to match."""
    order, remap = [], {}
    for m in sc.slots:
        if m >= 0 and m not in remap:
            remap[m] = len(order)
            order.append(sc.materials[m])
    return dataclasses.replace(sc, materials=order, slots=[remap[m] if m >= 0 else -1 for m in sc.slots])


@pytest.fixture(scope="module")
def dropin(lib_built, ref_built):
    if not ref_built.available("dropin"):
        pytest.skip("drop-in check library not built (needs the reference tree at build time)")
    return ref_built


@pytest.mark.parametrize("make", [lambda: S.cornell(128, 128, 8),
                                  lambda: S.hair(96, 54, 4, 10, n_strands=5000),
                                  lambda: S.throughput(96, 54, 4, 12, n_spheres=64),
                                  # the directional light is recovered by probing, an ulp
                                  # away from the description's: left out of the digest
                                  lambda: dataclasses.replace(S.glass(96, 72, 4), dir_lights=[]),
                                  lambda: S.motion(64, 48, 2)],
                         ids=["cornell", "hair", "throughput_small", "glass", "motion"])
def test_dropin_prepares_the_same_layout(dropin, make):
    sc = make()
    rs = dropin.RefScene(sc, variant="dropin")
    p = C.c_void_p(rs.dropin_prepare())
    try:
        L = api.lib()
        mine = api.Prepared(slot_ordered(sc))
        assert L.ana_prepared_bytes(p) == mine.nbytes
        assert L.ana_prepared_digest(p) == mine.digest
    finally:
        api.lib().ana_prepared_free(p)


def test_dropin_rejects_unsupported_content(dropin):
    sc = S.throughput(32, 32, 1, 4, n_spheres=8)
    rs = dropin.RefScene(sc, variant="dropin")
    with pytest.raises(RuntimeError, match="another film size"):
        rs.dropin_prepare(size=(48, 32))
