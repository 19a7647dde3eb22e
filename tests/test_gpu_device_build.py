"""ana_upload_scene_device: BVHBackend::commit's triangle setup and SAH build
(src/accel/BVHBackend.cpp:17-228) and the 4-wide collapse run on the device
must upload the bytes the host path uploads (FNV-1a of the whole arena), and
render the same film."""
import time

import numpy as np
import pytest

from anacapa_b200 import api
from anacapa_b200 import scenes as S

pytestmark = pytest.mark.gpu


def one_triangle():
    sc = S.cornell(16, 16, 1)
    pos = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.2], [0.0, 1.0, 0.4]], np.float32)
    sc.positions = pos
    sc.normals = np.zeros_like(pos)
    sc.uvs = np.zeros((3, 2), np.float32)
    sc.indices = np.array([[0, 1, 2]], np.uint32)
    sc.mesh_vert_offset = np.array([0, 3], np.uint32)
    sc.mesh_tri_offset = np.array([0, 1], np.uint32)
    sc.mesh_has_normals = np.zeros(1, np.uint8)
    sc.slots = [sc.slots[0]]
    return sc


CASES = {
    "cornell": lambda: S.cornell(),
    "throughput_small": lambda: S.throughput(96, 54, 4, 12, n_spheres=256),
    "hair_curves_on_host": lambda: S.hair(96, 54, 4, 10, n_strands=2000),
    "glass": lambda: S.glass(96, 72, 4),
    "leaf_size_8": lambda: S.throughput(64, 36, 1, 4, n_spheres=64, subdiv=2),
    "one_triangle_root_leaf": one_triangle,
}


@pytest.mark.parametrize("case", list(CASES))
def test_device_build_uploads_the_host_bytes(gpu, case):
    sc = CASES[case]()
    kw = {"max_leaf_tris": 8} if case == "leaf_size_8" else {}
    host = api.Prepared(sc, **kw)
    r = api.Renderer()
    try:
        r.upload(sc, device_build=True, **kw)
        assert r.scene_digest() == host.digest
        r.upload(host)
        assert r.scene_digest() == host.digest
    finally:
        r.close()


def test_device_build_renders_the_same_film(gpu):
    sc = S.sunlit(96, 72, 4)
    r = api.Renderer()
    try:
        r.upload(sc)
        r.render_scene(sc)
        a = r.film(sc.width, sc.height)
        r.upload(sc, device_build=True)
        r.render_scene(sc)
        b = r.film(sc.width, sc.height)
    finally:
        r.close()
    assert np.array_equal(a, b)


def test_device_build_full_throughput_scene(gpu):
    """5,242,882 triangles: the same bytes, built in a fraction of the host time."""
    sc = S.throughput()
    t0 = time.perf_counter()
    host = api.Prepared(sc)
    t_host = time.perf_counter() - t0
    r = api.Renderer()
    try:
        r.upload(sc, device_build=True)  # first call: context warm-up
        t0 = time.perf_counter()
        r.upload(sc, device_build=True)
        t_dev = time.perf_counter() - t0
        assert r.scene_digest() == host.digest
    finally:
        r.close()
    print(f"host prepare {t_host:.3f} s, device upload {t_dev:.3f} s")
    assert t_dev < t_host


def test_device_build_rejects_bad_meshes(gpu):
    bad = S.cornell()
    bad.indices = bad.indices.copy()
    bad.indices[5, 1] = 10_000
    r = api.Renderer()
    try:
        with pytest.raises(api.AnaError, match="index"):
            r.upload(bad, device_build=True)
        nan = S.cornell()
        nan.positions = nan.positions.copy()
        nan.positions[7, 2] = np.nan
        with pytest.raises(api.AnaError, match="non-finite"):
            r.upload(nan, device_build=True)
    finally:
        r.close()
