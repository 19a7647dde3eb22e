"""The C ABI boundary without a GPU: the library loads, exports every symbol
include/anacapa_b200.h declares, and the host-side scene preparation (BVH
builds, validation, error codes) behaves."""
import ctypes as C
import dataclasses
import os
import re

import numpy as np
import pytest

from anacapa_b200 import api
from anacapa_b200 import scenes as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "anacapa_b200.h")).read()
    return sorted(set(re.findall(r"\b(ana_[a-z_0-9]+)\s*\(", src)))


def test_header_declares_what_the_binding_lists():
    assert declared_symbols() == sorted(api.EXPORTS)


def test_library_exports_every_declared_symbol(lib_built):
    for name in declared_symbols():
        assert hasattr(lib_built, name), name
    assert lib_built.ana_version() >= 100


def test_struct_layouts_match_header(lib_built):
    # the sizes the binding assumes for the structs it passes by pointer
    assert C.sizeof(api.AnaFilmPixel) == 20
    assert C.sizeof(api.AnaHit) == 32
    assert C.sizeof(api.AnaRenderDesc) == 40


def _no_cuda():
    try:
        import torch
        return not torch.cuda.is_available()
    except Exception:
        return True


@pytest.mark.skipif(not _no_cuda(), reason="checks the no-device error path")
def test_create_without_device_fails_cleanly(lib_built):
    h = C.c_void_p()
    rc = lib_built.ana_create(C.byref(h), None)
    assert rc == api.ANA_ERR_CUDA and not h.value
    assert "CUDA" in api.last_error() or "device" in api.last_error()


def test_prepare_valid_scenes(lib_built):
    p = api.Prepared(S.cornell())
    assert p.nbytes > 36 * (48 + 64)
    p = api.Prepared(S.hair(64, 36, 1, n_strands=500))
    assert p.nbytes > 2000 * 80
    p = api.Prepared(S.throughput(64, 36, 1, 2, n_spheres=16, subdiv=1))
    assert p.nbytes > 16 * 80 * 48


def _prepare_rc(sc, **kw):
    d = api.SceneDesc(sc, **kw)
    h = C.c_void_p()
    rc = api.lib().ana_prepare_scene(C.byref(d.desc), C.byref(h))
    if h.value:
        api.lib().ana_prepared_free(h)
    return rc


def test_prepare_rejects_bad_input(lib_built):
    sc = S.cornell()
    bad = S.cornell()
    bad.indices = bad.indices.copy()
    bad.indices[0, 0] = 99
    assert _prepare_rc(bad) == api.ANA_ERR_INVALID_ARG
    assert "index" in api.last_error()
    bad = S.cornell()
    bad.positions = bad.positions.copy()
    bad.positions[3, 1] = np.nan
    assert _prepare_rc(bad) == api.ANA_ERR_INVALID_ARG
    bad = S.cornell()
    bad.slots = list(bad.slots)
    bad.slots[0] = 17
    assert _prepare_rc(bad) == api.ANA_ERR_INVALID_ARG
    glass = S.cornell()
    glass.materials = list(glass.materials)
    glass.materials[0] = S.Material(S.MAT_STANDARD, transmission=1.0, roughness=0.0)
    assert _prepare_rc(glass) == api.ANA_OK
    weird = S.cornell()
    weird.materials = list(weird.materials)
    weird.materials[0] = dataclasses.replace(weird.materials[0], type=7)
    assert _prepare_rc(weird) == api.ANA_ERR_INVALID_ARG
    assert _prepare_rc(sc, max_leaf_tris=65) == api.ANA_ERR_INVALID_ARG
    assert _prepare_rc(sc, max_leaf_tris=8) == api.ANA_OK
    h = C.c_void_p()
    assert api.lib().ana_prepare_scene(None, C.byref(h)) == api.ANA_ERR_INVALID_ARG


def test_prepare_is_deterministic(lib_built):
    sc = S.throughput(64, 36, 1, 2, n_spheres=64, subdiv=2)
    a = api.Prepared(sc)
    b = api.Prepared(sc)
    assert a.nbytes == b.nbytes
    # identical layouts: the parallel subtree build does not change the result
    L = api.lib()
    assert L.ana_prepared_digest(a.h) == L.ana_prepared_digest(b.h) != 0
    c = api.Prepared(sc, max_leaf_tris=8)
    assert L.ana_prepared_digest(c.h) != L.ana_prepared_digest(a.h)


def test_calls_on_null_context_are_rejected(lib_built):
    L = lib_built
    assert L.ana_render(None, None) == api.ANA_ERR_INVALID_ARG
    assert L.ana_trace_batch(None, None, 0, None, 0, 0) == api.ANA_ERR_INVALID_ARG
    assert L.ana_film_read(None, None, 0) == api.ANA_ERR_INVALID_ARG
    st = api.AnaStats()
    assert L.ana_get_stats(None, C.byref(st)) == api.ANA_ERR_INVALID_ARG


def test_prepare_motion_meshes(lib_built):
    """Motion keys (MeshDesc::motionKeys): a scene with keys prepares; a
    non-finite key is rejected; the time-expanded bounds make the layout
    differ from the same scene with the keys removed."""
    sc = S.motion(32, 24, 1)
    assert _prepare_rc(sc) == api.ANA_OK
    static = dataclasses.replace(sc, mesh_motion=None)
    assert api.Prepared(sc).digest != api.Prepared(static).digest
    keys = [list(k) if k else k for k in sc.mesh_motion]
    t, M = keys[1][0]
    M = np.array(M, np.float32)
    M[0, 3] = np.nan
    keys[1][0] = (t, M)
    assert _prepare_rc(dataclasses.replace(sc, mesh_motion=keys)) == api.ANA_ERR_INVALID_ARG
    assert "motion key" in api.last_error()


def test_prepare_glass_and_alpha_materials(lib_built):
    """Transmission and alpha masks prepare (glass lobes, tinted shadow rays);
    the layout depends on the opacity of an alpha-masked material."""
    sc = S.glass(32, 24, 1)
    assert _prepare_rc(sc) == api.ANA_OK
    mats = [dataclasses.replace(m, opacity=0.7) if m.alpha_mask and m.opacity > 0 else m for m in sc.materials]
    assert api.Prepared(sc).digest != api.Prepared(dataclasses.replace(sc, materials=mats)).digest
