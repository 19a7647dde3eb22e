"""TEST INFRASTRUCTURE — ctypes binding of oracle/_ref/libanacapa_ref*.so.

The library is the reference renderer's own hot-path code (compiled from its
sources by oracle/Makefile) plus oracle/ref_harness.cpp. Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg use it, as the checker
and as the timed CPU baseline; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_P = C.c_void_p
_F = C.POINTER(C.c_float)
_U32 = C.POINTER(C.c_uint32)
_I32 = C.POINTER(C.c_int32)
_U8 = C.POINTER(C.c_uint8)


def _fp(a):
    return a.ctypes.data_as(_F) if a is not None else None


def build(reference=None, quiet=True):
    """Compile the reference variants and, when the CUDA library exists, the
    drop-in check from the reference tree at `reference` (default: the
    ANACAPA_REFERENCE environment variable). Without a tree it only reports
    whether the libraries are already built."""
    libs = [os.path.join(REF_DIR, n) for n in ("libanacapa_ref.so", "libanacapa_ref_nocontract.so")]
    reference = reference or os.environ.get("ANACAPA_REFERENCE")
    if not reference or not os.path.isdir(reference):
        return all(os.path.exists(p) for p in libs)
    subprocess.run(["make", "-C", HERE, "ref", f"REF={reference}"], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)
    if os.path.exists(os.path.join(os.path.dirname(HERE), "anacapa_b200", "libanacapa_b200.so")):
        subprocess.run(["make", "-C", HERE, "dropin", f"REF={reference}"], check=True,
                       stdout=subprocess.DEVNULL if quiet else None)
    return True


def available(variant="record"):
    return os.path.exists(_libpath(variant))


def _libpath(variant):
    return os.path.join(REF_DIR, {"record": "libanacapa_ref.so",
                                  "nocontract": "libanacapa_ref_nocontract.so",
                                  "dropin": "libanacapa_ref_dropin.so"}[variant])


_LIBS = {}


def lib(variant="record"):
    if variant in _LIBS:
        return _LIBS[variant]
    L = C.CDLL(_libpath(variant))
    L.ref_scene_new.restype = _P
    L.ref_scene_free.argtypes = [_P]
    L.ref_add_mesh.argtypes = [_P, _F, _F, _F, C.c_uint32, _U32, C.c_uint32]
    L.ref_add_mesh_motion.argtypes = [_P, _F, _F, _F, C.c_uint32, _U32, C.c_uint32, _F, C.c_uint32]
    L.ref_set_shutter.argtypes = [_P, C.c_float, C.c_float]
    L.ref_add_strand.argtypes = [_P, _F, C.c_uint32, _F, C.c_uint32, C.c_uint32, _F]
    L.ref_mat_lambert.argtypes = [_P, _F]
    L.ref_mat_emissive.argtypes = [_P, _F, _F]
    L.ref_mat_standard.argtypes = [_P, _F]
    L.ref_mat_marschner.argtypes = [_P, C.c_float, _F, C.c_float, C.c_float, C.c_float]
    L.ref_set_slot.argtypes = [_P, C.c_uint32, C.c_int]
    L.ref_light_area.argtypes = [_P, _F, _F, _F, _F]
    L.ref_light_directional.argtypes = [_P, _F, _F, C.c_float]
    L.ref_light_dome.argtypes = [_P, _F, C.c_uint32, C.c_uint32, C.c_float, C.c_int]
    L.ref_set_env_radiance.argtypes = [_P, _F]
    L.ref_set_camera.argtypes = [_P, _F, _F, _F, C.c_float, C.c_uint32, C.c_uint32]
    L.ref_commit.argtypes = [_P]
    L.ref_trace.argtypes = [_P, _F, _F, C.c_uint64, _I32, _F, C.c_int]
    L.ref_render_rows.argtypes = [_P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int,
                                  _U32, C.c_uint32, _F, _F]
    L.ref_render_rows.restype = C.c_double
    L.ref_occluded.argtypes = [_P, _F, _F, C.c_uint64, _U8, C.c_int]
    L.ref_render.argtypes = [_P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                             C.c_int, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, _F, _F]
    L.ref_render.restype = C.c_double
    L.ref_render_aov.argtypes = [_P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int,
                                 _F, _F]
    L.ref_li.argtypes = [_P, C.c_uint32, C.c_uint32, C.c_uint32, _U32, C.c_uint64, _F, C.c_int]
    L.ref_dim_log.argtypes = [_P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                              C.c_uint32, _I32, C.c_int]
    L.ref_camera_rays.argtypes = [_P, C.c_uint32, C.c_uint32, _U32, C.c_uint64, _F]
    L.ref_camera_basis.argtypes = [_P, C.c_uint32, C.c_uint32, _F]
    L.ref_halton.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint32, _F]
    L.ref_pcg.argtypes = [C.c_uint64, C.c_uint32, _U32]
    L.ref_mat_evaluate.argtypes = [_P, C.c_int, _F, _F, _F, _F, _F]
    L.ref_mh_evaluate.argtypes = [_P, C.c_int, _F, _F, _F, _F, _F]
    L.ref_mh_sample.argtypes = [_P, C.c_int, _F, _F, _F, _F, C.c_float, _F]
    L.ref_mh_functions.argtypes = [_F, C.c_uint32, C.c_float, _F, _F]
    L.ref_mat_sample.argtypes = [_P, C.c_int, _F, _F, _F, _F, C.c_float, _F]
    L.ref_mat_le.argtypes = [_P, C.c_int, _F, _F, _F, _F]
    L.ref_ggx_D.argtypes = [C.c_float, C.c_float]
    L.ref_ggx_D.restype = C.c_float
    L.ref_light_sample.argtypes = [_P, C.c_int, _F, _F, _F, _F]
    L.ref_light_pdf.argtypes = [_P, C.c_int, _F, _F]
    L.ref_light_pdf.restype = C.c_float
    L.ref_light_le.argtypes = [_P, C.c_int, _F, _F]
    L.ref_light_sample_le.argtypes = [_P, C.c_int, _F, _F, _F]
    L.ref_dist1d.argtypes = [_F, C.c_uint32, _F, C.c_uint32, _F, _F]
    if variant == "dropin":
        L.ref_dropin_render.argtypes = [_P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int,
                                        _F, _F, C.c_char_p, C.c_int]
        L.ref_dropin_prepare.argtypes = [_P, C.c_uint32, C.c_uint32, C.c_char_p, C.c_int]
        L.ref_dropin_write.argtypes = [_P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, C.c_char_p,
                                       C.c_char_p, C.c_float, C.c_char_p, C.c_int]
        L.ref_dropin_prepare.restype = _P
    _LIBS[variant] = L
    return L


def f32(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.float32))


class RefScene:
    """The reference's scene objects (GeometryPool, CurvePool, materials,
    lights, CurveBrute accel, SceneView) built from a scenes.Scene."""

    def __init__(self, scene, variant="record", commit=True):
        from anacapa_b200 import scenes as S
        self.L = lib(variant)
        self.scene = scene
        self.h = self.L.ref_scene_new()
        L, h = self.L, self.h
        mats = []
        for m in scene.materials:
            if m.type == S.MAT_LAMBERT:
                mats.append(L.ref_mat_lambert(h, _fp(f32(m.albedo))))
            elif m.type == S.MAT_EMISSIVE:
                mats.append(L.ref_mat_emissive(h, _fp(f32(m.albedo)), _fp(f32(m.emission))))
            elif m.type == S.MAT_STANDARD:
                mats.append(L.ref_mat_standard(h, _fp(m.standard_packed())))
            elif m.type == S.MAT_HAIR:
                mats.append(L.ref_mat_marschner(h, m.eta, _fp(f32(m.sigma_a)), m.beta_m,
                                                m.beta_n, m.alpha_deg))
            else:
                raise ValueError(m.type)
        self.mat_handles = mats
        vo, to = scene.mesh_vert_offset, scene.mesh_tri_offset
        for i in range(scene.num_meshes):
            p = f32(scene.positions[vo[i]:vo[i + 1]])
            n = f32(scene.normals[vo[i]:vo[i + 1]]) if scene.mesh_has_normals[i] else None
            uv = f32(scene.uvs[vo[i]:vo[i + 1]]) if scene.uvs is not None else None
            idx = np.ascontiguousarray(scene.indices[to[i]:to[i + 1]], dtype=np.uint32)
            keys = scene.mesh_motion[i] if scene.mesh_motion is not None else None
            if keys:
                k17 = f32([[t, *np.asarray(M, np.float32).reshape(16)] for t, M in keys])
                L.ref_add_mesh_motion(h, _fp(p), _fp(n), _fp(uv), len(p), idx.ctypes.data_as(_U32), len(idx),
                                      _fp(k17), len(keys))
            else:
                L.ref_add_mesh(h, _fp(p), _fp(n), _fp(uv), len(p), idx.ctypes.data_as(_U32), len(idx))
        co, wo_ = scene.strand_cp_offset, scene.strand_width_offset
        cps = f32(scene.control_points)
        wds = f32(scene.widths)
        cols = f32(scene.strand_color)
        for s in range(scene.num_strands):
            L.ref_add_strand(h, _fp(cps[co[s]:co[s + 1]]), int(co[s + 1] - co[s]),
                             _fp(wds[wo_[s]:wo_[s + 1]]), int(wo_[s + 1] - wo_[s]),
                             int(scene.strand_slot[s]), _fp(cols[s]))
        for slot, mi in enumerate(scene.slots):
            L.ref_set_slot(h, slot, mats[mi] if mi >= 0 else -1)
        self.light_handles = []
        for a in scene.area_lights:
            self.light_handles.append(L.ref_light_area(h, _fp(f32(a.center)), _fp(f32(a.u)),
                                                       _fp(f32(a.v)), _fp(f32(a.Le))))
        for a in scene.dir_lights:
            self.light_handles.append(L.ref_light_directional(h, _fp(f32(a.direction)), _fp(f32(a.Le)),
                                                              float(a.half_angle_deg)))
        if scene.dome_rgb is not None:
            d = f32(scene.dome_rgb)
            self.light_handles.append(L.ref_light_dome(h, _fp(d), d.shape[1], d.shape[0],
                                                       scene.dome_intensity, 1))
        L.ref_set_env_radiance(h, _fp(f32(scene.env_radiance)))
        L.ref_set_camera(h, _fp(f32(scene.cam_from)), _fp(f32(scene.cam_at)),
                         _fp(f32(scene.cam_up)), scene.vfov, scene.width, scene.height)
        L.ref_set_shutter(h, float(scene.shutter[0]), float(scene.shutter[1]))
        if commit:
            L.ref_commit(h)

    def __del__(self):
        try:
            self.L.ref_scene_free(self.h)
        except Exception:
            pass

    def trace(self, rays, nthreads=0, times=None):
        rays = f32(rays).reshape(-1, 8)
        n = len(rays)
        ids = np.zeros((n, 4), np.int32)
        t = np.zeros(n, np.float32)
        tm = None if times is None else f32(times)
        self.L.ref_trace(self.h, _fp(rays), _fp(tm), n, ids.ctypes.data_as(_I32), _fp(t), nthreads)
        return ids, t

    def occluded(self, rays, nthreads=0, times=None):
        rays = f32(rays).reshape(-1, 8)
        out = np.zeros(len(rays), np.uint8)
        tm = None if times is None else f32(times)
        self.L.ref_occluded(self.h, _fp(rays), _fp(tm), len(rays), out.ctypes.data_as(_U8), nthreads)
        return out.astype(bool)

    def render(self, spp=None, sample_start=0, max_depth=None, nthreads=0, rect=None):
        s = self.scene
        W, H = s.width, s.height
        spp = s.spp if spp is None else spp
        md = s.max_depth if max_depth is None else max_depth
        x0, y0, x1, y1 = rect if rect is not None else (0, 0, W, H)
        rgbw = np.zeros((H, W, 4), np.float32)
        lsq = np.zeros((H, W), np.float32)
        secs = self.L.ref_render(self.h, W, H, spp, sample_start, md, nthreads, x0, y0, x1, y1,
                                 _fp(rgbw), _fp(lsq))
        return rgbw, lsq, secs

    def render_rows(self, bands, spp=None, sample_start=0, max_depth=None, nthreads=0):
        """render() over full-width row bands [(y0, y1), ...] in one thread
        pool dispatch; returns (rgbw, lsq, seconds)."""
        s = self.scene
        W, H = s.width, s.height
        rows = np.ascontiguousarray(np.asarray(bands, np.uint32).reshape(-1, 2))
        rgbw = np.zeros((H, W, 4), np.float32)
        lsq = np.zeros((H, W), np.float32)
        secs = self.L.ref_render_rows(self.h, W, H, s.spp if spp is None else spp, sample_start,
                                      s.max_depth if max_depth is None else max_depth, nthreads,
                                      rows.ctypes.data_as(_U32), len(rows), _fp(rgbw), _fp(lsq))
        return rgbw, lsq, secs

    def render_aov(self, spp=None, sample_start=0, max_depth=None, nthreads=0):
        """The frame's albedo and normal AOV accumulators, (H, W, 4) each
        (sum of per-tile averages, weight)."""
        s = self.scene
        al = np.zeros((s.height, s.width, 4), np.float32)
        nr = np.zeros((s.height, s.width, 4), np.float32)
        self.L.ref_render_aov(self.h, s.width, s.height, s.spp if spp is None else spp, sample_start,
                              s.max_depth if max_depth is None else max_depth, nthreads, _fp(al), _fp(nr))
        return al, nr

    def dropin_render(self, spp=None, passes=1, max_depth=None):
        """Render through this repository's B200PathIntegrator driven by the
        reference's SceneView and Film (variant "dropin" only). Returns the
        resolved RGB image and Film::varianceAt."""
        s = self.scene
        rgb = np.zeros((s.height, s.width, 3), np.float32)
        var = np.zeros((s.height, s.width), np.float32)
        err = C.create_string_buffer(512)
        rc = self.L.ref_dropin_render(self.h, s.width, s.height, s.spp if spp is None else spp,
                                      s.max_depth if max_depth is None else max_depth, passes,
                                      _fp(rgb), _fp(var), err, len(err))
        if rc:
            raise RuntimeError(f"drop-in render failed ({rc}): {err.value.decode()}")
        return rgb, var

    def dropin_write(self, exr, png, spp=None, passes=1, exposure=0.0, max_depth=None):
        """Render through the drop-in into a reference Film and write it with
        Film::writeEXR (AOV layers) and Film::writePNG (variant "dropin")."""
        s = self.scene
        err = C.create_string_buffer(512)
        rc = self.L.ref_dropin_write(self.h, s.width, s.height, s.spp if spp is None else spp,
                                     s.max_depth if max_depth is None else max_depth, passes,
                                     str(exr).encode(), str(png).encode(), exposure, err, len(err))
        if rc:
            raise RuntimeError(f"drop-in write failed ({rc}): {err.value.decode()}")

    def dropin_prepare(self, size=None):
        """The drop-in's host-side prepare of this scene (variant "dropin"
        only) for a film of `size` (default: the scene's): a raw ana_prepared
        handle, freed by the caller."""
        s = self.scene
        w, h = size if size is not None else (s.width, s.height)
        err = C.create_string_buffer(512)
        p = self.L.ref_dropin_prepare(self.h, w, h, err, len(err))
        if not p:
            raise RuntimeError(f"drop-in prepare failed: {err.value.decode()}")
        return p

    def camera_basis(self):
        """The scene's Camera as this build computed it (22 floats, the layout
        of Scene.cam_basis)."""
        s = self.scene
        out = np.zeros(22, np.float32)
        self.L.ref_camera_basis(self.h, s.width, s.height, _fp(out))
        return tuple(out.tolist())

    def li(self, pxy_s, max_depth=None, nthreads=0):
        s = self.scene
        q = np.ascontiguousarray(np.asarray(pxy_s, np.uint32).reshape(-1, 3))
        out = np.zeros((len(q), 3), np.float32)
        self.L.ref_li(self.h, s.width, s.height, s.max_depth if max_depth is None else max_depth,
                      q.ctypes.data_as(_U32), len(q), _fp(out), nthreads)
        return out

    def dim_log(self, px, py, sidx, max_depth=None):
        s = self.scene
        buf = np.zeros(4096, np.int32)
        n = self.L.ref_dim_log(self.h, s.width, s.height,
                               s.max_depth if max_depth is None else max_depth, px, py, sidx,
                               buf.ctypes.data_as(_I32), len(buf))
        return buf[:min(n, len(buf))].tolist()

    def camera_rays(self, pxy_s):
        s = self.scene
        q = np.ascontiguousarray(np.asarray(pxy_s, np.uint32).reshape(-1, 3))
        out = np.zeros((len(q), 6), np.float32)
        self.L.ref_camera_rays(self.h, s.width, s.height, q.ctypes.data_as(_U32), len(q), _fp(out))
        return out


# ana_bsdf_query / ana_bsdf_result layouts (include/anacapa_b200.h)
BSDF_QUERY = np.dtype([("n", "<f4", 3), ("t", "<f4", 3), ("color", "<f4", 3), ("wo", "<f4", 3),
                       ("wi", "<f4", 3), ("u", "<f4", 2), ("u_comp", "<f4"), ("is_curve", "<u4")])
BSDF_RESULT = np.dtype([("f", "<f4", 3), ("pdf", "<f4"), ("sample_f", "<f4", 3), ("sample_pdf", "<f4"),
                        ("sample_wi", "<f4", 3), ("sample_flags", "<u4")])


class RefMaterial:
    """One of the reference's material objects, outside any scene, for BSDF
    queries: IMaterial::evaluate / sample (the Kajiya-Kay lobe for hair, as
    the reference executes it), or for a hair material with
    marschner=True the Marschner branches of MarschnerHair.h (242-257,
    284-375) through ref_mh_evaluate / ref_mh_sample."""

    def __init__(self, m, variant="nocontract"):
        from anacapa_b200 import scenes as S
        L = self.L = lib(variant)
        self.h = L.ref_scene_new()
        if m.type == S.MAT_LAMBERT:
            self.mat = L.ref_mat_lambert(self.h, _fp(f32(m.albedo)))
        elif m.type == S.MAT_EMISSIVE:
            self.mat = L.ref_mat_emissive(self.h, _fp(f32(m.albedo)), _fp(f32(m.emission)))
        elif m.type == S.MAT_STANDARD:
            self.mat = L.ref_mat_standard(self.h, _fp(m.standard_packed()))
        elif m.type == S.MAT_HAIR:
            self.mat = L.ref_mat_marschner(self.h, m.eta, _fp(f32(m.sigma_a)), m.beta_m, m.beta_n, m.alpha_deg)
        else:
            raise ValueError(m.type)
        self.marschner = m.type == S.MAT_HAIR and m.hair_mode == 1

    def __del__(self):
        try:
            self.L.ref_scene_free(self.h)
        except Exception:
            pass

    def query(self, queries):
        q = np.ascontiguousarray(queries, BSDF_QUERY)
        out = np.zeros(len(q), BSDF_RESULT)
        L = self.L
        ev = np.zeros(5, np.float32)
        sm = np.zeros(8, np.float32)
        for k, r in enumerate(q):
            si = np.zeros(16, np.float32)
            si[3:6] = r["n"]
            si[6:9] = r["n"]
            si[9:12] = r["t"]
            si[12:15] = r["color"]
            si[15] = float(r["is_curve"])
            ray_dir = f32(-r["wo"])
            wo, wi, u = f32(r["wo"]), f32(r["wi"]), f32(r["u"])
            if self.marschner:
                L.ref_mh_evaluate(self.h, self.mat, _fp(si), _fp(ray_dir), _fp(wo), _fp(wi), _fp(ev))
                L.ref_mh_sample(self.h, self.mat, _fp(si), _fp(ray_dir), _fp(wo), _fp(u), float(r["u_comp"]),
                                _fp(sm))
                valid = sm[7] != 0.0
                flags = 2 | 8 | 16
            else:
                L.ref_mat_evaluate(self.h, self.mat, _fp(si), _fp(ray_dir), _fp(wo), _fp(wi), _fp(ev))
                L.ref_mat_sample(self.h, self.mat, _fp(si), _fp(ray_dir), _fp(wo), _fp(u), float(r["u_comp"]),
                                 _fp(sm))
                valid = sm[6] > 0.0 and np.any(sm[0:3] != 0.0)
                flags = int(sm[7])
            o = out[k]
            o["f"] = ev[0:3]
            o["pdf"] = ev[3]
            if valid:
                o["sample_f"] = sm[0:3]
                o["sample_wi"] = sm[3:6]
                o["sample_pdf"] = sm[6]
                o["sample_flags"] = flags
        return out


def mh_functions(inputs, eta, sigma_a, variant="nocontract"):
    """The reference's public Marschner lobe functions (MarschnerHair.h:
    88-187) over rows of (cosI, sinI, cosR, sinR, v, x, s, u, h, cosO); see
    ref_mh_functions for the 16 outputs per row."""
    x = f32(inputs).reshape(-1, 10)
    out = np.zeros((len(x), 16), np.float32)
    lib(variant).ref_mh_functions(_fp(x), len(x), float(eta), _fp(f32(sigma_a)), _fp(out))
    return out


def halton(px, py, sample_index, ndims, seed=0, variant="record"):
    out = np.zeros(ndims, np.float32)
    lib(variant).ref_halton(px, py, sample_index, seed, ndims, _fp(out))
    return out


def pcg(seed, n, variant="record"):
    out = np.zeros(n, np.uint32)
    lib(variant).ref_pcg(seed, n, out.ctypes.data_as(_U32))
    return out


def dist1d(vals, us, variant="record"):
    vals, us = f32(vals), f32(us)
    out = np.zeros((len(us), 3), np.float32)
    integ = np.zeros(1, np.float32)
    lib(variant).ref_dist1d(_fp(vals), len(vals), _fp(us), len(us), _fp(out), _fp(integ))
    return out, float(integ[0])
