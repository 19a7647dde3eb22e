"""TEST INFRASTRUCTURE — ctypes binding of the CPU restatement
(oracle/restate/pt_oracle.cpp, built by `make -C oracle restate` into
oracle/_build/libpt_oracle.so). precision=32 reproduces the reference's float
arithmetic; precision=64 is the FP64 oracle. It covers opaque, glass and
alpha-masked materials and motion-blurred meshes."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libpt_oracle.so")

_F = C.POINTER(C.c_float)
_D = C.POINTER(C.c_double)
_U32 = C.POINTER(C.c_uint32)
_I32 = C.POINTER(C.c_int32)
_P = C.c_void_p
_lib = None


def build():
    srcs = [os.path.join(HERE, "restate", n) for n in ("pt_oracle.cpp", "pt_oracle.h")]
    if os.path.exists(LIB) and all(os.path.getmtime(s) <= os.path.getmtime(LIB) for s in srcs):
        return
    subprocess.run(["make", "-C", HERE, "restate"], check=True, stdout=subprocess.DEVNULL)


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        L.po_scene_new.restype = _P
        L.po_scene_new.argtypes = [C.c_int]
        L.po_scene_free.argtypes = [_P]
        L.po_add_mesh.argtypes = [_P, C.c_uint32, _F, _F, C.c_uint32, _U32, C.c_uint32]
        L.po_add_strand.argtypes = [_P, _F, C.c_uint32, _F, C.c_uint32, C.c_uint32, _F]
        L.po_add_mesh_motion.argtypes = [_P, C.c_uint32, _F, _F, C.c_uint32, _U32, C.c_uint32, _F, C.c_uint32]
        L.po_set_shutter.argtypes = [_P, C.c_float, C.c_float]
        L.po_add_material.argtypes = [_P, C.c_int, _F, _F, _F, _F]
        L.po_set_slots.argtypes = [_P, _I32, C.c_uint32]
        L.po_light_area.argtypes = [_P, _F, _F, _F, _F]
        L.po_light_directional.argtypes = [_P, _F, _F, C.c_float]
        L.po_light_dome.argtypes = [_P, _F, C.c_uint32, C.c_uint32, C.c_float]
        L.po_set_env_radiance.argtypes = [_P, _F]
        L.po_set_camera.argtypes = [_P, _F, _F, _F, C.c_float, C.c_uint32, C.c_uint32]
        L.po_commit.argtypes = [_P]
        L.po_trace.argtypes = [_P, _F, C.c_uint64, _I32, _D, C.c_int]
        L.po_render.argtypes = [_P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int,
                                C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, _D, _D]
        L.po_li.argtypes = [_P, _U32, C.c_uint64, C.c_uint32, C.c_uint64, _D, C.c_int]
        L.po_halton.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint32, _F]
        L.po_pcg.argtypes = [C.c_uint64, C.c_uint32, _U32]
        L.po_mh_functions.argtypes = [_F, C.c_uint32, C.c_float, _F, _F]
        L.po_ggx_D.argtypes = [C.c_float, C.c_float]
        L.po_ggx_D.restype = C.c_float
        L.po_num_params.argtypes = [_P]
        L.po_num_params.restype = C.c_uint64
        L.po_adjoint.argtypes = [_P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64,
                                 _F, C.c_int, _D]
        _lib = L
    return _lib


def f32(x):
    return np.ascontiguousarray(np.asarray(x, np.float32))


def _fp(a):
    return None if a is None else a.ctypes.data_as(_F)


class PoScene:
    def __init__(self, scene, precision=64):
        from anacapa_b200 import scenes as S
        L = self.L = lib()
        self.scene = scene
        h = self.h = L.po_scene_new(precision)
        for m in scene.materials:
            if m.type in (S.MAT_LAMBERT, S.MAT_EMISSIVE):
                L.po_add_material(h, m.type, _fp(f32(m.albedo)), _fp(f32(m.emission)), None, None)
            elif m.type == S.MAT_STANDARD:
                L.po_add_material(h, m.type, None, None, _fp(m.standard_packed()), None)
            else:
                hv = f32([m.eta, *m.sigma_a, m.beta_m, m.beta_n, m.alpha_deg, m.hair_mode])
                L.po_add_material(h, m.type, None, None, None, _fp(hv))
        vo, to = scene.mesh_vert_offset, scene.mesh_tri_offset
        for i in range(scene.num_meshes):
            p = f32(scene.positions[vo[i]:vo[i + 1]])
            n = f32(scene.normals[vo[i]:vo[i + 1]]) if scene.mesh_has_normals[i] else None
            idx = np.ascontiguousarray(scene.indices[to[i]:to[i + 1]], np.uint32)
            keys = scene.mesh_motion[i] if scene.mesh_motion is not None else None
            if keys:
                k17 = f32([[t, *np.asarray(M, np.float32).reshape(16)] for t, M in keys])
                L.po_add_mesh_motion(h, i, _fp(p), _fp(n), len(p), idx.ctypes.data_as(_U32), len(idx),
                                     _fp(k17), len(keys))
            else:
                L.po_add_mesh(h, i, _fp(p), _fp(n), len(p), idx.ctypes.data_as(_U32), len(idx))
        co, wo = scene.strand_cp_offset, scene.strand_width_offset
        cps, wds, cols = f32(scene.control_points), f32(scene.widths), f32(scene.strand_color)
        for s in range(scene.num_strands):
            L.po_add_strand(h, _fp(cps[co[s]:co[s + 1]]), int(co[s + 1] - co[s]), _fp(wds[wo[s]:wo[s + 1]]),
                            int(wo[s + 1] - wo[s]), int(scene.strand_slot[s]), _fp(cols[s]))
        slots = np.ascontiguousarray(np.asarray(scene.slots, np.int32))
        L.po_set_slots(h, slots.ctypes.data_as(_I32), len(slots))
        for a in scene.area_lights:
            L.po_light_area(h, _fp(f32(a.center)), _fp(f32(a.u)), _fp(f32(a.v)), _fp(f32(a.Le)))
        for a in scene.dir_lights:
            L.po_light_directional(h, _fp(f32(a.direction)), _fp(f32(a.Le)), float(a.half_angle_deg))
        if scene.dome_rgb is not None:
            d = f32(scene.dome_rgb)
            L.po_light_dome(h, _fp(d), d.shape[1], d.shape[0], scene.dome_intensity)
        L.po_set_env_radiance(h, _fp(f32(scene.env_radiance)))
        L.po_set_camera(h, _fp(f32(scene.cam_from)), _fp(f32(scene.cam_at)), _fp(f32(scene.cam_up)),
                        scene.vfov, scene.width, scene.height)
        L.po_set_shutter(h, float(scene.shutter[0]), float(scene.shutter[1]))
        L.po_commit(h)

    def __del__(self):
        try:
            self.L.po_scene_free(self.h)
        except Exception:
            pass

    def trace(self, rays, threads=0):
        rays = f32(rays).reshape(-1, 8)
        ids = np.zeros((len(rays), 4), np.int32)
        t = np.zeros(len(rays), np.float64)
        self.L.po_trace(self.h, _fp(rays), len(rays), ids.ctypes.data_as(_I32), t.ctypes.data_as(_D), threads)
        return ids, t

    def render(self, spp=None, sample_start=0, max_depth=None, threads=0, rect=None, seed=0):
        s = self.scene
        W, H = s.width, s.height
        x0, y0, x1, y1 = rect if rect is not None else (0, 0, W, H)
        rgbw = np.zeros((H, W, 4), np.float64)
        lsq = np.zeros((H, W), np.float64)
        self.L.po_render(self.h, W, H, s.spp if spp is None else spp, sample_start,
                         s.max_depth if max_depth is None else max_depth, threads, x0, y0, x1, y1, seed,
                         rgbw.ctypes.data_as(_D), lsq.ctypes.data_as(_D))
        return rgbw, lsq

    def adjoint(self, d_image, spp=None, sample_start=0, max_depth=None, seed=0, threads=0):
        """Reference dLoss/d theta (float64) of the frame for dLoss/d image
        (H, W, 3): forward-mode along every path, parameters laid out 8 per
        material (albedo rgb, roughness, emission rgb, -), 4 per light."""
        s = self.scene
        g = np.ascontiguousarray(np.asarray(d_image, np.float32).reshape(s.height, s.width, 3))
        out = np.zeros(int(self.L.po_num_params(self.h)), np.float64)
        self.L.po_adjoint(self.h, s.width, s.height, s.spp if spp is None else spp, sample_start,
                          s.max_depth if max_depth is None else max_depth, seed, _fp(g), threads,
                          out.ctypes.data_as(_D))
        return out

    def li(self, q, max_depth=None, seed=0, threads=0):
        q = np.ascontiguousarray(np.asarray(q, np.uint32).reshape(-1, 3))
        out = np.zeros((len(q), 3), np.float64)
        self.L.po_li(self.h, q.ctypes.data_as(_U32), len(q),
                     self.scene.max_depth if max_depth is None else max_depth, seed,
                     out.ctypes.data_as(_D), threads)
        return out


def halton(px, py, s, n, seed=0):
    out = np.zeros(n, np.float32)
    lib().po_halton(px, py, s, seed, n, out.ctypes.data_as(_F))
    return out


def mh_functions(inputs, eta, sigma_a):
    """The restatement's Marschner lobe functions in float (the layout of
    oracle.refbind.mh_functions)."""
    x = f32(inputs).reshape(-1, 10)
    out = np.zeros((len(x), 16), np.float32)
    lib().po_mh_functions(_fp(x), len(x), float(eta), _fp(f32(sigma_a)), _fp(out))
    return out


def pcg(seed, n):
    out = np.zeros(n, np.uint32)
    lib().po_pcg(seed, n, out.ctypes.data_as(_U32))
    return out
