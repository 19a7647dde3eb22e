"""ctypes binding of libanacapa_b200.so (include/anacapa_b200.h).

The library is the only compute path: importing a renderer on a machine where
the shared object is missing raises instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

from . import scenes as S

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libanacapa_b200.so")

ANA_OK = 0
ANA_ERR_INVALID_ARG = 1
ANA_ERR_CUDA = 2
ANA_ERR_OOM = 3
ANA_ERR_TIMEOUT = 4
ANA_ERR_UNSUPPORTED = 5
ANA_ERR_STATE = 6
ANA_ERR_DEVICE_CHECK = 7
ANA_RENDER_CLEAR_FILM = 1
ANA_RENDER_COUNT_WORK = 2
ANA_RENDER_AOVS = 8
ANA_TRAVERSAL_DEFAULT = 0
ANA_TRAVERSAL_PERSISTENT = 1
ANA_TRAVERSAL_PER_RAY = 2
TRACE_NOALLOC_MAX_RAYS = 65536  # ANA_TRACE_NOALLOC_MAX_RAYS

F3 = C.c_float * 3

# ana_bsdf_query / ana_bsdf_result as numpy records
BSDF_QUERY = np.dtype([("n", "<f4", 3), ("t", "<f4", 3), ("color", "<f4", 3), ("wo", "<f4", 3),
                       ("wi", "<f4", 3), ("u", "<f4", 2), ("u_comp", "<f4"), ("is_curve", "<u4")])
BSDF_RESULT = np.dtype([("f", "<f4", 3), ("pdf", "<f4"), ("sample_f", "<f4", 3), ("sample_pdf", "<f4"),
                        ("sample_wi", "<f4", 3), ("sample_flags", "<u4")])


class AnaMaterial(C.Structure):
    _fields_ = [("type", C.c_uint32), ("albedo", F3), ("emission", F3), ("base_color", F3),
                ("base", C.c_float), ("metalness", C.c_float), ("roughness", C.c_float),
                ("specular", C.c_float), ("specular_color", F3), ("specular_ior", C.c_float),
                ("coat", C.c_float), ("coat_roughness", C.c_float), ("transmission", C.c_float),
                ("emission_weight", C.c_float), ("emission_color", F3), ("alpha_mask", C.c_uint32),
                ("eta", C.c_float), ("sigma_a", F3), ("beta_m", C.c_float), ("beta_n", C.c_float),
                ("alpha_deg", C.c_float), ("hair_mode", C.c_uint32), ("opacity", C.c_float)]


class AnaLight(C.Structure):
    _fields_ = [("type", C.c_uint32), ("center", F3), ("u", F3), ("v", F3), ("Le", F3),
                ("half_angle_deg", C.c_float)]


class AnaCamera(C.Structure):
    _fields_ = [("from_", F3), ("at", F3), ("up", F3), ("vfov_deg", C.c_float),
                ("aperture_radius", C.c_float), ("focal_distance", C.c_float),
                ("shutter_open", C.c_float), ("shutter_close", C.c_float),
                ("explicit_basis", C.c_uint32), ("origin", F3), ("lower_left", F3),
                ("horizontal", F3), ("vertical", F3), ("basis_u", F3), ("basis_v", F3)]


_P = C.c_void_p


class AnaSceneDesc(C.Structure):
    _fields_ = [("num_meshes", C.c_uint32), ("mesh_vert_offset", _P), ("mesh_tri_offset", _P),
                ("mesh_has_normals", _P), ("positions", _P), ("normals", _P), ("indices", _P),
                ("num_strands", C.c_uint32), ("strand_cp_offset", _P), ("control_points", _P),
                ("strand_width_offset", _P), ("widths", _P), ("strand_slot", _P),
                ("strand_color", _P),
                ("num_materials", C.c_uint32), ("materials", _P), ("num_slots", C.c_uint32),
                ("slot_material", _P), ("num_lights", C.c_uint32), ("lights", _P),
                ("env_rgb", _P), ("env_width", C.c_uint32), ("env_height", C.c_uint32),
                ("env_intensity", C.c_float), ("env_radiance", F3), ("camera", AnaCamera),
                ("max_leaf_tris", C.c_uint32), ("max_leaf_segments", C.c_uint32),
                ("mesh_motion_offset", _P), ("motion_keys", _P)]


class AnaRenderDesc(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("sample_start", C.c_uint32),
                ("sample_count", C.c_uint32), ("max_depth", C.c_uint32), ("min_depth", C.c_uint32),
                ("seed", C.c_uint64), ("flags", C.c_uint32)]


class AnaFilmPixel(C.Structure):
    _fields_ = [("r", C.c_float), ("g", C.c_float), ("b", C.c_float), ("w", C.c_float),
                ("sum_lum_sq", C.c_float)]


class AnaHit(C.Structure):
    _fields_ = [("hit", C.c_int32), ("mesh_id", C.c_int32), ("prim_id", C.c_int32),
                ("strand_id", C.c_int32), ("t", C.c_float), ("u", C.c_float), ("v", C.c_float),
                ("pad", C.c_float)]


class AnaStats(C.Structure):
    _fields_ = [("paths", C.c_uint64), ("extend_rays", C.c_uint64), ("shadow_rays", C.c_uint64),
                ("mis_rays", C.c_uint64), ("render_ms", C.c_float), ("extend_ms", C.c_float),
                ("shade_ms", C.c_float), ("shadow_ms", C.c_float), ("mis_ms", C.c_float),
                ("film_ms", C.c_float), ("bounces", C.c_uint32), ("chunks", C.c_uint32),
                ("kernel_launches", C.c_uint64), ("extend_launches", C.c_uint64),
                ("node_fetches", C.c_uint64), ("tri_tests", C.c_uint64), ("seg_tests", C.c_uint64),
                ("curve_node_fetches", C.c_uint64),
                ("upload_ms", C.c_float), ("build_ms", C.c_float * 4), ("build_levels", C.c_uint32)]


class AnaTile(C.Structure):
    _fields_ = [("x0", C.c_uint32), ("y0", C.c_uint32), ("width", C.c_uint32), ("height", C.c_uint32),
                ("sample_start", C.c_uint32), ("sample_count", C.c_uint32)]


class AnaDiffParams(C.Structure):
    _fields_ = [("albedo", _P), ("roughness", _P), ("emission", _P), ("light_le", _P)]


class AnaDeviceOpts(C.Structure):
    _fields_ = [("device", C.c_int), ("chunk_paths", C.c_uint32), ("block_size", C.c_uint32),
                ("timing", C.c_uint32), ("traversal", C.c_uint32)]


HIT_DTYPE = np.dtype([("hit", "<i4"), ("mesh_id", "<i4"), ("prim_id", "<i4"),
                      ("strand_id", "<i4"), ("t", "<f4"), ("u", "<f4"), ("v", "<f4"),
                      ("pad", "<f4")])

# Every symbol include/anacapa_b200.h declares.
EXPORTS = ["ana_create", "ana_destroy", "ana_upload_scene", "ana_prepare_scene",
           "ana_upload_prepared", "ana_prepared_bytes", "ana_prepared_free", "ana_render",
           "ana_film_clear", "ana_film_read", "ana_film_device_ptr", "ana_trace_batch",
           "ana_get_stats", "ana_last_error", "ana_version", "ana_batch_create", "ana_batch_free",
           "ana_batch_bytes", "ana_upload_batch", "ana_render_batch", "ana_batch_film_read",
           "ana_prepared_digest", "ana_trace_batch_noalloc", "ana_diff_counts", "ana_diff_get_params",
           "ana_forward", "ana_backward", "ana_render_tiles", "ana_render_adaptive",
           "ana_upload_scene_device", "ana_scene_digest", "ana_aov_read", "ana_film_write_exr",
           "ana_film_write_png", "ana_image_write_exr", "ana_image_write_png", "ana_trace_batch_timed",
           "ana_bsdf_batch"]
ANA_RENDER_GRAPH = 4

_lib = None


class AnaError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"anacapa_b200 error {code}: {msg}")
        self.code = code


def lib():
    """Load the in-tree shared library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: run `python -m anacapa_b200.build`")
    L = C.CDLL(LIB_PATH)
    L.ana_create.argtypes = [C.POINTER(_P), C.POINTER(AnaDeviceOpts)]
    L.ana_destroy.argtypes = [_P]
    L.ana_destroy.restype = None
    L.ana_upload_scene.argtypes = [_P, C.POINTER(AnaSceneDesc)]
    L.ana_upload_scene_device.argtypes = [_P, C.POINTER(AnaSceneDesc)]
    L.ana_scene_digest.argtypes = [_P, C.POINTER(C.c_uint64)]
    L.ana_aov_read.argtypes = [_P, _P, _P, C.c_size_t]
    L.ana_film_write_exr.argtypes = [_P, C.c_uint32, C.c_uint32, C.c_char_p, C.c_int]
    L.ana_film_write_png.argtypes = [_P, C.c_uint32, C.c_uint32, C.c_char_p, C.c_float]
    L.ana_image_write_exr.argtypes = [C.c_char_p, C.c_uint32, C.c_uint32, _P, _P, _P]
    L.ana_image_write_png.argtypes = [C.c_char_p, C.c_uint32, C.c_uint32, _P, C.c_float]
    L.ana_trace_batch_timed.argtypes = [_P, _P, _P, C.c_size_t, _P, C.c_int, C.c_int]
    L.ana_prepare_scene.argtypes = [C.POINTER(AnaSceneDesc), C.POINTER(_P)]
    L.ana_upload_prepared.argtypes = [_P, _P]
    L.ana_prepared_bytes.argtypes = [_P]
    L.ana_prepared_bytes.restype = C.c_uint64
    L.ana_prepared_free.argtypes = [_P]
    L.ana_prepared_free.restype = None
    L.ana_render.argtypes = [_P, C.POINTER(AnaRenderDesc)]
    L.ana_film_clear.argtypes = [_P, C.c_uint32, C.c_uint32]
    L.ana_film_read.argtypes = [_P, _P, C.c_size_t]
    L.ana_film_device_ptr.argtypes = [_P, C.POINTER(_P)]
    L.ana_trace_batch.argtypes = [_P, _P, C.c_size_t, _P, C.c_int, C.c_int]
    L.ana_trace_batch_noalloc.argtypes = [_P, _P, C.c_size_t, _P, C.c_int]
    L.ana_get_stats.argtypes = [_P, C.POINTER(AnaStats)]
    L.ana_last_error.argtypes = [_P, C.c_char_p, C.c_size_t]
    L.ana_version.restype = C.c_int
    L.ana_batch_create.argtypes = [C.POINTER(_P), C.c_uint32, C.POINTER(_P)]
    L.ana_batch_free.argtypes = [_P]
    L.ana_batch_free.restype = None
    L.ana_batch_bytes.argtypes = [_P]
    L.ana_batch_bytes.restype = C.c_uint64
    L.ana_upload_batch.argtypes = [_P, _P]
    L.ana_render_batch.argtypes = [_P, C.POINTER(AnaRenderDesc), C.c_uint32, C.c_uint32]
    L.ana_batch_film_read.argtypes = [_P, C.c_uint32, _P, C.c_size_t]
    L.ana_prepared_digest.argtypes = [_P]
    L.ana_prepared_digest.restype = C.c_uint64
    L.ana_render_tiles.argtypes = [_P, C.POINTER(AnaRenderDesc), C.POINTER(AnaTile), C.c_uint32]
    L.ana_render_adaptive.argtypes = [_P, C.POINTER(AnaRenderDesc), C.c_uint32, C.c_uint32, _P, C.c_uint32]
    L.ana_diff_counts.argtypes = [_P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
    L.ana_diff_get_params.argtypes = [_P, C.POINTER(AnaDiffParams)]
    L.ana_forward.argtypes = [_P, C.POINTER(AnaRenderDesc), C.POINTER(AnaDiffParams), _P]
    L.ana_backward.argtypes = [_P, _P, C.POINTER(AnaDiffParams)]
    L.ana_bsdf_batch.argtypes = [_P, C.POINTER(AnaMaterial), _P, C.c_size_t, _P]
    _lib = L
    return L


def last_error(ctx=None) -> str:
    buf = C.create_string_buffer(1024)
    lib().ana_last_error(ctx, buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc, ctx=None):
    if rc != ANA_OK:
        raise AnaError(rc, last_error(ctx))


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data


def material_struct(m: S.Material) -> AnaMaterial:
    s = AnaMaterial()
    s.type = m.type
    s.albedo[:] = m.albedo
    s.emission[:] = m.emission
    s.base_color[:] = m.base_color
    s.base = m.base
    s.metalness = m.metalness
    s.roughness = m.roughness
    s.specular = m.specular
    s.specular_color[:] = m.specular_color
    s.specular_ior = m.specular_ior
    s.coat = m.coat
    s.coat_roughness = m.coat_roughness
    s.transmission = m.transmission
    s.emission_weight = m.emission_w
    s.emission_color[:] = m.emission_color
    s.alpha_mask = 1 if m.alpha_mask else 0
    s.opacity = m.opacity
    s.eta = m.eta
    s.sigma_a[:] = m.sigma_a
    s.beta_m = m.beta_m
    s.beta_n = m.beta_n
    s.alpha_deg = m.alpha_deg
    s.hair_mode = m.hair_mode
    return s


class SceneDesc:
    """An AnaSceneDesc plus the numpy arrays it points into (kept alive)."""

    def __init__(self, sc: S.Scene, max_leaf_tris=0, max_leaf_segments=0):
        keep = []

        def arr(x, dt):
            a = np.ascontiguousarray(np.asarray(x, dtype=dt))
            keep.append(a)
            return a

        d = AnaSceneDesc()
        d.num_meshes = sc.num_meshes
        d.mesh_vert_offset = _ptr(arr(sc.mesh_vert_offset, np.uint32))
        d.mesh_tri_offset = _ptr(arr(sc.mesh_tri_offset, np.uint32))
        d.mesh_has_normals = _ptr(arr(sc.mesh_has_normals, np.uint8))
        d.positions = _ptr(arr(sc.positions, np.float32))
        d.normals = _ptr(arr(sc.normals, np.float32)) if sc.normals is not None else None
        d.indices = _ptr(arr(sc.indices, np.uint32))
        d.num_strands = sc.num_strands
        d.strand_cp_offset = _ptr(arr(sc.strand_cp_offset, np.uint32))
        d.control_points = _ptr(arr(sc.control_points, np.float32))
        d.strand_width_offset = _ptr(arr(sc.strand_width_offset, np.uint32))
        d.widths = _ptr(arr(sc.widths, np.float32))
        d.strand_slot = _ptr(arr(sc.strand_slot, np.uint32))
        d.strand_color = _ptr(arr(sc.strand_color, np.float32))
        mats = (AnaMaterial * max(1, len(sc.materials)))(*[material_struct(m) for m in sc.materials])
        keep.append(mats)
        d.num_materials = len(sc.materials)
        d.materials = C.addressof(mats)
        d.num_slots = len(sc.slots)
        d.slot_material = _ptr(arr(sc.slots, np.int32))
        lights = []
        for a in sc.area_lights:
            l = AnaLight()
            l.type = S.LIGHT_AREA
            l.center[:] = a.center
            l.u[:] = a.u
            l.v[:] = a.v
            l.Le[:] = a.Le
            lights.append(l)
        for a in sc.dir_lights:
            l = AnaLight()
            l.type = S.LIGHT_DIRECTIONAL
            l.u[:] = a.direction
            l.Le[:] = a.Le
            l.half_angle_deg = a.half_angle_deg
            lights.append(l)
        if sc.dome_rgb is not None:
            l = AnaLight()
            l.type = S.LIGHT_DOME
            lights.append(l)
        la = (AnaLight * max(1, len(lights)))(*lights)
        keep.append(la)
        d.num_lights = len(lights)
        d.lights = C.addressof(la)
        if sc.dome_rgb is not None:
            env = arr(sc.dome_rgb, np.float32)
            d.env_rgb = _ptr(env)
            d.env_width = env.shape[1]
            d.env_height = env.shape[0]
            d.env_intensity = sc.dome_intensity
        d.env_radiance[:] = sc.env_radiance
        cam = AnaCamera()
        cam.from_[:] = sc.cam_from
        cam.at[:] = sc.cam_at
        cam.up[:] = sc.cam_up
        cam.vfov_deg = sc.vfov
        cam.shutter_open, cam.shutter_close = sc.shutter
        if sc.cam_basis is not None:
            b = [float(x) for x in sc.cam_basis]
            cam.explicit_basis = 1
            cam.origin[:], cam.lower_left[:], cam.horizontal[:] = b[0:3], b[3:6], b[6:9]
            cam.vertical[:], cam.basis_u[:], cam.basis_v[:] = b[9:12], b[12:15], b[15:18]
            cam.aperture_radius, cam.focal_distance, cam.shutter_open, cam.shutter_close = b[18:22]
        d.camera = cam
        d.max_leaf_tris = max_leaf_tris
        d.max_leaf_segments = max_leaf_segments
        if sc.mesh_motion is not None and any(k for k in sc.mesh_motion):
            off = np.zeros(sc.num_meshes + 1, np.uint32)
            rows = []
            for m in range(sc.num_meshes):
                keys = sc.mesh_motion[m] or []
                off[m + 1] = off[m] + len(keys)
                rows += [[t, *np.asarray(M, np.float32).reshape(16)] for t, M in keys]
            d.mesh_motion_offset = _ptr(arr(off, np.uint32))
            d.motion_keys = _ptr(arr(np.asarray(rows, np.float32).reshape(-1, 17), np.float32))
        self.desc = d
        self._keep = keep


class Prepared:
    """Host-prepared scene (BVHs built, device layout flattened into one blob)."""

    def __init__(self, sc: S.Scene, **kw):
        self.desc = SceneDesc(sc, **kw)
        h = _P()
        check(lib().ana_prepare_scene(C.byref(self.desc.desc), C.byref(h)))
        self.h = h

    @property
    def nbytes(self) -> int:
        return int(lib().ana_prepared_bytes(self.h))

    @property
    def digest(self) -> int:
        """FNV-1a of the device layout (BVHs, primitives, materials, lights, dome)."""
        return int(lib().ana_prepared_digest(self.h))

    def __del__(self):
        try:
            if self.h:
                lib().ana_prepared_free(self.h)
        except Exception:
            pass


class Renderer:
    """One ana_ctx (one CUDA stream) on one device."""

    def __init__(self, device=0, chunk_paths=0, block_size=0, timing=False, traversal=0):
        o = AnaDeviceOpts(device, chunk_paths, block_size, 1 if timing else 0, traversal)
        h = _P()
        check(lib().ana_create(C.byref(h), C.byref(o)))
        self.h = h
        self.scene: Optional[S.Scene] = None

    def close(self):
        if self.h:
            lib().ana_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        check(rc, self.h)

    def upload(self, sc_or_prep, device_build=False, **kw):
        """ana_upload_scene (host BVH build), ana_upload_scene_device with
        device_build, or ana_upload_prepared for a Prepared scene."""
        if isinstance(sc_or_prep, Prepared):
            self._check(lib().ana_upload_prepared(self.h, sc_or_prep.h))
        else:
            d = SceneDesc(sc_or_prep, **kw)
            fn = lib().ana_upload_scene_device if device_build else lib().ana_upload_scene
            self._check(fn(self.h, C.byref(d.desc)))
            self.scene = sc_or_prep

    def scene_digest(self) -> int:
        """ana_scene_digest: FNV-1a 64 of the uploaded scene arena."""
        out = C.c_uint64()
        self._check(lib().ana_scene_digest(self.h, C.byref(out)))
        return int(out.value)

    def render(self, width, height, spp, max_depth, sample_start=0, min_depth=2, seed=0, clear=True,
               count_work=False, aovs=False):
        flags = ((ANA_RENDER_CLEAR_FILM if clear else 0) | (ANA_RENDER_COUNT_WORK if count_work else 0)
                 | (ANA_RENDER_AOVS if aovs else 0))
        r = AnaRenderDesc(width, height, sample_start, spp, max_depth, min_depth, seed, flags)
        self._check(lib().ana_render(self.h, C.byref(r)))

    def render_scene(self, sc: S.Scene, spp=None, clear=True, sample_start=0, seed=0, count_work=False,
                     aovs=False):
        self.render(sc.width, sc.height, sc.spp if spp is None else spp, sc.max_depth,
                    sample_start=sample_start, seed=seed, clear=clear, count_work=count_work, aovs=aovs)

    def aovs(self, width, height):
        """ana_aov_read: resolved first-hit albedo and shading normal, (H, W, 3) each."""
        al = np.zeros((height, width, 3), np.float32)
        nr = np.zeros((height, width, 3), np.float32)
        self._check(lib().ana_aov_read(self.h, al.ctypes.data, nr.ctypes.data, width * height))
        return al, nr

    def write_exr(self, path, width, height, aovs=True):
        """ana_film_write_exr (Film::writeEXR)."""
        self._check(lib().ana_film_write_exr(self.h, width, height, str(path).encode(), 1 if aovs else 0))

    def write_png(self, path, width, height, exposure=0.0):
        """ana_film_write_png (Film::writePNG)."""
        self._check(lib().ana_film_write_png(self.h, width, height, str(path).encode(), exposure))

    def render_tiles(self, width, height, max_depth, tiles, clear=False, min_depth=2, seed=0, aovs=False):
        """ana_render_tiles: tiles = [(x0, y0, w, h, sample_start, sample_count), ...]
        of one width x height frame, accumulated into the film."""
        arr = (AnaTile * max(1, len(tiles)))(*[AnaTile(*map(int, t)) for t in tiles])
        r = AnaRenderDesc(width, height, 0, 0, max_depth, min_depth, seed,
                          (ANA_RENDER_CLEAR_FILM if clear else 0) | (ANA_RENDER_AOVS if aovs else 0))
        self._check(lib().ana_render_tiles(self.h, C.byref(r), arr, len(tiles)))

    def render_adaptive(self, width, height, spp, max_depth, tile_size=64, base_spp=0, min_depth=2, seed=0,
                        aovs=False):
        """ana_render_adaptive: the two-pass tile-adaptive schedule; returns the
        extra samples given to each tile (row-major)."""
        nt = (-(-width // tile_size)) * (-(-height // tile_size))
        extra = np.zeros(nt, np.uint32)
        r = AnaRenderDesc(width, height, 0, spp, max_depth, min_depth, seed,
                          ANA_RENDER_CLEAR_FILM | (ANA_RENDER_AOVS if aovs else 0))
        self._check(lib().ana_render_adaptive(self.h, C.byref(r), tile_size, base_spp, extra.ctypes.data, nt))
        return extra

    def film(self, width, height) -> np.ndarray:
        """(H, W, 5) float32: pre-weighted r, g, b, weight, sum of lum^2."""
        out = np.zeros((height, width, 5), np.float32)
        self._check(lib().ana_film_read(self.h, out.ctypes.data, width * height))
        return out

    def image(self, width, height) -> np.ndarray:
        f = self.film(width, height)
        return f[..., :3] / np.maximum(f[..., 3:4], 1e-30)

    # ---- differentiable rendering (ana_forward / ana_backward) ----
    def diff_counts(self):
        nm, nl = C.c_uint32(), C.c_uint32()
        self._check(lib().ana_diff_counts(self.h, C.byref(nm), C.byref(nl)))
        return nm.value, nl.value

    def _diff_arrays(self):
        nm, nl = self.diff_counts()
        return {"albedo": np.zeros((nm, 3), np.float32), "roughness": np.zeros(nm, np.float32),
                "emission": np.zeros((nm, 3), np.float32), "light_le": np.zeros((nl, 3), np.float32)}

    @staticmethod
    def _diff_struct(d):
        st = AnaDiffParams()
        for k in ("albedo", "roughness", "emission", "light_le"):
            a = d.get(k)
            setattr(st, k, None if a is None else a.ctypes.data)
        return st

    def diff_params(self):
        """Current differentiable parameters: albedo (M,3), roughness (M,),
        emission (M,3), light_le (L,3), by uploaded material / light index."""
        d = self._diff_arrays()
        st = self._diff_struct(d)
        self._check(lib().ana_diff_get_params(self.h, C.byref(st)))
        return d

    def forward(self, width, height, spp, max_depth, params=None, sample_start=0, min_depth=2, seed=0):
        """ana_forward: set `params` (dict of arrays, missing keys unchanged),
        render, return the (H, W, 3) image."""
        keep = None
        st = None
        if params is not None:
            keep = {k: np.ascontiguousarray(np.asarray(v, np.float32)) for k, v in params.items()
                    if v is not None}
            st = self._diff_struct(keep)
        r = AnaRenderDesc(width, height, sample_start, spp, max_depth, min_depth, seed, ANA_RENDER_CLEAR_FILM)
        img = np.zeros((height, width, 3), np.float32)
        self._check(lib().ana_forward(self.h, C.byref(r), C.byref(st) if st is not None else None,
                                      img.ctypes.data))
        del keep
        return img

    def backward(self, d_image):
        """ana_backward: dLoss/d image (H, W, 3) -> dict of dLoss/d parameters."""
        g = np.ascontiguousarray(np.asarray(d_image, np.float32))
        d = self._diff_arrays()
        st = self._diff_struct(d)
        self._check(lib().ana_backward(self.h, g.ctypes.data, C.byref(st)))
        return d

    def bsdf(self, material: S.Material, queries: np.ndarray) -> np.ndarray:
        """IMaterial::evaluate and sample of `material` on the device for a
        BSDF_QUERY record array; returns BSDF_RESULT records."""
        q = np.ascontiguousarray(queries, BSDF_QUERY)
        out = np.zeros(len(q), BSDF_RESULT)
        m = material_struct(material)
        self._check(lib().ana_bsdf_batch(self.h, C.byref(m), _ptr(q), len(q), _ptr(out)))
        return out

    def stats(self) -> AnaStats:
        s = AnaStats()
        self._check(lib().ana_get_stats(self.h, C.byref(s)))
        return s

    def trace(self, rays: np.ndarray, occlusion=False, times=None) -> np.ndarray:
        """ana_trace_batch (ana_trace_batch_timed with per-ray `times`)."""
        rays = np.ascontiguousarray(np.asarray(rays, np.float32).reshape(-1, 8))
        out = np.zeros(len(rays), HIT_DTYPE)
        if times is None:
            self._check(lib().ana_trace_batch(self.h, rays.ctypes.data, len(rays), out.ctypes.data,
                                              1 if occlusion else 0, 0))
        else:
            tm = np.ascontiguousarray(np.asarray(times, np.float32).reshape(-1))
            assert len(tm) == len(rays)
            self._check(lib().ana_trace_batch_timed(self.h, rays.ctypes.data, tm.ctypes.data, len(rays),
                                                    out.ctypes.data, 1 if occlusion else 0, 0))
        return out

    def trace_noalloc(self, rays: np.ndarray, occlusion=False) -> np.ndarray:
        """ana_trace_batch_noalloc: the same query staged in the library's fixed
        device scratch (at most TRACE_NOALLOC_MAX_RAYS rays, no device
        allocation), for callers that must not allocate while tracing."""
        rays = np.ascontiguousarray(np.asarray(rays, np.float32).reshape(-1, 8))
        out = np.zeros(len(rays), HIT_DTYPE)
        self._check(lib().ana_trace_batch_noalloc(self.h, rays.ctypes.data, len(rays), out.ctypes.data,
                                                  1 if occlusion else 0))
        return out

    # ---- batches -------------------------------------------------------------
    def upload_batch(self, batch: "Batch"):
        self._check(lib().ana_upload_batch(self.h, batch.h))

    def render_batch(self, descs, clear=True, graph=False):
        """descs: list of (width, height, spp, max_depth[, sample_start, min_depth, seed])."""
        flags = (ANA_RENDER_CLEAR_FILM if clear else 0) | (ANA_RENDER_GRAPH if graph else 0)
        arr = (AnaRenderDesc * len(descs))()
        for k, d in enumerate(descs):
            w, h, spp, depth = d[:4]
            start = d[4] if len(d) > 4 else 0
            mind = d[5] if len(d) > 5 else 2
            seed = d[6] if len(d) > 6 else 0
            arr[k] = AnaRenderDesc(w, h, start, spp, depth, mind, seed, 0)
        self._check(lib().ana_render_batch(self.h, arr, len(descs), flags))

    def batch_film(self, item, width, height) -> np.ndarray:
        out = np.zeros((height, width, 5), np.float32)
        self._check(lib().ana_batch_film_read(self.h, item, out.ctypes.data, width * height))
        return out


class Batch:
    """Several prepared scenes concatenated into one device arena."""

    def __init__(self, prepared):
        self.items = list(prepared)
        arr = (_P * len(self.items))(*[p.h for p in self.items])
        h = _P()
        check(lib().ana_batch_create(arr, len(self.items), C.byref(h)))
        self.h = h

    @property
    def nbytes(self) -> int:
        return int(lib().ana_batch_bytes(self.h))

    def __del__(self):
        try:
            if self.h:
                lib().ana_batch_free(self.h)
        except Exception:
            pass


def scene_desc_tuple(sc: S.Scene, sample_start=0, seed=0):
    return (sc.width, sc.height, sc.spp, sc.max_depth, sample_start, 2, seed)


def image_write_exr(path, rgb, albedo=None, normal=None):
    """ana_image_write_exr: (H, W, 3) float images to a ZIP-compressed EXR."""
    rgb = np.ascontiguousarray(rgb, np.float32)
    h, w = rgb.shape[:2]
    al = None if albedo is None else np.ascontiguousarray(albedo, np.float32)
    nr = None if normal is None else np.ascontiguousarray(normal, np.float32)
    check(lib().ana_image_write_exr(str(path).encode(), w, h, rgb.ctypes.data,
                                    al.ctypes.data if al is not None else None,
                                    nr.ctypes.data if nr is not None else None))


def image_write_png(path, rgb, exposure=0.0):
    """ana_image_write_png: (H, W, 3) linear float image to 8-bit sRGB PNG."""
    rgb = np.ascontiguousarray(rgb, np.float32)
    h, w = rgb.shape[:2]
    check(lib().ana_image_write_png(str(path).encode(), w, h, rgb.ctypes.data, exposure))
