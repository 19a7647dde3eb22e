"""Synthetic scenes for the path-tracing hot path.

Every scene is generated deterministically from numpy's PCG64 generator, so the
CUDA renderer and the CPU reference integrator receive byte-identical input.
The scene model mirrors the reference's input format:

* triangle meshes as in ``MeshDesc`` (include/anacapa/accel/GeometryPool.h:28-77):
  positions, optional per-vertex normals and uvs, triangle indices; mesh i is
  ``meshID`` i;
* hair strands as in ``StrandDesc`` (include/anacapa/accel/CurvePool.h:27-55):
  endpoint-sharing cubic Bezier control points, a width list, a material slot
  and a per-strand colour;
* ``slots``: ``SceneView::materials`` (include/anacapa/integrator/IIntegrator.h:150-157),
  indexed by meshID and by ``StrandDesc::materialIndex``;
* lights in ``SceneView::lights`` order: area quads (src/shading/lights/AreaLight.h)
  and at most one equirect dome (src/shading/lights/DomeLight.h), which is also
  ``SceneView::envLight``;
* a pinhole camera as ``Camera::makePinhole`` (IIntegrator.h:49-74).
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional

import numpy as np

# Material type codes (match include/anacapa_b200.h)
MAT_LAMBERT = 0
MAT_EMISSIVE = 1
MAT_STANDARD = 2
MAT_HAIR = 3

LIGHT_AREA = 0
LIGHT_DOME = 1
LIGHT_DIRECTIONAL = 2


@dataclasses.dataclass
class Material:
    type: int
    albedo: tuple = (0.8, 0.8, 0.8)
    emission: tuple = (0.0, 0.0, 0.0)
    # standard_surface (src/shading/StandardSurface.h:117-148 defaults)
    base_color: tuple = (0.8, 0.8, 0.8)
    base: float = 1.0
    metalness: float = 0.0
    roughness: float = 0.5
    specular: float = 1.0
    specular_color: tuple = (1.0, 1.0, 1.0)
    specular_ior: float = 1.5
    coat: float = 0.0
    coat_roughness: float = 0.1
    transmission: float = 0.0
    alpha_mask: bool = False
    opacity: float = 1.0
    emission_w: float = 0.0
    emission_color: tuple = (0.0, 0.0, 0.0)
    # hair (src/shading/MarschnerHair.h:192-198 defaults)
    eta: float = 1.55
    sigma_a: tuple = (0.40, 0.65, 1.35)
    beta_m: float = 0.30
    beta_n: float = 0.30
    alpha_deg: float = 2.0
    hair_mode: int = 0  # 0: as the reference executes it (Kajiya-Kay); 1: Marschner lobes

    def standard_packed(self) -> np.ndarray:
        """20-float packing used by the reference harness (the restatement
        reads the first 18)."""
        return np.array([*self.base_color, self.base, self.metalness, self.roughness,
                         self.specular, *self.specular_color, self.specular_ior, self.coat,
                         self.coat_roughness, self.transmission, self.emission_w,
                         *self.emission_color, float(self.alpha_mask), self.opacity],
                        dtype=np.float32)


@dataclasses.dataclass
class AreaLight:
    center: tuple
    u: tuple
    v: tuple
    Le: tuple


@dataclasses.dataclass
class DirLight:
    """DirectionalLight (src/shading/lights/DirectionalLight.h): direction
    toward the light, radiance, angular radius in degrees (0: hard shadows)."""
    direction: tuple
    Le: tuple
    half_angle_deg: float = 0.0


@dataclasses.dataclass
class Scene:
    name: str
    # meshes, concatenated: vertex/triangle ranges per mesh
    positions: np.ndarray          # (V,3) f32
    normals: Optional[np.ndarray]  # (V,3) f32 or None
    uvs: Optional[np.ndarray]      # (V,2) f32 or None
    indices: np.ndarray            # (T,3) u32, local to the mesh's vertex range
    mesh_vert_offset: np.ndarray   # (M+1,) u32
    mesh_tri_offset: np.ndarray    # (M+1,) u32
    mesh_has_normals: np.ndarray   # (M,) u8
    # strands, concatenated
    strand_cp_offset: np.ndarray   # (S+1,) u32
    control_points: np.ndarray     # (C,3) f32
    strand_width_offset: np.ndarray  # (S+1,) u32
    widths: np.ndarray             # (Wd,) f32
    strand_slot: np.ndarray        # (S,) u32
    strand_color: np.ndarray       # (S,3) f32
    materials: List[Material]
    slots: List[int]               # slot -> material index (-1: none)
    area_lights: List[AreaLight]
    dome_rgb: Optional[np.ndarray] = None   # (H,W,3) f32, row 0 = zenith
    dome_intensity: float = 1.0
    env_radiance: tuple = (0.0, 0.0, 0.0)
    cam_from: tuple = (0.0, 0.0, -2.5)
    cam_at: tuple = (0.0, 0.0, 1.0)
    cam_up: tuple = (0.0, 1.0, 0.0)
    vfov: float = 50.0
    width: int = 256
    height: int = 256
    spp: int = 16
    max_depth: int = 8
    # An already built Camera for width x height (ana_camera.explicit_basis):
    # origin, lowerLeftCorner, horizontal, vertical, basisU, basisV (3 floats
    # each), apertureRadius, focalDistance, shutterOpen, shutterClose. None:
    # built from cam_from/cam_at/cam_up/vfov.
    cam_basis: Optional[tuple] = None
    # SceneView::lights after the area lights, before the dome
    dir_lights: List[DirLight] = dataclasses.field(default_factory=list)
    # Motion blur: per mesh None (static, world space) or a list of
    # (time, 4x4 row-major objectToWorld) keys sorted by time (MeshDesc::
    # motionKeys), the mesh's positions then in object space
    mesh_motion: Optional[list] = None
    # Camera::shutterOpen / shutterClose (normalized), when cam_basis is None
    shutter: tuple = (0.0, 0.0)

    @property
    def num_meshes(self) -> int:
        return len(self.mesh_vert_offset) - 1

    @property
    def num_triangles(self) -> int:
        return int(self.mesh_tri_offset[-1])

    @property
    def num_strands(self) -> int:
        return len(self.strand_cp_offset) - 1

    @property
    def num_segments(self) -> int:
        n = np.diff(self.strand_cp_offset.astype(np.int64))
        return int(np.where(n >= 4, (n - 1) // 3, 0).sum())

    @property
    def num_paths(self) -> int:
        return self.width * self.height * self.spp


class _Builder:
    def __init__(self):
        self.pos: List[np.ndarray] = []
        self.nrm: List[np.ndarray] = []
        self.uv: List[np.ndarray] = []
        self.idx: List[np.ndarray] = []
        self.has_n: List[int] = []
        self.materials: List[Material] = []
        self.slots: List[int] = []

    def material(self, m: Material) -> int:
        self.materials.append(m)
        return len(self.materials) - 1

    def mesh(self, pos, idx, mat: int, nrm=None, uv=None) -> int:
        pos = np.ascontiguousarray(pos, dtype=np.float32).reshape(-1, 3)
        self.pos.append(pos)
        self.nrm.append(np.zeros_like(pos) if nrm is None
                        else np.ascontiguousarray(nrm, dtype=np.float32).reshape(-1, 3))
        self.uv.append(np.zeros((len(pos), 2), np.float32) if uv is None
                       else np.ascontiguousarray(uv, dtype=np.float32).reshape(-1, 2))
        self.idx.append(np.ascontiguousarray(idx, dtype=np.uint32).reshape(-1, 3))
        self.has_n.append(0 if nrm is None else 1)
        self.slots.append(mat)
        return len(self.pos) - 1

    def quad(self, v0, v1, v2, v3, normal, mat: int) -> int:
        n = np.asarray(normal, np.float32)
        n = n / np.linalg.norm(n)
        return self.mesh([v0, v1, v2, v3], [[0, 1, 2], [0, 2, 3]], mat,
                         nrm=np.tile(n, (4, 1)),
                         uv=[[0, 0], [1, 0], [1, 1], [0, 1]])

    def scene(self, name, **kw) -> Scene:
        nv = np.array([0] + [len(p) for p in self.pos], np.int64).cumsum()
        nt = np.array([0] + [len(i) for i in self.idx], np.int64).cumsum()
        strands = kw.pop("strands", None)
        if strands is None:
            strands = dict(strand_cp_offset=np.zeros(1, np.uint32),
                           control_points=np.zeros((0, 3), np.float32),
                           strand_width_offset=np.zeros(1, np.uint32),
                           widths=np.zeros(0, np.float32),
                           strand_slot=np.zeros(0, np.uint32),
                           strand_color=np.zeros((0, 3), np.float32))
        slots = kw.pop("slots", None) or list(self.slots)
        return Scene(
            name=name,
            positions=np.concatenate(self.pos) if self.pos else np.zeros((0, 3), np.float32),
            normals=np.concatenate(self.nrm) if self.nrm else None,
            uvs=np.concatenate(self.uv) if self.uv else None,
            indices=np.concatenate(self.idx) if self.idx else np.zeros((0, 3), np.uint32),
            mesh_vert_offset=nv.astype(np.uint32), mesh_tri_offset=nt.astype(np.uint32),
            mesh_has_normals=np.array(self.has_n, np.uint8),
            materials=list(self.materials), slots=slots, **strands, **kw)


def _rot_y(p, pivot, deg):
    a = math.radians(deg)
    c, s = math.cos(a), math.sin(a)
    d = np.asarray(p, np.float64) - pivot
    return np.array([c * d[0] + s * d[2], d[1], -s * d[0] + c * d[2]]) + pivot


def _box(b: _Builder, lo, hi, ydeg, mat):
    """12-triangle box rotated about its vertical centre axis."""
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    pivot = np.array([(lo[0] + hi[0]) / 2, lo[1], (lo[2] + hi[2]) / 2])
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    faces = [
        ([x0, y0, z0], [x1, y0, z0], [x1, y0, z1], [x0, y0, z1], [0, -1, 0]),
        ([x0, y1, z1], [x1, y1, z1], [x1, y1, z0], [x0, y1, z0], [0, 1, 0]),
        ([x0, y0, z0], [x0, y1, z0], [x1, y1, z0], [x1, y0, z0], [0, 0, -1]),
        ([x1, y0, z1], [x1, y1, z1], [x0, y1, z1], [x0, y0, z1], [0, 0, 1]),
        ([x0, y0, z1], [x0, y1, z1], [x0, y1, z0], [x0, y0, z0], [-1, 0, 0]),
        ([x1, y0, z0], [x1, y1, z0], [x1, y1, z1], [x1, y0, z1], [1, 0, 0]),
    ]
    pos, nrm, idx = [], [], []
    for k, (a, bb, c, d, n) in enumerate(faces):
        for v in (a, bb, c, d):
            pos.append(_rot_y(v, pivot, ydeg))
            nrm.append(_rot_y(np.asarray(n, float) + pivot, pivot, ydeg) - pivot)
        idx += [[4 * k, 4 * k + 1, 4 * k + 2], [4 * k, 4 * k + 2, 4 * k + 3]]
    return b.mesh(np.array(pos), idx, mat, nrm=np.array(nrm))


CORNELL_LIGHT_LE = (17.0, 12.0, 4.0)


def cornell(width=256, height=256, spp=16, max_depth=8, *, wall_jitter=None,
            box_rot=(-17.0, 17.0), extra=None) -> Scene:
    """Unit-box Cornell scene: 5 walls (10 tris), two 12-tri boxes 0.3 and 0.6
    tall rotated -17/+17 deg about Y, a 0.25 x 0.2 ceiling light carried both as
    an emissive quad and as an AreaLight with emission (17,12,4), Lambert
    materials, pinhole camera with 40 deg vertical FOV. 36 triangles."""
    b = _Builder()
    white = (0.725, 0.71, 0.68)
    red = (0.63, 0.065, 0.05)
    green = (0.14, 0.45, 0.09)
    if wall_jitter is not None:
        white, red, green = (tuple(np.clip(np.asarray(c) + j, 0.0, 0.95))
                             for c, j in zip((white, red, green), wall_jitter))
    mw = b.material(Material(MAT_LAMBERT, albedo=tuple(white)))
    mr = b.material(Material(MAT_LAMBERT, albedo=tuple(red)))
    mg = b.material(Material(MAT_LAMBERT, albedo=tuple(green)))
    ml = b.material(Material(MAT_EMISSIVE, albedo=(0.0, 0.0, 0.0), emission=CORNELL_LIGHT_LE))
    b.quad([0, 0, 0], [1, 0, 0], [1, 0, 1], [0, 0, 1], [0, 1, 0], mw)      # floor
    b.quad([0, 1, 1], [1, 1, 1], [1, 1, 0], [0, 1, 0], [0, -1, 0], mw)     # ceiling
    b.quad([0, 0, 1], [0, 1, 1], [1, 1, 1], [1, 0, 1], [0, 0, -1], mw)     # back
    b.quad([0, 0, 1], [0, 1, 1], [0, 1, 0], [0, 0, 0], [1, 0, 0], mr)      # left
    b.quad([1, 0, 0], [1, 1, 0], [1, 1, 1], [1, 0, 1], [-1, 0, 0], mg)     # right
    ly, cx, cz, hu, hv = 0.999, 0.5, 0.5, 0.125, 0.1
    b.quad([cx - hu, ly, cz - hv], [cx + hu, ly, cz - hv], [cx + hu, ly, cz + hv],
           [cx - hu, ly, cz + hv], [0, -1, 0], ml)
    _box(b, [0.13, 0.0, 0.37], [0.43, 0.3, 0.67], box_rot[0], mw)           # short box
    _box(b, [0.53, 0.0, 0.25], [0.83, 0.6, 0.55], box_rot[1], mw)           # tall box
    if extra is not None:
        extra(b)
    lights = [AreaLight((cx, ly, cz), (hu, 0.0, 0.0), (0.0, 0.0, hv), CORNELL_LIGHT_LE)]
    return b.scene("cornell", area_lights=lights, cam_from=(0.5, 0.5, -1.4),
                   cam_at=(0.5, 0.5, 0.5), cam_up=(0.0, 1.0, 0.0), vfov=40.0,
                   width=width, height=height, spp=spp, max_depth=max_depth)


def icosphere(subdiv: int):
    """Unit icosphere by midpoint subdivision: 20 * 4**subdiv triangles."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = [[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t],
         [0, -1, -t], [0, 1, -t], [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]]
    f = [[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4],
         [11, 10, 2], [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8],
         [3, 8, 9], [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]]
    verts = [np.asarray(p, np.float64) / np.linalg.norm(p) for p in v]
    faces = np.array(f, np.int64)
    for _ in range(subdiv):
        cache = {}

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b_, c in faces:
            ab, bc, ca = mid(a, b_), mid(b_, c), mid(c, a)
            nf += [[a, ab, ca], [b_, bc, ab], [c, ca, bc], [ab, bc, ca]]
        faces = np.array(nf, np.int64)
    return np.array(verts), faces.astype(np.uint32)


def sky_dome(width=1024, height=512, sun_elev_deg=35.0, sun_azim_deg=40.0,
             sun_radius_deg=0.25, sun_intensity=1.0e4) -> np.ndarray:
    """Procedural equirect (row 0 = zenith, DomeLight.h:190-201 convention):
    a zenith-to-horizon sky gradient, a dim ground below the horizon and a
    0.5 deg sun disc of radiance 1e4."""
    v = (np.arange(height) + 0.5) / height
    u = (np.arange(width) + 0.5) / width
    theta = v[:, None] * math.pi
    phi = u[None, :] * 2.0 * math.pi
    d = np.stack([np.sin(theta) * np.sin(phi), np.cos(theta) * np.ones_like(phi),
                  np.sin(theta) * np.cos(phi)], -1)
    up = np.clip(d[..., 1], -1.0, 1.0)
    zen = np.array([0.25, 0.45, 0.95])
    hor = np.array([0.85, 0.90, 1.00])
    gnd = np.array([0.20, 0.18, 0.16])
    t = np.clip(up, 0.0, 1.0)[..., None] ** 0.5
    img = np.where(up[..., None] >= 0.0, hor * (1 - t) + zen * t, gnd * np.ones_like(t))
    el, az = math.radians(sun_elev_deg), math.radians(sun_azim_deg)
    s = np.array([math.cos(el) * math.sin(az), math.sin(el), math.cos(el) * math.cos(az)])
    cosang = (d * s).sum(-1)
    img[cosang >= math.cos(math.radians(sun_radius_deg))] = sun_intensity
    return np.ascontiguousarray(img.astype(np.float32))


def throughput(width=1920, height=1080, spp=64, max_depth=12, n_spheres=4096,
               subdiv=3, dome_size=(1024, 512), seed=0) -> Scene:
    """n_spheres icospheres (subdivision 3: 1280 tris each) with centres
    U[-10,10]^3 and radii U[0.1,0.6], smooth vertex normals, plus a ground quad;
    GGX standard_surface: base colour U[0,1]^3, roughness U[0.05,1],
    metalness Bernoulli(0.3), coat 0; procedural 1024x512 HDR dome with a 0.5
    deg sun at 1e4, importance-sampled; 1920x1080, 64 spp, depth 12."""
    rng = np.random.default_rng(seed)
    b = _Builder()
    uv_, f_ = icosphere(subdiv)
    centers = rng.uniform(-10.0, 10.0, (n_spheres, 3))
    radii = rng.uniform(0.1, 0.6, n_spheres)
    base = rng.uniform(0.0, 1.0, (n_spheres, 3))
    rough = rng.uniform(0.05, 1.0, n_spheres)
    metal = (rng.uniform(0.0, 1.0, n_spheres) < 0.3).astype(np.float64)
    for i in range(n_spheres):
        m = b.material(Material(MAT_STANDARD, base_color=tuple(base[i]), roughness=float(rough[i]),
                                metalness=float(metal[i]), coat=0.0))
        b.mesh(centers[i] + radii[i] * uv_, f_, m, nrm=uv_)
    mg = b.material(Material(MAT_STANDARD, base_color=(0.45, 0.45, 0.45), roughness=0.7))
    # The ground rises 0.1 over its 120-unit depth. An exactly level quad at
    # |y| = 10.6 has a zero-thickness box once the reference's 1e-7 padding
    # (BVHBackend.cpp, sahSplit) is rounded away, so its slab test never
    # passes and the plane would be invisible to the reference and to us.
    g, y0, y1 = 60.0, -10.6, -10.5
    gn = np.array([0.0, 2.0 * g, -(y1 - y0)])
    gn /= np.linalg.norm(gn)
    b.quad([-g, y0, -g], [-g, y1, g], [g, y1, g], [g, y0, -g], gn, mg)
    dome = sky_dome(*dome_size)
    return b.scene("throughput", area_lights=[], dome_rgb=dome, dome_intensity=1.0,
                   cam_from=(0.0, 6.0, -32.0), cam_at=(0.0, -1.0, 0.0), cam_up=(0.0, 1.0, 0.0),
                   vfov=40.0, width=width, height=height, spp=spp, max_depth=max_depth)


def hair(width=1280, height=720, spp=32, max_depth=10, n_strands=200_000, seed=0,
         hair_mode=0) -> Scene:
    """n_strands cubic Bezier strands of 4 segments (13 CVs), roots uniform on
    the unit sphere, length U[0.3,0.6] with a random bend, width 0.002 at the
    root tapering to 0.0005 (2-entry width list), per-strand absorption
    sigma_a U[0.05,2]^3 (carried as the strand colour c = exp(-sigma_a)^(1/2.2),
    which MarschnerHair.h:430-450 inverts), eta 1.55, beta_m = beta_n = 0.3,
    alpha 2 deg; one area light quad (with matching emissive geometry)."""
    rng = np.random.default_rng(seed)
    b = _Builder()
    mh = b.material(Material(MAT_HAIR, eta=1.55, sigma_a=(0.4, 0.65, 1.35), beta_m=0.3,
                             beta_n=0.3, alpha_deg=2.0, hair_mode=hair_mode))
    le = (30.0, 30.0, 30.0)
    ml = b.material(Material(MAT_EMISSIVE, albedo=(0.0, 0.0, 0.0), emission=le))
    c = np.array([1.6, 2.4, -1.8])
    u = np.array([0.5, 0.0, 0.0])
    w_ = np.array([0.0, 0.30, 0.40])
    b.quad(c - u - w_, c + u - w_, c + u + w_, c - u + w_, np.cross(u, w_), ml)
    # strands
    z = rng.uniform(-1.0, 1.0, n_strands)
    ph = rng.uniform(0.0, 2.0 * math.pi, n_strands)
    r = np.sqrt(1.0 - z * z)
    root = np.stack([r * np.cos(ph), z, r * np.sin(ph)], -1)
    length = rng.uniform(0.3, 0.6, n_strands)
    bend = rng.normal(0.0, 1.0, (n_strands, 3))
    bend -= (bend * root).sum(-1, keepdims=True) * root
    bend *= 0.35
    ts = np.linspace(0.0, 1.0, 13)
    # quadratic bend profile along the strand, then sampled at 13 CVs
    cps = (root[:, None, :] * (1.0 + length[:, None, None] * ts[None, :, None])
           + bend[:, None, :] * (length[:, None, None] * ts[None, :, None] ** 2))
    cps = cps.astype(np.float32).reshape(-1, 3)
    sigma = rng.uniform(0.05, 2.0, (n_strands, 3))
    color = np.exp(-sigma) ** (1.0 / 2.2)
    strands = dict(
        strand_cp_offset=(np.arange(n_strands + 1, dtype=np.int64) * 13).astype(np.uint32),
        control_points=np.ascontiguousarray(cps),
        strand_width_offset=(np.arange(n_strands + 1, dtype=np.int64) * 2).astype(np.uint32),
        widths=np.tile(np.array([0.002, 0.0005], np.float32), n_strands),
        strand_slot=np.full(n_strands, 1, np.uint32),
        strand_color=color.astype(np.float32))
    # slot 0 = light mesh, slot 1 = hair material
    return b.scene("hair", strands=strands, slots=[ml, mh],
                   area_lights=[AreaLight(tuple(c), tuple(u), tuple(w_), le)],
                   cam_from=(0.0, 0.3, -4.2), cam_at=(0.0, 0.0, 0.0), cam_up=(0.0, 1.0, 0.0),
                   vfov=40.0, width=width, height=height, spp=spp, max_depth=max_depth)


def batched_variants(n=64, seed=0):
    """n Cornell variants: wall albedos jittered +-0.1, inner-box rotation
    U[0,90] deg, resolution from {64,128,256,384,512}^2, spp from
    {4,8,16,32,64}, max depth U{4..16}."""
    rng = np.random.default_rng(seed)
    res = [64, 128, 256, 384, 512]
    spps = [4, 8, 16, 32, 64]
    out = []
    for _ in range(n):
        jit = rng.uniform(-0.1, 0.1, (3, 3))
        rot = rng.uniform(0.0, 90.0, 2)
        r = int(rng.choice(res))
        s = int(rng.choice(spps))
        d = int(rng.integers(4, 17))
        out.append(cornell(r, r, s, d, wall_jitter=jit, box_rot=(float(rot[0]), float(rot[1]))))
    return out


def differentiable(width=512, height=512, spp=16, max_depth=8, subdiv=5,
                   params=None) -> Scene:
    """Cornell box with a subdivided-icosphere centrepiece (subdivision 5:
    20,480 triangles) and 6 standard_surface materials (white walls, red, green,
    short box, tall box, sphere) whose RGB albedo and roughness are the
    differentiable parameters; the light emission RGB is a parameter shared by
    the emissive quad and the AreaLight."""
    if params is None:
        params = default_diff_params()
    alb, rough, emis = params["albedo"], params["roughness"], params["emission"]
    b = _Builder()
    mats = [b.material(Material(MAT_STANDARD, base_color=tuple(map(float, alb[k])),
                                roughness=float(rough[k]), metalness=0.0, specular=1.0))
            for k in range(6)]
    ml = b.material(Material(MAT_EMISSIVE, albedo=(0.0, 0.0, 0.0), emission=tuple(map(float, emis))))
    b.quad([0, 0, 0], [1, 0, 0], [1, 0, 1], [0, 0, 1], [0, 1, 0], mats[0])
    b.quad([0, 1, 1], [1, 1, 1], [1, 1, 0], [0, 1, 0], [0, -1, 0], mats[0])
    b.quad([0, 0, 1], [0, 1, 1], [1, 1, 1], [1, 0, 1], [0, 0, -1], mats[0])
    b.quad([0, 0, 1], [0, 1, 1], [0, 1, 0], [0, 0, 0], [1, 0, 0], mats[1])
    b.quad([1, 0, 0], [1, 1, 0], [1, 1, 1], [1, 0, 1], [-1, 0, 0], mats[2])
    ly, cx, cz, hu, hv = 0.999, 0.5, 0.5, 0.125, 0.1
    b.quad([cx - hu, ly, cz - hv], [cx + hu, ly, cz - hv], [cx + hu, ly, cz + hv],
           [cx - hu, ly, cz + hv], [0, -1, 0], ml)
    _box(b, [0.13, 0.0, 0.37], [0.43, 0.3, 0.67], -17.0, mats[3])
    _box(b, [0.53, 0.0, 0.25], [0.83, 0.6, 0.55], 17.0, mats[4])
    v, f = icosphere(subdiv)
    ctr, rad = np.array([0.3, 0.45, 0.22]), 0.14
    b.mesh(ctr + rad * v, f, mats[5], nrm=v)
    lights = [AreaLight((cx, ly, cz), (hu, 0.0, 0.0), (0.0, 0.0, hv), tuple(map(float, emis)))]
    return b.scene("differentiable", area_lights=lights, cam_from=(0.5, 0.5, -1.4),
                   cam_at=(0.5, 0.5, 0.5), cam_up=(0.0, 1.0, 0.0), vfov=40.0,
                   width=width, height=height, spp=spp, max_depth=max_depth)


def default_diff_params():
    return {
        "albedo": np.array([[0.725, 0.71, 0.68], [0.63, 0.065, 0.05], [0.14, 0.45, 0.09],
                            [0.70, 0.70, 0.70], [0.60, 0.60, 0.65], [0.80, 0.55, 0.30]],
                           np.float32),
        "roughness": np.array([0.9, 0.8, 0.8, 0.6, 0.4, 0.3], np.float32),
        "emission": np.array(CORNELL_LIGHT_LE, np.float32),
    }


def perturbed_diff_params(seed=1):
    rng = np.random.default_rng(seed)
    p = default_diff_params()
    p["albedo"] = np.clip(p["albedo"] + rng.uniform(-0.2, 0.2, p["albedo"].shape), 0.02, 0.95
                          ).astype(np.float32)
    p["roughness"] = np.clip(p["roughness"] + rng.uniform(-0.15, 0.15, 6), 0.05, 1.0
                             ).astype(np.float32)
    return p


def sunlit(width=256, height=192, spp=16, max_depth=8, half_angle_deg=0.0, n_spheres=12, seed=3) -> Scene:
    """A ground quad and n_spheres subdivision-2 icospheres (standard_surface,
    random base colour and roughness, a third metallic) lit by a
    DirectionalLight (DirectionalLight.h; half_angle_deg 0: hard shadows, else a
    soft cone) and a small area light, under a constant environment radiance.
    Light selection alternates between a delta light (no BSDF-sampled MIS ray)
    and an area light (with one)."""
    rng = np.random.default_rng(seed)
    b = _Builder()
    mg = b.material(Material(MAT_LAMBERT, albedo=(0.5, 0.5, 0.5)))
    # The ground rises 0.1 over its depth and the area light tilts by 0.02:
    # an exactly level quad has a zero-thickness box once the reference's
    # 1e-7 padding (BVHBackend.cpp, sahSplit) rounds away against |y| - |oy|,
    # and its slab test then rejects every ray.
    g, y0, y1 = 6.0, 0.0, 0.1
    gn = np.array([0.0, 2.0 * g, -(y1 - y0)])
    gn /= np.linalg.norm(gn)
    b.quad([-g, y0, -g], [-g, y1, g], [g, y1, g], [g, y0, -g], gn, mg)
    v, f = icosphere(2)
    for _ in range(n_spheres):
        m = b.material(Material(MAT_STANDARD, base_color=tuple(map(float, rng.uniform(0.1, 0.9, 3))),
                                roughness=float(rng.uniform(0.1, 0.9)),
                                metalness=float(rng.uniform() < 0.33)))
        r = float(rng.uniform(0.3, 0.8))
        c = np.array([rng.uniform(-3, 3), r + 0.05, rng.uniform(-3, 3)])
        b.mesh(c + r * v, f, m, nrm=v)
    le = (6.0, 5.0, 4.0)
    ml = b.material(Material(MAT_EMISSIVE, albedo=(0.0, 0.0, 0.0), emission=le))
    lc, lu, lv = np.array([2.0, 3.5, 1.0]), np.array([0.4, 0.0, 0.0]), np.array([0.0, 0.02, 0.3])
    ln = np.cross(lu, lv)
    ln /= np.linalg.norm(ln)
    b.quad(lc - lu - lv, lc + lu - lv, lc + lu + lv, lc - lu + lv, ln, ml)
    return b.scene("sunlit", area_lights=[AreaLight(tuple(lc), tuple(lu), tuple(lv), le)],
                   dir_lights=[DirLight((-0.4, 0.8, -0.3), (3.0, 2.8, 2.5), half_angle_deg)],
                   env_radiance=(0.05, 0.07, 0.1),
                   cam_from=(0.0, 4.0, -9.0), cam_at=(0.0, 0.5, 0.0), cam_up=(0.0, 1.0, 0.0),
                   vfov=45.0, width=width, height=height, spp=spp, max_depth=max_depth)


def glass(width=192, height=144, spp=16, max_depth=8, seed=5) -> Scene:
    """Transmission and alpha testing (StandardSurface.h:197-414,
    PathIntegrator.cpp:103-118, ShadowRay.h): on the tilted ground of `sunlit`,
    a smooth glass sphere (IOR 1.5, delta), a rough glass sphere (roughness
    0.3, GGX transmission), a smooth tinted water sphere (IOR 1.33), a smooth
    mirror (roughness 0, metal: a delta opaque material), two alpha-masked
    cards (opacity 0.4: stochastic, one sample dimension per test; opacity 0:
    cut out without one) and two glass panes, lit by an area light, a
    directional light and a constant environment. Cards and panes are turned
    about y so that no box is flat."""
    rng = np.random.default_rng(seed)
    b = _Builder()
    mg = b.material(Material(MAT_LAMBERT, albedo=(0.55, 0.5, 0.45)))
    g, y0, y1 = 6.0, 0.0, 0.1
    gn = np.array([0.0, 2.0 * g, -(y1 - y0)])
    gn /= np.linalg.norm(gn)
    b.quad([-g, y0, -g], [-g, y1, g], [g, y1, g], [g, y0, -g], gn, mg)
    v, f = icosphere(3)
    spheres = [
        (Material(MAT_STANDARD, base_color=(1.0, 1.0, 1.0), roughness=0.0, transmission=1.0,
                  specular_ior=1.5), (-1.6, 0.8, 0.2), 0.75),
        (Material(MAT_STANDARD, base_color=(0.9, 0.95, 1.0), roughness=0.3, transmission=1.0,
                  specular_ior=1.5), (0.4, 0.7, 0.9), 0.6),
        (Material(MAT_STANDARD, base_color=(0.7, 0.9, 0.8), roughness=0.0, transmission=0.9,
                  specular_ior=1.33), (1.9, 0.55, -0.6), 0.5),
        (Material(MAT_STANDARD, base_color=(0.9, 0.85, 0.7), roughness=0.0, metalness=1.0),
         (-0.2, 0.45, -1.3), 0.4),
        (Material(MAT_STANDARD, base_color=(0.8, 0.3, 0.2), roughness=0.4), (2.6, 0.5, 1.8), 0.45),
    ]
    for m, c, r in spheres:
        b.mesh(np.asarray(c) + r * v, f, b.material(m), nrm=v)

    def card(mat, c, half_w, half_h, yaw_deg):
        a = np.radians(yaw_deg)
        u = np.array([np.cos(a), 0.0, np.sin(a)]) * half_w
        w = np.array([0.05, 1.0, 0.03]) * half_h
        c = np.asarray(c, np.float64)
        n = np.cross(u, w)
        b.quad(c - u - w, c + u - w, c + u + w, c - u + w, n / np.linalg.norm(n), mat)

    leaf = b.material(Material(MAT_STANDARD, base_color=(0.3, 0.6, 0.2), roughness=0.6, alpha_mask=True,
                               opacity=0.4))
    cutout = b.material(Material(MAT_STANDARD, base_color=(0.9, 0.1, 0.1), roughness=0.5, alpha_mask=True,
                                 opacity=0.0))
    pane = b.material(Material(MAT_STANDARD, base_color=(0.95, 0.9, 0.8), roughness=0.0, transmission=1.0,
                               specular_ior=1.5))
    frosted = b.material(Material(MAT_STANDARD, base_color=(0.9, 0.9, 1.0), roughness=0.15, transmission=1.0,
                                  specular_ior=1.5))
    card(leaf, (-0.6, 1.0, -2.4), 0.8, 0.9, 25.0)
    card(cutout, (1.2, 0.9, -2.2), 0.6, 0.8, -30.0)
    card(pane, (0.9, 1.1, 2.6), 1.1, 1.0, 15.0)
    card(frosted, (-2.4, 1.0, 1.9), 0.8, 0.9, -40.0)
    for _ in range(6):
        m = b.material(Material(MAT_STANDARD, base_color=tuple(map(float, rng.uniform(0.1, 0.9, 3))),
                                roughness=float(rng.uniform(0.1, 0.9))))
        r = float(rng.uniform(0.2, 0.35))
        c = np.array([rng.uniform(-4, 4), r + 0.05, rng.uniform(-4, 4)])
        b.mesh(c + r * icosphere(1)[0], icosphere(1)[1], m, nrm=icosphere(1)[0])
    le = (7.0, 6.0, 5.0)
    ml = b.material(Material(MAT_EMISSIVE, albedo=(0.0, 0.0, 0.0), emission=le))
    lc, lu, lv = np.array([-1.0, 3.2, -0.5]), np.array([0.5, 0.0, 0.0]), np.array([0.0, 0.03, 0.4])
    ln = np.cross(lu, lv)
    ln /= np.linalg.norm(ln)
    b.quad(lc - lu - lv, lc + lu - lv, lc + lu + lv, lc - lu + lv, ln, ml)
    return b.scene("glass", area_lights=[AreaLight(tuple(lc), tuple(lu), tuple(lv), le)],
                   dir_lights=[DirLight((0.5, 0.7, -0.4), (2.5, 2.4, 2.2), 1.5)],
                   env_radiance=(0.15, 0.18, 0.25),
                   cam_from=(0.0, 3.2, -7.5), cam_at=(0.0, 0.6, 0.0), cam_up=(0.0, 1.0, 0.0),
                   vfov=45.0, width=width, height=height, spp=spp, max_depth=max_depth)


def _trs(t, yaw_deg=0.0, s=1.0):
    """Row-major objectToWorld: translate(t) * rotate_y(yaw) * scale(s)."""
    a = np.radians(yaw_deg)
    c, n = np.cos(a), np.sin(a)
    M = np.array([[c * s, 0.0, n * s, t[0]], [0.0, s, 0.0, t[1]], [-n * s, 0.0, c * s, t[2]],
                  [0.0, 0.0, 0.0, 1.0]], np.float32)
    return M


def motion(width=128, height=96, spp=16, max_depth=6, shutter=(0.0, 1.0), seed=9) -> Scene:
    """Motion blur (MeshDesc::motionKeys, BVHBackend.cpp:35-50, 86-95, 356-367):
    on the tilted ground of `sunlit`, spheres kept in object space with 2 keys
    (a translation), 3 keys (translation with a yaw; keys at 0, 0.4, 1) and a
    growing scale, a moving box, and static spheres, lit by an area light and a
    constant environment; the camera's shutter samples each path's time."""
    rng = np.random.default_rng(seed)
    b = _Builder()
    mg = b.material(Material(MAT_LAMBERT, albedo=(0.5, 0.5, 0.5)))
    g, y0, y1 = 6.0, 0.0, 0.1
    gn = np.array([0.0, 2.0 * g, -(y1 - y0)])
    gn /= np.linalg.norm(gn)
    b.quad([-g, y0, -g], [-g, y1, g], [g, y1, g], [g, y0, -g], gn, mg)
    v, f = icosphere(2)
    keys = [None]
    movers = [
        [(0.0, _trs((-2.0, 0.6, 0.0), 0.0, 0.5)), (1.0, _trs((-0.8, 0.6, 0.3), 0.0, 0.5))],
        [(0.0, _trs((0.5, 0.7, 1.0), 0.0, 0.6)), (0.4, _trs((0.9, 1.1, 1.2), 40.0, 0.6)),
         (1.0, _trs((1.6, 0.7, 1.0), 90.0, 0.6))],
        [(0.0, _trs((1.8, 0.5, -1.2), 0.0, 0.3)), (1.0, _trs((1.8, 0.75, -1.2), 0.0, 0.55))],
    ]
    for mk in movers:
        m = b.material(Material(MAT_STANDARD, base_color=tuple(map(float, rng.uniform(0.2, 0.9, 3))),
                                roughness=float(rng.uniform(0.2, 0.7))))
        b.mesh(v, f, m, nrm=v)
        keys.append(mk)
    # a box, turned and moving
    bv = np.array([[x, y, z] for x in (-0.4, 0.4) for y in (-0.4, 0.4) for z in (-0.4, 0.4)], np.float32)
    bf = np.array([[0, 1, 3], [0, 3, 2], [4, 6, 7], [4, 7, 5], [0, 4, 5], [0, 5, 1],
                   [2, 3, 7], [2, 7, 6], [0, 2, 6], [0, 6, 4], [1, 5, 7], [1, 7, 3]], np.uint32)
    mb = b.material(Material(MAT_STANDARD, base_color=(0.8, 0.7, 0.3), roughness=0.35, metalness=1.0))
    b.mesh(bv, bf, mb)
    keys.append([(0.0, _trs((-1.5, 0.5, -1.5), 20.0)), (1.0, _trs((-1.0, 0.5, -1.7), 50.0))])
    for _ in range(4):
        m = b.material(Material(MAT_STANDARD, base_color=tuple(map(float, rng.uniform(0.1, 0.9, 3))),
                                roughness=float(rng.uniform(0.2, 0.9))))
        r = float(rng.uniform(0.3, 0.5))
        c = np.array([rng.uniform(-3, 3), r + 0.05, rng.uniform(1.5, 3.5)])
        b.mesh(c + r * v, f, m, nrm=v)
        keys.append(None)
    le = (6.0, 5.0, 4.0)
    ml = b.material(Material(MAT_EMISSIVE, albedo=(0.0, 0.0, 0.0), emission=le))
    lc, lu, lv = np.array([0.5, 3.5, -0.5]), np.array([0.6, 0.0, 0.0]), np.array([0.0, 0.02, 0.5])
    ln = np.cross(lu, lv)
    ln /= np.linalg.norm(ln)
    b.quad(lc - lu - lv, lc + lu - lv, lc + lu + lv, lc - lu + lv, ln, ml)
    keys.append(None)
    return b.scene("motion", area_lights=[AreaLight(tuple(lc), tuple(lu), tuple(lv), le)],
                   env_radiance=(0.1, 0.12, 0.16),
                   cam_from=(0.0, 3.5, -7.0), cam_at=(0.0, 0.6, 0.0), cam_up=(0.0, 1.0, 0.0),
                   vfov=45.0, width=width, height=height, spp=spp, max_depth=max_depth,
                   mesh_motion=keys, shutter=tuple(shutter))
