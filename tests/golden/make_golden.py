"""Generates the committed golden fixtures from the reference's own code.

    python tests/golden/make_golden.py              # reference_vectors.npz
    python tests/golden/make_golden.py --features   # feature_vectors.npz
    python tests/golden/make_golden.py --bsdf       # bsdf_vectors.npz

Runs here (where the reference tree was compiled into oracle/_ref by
oracle/Makefile); the resulting .npz files travel with the repository, so the
tests that read them need neither the reference tree nor a rebuild. Every
array is produced by the reference build without FMA contraction
(-ffp-contract=off), except where a name says `record` (the reference's
Release flags of record).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from anacapa_b200 import scenes as S  # noqa: E402
from oracle import refbind as R  # noqa: E402


def seeded_rays(seed, n, lo, hi):
    rng = np.random.default_rng(seed)
    o = rng.uniform(lo, hi, (n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((n, 8), np.float32)
    r[:, :3] = o
    r[:, 3] = 1e-4
    r[:, 4:7] = d
    r[:, 7] = np.inf
    return r


def main():
    R.build()
    out = {}
    # --- sampler: HaltonSampler (src/sampling/HaltonSampler.h) and PCG32 ---
    pts = [(0, 0, 0), (1, 0, 0), (0, 1, 0), (17, 33, 5), (255, 255, 15), (1919, 1079, 63),
           (640, 360, 1000), (3, 7, 123456)]
    out["halton_pts"] = np.array(pts, np.uint32)
    out["halton_vals"] = np.stack([R.halton(x, y, s, 140, variant="nocontract") for x, y, s in pts])
    out["pcg_seeds"] = np.array([0, 42, 12345, 2 ** 40 + 7], np.uint64)
    out["pcg_vals"] = np.stack([R.pcg(int(s), 16, variant="nocontract") for s in out["pcg_seeds"]])
    # --- Distribution1D (DomeLight.h:146-182), the reference unit test's input ---
    us = np.linspace(0.0, 0.999, 64).astype(np.float32)
    d, integ = R.dist1d([1.0, 3.0, 2.0, 4.0], us, variant="nocontract")
    out["dist_u"] = us
    out["dist_out"] = d
    out["dist_integral"] = np.float32(integ)
    # --- closest-hit ids on the Cornell scene (1024 seeded rays) ---
    sc = S.cornell()
    rays = seeded_rays(7, 1024, 0.0, 1.0)
    rs = R.RefScene(sc, variant="nocontract")
    ids, t = rs.trace(rays, nthreads=1)
    out["cornell_rays"] = rays
    out["cornell_ids"] = ids
    out["cornell_t"] = t
    occ_rays = rays.copy()
    occ_rays[:, 7] = 0.5
    out["cornell_occ"] = rs.occluded(occ_rays, nthreads=1)
    # --- camera rays and per-sample radiance on Cornell (PathIntegrator::Li) ---
    q = np.array([[x, y, s] for x, y in [(128, 128), (40, 200), (200, 60), (90, 30), (150, 230)]
                  for s in range(8)], np.uint32)
    out["cornell_li_q"] = q
    out["cornell_li"] = rs.li(q, nthreads=1)
    out["cornell_cam"] = rs.camera_rays(q)
    # --- hair scene: closest-hit ids (small strand count) ---
    hs = S.hair(width=64, height=36, spp=1, n_strands=2000)
    hrays = seeded_rays(11, 1024, -1.6, 1.6)
    hr = R.RefScene(hs, variant="nocontract")
    hid, ht = hr.trace(hrays, nthreads=1)
    out["hair_rays"] = hrays
    out["hair_ids"] = hid
    out["hair_t"] = ht
    # --- a small Cornell film at 4 spp (renderTile + merge) ---
    small = S.cornell(width=32, height=32, spp=4)
    sr = R.RefScene(small, variant="nocontract")
    rgbw, lsq, _ = sr.render(nthreads=1)
    out["cornell32_rgbw"] = rgbw
    out["cornell32_lumsq"] = lsq
    np.savez_compressed(os.path.join(HERE, "reference_vectors.npz"), **out)
    print("wrote", os.path.join(HERE, "reference_vectors.npz"))


def feature_queries():
    """The (pixel, sample) queries, rays and ray times of the feature
    fixtures: deterministic, so tests rebuild them from the same seeds."""
    rng = np.random.default_rng(2024)
    q = {}
    for name, (w, h) in {"sunlit": (96, 72), "glass": (96, 72), "motion": (96, 72)}.items():
        q[name] = np.stack([rng.integers(0, w, 256), rng.integers(0, h, 256), rng.integers(0, 4, 256)],
                           1).astype(np.uint32)
    rays = seeded_rays(29, 2048, -2.5, 2.5)
    rays[:, 1] = np.abs(rays[:, 1])
    times = rng.uniform(-0.1, 1.1, len(rays)).astype(np.float32)
    return q, rays, times


def feature_scenes():
    return {"sunlit": S.sunlit(96, 72, 1, 8, half_angle_deg=2.0), "glass": S.glass(96, 72, 1, 8),
            "motion": S.motion(96, 72, 1, 6)}


def features():
    """feature_vectors.npz: per-sample radiance (PathIntegrator::Li) of the
    directional-light, glass / alpha-mask and motion-blur scenes, and timed
    closest hits against the motion scene (BVHBackend with Ray::time)."""
    R.build()
    q, rays, times = feature_queries()
    out = {}
    for name, sc in feature_scenes().items():
        rs = R.RefScene(sc, variant="nocontract")
        out[name + "_li"] = rs.li(q[name], nthreads=1)
        if name == "motion":
            ids, t = rs.trace(rays, nthreads=1, times=times)
            out["motion_ids"] = ids
            out["motion_t"] = t
    np.savez_compressed(os.path.join(HERE, "feature_vectors.npz"), **out)
    print("wrote", os.path.join(HERE, "feature_vectors.npz"))


def bsdf_materials():
    """The materials of the BSDF fixtures: Lambert, standard_surface over
    roughness / metalness / coat, and hair in both modes over eta, sigma_a,
    beta_m, beta_n and the cuticle tilt."""
    M = S.Material
    mats = [M(S.MAT_LAMBERT, albedo=(0.7, 0.4, 0.2))]
    for rough, metal, coat in [(0.05, 0.0, 0.0), (0.3, 0.0, 0.0), (0.6, 1.0, 0.0), (1.0, 0.0, 0.5),
                               (0.15, 1.0, 0.3)]:
        mats.append(M(S.MAT_STANDARD, base_color=(0.8, 0.5, 0.3), roughness=rough, metalness=metal, coat=coat))
    for mode in (0, 1):
        for eta, sa, bm, bn, al in [(1.55, (0.4, 0.65, 1.35), 0.3, 0.3, 2.0), (1.4, (0.05, 0.5, 2.0), 0.15, 0.6, 3.0),
                                    (1.6, (1.5, 1.0, 0.2), 0.6, 0.2, 0.0), (1.55, (0.2, 0.2, 0.2), 0.08, 0.9, 4.0)]:
            mats.append(M(S.MAT_HAIR, eta=eta, sigma_a=sa, beta_m=bm, beta_n=bn, alpha_deg=al, hair_mode=mode))
    return mats


def bsdf_queries(material, n, seed):
    """Seeded shading frames: for hair a unit fiber tangent t and a ribbon
    normal n perpendicular to it, wo on n's side, strand colours white (the
    material's sigma_a) or coloured; for surfaces a normal with wo mostly
    above it; wi anywhere on the sphere; uniform 2-D and component samples."""
    from oracle import refbind as Rb
    rng = np.random.default_rng(seed)

    def unit(k):
        v = rng.normal(size=(k, 3))
        return v / np.linalg.norm(v, axis=1, keepdims=True)

    q = np.zeros(n, Rb.BSDF_QUERY)
    nrm = unit(n)
    hair = material.type == S.MAT_HAIR
    if hair:
        t = unit(n)
        nrm = nrm - t * np.sum(nrm * t, 1, keepdims=True)
        nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
        q["t"] = t
        q["is_curve"] = 1
        col = np.ones((n, 3))
        coloured = rng.random(n) < 0.5
        col[coloured] = rng.uniform(0.05, 0.95, (int(coloured.sum()), 3))
        q["color"] = col
    else:
        q["color"] = 1.0
    wo = unit(n)
    flip = np.sum(wo * nrm, 1) < 0
    if hair:
        wo[flip] = -wo[flip]
    else:  # one in eight below the surface
        below = rng.random(n) < 0.125
        wo[flip != below] = -wo[flip != below]
    q["n"] = nrm
    q["wo"] = wo
    q["wi"] = unit(n)
    q["u"] = rng.random((n, 2))
    q["u_comp"] = rng.random(n)
    return q


def bsdf():
    """bsdf_vectors.npz: IMaterial::evaluate / sample of the reference's
    material classes on seeded shading frames (hair in Kajiya-Kay mode as the
    reference executes it, and through the Marschner branches of
    MarschnerHair.h for hair_mode 1), plus the public Marschner lobe functions
    over a seeded grid. Built without FMA contraction."""
    from oracle import refbind as Rb
    R.build()
    out = {}
    for k, m in enumerate(bsdf_materials()):
        q = bsdf_queries(m, 512, 100 + k)
        out[f"m{k}_query"] = q
        out[f"m{k}_result"] = Rb.RefMaterial(m, variant="nocontract").query(q)
    rng = np.random.default_rng(77)
    n = 4096
    thI = rng.uniform(-np.pi / 2, np.pi / 2, n)
    thR = rng.uniform(-np.pi / 2, np.pi / 2, n)
    v = np.exp(rng.uniform(np.log(2e-3), np.log(1.5), n))
    x = rng.uniform(-np.pi, np.pi, n)
    s = rng.uniform(0.05, 1.2, n)
    u = rng.random(n)
    h = rng.uniform(-0.999, 0.999, n)
    cosO = np.cos(rng.uniform(-1.5, 1.5, n))
    grid = np.stack([np.cos(thI), np.sin(thI), np.cos(thR), np.sin(thR), v, x, s, u, h, cosO], 1).astype(np.float32)
    out["mh_grid"] = grid
    out["mh_eta"] = np.float32(1.55)
    out["mh_sigma_a"] = np.array([0.4, 0.65, 1.35], np.float32)
    out["mh_out"] = Rb.mh_functions(grid, 1.55, out["mh_sigma_a"], variant="nocontract")
    np.savez_compressed(os.path.join(HERE, "bsdf_vectors.npz"), **out)
    print("wrote", os.path.join(HERE, "bsdf_vectors.npz"))


if __name__ == "__main__":
    if "--bsdf" in sys.argv:
        bsdf()
    elif "--features" in sys.argv:
        features()
    else:
        main()
