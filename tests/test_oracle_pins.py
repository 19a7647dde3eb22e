"""Pins the oracles before they are trusted (CPU only).

1. The reference's own unit-test assertions (tests/unit/test_bvh.cpp,
   test_sampler.cpp, test_phase4.cpp), restated, run against the reference
   compiled from its sources (oracle/_ref) and against the CPU restatement
   (oracle/restate) in float and double.
2. The committed golden vectors (tests/golden/make_golden.py, produced by the
   reference build without FMA contraction) against the restatement: float
   mode must reproduce them bit for bit, double mode within 1e-5.
"""
import math

import numpy as np
import pytest

from anacapa_b200 import scenes as S

GOLD = np.load(__import__("os").path.join(__import__("os").path.dirname(__file__), "golden",
                                          "reference_vectors.npz"))


def tri_scene(positions, indices):
    """A one-mesh Lambert scene (the unit tests' GeometryPool)."""
    b = S._Builder()
    m = b.material(S.Material(S.MAT_LAMBERT))
    b.mesh(np.array(positions, np.float32), np.array(indices, np.uint32).reshape(-1, 3), m)
    return b.scene("unit", area_lights=[])


def ray(o, d, tmin=1e-4, tmax=np.inf):
    return np.array([[*o, tmin, *d, tmax]], np.float32)


def oracles(ref_built):
    from oracle import restatebind as P
    R = ref_built

    def ref(sc):
        rs = R.RefScene(sc, variant="record")
        return rs.trace, rs.occluded

    def po(prec):
        def make(sc):
            ps = P.PoScene(sc, prec)

            def occ(r):
                rr = np.array(r, np.float32)
                ids, _ = ps.trace(rr)
                return ids[:, 0] == 1
            return ps.trace, occ
        return make
    return {"reference": ref, "restate32": po(32), "restate64": po(64)}


# ---- tests/unit/test_bvh.cpp -------------------------------------------------
@pytest.mark.parametrize("which", ["reference", "restate32", "restate64"])
def test_bvh_unit(ref_built, which):
    make = oracles(ref_built)[which]
    tr, occ = make(tri_scene([[-1, 0, 0], [1, 0, 0], [0, 1, 0]], [0, 1, 2]))
    ids, t = tr(ray([0, 0.4, -1], [0, 0, 1]))            # SingleTriangleHit (8-25)
    assert ids[0, 0] == 1 and abs(float(t[0]) - 1.0) < 1e-4
    ids, _ = tr(ray([5, 5, -1], [0, 0, 1]))              # SingleTriangleMiss (27-42)
    assert ids[0, 0] == 0
    assert occ(ray([0, 0.3, -2], [0, 0, 1], 1e-4, 5.0))[0]        # OcclusionTest (44-60)
    assert not occ(ray([5, 5, -2], [0, 0, 1], 1e-4, 5.0))[0]
    tr2, _ = make(tri_scene([[-2, 0, 0], [-0.1, 0, 0], [-1, 1, 0], [0.1, 0, 0], [2, 0, 0], [1, 1, 0]],
                            [0, 1, 2, 3, 4, 5]))                  # MultipleTriangles (62-89)
    assert tr2(ray([-1, 0.2, -1], [0, 0, 1]))[0][0, 0] == 1
    assert tr2(ray([1, 0.2, -1], [0, 0, 1]))[0][0, 0] == 1
    assert tr2(ray([0, 0.5, -1], [0, 0, 1]))[0][0, 0] == 0


# ---- tests/unit/test_sampler.cpp ---------------------------------------------
@pytest.mark.parametrize("which", ["reference", "restate"])
def test_sampler_unit(ref_built, which):
    from oracle import restatebind as P
    halton = ref_built.halton if which == "reference" else (lambda x, y, s, n: P.halton(x, y, s, n))
    pcg = ref_built.pcg if which == "reference" else P.pcg
    v = pcg(42, 10000).astype(np.float64) * 2.3283064365386963e-10     # ValuesInRange (9-16)
    assert (v >= 0).all() and (v < 1).all()
    assert np.array_equal(pcg(12345, 100), pcg(12345, 100))          # Reproducible (18-22)
    vals = np.array([halton(0, 0, i, 1)[0] for i in range(1000)])    # Uniformity1D (25-52)
    assert (vals >= 0).all() and (vals < 1).all()
    bins = np.bincount(np.minimum((vals * 10).astype(int), 9), minlength=10)
    chi2 = float(((bins - 100.0) ** 2 / 100.0).sum())
    assert chi2 < 27.88
    v00 = halton(0, 0, 0, 1)[0]                                      # DifferentPixelsDiffer (54-69)
    assert v00 != halton(1, 0, 0, 1)[0] and v00 != halton(0, 1, 0, 1)[0]


# ---- tests/unit/test_phase4.cpp ----------------------------------------------
def test_ggx_ndf_integral(ref_built):
    from oracle import restatebind as P
    a2 = (0.5 * 0.5) ** 2
    for D in (ref_built.lib().ref_ggx_D, P.lib().po_ggx_D):          # NDF_IntegralApproximatelyOne (30-48)
        s = sum(D((i + 0.5) / 512, a2) * ((i + 0.5) / 512) / 512 for i in range(512)) * 2 * math.pi
        assert abs(s - 1.0) < 0.05


def _ref_material_scene(ref_built, mat):
    sc = tri_scene([[-1, 0, 0], [1, 0, 0], [0, 1, 0]], [0, 1, 2])
    sc.materials = [mat]
    return ref_built.RefScene(sc, variant="record", commit=False)


def _flat_si():
    # ShadingContext facing +Z (test_phase4.cpp:15-22): p=0, n=ng=(0,0,1)
    return np.array([0, 0, 0, 0, 0, 1, 0, 0, 1, 1, 0, 0, 1, 1, 1, 0], np.float32)


def test_standard_surface_unit(ref_built):
    L = ref_built.lib()
    fp = lambda a: np.ascontiguousarray(a, np.float32).ctypes.data_as(__import__("ctypes").POINTER(
        __import__("ctypes").c_float))
    si = _flat_si()
    ray_dir = np.array([0, 0, -1], np.float32)
    # DiffuseEnergyConservation (54-89)
    m = S.Material(S.MAT_STANDARD, base_color=(1, 1, 1), metalness=0.0, roughness=1.0, specular=0.0, coat=0.0)
    rs = _ref_material_scene(ref_built, m)
    out = np.zeros(5, np.float32)
    acc = np.zeros(3)
    N = 4096
    wo = np.array([0, 0, 1], np.float32)
    for i in range(N):
        th = math.acos(1 - (i + 0.5) / N)
        ph = 2 * math.pi * 0.618033 * i
        wi = np.array([math.sin(th) * math.cos(ph), math.sin(th) * math.sin(ph), math.cos(th)], np.float32)
        L.ref_mat_evaluate(rs.h, rs.mat_handles[0], fp(si), fp(ray_dir), fp(wo), fp(wi), fp(out))
        acc += out[:3] * abs(wi[2]) * (2 * math.pi / N)
    assert np.all(np.abs(acc - 1.0) < 0.05)
    # SampleReturnsValid (94-118)
    m = S.Material(S.MAT_STANDARD, base_color=(0.8, 0.3, 0.1), metalness=0.5, roughness=0.3)
    rs = _ref_material_scene(ref_built, m)
    wo = np.array([0.1, 0.1, 1.0], np.float32)
    wo /= np.linalg.norm(wo)
    valid = 0
    o8 = np.zeros(8, np.float32)
    for i in range(128):
        ui = (i + 0.5) / 128
        u = np.array([ui, math.fmod(ui * 137, 1)], np.float32)
        L.ref_mat_sample(rs.h, rs.mat_handles[0], fp(si), fp(ray_dir), fp(wo), fp(u),
                         math.fmod(ui * 31, 1), fp(o8))
        if o8[6] > 0 and np.any(o8[:3] != 0):
            assert not np.isnan(o8[:3]).any()
            valid += 1
    assert valid > 89
    # Emission (123-135)
    m = S.Material(S.MAT_STANDARD, emission_w=2.0, emission_color=(1.0, 0.5, 0.0))
    rs = _ref_material_scene(ref_built, m)
    le = np.zeros(3, np.float32)
    L.ref_mat_le(rs.h, rs.mat_handles[0], fp(si), fp(ray_dir), fp(np.array([0, 0, 1], np.float32)), fp(le))
    assert np.allclose(le, [2.0, 1.0, 0.0], atol=1e-5)
    # DiffusePdfSymmetry (140-163)
    m = S.Material(S.MAT_STANDARD, metalness=0.0, roughness=1.0, specular=0.0, coat=0.0)
    rs = _ref_material_scene(ref_built, m)
    a = np.array([0.3, 0.1, 0.9], np.float32)
    a /= np.linalg.norm(a)
    b = np.array([-0.2, 0.4, 0.8], np.float32)
    b /= np.linalg.norm(b)
    eab, eba = np.zeros(5, np.float32), np.zeros(5, np.float32)
    L.ref_mat_evaluate(rs.h, rs.mat_handles[0], fp(si), fp(ray_dir), fp(a), fp(b), fp(eab))
    L.ref_mat_evaluate(rs.h, rs.mat_handles[0], fp(si), fp(ray_dir), fp(b), fp(a), fp(eba))
    assert abs(eab[3] - eba[4]) < 1e-4 and abs(eba[3] - eab[4]) < 1e-4


def test_distribution1d_unit(ref_built):
    out, integ = ref_built.dist1d([1, 3, 2, 4], [0.95])                  # IntegralAndSample (168-181)
    assert abs(integ - 10.0) < 1e-5 and out[0, 0] == 3 and abs(out[0, 1] - 0.4) < 1e-4
    us = np.arange(10000, dtype=np.float32) / 10000                      # SampleConvergesToExpected (183-199)
    out, _ = ref_built.dist1d([1, 1], us)
    assert abs((out[:, 0] == 0).mean() - 0.5) < 0.02
    # golden: the same sampler over 64 u values
    o2, i2 = ref_built.dist1d([1, 3, 2, 4], GOLD["dist_u"], variant="nocontract")
    assert np.array_equal(o2, GOLD["dist_out"]) and i2 == float(GOLD["dist_integral"])


def test_dome_unit(ref_built):
    import ctypes as C
    L = ref_built.lib()
    fp = lambda a: np.ascontiguousarray(a, np.float32).ctypes.data_as(C.POINTER(C.c_float))
    sc = tri_scene([[-1, 0, 0], [1, 0, 0], [0, 1, 0]], [0, 1, 2])
    for intensity, le_expect in ((1.0, None), (2.0, 2.0)):
        rs = ref_built.RefScene(sc, variant="record", commit=False)
        h = L.ref_light_dome(rs.h, None, 0, 0, intensity, 1)    # DomeLight("") 1x1 fallback
        out = np.zeros(8, np.float32)
        L.ref_light_sample(rs.h, h, fp([0, 0, 0]), fp([0, 0, 1]), fp([0.3, 0.7]), fp(out))
        assert out[6] > 0 and not np.isnan(out[:3]).any() and out[7] == np.float32(1e10)   # (204-215)
        assert L.ref_light_pdf(rs.h, h, fp([0, 0, 0]), fp([1, 0, 0])) > 0                  # (217-227)
        assert L.ref_light_pdf(rs.h, h, fp([0, 0, 0]), fp([0, 1, 0])) > 0
        o6 = np.zeros(6, np.float32)
        L.ref_light_sample_le(rs.h, h, fp([0.25, 0.75]), fp([0.1, 0.9]), fp(o6))            # (229-238)
        assert o6[0] > 0 and o6[1] > 0 and o6[2] > 0
        if le_expect is not None:                                                           # (240-245)
            le = np.zeros(3, np.float32)
            L.ref_light_le(rs.h, h, fp([0, 1, 0]), fp(le))
            assert np.all(np.abs(le - le_expect) < 0.1)


# ---- golden vectors vs the restatement -----------------------------------------------
def test_restatement_matches_golden_bit_exact(ref_built):
    from oracle import restatebind as P
    hv = np.stack([P.halton(int(x), int(y), int(s), 140) for x, y, s in GOLD["halton_pts"]])
    assert np.array_equal(hv, GOLD["halton_vals"])
    pv = np.stack([P.pcg(int(s), 16) for s in GOLD["pcg_seeds"]])
    assert np.array_equal(pv, GOLD["pcg_vals"])
    ps = P.PoScene(S.cornell(), 32)
    li = ps.li(GOLD["cornell_li_q"])
    assert np.array_equal(li.astype(np.float32), GOLD["cornell_li"])
    ps = P.PoScene(S.cornell(32, 32, 4), 32)
    rgbw, lsq = ps.render(threads=1)
    assert np.array_equal(rgbw.astype(np.float32), GOLD["cornell32_rgbw"])
    assert np.array_equal(lsq.astype(np.float32), GOLD["cornell32_lumsq"])


def _tie_or_equal(ids, t, gids, gt):
    """Rows agree, or both hit and their distances are within 1e-6 relative (a
    tie between two surfaces: coplanar faces, shared edges)."""
    same = (ids == gids).all(1)
    tie = (ids[:, 0] == 1) & (gids[:, 0] == 1) & (np.abs(t - gt) <= 1e-6 * np.maximum(np.abs(gt), 1e-30))
    return same | tie


@pytest.mark.parametrize("prec", [32, 64])
def test_restatement_hits_match_golden(ref_built, prec):
    from oracle import restatebind as P
    for sc, rk, ik, tk in [(S.cornell(), "cornell_rays", "cornell_ids", "cornell_t"),
                           (S.hair(64, 36, 1, n_strands=2000), "hair_rays", "hair_ids", "hair_t")]:
        ids, t = P.PoScene(sc, prec).trace(GOLD[rk])
        assert _tie_or_equal(ids, t, GOLD[ik], GOLD[tk].astype(np.float64)).all()
        hit = GOLD[ik][:, 0] == 1
        if prec == 32:
            same = (ids == GOLD[ik]).all(1) & hit
            assert np.array_equal(t[same].astype(np.float32), GOLD[tk][same])
        else:
            assert np.max(np.abs(t[hit] - GOLD[tk][hit]) / np.abs(t[hit])) < 1e-5


def test_restatement64_radiance_close(ref_built):
    from oracle import restatebind as P
    li = P.PoScene(S.cornell(), 64).li(GOLD["cornell_li_q"])
    assert np.max(np.abs(li - GOLD["cornell_li"])) < 1e-5 * max(1.0, float(np.abs(GOLD["cornell_li"]).max()))


@pytest.mark.parametrize("half_angle", [0.0, 2.0], ids=["hard", "cone"])
def test_restatement_directional_light_matches_reference(ref_built, half_angle):
    """The restatement's DirectionalLight and its skipped BSDF-sampling branch
    (PathIntegrator.cpp:210) against the reference built without FMA
    contraction: per-sample radiance bit for bit."""
    from oracle import restatebind as P
    sc = S.sunlit(64, 48, 1, 8, half_angle_deg=half_angle)
    rng = np.random.default_rng(11)
    q = np.stack([rng.integers(0, sc.width, 300), rng.integers(0, sc.height, 300),
                  rng.integers(0, 8, 300)], 1).astype(np.uint32)
    ref = ref_built.RefScene(sc, variant="nocontract").li(q)
    li = P.PoScene(sc, 32).li(q).astype(np.float32)
    assert np.array_equal(li, ref)
