"""Synthetic workload generators: sizes stated by the configs, determinism."""
import numpy as np

from anacapa_b200 import scenes as S


def test_cornell():
    sc = S.cornell()
    assert sc.num_triangles == 36 and sc.num_meshes == 8
    assert (sc.width, sc.height, sc.spp, sc.max_depth) == (256, 256, 16, 8)
    assert sc.num_paths == 1_048_576
    assert sc.area_lights[0].Le == (17.0, 12.0, 4.0)
    # the emissive quad coincides with the area light: 0.25 x 0.2
    a = sc.area_lights[0]
    assert abs(2 * a.u[0] - 0.25) < 1e-7 and abs(2 * a.v[2] - 0.2) < 1e-7


def test_throughput_sizes():
    sc = S.throughput()
    assert sc.num_triangles == 4096 * 1280 + 2
    assert (sc.width, sc.height, sc.spp, sc.max_depth) == (1920, 1080, 64, 12)
    assert sc.num_paths == 132_710_400
    assert sc.dome_rgb.shape == (512, 1024, 3) and sc.dome_rgb.max() == np.float32(1e4)
    assert sum(m.metalness for m in sc.materials) > 0.2 * 4096
    rough = np.array([m.roughness for m in sc.materials[:4096]])
    assert rough.min() >= 0.05 and rough.max() <= 1.0


def test_hair_sizes():
    sc = S.hair()
    assert sc.num_strands == 200_000 and sc.num_segments == 800_000
    assert sc.control_points.shape == (200_000 * 13, 3)
    assert (sc.width, sc.height, sc.spp, sc.max_depth) == (1280, 720, 32, 10)
    roots = sc.control_points[::13]
    assert np.allclose(np.linalg.norm(roots, axis=1), 1.0, atol=1e-5)
    # per-strand sigma_a recovered by MarschnerHair.h:430-450 lies in [0.05, 2]
    sig = -np.log(np.maximum(sc.strand_color.astype(np.float64) ** 2.2, 1e-3))
    assert sig.min() > 0.04 and sig.max() < 2.01


def test_batched_variants():
    vs = S.batched_variants()
    assert len(vs) == 64
    assert {v.width for v in vs} <= {64, 128, 256, 384, 512}
    assert {v.spp for v in vs} <= {4, 8, 16, 32, 64}
    assert all(4 <= v.max_depth <= 16 for v in vs)


def test_differentiable_sizes():
    sc = S.differentiable()
    assert sc.num_triangles == 36 + 20480
    assert (sc.width, sc.height, sc.spp) == (512, 512, 16)


def test_determinism():
    a, b = S.throughput(n_spheres=8), S.throughput(n_spheres=8)
    assert np.array_equal(a.positions, b.positions)
    h1, h2 = S.hair(n_strands=100), S.hair(n_strands=100)
    assert np.array_equal(h1.control_points, h2.control_points)
