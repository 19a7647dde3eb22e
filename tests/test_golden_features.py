"""The feature fixtures (tests/golden/feature_vectors.npz, made by
tests/golden/make_golden.py --features from the reference's own code) are
pinned: rebuilt from the compiled reference they come out identical. The GPU
side of these fixtures is tests/test_gpu_golden_features.py."""
import importlib.util
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def golden_module():
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(HERE, "golden", "make_golden.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def test_feature_fixtures_reproduce_from_the_reference(ref_built):
    G = golden_module()
    gold = np.load(os.path.join(HERE, "golden", "feature_vectors.npz"))
    q, rays, times = G.feature_queries()
    for name, sc in G.feature_scenes().items():
        rs = ref_built.RefScene(sc, variant="nocontract")
        assert np.array_equal(rs.li(q[name], nthreads=1), gold[name + "_li"]), name
        assert np.abs(gold[name + "_li"]).sum() > 0
        if name == "motion":
            ids, t = rs.trace(rays, nthreads=1, times=times)
            assert np.array_equal(ids, gold["motion_ids"]) and np.array_equal(t, gold["motion_t"])
            assert (ids[:, 0] == 1).sum() > 200


def test_restatement_lights_glass_motion_match_the_reference_fixtures(restate_built):
    """The CPU restatement in float (oracle/restate) reproduces the
    reference's per-sample radiance bit for bit on the directional-light,
    glass / alpha-mask and motion-blur scenes: the FP64 windows of those
    frames come from the same code in double."""
    G = golden_module()
    gold = np.load(os.path.join(HERE, "golden", "feature_vectors.npz"))
    q, _, _ = G.feature_queries()
    for name, sc in G.feature_scenes().items():
        li = restate_built.PoScene(sc, 32).li(q[name], threads=1)
        assert np.array_equal(li.astype(np.float32), gold[name + "_li"]), name
