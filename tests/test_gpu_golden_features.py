"""The CUDA path against the committed feature fixtures (no reference build
needed at run time): per-sample radiance of the directional-light (cone),
glass / alpha-mask and motion-blur scenes against PathIntegrator::Li, and
timed closest hits of the motion scene against BVHBackend (ids bit-exact
except ties, distances bit-exact where the ids agree)."""
import os

import numpy as np
import pytest

from anacapa_b200 import api

from test_golden_features import golden_module
from test_gpu_trace import excluded_ties, gpu_ids

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def renderer(gpu):
    r = api.Renderer()
    yield r
    r.close()


@pytest.fixture(scope="module")
def fixtures():
    G = golden_module()
    return G, np.load(os.path.join(HERE, "golden", "feature_vectors.npz"))


@pytest.mark.parametrize("name", ["sunlit", "glass", "motion"])
def test_per_sample_radiance_matches_fixture(renderer, fixtures, name):
    G, gold = fixtures
    sc = G.feature_scenes()[name]
    q = G.feature_queries()[0][name]
    renderer.upload(sc)
    got = np.zeros((len(q), 3), np.float32)
    for s in np.unique(q[:, 2]):
        renderer.render(sc.width, sc.height, 1, sc.max_depth, sample_start=int(s))
        img = renderer.image(sc.width, sc.height)
        sel = q[:, 2] == s
        got[sel] = img[q[sel, 1], q[sel, 0]]
    ref = gold[name + "_li"]
    close = np.all(np.abs(got - ref) <= 1e-4 * np.maximum(np.abs(ref), 1.0), axis=1)
    assert close.mean() >= 0.95, close.mean()


def test_timed_hits_match_fixture(renderer, fixtures):
    G, gold = fixtures
    _, rays, times = G.feature_queries()
    renderer.upload(G.feature_scenes()["motion"])
    g = renderer.trace(rays, times=times)
    ids, t = gold["motion_ids"], gold["motion_t"]
    same = (gpu_ids(g) == ids).all(1)
    assert not (~(same | excluded_ties(g, ids, t))).any()
    hit = ids[:, 0] == 1
    assert np.array_equal(g["t"][hit & same], t[hit & same])
