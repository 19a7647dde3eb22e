"""Batched renders: several scenes with different resolutions, spp and depths
in one launch sequence (optionally replayed from a CUDA graph) give each item
the same film as rendering it alone."""
import numpy as np
import pytest

from anacapa_b200 import api
from anacapa_b200 import scenes as S

pytestmark = pytest.mark.gpu


def small_variants():
    vs = S.batched_variants(n=6, seed=3)
    # keep the test quick: cap the resolution and spp of the drawn variants
    for v in vs:
        v.width = v.height = min(v.width, 128)
        v.spp = min(v.spp, 8)
    return vs


@pytest.mark.parametrize("graph", [False, True])
def test_batch_matches_plain(gpu, graph):
    vs = small_variants()
    preps = [api.Prepared(v) for v in vs]
    r = api.Renderer(chunk_paths=1 << 16)  # small chunks: items straddle chunk boundaries
    plain = []
    for v, p in zip(vs, preps):
        r.upload(p)
        r.render_scene(v)
        plain.append(r.film(v.width, v.height))
    batch = api.Batch(preps)
    r.upload_batch(batch)
    descs = [api.scene_desc_tuple(v) for v in vs]
    for rep in range(2 if graph else 1):
        r.render_batch(descs, graph=graph)
        for k, v in enumerate(vs):
            f = r.batch_film(k, v.width, v.height)
            assert np.array_equal(f[..., 3], plain[k][..., 3])
            assert np.allclose(f, plain[k], rtol=1e-6, atol=1e-7), (k, rep)
    st = r.stats()
    assert st.paths == sum(v.num_paths for v in vs)
    r.close()


def test_batch_rejects_mismatched_descs(gpu):
    vs = small_variants()[:2]
    r = api.Renderer()
    r.upload_batch(api.Batch([api.Prepared(v) for v in vs]))
    with pytest.raises(api.AnaError) as e:
        r.render_batch([api.scene_desc_tuple(vs[0])])
    assert e.value.code == api.ANA_ERR_INVALID_ARG
    with pytest.raises(api.AnaError) as e:
        r.render(64, 64, 1, 4)
    assert e.value.code == api.ANA_ERR_STATE
    r.close()


def test_graph_replay_matches_eager(gpu):
    sc = S.cornell(96, 96, 8)
    r = api.Renderer()
    r.upload(sc)
    r.render_scene(sc)
    eager = r.film(96, 96)
    descs = [api.scene_desc_tuple(sc)]
    for _ in range(3):
        r.render_batch(descs, graph=True)
        assert np.array_equal(r.film(96, 96)[..., 3], eager[..., 3])
        assert np.allclose(r.film(96, 96), eager, rtol=1e-6, atol=1e-7)
    r.close()
