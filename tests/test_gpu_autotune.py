"""The autotuner (anacapa_b200/autotune.py) on a small batch: it measures
every point of the space it is given, returns the fastest (under its 2 %
switching rule), and every configuration renders the same films (no launch
configuration changes the estimator)."""
import dataclasses

import numpy as np
import pytest

from anacapa_b200 import api
from anacapa_b200 import autotune as A
from anacapa_b200 import scenes as S

pytestmark = pytest.mark.gpu


def films(cfg, scenes):
    r = api.Renderer(chunk_paths=cfg.chunk_paths, block_size=cfg.block_size, traversal=cfg.traversal)
    try:
        batch = api.Batch([api.Prepared(s, max_leaf_tris=cfg.max_leaf_tris) for s in scenes])
        r.upload_batch(batch)
        descs = [api.scene_desc_tuple(s) for s in scenes]
        r.render_batch(descs, graph=True)
        return [r.batch_film(k, s.width, s.height) for k, s in enumerate(scenes)]
    finally:
        r.close()


def test_tuner_picks_the_faster_point_with_identical_films(gpu):
    scenes = S.batched_variants(6, seed=3)
    start = A.Config(chunk_paths=1 << 16, block_size=256, traversal=api.ANA_TRAVERSAL_PERSISTENT, max_leaf_tris=4)
    space = {"chunk_paths": [1 << 16, 1 << 22]}
    t = A.Tuner(scenes, repeats=2)
    best = t.tune(start=start, rounds=1, space=space)
    assert len(t.table) == 2 and all("error" not in row for row in t.table)
    ms = {row["chunk_paths"]: row["ms"] for row in t.table}
    other = 1 << 22
    expect = other if ms[other] < ms[1 << 16] * 0.98 else 1 << 16
    assert best.chunk_paths == expect, t.table
    assert t.best_ms == ms[expect]
    # a 64K-path chunk runs the 6 variants in many chunks, a 4M one in one:
    # the films are bit-identical
    a = films(start, scenes)
    b = films(dataclasses.replace(start, chunk_paths=other), scenes)
    for fa, fb in zip(a, b):
        assert np.array_equal(fa, fb)


def test_tuned_point_reads_the_recorded_table():
    p = A.tuned_point("batched")
    assert set(p) >= {"chunk", "block", "traversal", "leaf"}
    assert p["block"] in A.SPACE["block_size"] and p["leaf"] in A.SPACE["max_leaf_tris"]
