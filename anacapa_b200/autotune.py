"""Autotuner for the wavefront launch configuration.

Searches, by coordinate descent on measured device time, over
  * chunk capacity (paths in flight per wavefront chunk, i.e. queue size),
  * the block size of the shading/generation kernels,
  * the traversal schedule (persistent warps with refill, or thread per ray),
  * the BVH leaf width (maximum triangles per leaf; rebuilds the BVHs).
Each candidate renders the given workload once after one warm-up render, and
the fastest configuration is returned with the full table of measurements.
Results are identical across configurations (none changes the estimator).
"""
from __future__ import annotations

import dataclasses
import time
from typing import Dict, List, Sequence

from . import api
from . import scenes as S


@dataclasses.dataclass(frozen=True)
class Config:
    chunk_paths: int = 1 << 25
    block_size: int = 256
    traversal: int = api.ANA_TRAVERSAL_PERSISTENT
    max_leaf_tris: int = 4


SPACE = {
    "chunk_paths": [1 << 21, 1 << 22, 1 << 23, 1 << 24, 1 << 25, 1 << 26],
    "block_size": [128, 256],  # the shading kernel's blocks (at most 256 threads)
    "traversal": [api.ANA_TRAVERSAL_PERSISTENT, api.ANA_TRAVERSAL_PER_RAY],
    "max_leaf_tris": [2, 4, 8],
}


class Tuner:
    """Times a batch of scenes (one item = a plain render) under configs."""

    def __init__(self, scenes: Sequence[S.Scene], device=0, graph=True, repeats=1):
        self.scenes = list(scenes)
        self.device = device
        self.graph = graph
        self.repeats = repeats
        self._prep: Dict[int, List[api.Prepared]] = {}
        self.table: List[dict] = []

    def _prepared(self, leaf):
        if leaf not in self._prep:
            self._prep[leaf] = [api.Prepared(s, max_leaf_tris=leaf) for s in self.scenes]
        return self._prep[leaf]

    def measure(self, cfg: Config) -> float:
        """Device time of one render of the workload under cfg (inf if the
        configuration is rejected; the error is kept in the table)."""
        best, error = float("inf"), None
        r = None
        try:
            r = api.Renderer(device=self.device, chunk_paths=cfg.chunk_paths, block_size=cfg.block_size,
                             traversal=cfg.traversal)
            preps = self._prepared(cfg.max_leaf_tris)
            batch = api.Batch(preps)
            r.upload_batch(batch)
            descs = [api.scene_desc_tuple(s) for s in self.scenes]
            r.render_batch(descs, graph=self.graph)  # warm-up (and graph capture)
            for _ in range(self.repeats):
                r.render_batch(descs, graph=self.graph)
                best = min(best, r.stats().render_ms)
        except api.AnaError as e:
            error = str(e)
        finally:
            if r is not None:
                r.close()
        row = {**dataclasses.asdict(cfg), "ms": best}
        if error:
            row["error"] = error
        self.table.append(row)
        return best

    def tune(self, start: Config = Config(), rounds=2, space=SPACE) -> Config:
        cur = start
        cur_ms = self.measure(cur)
        for _ in range(rounds):
            improved = False
            for key, values in space.items():
                for v in values:
                    if getattr(cur, key) == v:
                        continue
                    cand = dataclasses.replace(cur, **{key: v})
                    ms = self.measure(cand)
                    if ms < cur_ms * 0.98:
                        cur, cur_ms, improved = cand, ms, True
            if not improved:
                break
        self.best = cur
        self.best_ms = cur_ms
        return cur


def tune(scenes, **kw):
    t = Tuner(scenes, **kw)
    t0 = time.time()
    best = t.tune()
    return best, t.best_ms, t.table, time.time() - t0
