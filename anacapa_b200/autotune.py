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

import argparse
import dataclasses
import json
import os
import sys
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
    "chunk_paths": [1 << k for k in range(20, 28)],  # 1M .. 128M paths in flight
    "block_size": [128, 256],  # the shading kernel's blocks (at most 256 threads)
    "traversal": [api.ANA_TRAVERSAL_PERSISTENT, api.ANA_TRAVERSAL_PER_RAY],
    "max_leaf_tris": [2, 4, 8],
}

HERE = os.path.dirname(os.path.abspath(__file__))
TABLES = os.path.join(os.path.dirname(HERE), "profiles")
# the point used when no tuning table has been recorded for a workload
DEFAULT_POINT = {"chunk": 8 << 20, "block": 256, "traversal": api.ANA_TRAVERSAL_PERSISTENT, "leaf": 2}


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


def table_path(workload):
    return os.path.join(TABLES, f"autotune_{workload}.json")


def tuned_point(workload):
    """The best point of the recorded tuning table of a workload
    (profiles/autotune_<workload>.json, written by this module's command
    line), else DEFAULT_POINT."""
    p = table_path(workload)
    if os.path.exists(p):
        with open(p) as f:
            b = json.load(f)["best"]
        return {"chunk": int(b["chunk_paths"]), "block": int(b["block_size"]), "traversal": int(b["traversal"]),
                "leaf": int(b["max_leaf_tris"]), "source": os.path.relpath(p, os.path.dirname(TABLES))}
    return dict(DEFAULT_POINT, source="default")


WORKLOADS = {"batched": lambda: S.batched_variants(64, seed=0)}


def main(argv=None):
    ap = argparse.ArgumentParser(description="Tune the launch configuration of a workload and record the table.")
    ap.add_argument("--workload", default="batched", choices=sorted(WORKLOADS))
    ap.add_argument("--out", default=None, help="table file (default profiles/autotune_<workload>.json)")
    ap.add_argument("--repeats", type=int, default=2)
    a = ap.parse_args(argv)
    scenes = WORKLOADS[a.workload]()
    best, ms, table, secs = tune(scenes, repeats=a.repeats)
    rec = {"workload": a.workload, "paths": sum(sc.num_paths for sc in scenes), "space": SPACE,
           "start": dataclasses.asdict(Config()), "best": dataclasses.asdict(best), "best_ms": ms,
           "tuning_seconds": secs, "table": table,
           "command": f"python -m anacapa_b200.autotune --workload {a.workload} --repeats {a.repeats}"}
    out = a.out or table_path(a.workload)
    with open(out, "w") as f:
        json.dump(rec, f, indent=1)
    print(json.dumps({"best": rec["best"], "best_ms": ms, "measurements": len(table), "seconds": secs}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
