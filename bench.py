#!/usr/bin/env python
"""Benchmark of the B200 path-tracing hot path.

Workload (one step = one frame): the throughput scene — 4096 subdivision-3
icospheres (5,242,880 triangles) plus a ground quad, GGX standard_surface
materials, a 1024x512 importance-sampled HDR dome with a 0.5 deg sun — rendered
at 1920x1080, 64 samples per pixel, max depth 12: 132,710,400 camera paths.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Prints one JSON line. `value` is path samples/s with the scene resident in HBM
(device time from CUDA events on the library's stream, max over ranks); `e2e`
is the same metric through the C ABI with host buffers: every step uploads
the prepared scene from pinned host memory, renders and reads the film back.
`--impl reference` times the reference's own CPU PathIntegrator (compiled from
its sources into oracle/_ref) on the host cores instead.

The same line carries the metric's two other parts, measured after the timed
region: "batched" (64 Cornell variants as one graph-replayed batch render vs
one launch sequence per scene, same samples, so equal RMSE) and "adjoint"
(ana_backward vs ana_forward device time on the differentiable scene);
"other_configs" times single frames of the Cornell and hair configurations,
of a 938-sphere (about 1.2M-triangle) throughput frame and of the glass /
alpha-mask and motion-blur scenes; "scene_setup" compares the host build of
the throughput scene (ana_prepare_scene) with the device build
(ana_upload_scene_device), whose uploaded bytes must be the same.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# the headline value is the throughput scene's samples/s; the batched-vs-plain
# and adjoint/forward parts of the metric are reported under "batched" and
# "adjoint" in the same line
METRIC = "path samples/s at equal RMSE vs FP64 image, batched vs plain; adjoint/fwd time"
UNIT = "samples/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n-spheres", type=int, default=4096)
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--spp", type=int, default=64)
    ap.add_argument("--depth", type=int, default=12)
    ap.add_argument("--cpu-seconds", type=float, default=15.0,
                    help="target CPU work of the reference sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--chunk-paths", type=int, default=1 << 27,
                    help="paths in flight per wavefront chunk; the default is the autotuner's best "
                         "point for this frame (all 132,710,400 paths in one chunk, ~31 GB of queues)")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batched-vs-plain and adjoint/forward measurements")
    ap.add_argument("--traversal", type=int, default=0,
                    help="0 library default, 1 persistent warps, 2 one thread per ray")
    ap.add_argument("--scene", default="throughput", choices=["throughput", "glass", "motion", "hair"],
                    help="the frame to time (profiling of the other scenes; the bench line's workload is "
                         "the throughput scene)")
    return ap.parse_args()


def make_scene(a):
    """The timed frame: the throughput scene, or (--scene) the glass /
    alpha-mask, motion-blur or hair scene at the same film size, spp and depth."""
    from anacapa_b200 import scenes as S
    if a.scene == "glass":
        return S.glass(a.width, a.height, a.spp, a.depth)
    if a.scene == "motion":
        return S.motion(a.width, a.height, a.spp, a.depth)
    if a.scene == "hair":
        return S.hair(a.width, a.height, a.spp, a.depth)
    return S.throughput(a.width, a.height, a.spp, a.depth, n_spheres=a.n_spheres)


def workload_config(a, scene):
    if a.scene != "throughput":
        return {"workload": f"{a.scene} scene, {scene.num_triangles} triangles, {scene.num_segments} curve "
                            f"segments; {a.width}x{a.height}, {a.spp} spp, max depth {a.depth}",
                "paths_per_step": scene.num_paths, "triangles": scene.num_triangles,
                "chunk_paths": min(a.chunk_paths, scene.num_paths)}
    return {
        "workload": (f"throughput scene: {a.n_spheres} icospheres (subdiv 3) + ground, "
                     f"{scene.num_triangles} triangles, GGX standard_surface, 1024x512 HDR dome; "
                     f"{a.width}x{a.height}, {a.spp} spp, max depth {a.depth}"),
        "paths_per_step": scene.num_paths,
        "triangles": scene.num_triangles,
        "l2": "inputs larger than L2 (706 MB of scene arrays + GBs of wavefront queues vs 126 MB L2)",
        "sampler": "scrambled Halton seed 0",
        "chunk_paths": min(a.chunk_paths, scene.num_paths),
        "launch": "stage block 256, persistent traversal, BVH leaves of 4 (the reference's)",
    }


# ---------------------------------------------------------------------------
def dist_setup(a):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
        pg = dist
    return ws, rank, local, pg


def barrier(pg, local):
    import torch
    if torch.cuda.is_available():
        torch.cuda.synchronize(local)
    if pg is not None:
        pg.barrier()
    if torch.cuda.is_available():
        torch.cuda.synchronize(local)


def allreduce_max(pg, x, local):
    if pg is None:
        return x
    import torch
    dev = f"cuda:{local}" if torch.cuda.is_available() else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


class Clocks:
    """nvidia-smi samples (every 200 ms) during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.f = None

    def start(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
                for n, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(n)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def extend_traffic_per_ray():
    """DRAM bytes per closest-hit ray of the extend kernel, from the committed
    ncu summary (profiles/extend_throughput.md), or None."""
    p = os.path.join(ROOT, "profiles", "extend_throughput.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("dram_bytes_per_ray:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


# ---------------------------------------------------------------------------
def cpu_reference_sample(scene, target_s, steps=1, warmup=0):
    """Time the reference's CPU PathIntegrator (oracle/_ref, flags of record)
    through its own ThreadPool on a band of image rows at the full spp. Returns
    (samples/s per step list, description, cores)."""
    from oracle import refbind as R
    if not R.available("record"):
        R.build()
    rs = R.RefScene(scene, variant="record")
    W, H = scene.width, scene.height
    cores = os.cpu_count() or 1
    # calibrate on 2 rows in the middle of the frame
    y0 = H // 2
    _, _, secs = rs.render(rect=(0, y0, W, y0 + 2))
    per_row = max(secs / 2.0, 1e-6)
    rows = int(max(1, min(H - y0, target_s / per_row)))
    for _ in range(warmup):
        rs.render(rect=(0, y0, W, y0 + rows))
    vals = []
    for _ in range(steps):
        _, _, secs = rs.render(rect=(0, y0, W, y0 + rows))
        vals.append(W * rows * scene.spp / secs)
    desc = (f"rows {y0}..{y0 + rows - 1} of the {W}x{H} frame at {scene.spp} spp "
            f"({W * rows * scene.spp} paths), reference PathIntegrator via its ThreadPool, "
            f"64x64 tiles, non-adaptive")
    return vals, desc, cores


def run_reference(a):
    ws, rank, local, pg = dist_setup(a)
    if rank != 0:
        return 0
    from anacapa_b200 import scenes as S
    scene = make_scene(a)
    vals, desc, cores = cpu_reference_sample(scene, a.cpu_seconds, steps=a.steps, warmup=a.warmup)
    v = statistics.mean(vals)
    paths = scene.num_paths
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": paths / v * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded numpy scene generator)",
        "config": workload_config(a, scene),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": desc},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def bench_batched(local, reps=3):
    """The batched workload: 64 Cornell variants (resolutions 64^2..512^2,
    4..64 spp, depth 4..16) as one batch render replayed from a CUDA graph,
    against the same 64 frames rendered one scene per launch sequence. Both
    forms run the same per-variant estimator (same samples), so their images
    and RMSE against the FP64 oracle are identical. Device time (CUDA events)
    per form; launch configuration from the autotuner's best point (8M-path
    chunks, 256-thread stage blocks, persistent traversal, leaves of 2)."""
    from anacapa_b200 import api
    from anacapa_b200 import scenes as S
    scenes = S.batched_variants(64, seed=0)
    preps = [api.Prepared(sc, max_leaf_tris=2) for sc in scenes]
    descs = [(sc.width, sc.height, sc.spp, sc.max_depth) for sc in scenes]
    paths = sum(sc.num_paths for sc in scenes)
    r = api.Renderer(device=local, chunk_paths=8 << 20, block_size=256)
    plain = []
    for it in range(reps + 1):
        ms = 0.0
        for pr, d in zip(preps, descs):
            r.upload(pr)
            r.render(*d)
            ms += r.stats().render_ms
        if it:
            plain.append(ms)
    batch = api.Batch(preps)
    r.upload_batch(batch)
    batched = []
    for it in range(reps + 1):
        r.render_batch(descs, graph=True)
        if it:
            batched.append(r.stats().render_ms)
    r.close()
    pm, bm = statistics.median(plain), statistics.median(batched)
    return {"workload": f"64 Cornell variants, {paths:,} paths", "paths": paths,
            "plain_ms": pm, "batched_graph_ms": bm,
            "plain_samples_per_s": paths / (pm / 1e3), "batched_samples_per_s": paths / (bm / 1e3),
            "speedup": pm / bm, "equal_rmse": "identical per-variant estimator and samples"}


def bench_frame(local, scene, reps=3, chunk_paths=0):
    """Device time of one frame of `scene` (median of reps after one warm-up)."""
    from anacapa_b200 import api
    r = api.Renderer(device=local, chunk_paths=chunk_paths)
    r.upload(api.Prepared(scene))
    times = []
    for it in range(reps + 1):
        r.render_scene(scene)
        if it:
            times.append(r.stats().render_ms)
    st = r.stats()
    r.close()
    ms = statistics.median(times)
    rays = st.extend_rays + st.shadow_rays + st.mis_rays
    return {"paths": scene.num_paths, "ms": ms, "samples_per_s": scene.num_paths / (ms / 1e3),
            "rays_per_s": rays / (ms / 1e3)}


def bench_configs(local):
    """The other single-frame configurations: Cornell 256x256x16 (depth 8),
    hair 200k strands 1280x720x32 (depth 10), and the throughput frame with
    938 spheres (about 1.2M triangles, the triangle count the throughput
    configuration states; its generator gives 5.24M with 4096 spheres)."""
    from anacapa_b200 import scenes as S
    out = {}
    cornell = S.cornell(256, 256, 16, 8)
    out["cornell_256x256x16"] = {"workload": "Cornell box, 36 triangles, Lambert, area light; depth 8",
                                 **bench_frame(local, cornell)}
    hair = S.hair(1280, 720, 32, 10)
    out["hair_1280x720x32"] = {"workload": f"hair: 200,000 strands, {hair.num_segments:,} cubic segments, "
                                           "Kajiya-Kay as the reference executes it, one area light; depth 10",
                               **bench_frame(local, hair, chunk_paths=1 << 25)}
    thr = S.throughput(n_spheres=938)
    out["throughput_938_spheres"] = {"workload": f"throughput scene with 938 spheres: {thr.num_triangles:,} "
                                                 "triangles, 1920x1080x64, depth 12",
                                     **bench_frame(local, thr, chunk_paths=1 << 27)}
    glass = S.glass(1280, 720, 16, 8)
    out["glass_1280x720x16"] = {"workload": "glass: smooth and rough dielectric spheres and panes, "
                                            "alpha-masked cards, directional + area light; depth 8",
                                **bench_frame(local, glass, chunk_paths=1 << 25)}
    mo = S.motion(1280, 720, 16, 6)
    out["motion_1280x720x16"] = {"workload": "motion blur: object-space meshes with 2-3 motion keys, "
                                             "shutter [0, 1]; depth 6",
                                 **bench_frame(local, mo, chunk_paths=1 << 25)}
    return out


def bench_aov_film_io(r, scene, start):
    """One frame of the timed workload with the denoising AOVs (device time
    against the frame without them), then Film::writeEXR (beauty + albedo +
    normals, ZIP) and Film::writePNG of it through the C ABI (wall time,
    device-to-host read included)."""
    W, H = scene.width, scene.height
    r.render(W, H, scene.spp, scene.max_depth, sample_start=start, clear=True)
    plain = r.stats().render_ms
    r.render(W, H, scene.spp, scene.max_depth, sample_start=start, clear=True, aovs=True)
    with_aov = r.stats().render_ms
    with tempfile.TemporaryDirectory() as d:
        t0 = time.perf_counter()
        r.write_exr(os.path.join(d, "f.exr"), W, H, aovs=True)
        t1 = time.perf_counter()
        r.write_png(os.path.join(d, "f.png"), W, H)
        t2 = time.perf_counter()
        exr_mb = os.path.getsize(os.path.join(d, "f.exr")) / 1e6
    return {"frame_ms": plain, "frame_with_aovs_ms": with_aov, "aov_overhead": with_aov / plain - 1.0,
            "write_exr_s": t1 - t0, "exr_mb": exr_mb, "write_png_s": t2 - t1}


def bench_scene_setup(local, scene, prep_s):
    """Host build (ana_prepare_scene, timed by the caller) against the device
    build (ana_upload_scene_device: triangle setup, SAH build and collapse on
    the GPU, the rest of the scene prepared on the host), second of two calls."""
    from anacapa_b200 import api
    r = api.Renderer(device=local)
    try:
        r.upload(scene, device_build=True)
        t0 = time.perf_counter()
        r.upload(scene, device_build=True)
        dev_s = time.perf_counter() - t0
        st = r.stats()
        digest = r.scene_digest()
    finally:
        r.close()
    return {"workload": f"throughput scene, {scene.num_triangles:,} triangles",
            "host_prepare_s": prep_s, "device_upload_s": dev_s,
            "device_build_ms": {"setup": st.build_ms[0], "sah_levels": st.build_ms[1],
                                "small_subtrees": st.build_ms[2], "collapse": st.build_ms[3]},
            "sah_levels": int(st.build_levels), "speedup": prep_s / dev_s, "digest": digest}


def bench_adjoint(local, reps=3):
    """Path-replay adjoint on the differentiable scene (Cornell + 20,480-
    triangle icosphere, 512x512, 16 spp, depth 8): device time of ana_forward
    and of ana_backward (primal + adjoint replay) for an L2 loss against a
    target rendered from perturbed parameters."""
    from anacapa_b200 import api
    from anacapa_b200 import scenes as S
    W = H = 512
    spp, depth = 16, 8
    r = api.Renderer(device=local)
    r.upload(S.differentiable(W, H, spp, depth, params=S.perturbed_diff_params(1)))
    target = r.forward(W, H, spp, depth)
    r.upload(S.differentiable(W, H, spp, depth))
    fwd, bwd = [], []
    for it in range(reps + 1):
        img = r.forward(W, H, spp, depth)
        f = r.stats().render_ms
        r.backward(2.0 * (img - target) / img.size)
        b = r.stats().render_ms
        if it:
            fwd.append(f)
            bwd.append(b)
    r.close()
    fm, bm = statistics.median(fwd), statistics.median(bwd)
    return {"workload": "differentiable Cornell + icosphere 512x512x16, depth 8, L2 loss",
            "forward_ms": fm, "backward_ms": bm, "adjoint_over_forward": bm / fm,
            "forward_samples_per_s": W * H * spp / (fm / 1e3)}


def run_ours(a):
    ws, rank, local, pg = dist_setup(a)
    import torch
    from anacapa_b200 import api
    from anacapa_b200 import scenes as S
    if torch.cuda.is_available():
        torch.cuda.set_device(local)
    scene = make_scene(a)
    t_prep = time.perf_counter()
    prep = api.Prepared(scene)
    t_prep = time.perf_counter() - t_prep
    r = api.Renderer(device=local, timing=True, traversal=a.traversal, chunk_paths=a.chunk_paths)
    r.upload(prep)
    W, H, spp = scene.width, scene.height, scene.spp
    start = rank * spp  # each rank renders its own disjoint sample range of the frame

    def step():
        r.render(W, H, spp, scene.max_depth, sample_start=start, clear=True)
        return r.stats()

    for _ in range(a.warmup):
        step()
    # instrumented pass (untimed): algorithmic work of the closest-hit stage
    r.render(W, H, spp, scene.max_depth, sample_start=start, clear=True, count_work=True)
    work = r.stats()
    # timed region
    clocks = Clocks(local)
    barrier(pg, local)
    clocks.start()
    stats = [step() for _ in range(a.steps)]
    barrier(pg, local)
    ck = clocks.stop()
    dev_ms = sum(s.render_ms for s in stats)
    dev_ms = allreduce_max(pg, dev_ms, local)
    ms_step = dev_ms / a.steps
    paths_step = scene.num_paths
    value = ws * paths_step / (ms_step / 1e3)
    rays = sum(s.extend_rays + s.shadow_rays + s.mis_rays for s in stats) / a.steps
    ext_ms = sum(s.extend_ms for s in stats) / a.steps
    shade_ms = sum(s.shade_ms for s in stats) / a.steps
    shadow_ms = sum(s.shadow_ms for s in stats) / a.steps
    mis_ms = sum(s.mis_ms for s in stats) / a.steps
    launches = int(sum(s.kernel_launches for s in stats))
    # roofline of the dominant kernel (closest-hit traversal)
    ext_launches = stats[0].extend_launches
    alg_bytes = (128 * work.node_fetches + 64 * work.curve_node_fetches + 48 * work.tri_tests + 80 * work.seg_tests
                 + (32 + 16) * work.extend_rays)
    peak, peak_kind = measured_peaks()
    achieved = (alg_bytes / ext_launches) / ((ext_ms / ext_launches) / 1e3) / 1e9 if ext_ms > 0 else None
    tpr = extend_traffic_per_ray() if a.scene == "throughput" else None  # measured on that scene
    traffic = (tpr * work.extend_rays / ext_launches) if tpr else None
    # end to end through the C ABI with host buffers
    e2e = None
    if not a.no_e2e:
        film = np.zeros((H, W, 5), np.float32)
        barrier(pg, local)
        t0 = time.perf_counter()
        for _ in range(a.steps):
            r.upload(prep)
            r.render(W, H, spp, scene.max_depth, sample_start=start, clear=True)
            api.check(api.lib().ana_film_read(r.h, film.ctypes.data, W * H), r.h)
        t1 = time.perf_counter()
        e2e_s = allreduce_max(pg, (t1 - t0) / a.steps, local)
        e2e = {"value": ws * paths_step / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": int(prep.nbytes), "d2h_bytes_per_step": int(W * H * 20)}
    extra = {}
    if not a.no_extras:  # the metric's other two parts, outside the timed region
        extra["batched"] = bench_batched(local)
        extra["adjoint"] = bench_adjoint(local)
        extra["other_configs"] = bench_configs(local)
        setup = bench_scene_setup(local, scene, t_prep)
        setup["same_bytes"] = setup.pop("digest") == prep.digest
        extra["scene_setup"] = setup
        extra["aov_film_io"] = bench_aov_film_io(r, scene, start)
    cpu = None
    if rank == 0 and ws == 1 and not a.no_cpu_baseline:
        try:
            vals, desc, cores = cpu_reference_sample(scene, a.cpu_seconds)
            cpu = {"value": vals[0], "unit": UNIT, "cores": cores, "kind": "reference", "sample": desc}
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"failed: {e}"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded numpy scene generator)",
            "config": workload_config(a, scene),
            "rays_per_s": ws * rays / (ms_step / 1e3),
            "extend_rays_per_step": int(stats[0].extend_rays),
            "stage_ms": {"extend": ext_ms, "shade": shade_ms, "shadow": shadow_ms, "mis": mis_ms},
            "roofline": {"bound": "hbm", "kernel": "k_extend (closest-hit BVH traversal)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None,
                         "peak_kind": peak_kind, "traffic": traffic,
                         "alg_bytes_per_launch": alg_bytes / ext_launches,
                         "launches_per_step": ext_launches},
            "gpu_launches": launches,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "clocks": ck,
            **extra,
        }
        print(json.dumps(line), flush=True)
    r.close()
    if pg is not None:
        pg.destroy_process_group()
    return 0


def main():
    a = parse()
    if a.impl == "reference":
        return run_reference(a)
    return run_ours(a)


if __name__ == "__main__":
    sys.exit(main())
