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
    ap.add_argument("--config-cpu-seconds", type=float, default=5.0,
                    help="target CPU work of each other configuration's reference sample")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--chunk-paths", type=int, default=1 << 27,
                    help="paths in flight per wavefront chunk; the default is the autotuner's best "
                         "point for this frame (all 132,710,400 paths in one chunk, ~31 GB of queues)")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batched-vs-plain and adjoint/forward measurements")
    ap.add_argument("--leaf-tris", type=int, default=0,
                    help="maximum triangles per BVH leaf (0: the reference's 4)")
    ap.add_argument("--leaf-segments", type=int, default=0,
                    help="maximum curve segments per BVH leaf (0: the reference's 4)")
    ap.add_argument("--traversal", type=int, default=0,
                    help="0 library default, 1 persistent warps, 2 one thread per ray")
    ap.add_argument("--hair-mode", type=int, default=0, choices=[0, 1],
                    help="hair scene: 0 Kajiya-Kay (as the reference executes it), 1 Marschner lobes")
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
        return S.hair(a.width, a.height, a.spp, a.depth, hair_mode=a.hair_mode)
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


def extend_profile_field(name):
    """A figure of the committed ncu summary of the extend kernel
    (profiles/extend_throughput.md, lines `name: value`), or None:
    dram_bytes_per_ray, lanes_active_per_instruction, l2_throughput_pct."""
    p = os.path.join(ROOT, "profiles", "extend_throughput.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith(name + ":"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


FP64_WINDOWS = os.path.join(ROOT, "tests", "golden", "config_windows_fp64.npz")
_fp64 = None


def rmse_vs_fp64(name, img):
    """RMSE of a rendered image (H, W, 3) against the FP64 converged windows
    of its frame (tests/golden/config_windows_fp64.npz, made by the CPU
    restatement in double precision at 4096 spp), window by window, beside the
    reference CPU integrator's RMSE at the same spp on the same window."""
    global _fp64
    if _fp64 is None:
        _fp64 = dict(np.load(FP64_WINDOWS)) if os.path.exists(FP64_WINDOWS) else {}
    out = {"windows": [], "rmse": [], "reference_cpu_rmse": [], "fp64_spp": int(_fp64.get("conv_spp", 0))}
    k = 0
    while f"{name}_{k}_image" in _fp64:
        x0, y0, x1, y1 = (int(v) for v in _fp64[f"{name}_{k}_rect"])
        conv = _fp64[f"{name}_{k}_image"].astype(np.float64)
        err = float(np.sqrt(np.mean((img[y0:y1, x0:x1].astype(np.float64) - conv) ** 2)))
        out["windows"].append([x0, y0, x1, y1])
        out["rmse"].append(err)
        out["reference_cpu_rmse"].append(float(_fp64[f"{name}_{k}_ref_rmse"]))
        k += 1
    return out if k else None


# ---------------------------------------------------------------------------
def row_bands(H, n_bands, rows):
    """n_bands bands of `rows` rows whose centres are spread evenly over the
    frame's height (band b centred on row (b + 1/2) H / n_bands)."""
    out = []
    for b in range(n_bands):
        c = int((b + 0.5) * H / n_bands)
        y0 = min(max(0, c - rows // 2), H - rows)
        out.append((y0, y0 + rows))
    return out


def cpu_reference_sample(scene, target_s, steps=1, warmup=0, n_bands=16):
    """Time the reference's CPU PathIntegrator (oracle/_ref, flags of record)
    through its own ThreadPool on a stratified sample of the frame: n_bands
    full-width bands of rows spread evenly over its height, all their 64x64
    tiles in one pool dispatch, at the frame's spp and depth. The band height
    is sized from a calibration pass (one row per band) so that one step takes
    about target_s. Returns (samples/s per step, seconds per step, paths per
    step, description, cores); frames small enough for target_s run whole."""
    from oracle import refbind as R
    if not R.available("record"):
        R.build()
    rs = R.RefScene(scene, variant="record")
    W, H = scene.width, scene.height
    cores = os.cpu_count() or 1
    n_bands = min(n_bands, H)
    _, _, secs = rs.render_rows(row_bands(H, n_bands, 1))
    per_row = max(secs / n_bands, 1e-6)
    rows = int(max(1, min(H // n_bands, round(target_s / (per_row * n_bands)))))
    bands = [(0, H)] if rows * n_bands >= H else row_bands(H, n_bands, rows)
    nrows = sum(b - a for a, b in bands)
    for _ in range(warmup):
        rs.render_rows(bands)
    vals, times = [], []
    for _ in range(steps):
        _, _, secs = rs.render_rows(bands)
        vals.append(W * nrows * scene.spp / secs)
        times.append(secs)
    paths = W * nrows * scene.spp
    if bands == [(0, H)]:
        what = f"the whole {W}x{H} frame"
    else:
        what = (f"{len(bands)} bands of {rows} rows spread evenly over the {W}x{H} frame "
                f"(rows {bands[0][0]}..{bands[0][1] - 1}, ..., {bands[-1][0]}..{bands[-1][1] - 1}; "
                f"{nrows / H:.1%} of its pixels)")
    desc = (f"{what} at {scene.spp} spp, depth {scene.max_depth} ({paths} paths per step), reference "
            f"PathIntegrator via its ThreadPool, 64x64 tiles in one dispatch, non-adaptive")
    return vals, times, paths, desc, cores


def run_reference(a):
    ws, rank, local, pg = dist_setup(a)
    if rank != 0:
        return 0
    scene = make_scene(a)
    # each step a bounded sample, so warm-up and timed steps end within a few minutes
    per_step = min(a.cpu_seconds, max(2.0, 150.0 / max(1, a.steps + a.warmup)))
    vals, times, paths, desc, cores = cpu_reference_sample(scene, per_step, steps=a.steps, warmup=a.warmup)
    v = statistics.mean(vals)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": statistics.mean(times) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded numpy scene generator)",
        "config": workload_config(a, scene),
        "sample_paths_per_step": paths,
        "frame_ms_at_this_rate": scene.num_paths / v * 1e3,
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": desc},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def batched_rmse(images):
    """Per-variant RMSE of the 64 batched frames against their FP64 centre
    windows (tests/golden/config_windows_fp64.npz, key `batched_*`)."""
    global _fp64
    if _fp64 is None:
        rmse_vs_fp64("none", None)
    if "batched_image" not in _fp64:
        return None
    out = []
    for k, img in enumerate(images):
        x0, y0, x1, y1 = (int(v) for v in _fp64["batched_rect"][k])
        conv = _fp64["batched_image"][k].astype(np.float64)
        out.append(float(np.sqrt(np.mean((img[y0:y1, x0:x1].astype(np.float64) - conv) ** 2))))
    return out


def bench_batched(local, reps=3):
    """The batched workload: 64 Cornell variants (resolutions 64^2..512^2,
    4..64 spp, depth 4..16) as one batch render replayed from a CUDA graph,
    against the same 64 frames rendered one scene per launch sequence. Device
    time (CUDA events) per form; launch configuration from the committed
    autotuner table (profiles/autotune_batched.json) when present. Each
    form's per-variant RMSE against the variant's FP64 centre window is
    measured on its own images."""
    from anacapa_b200 import api
    from anacapa_b200 import autotune
    from anacapa_b200 import scenes as S
    tuned = autotune.tuned_point("batched")
    scenes = S.batched_variants(64, seed=0)
    preps = [api.Prepared(sc, max_leaf_tris=tuned["leaf"]) for sc in scenes]
    descs = [(sc.width, sc.height, sc.spp, sc.max_depth) for sc in scenes]
    paths = sum(sc.num_paths for sc in scenes)
    r = api.Renderer(device=local, chunk_paths=tuned["chunk"], block_size=tuned["block"],
                     traversal=tuned["traversal"])
    plain, plain_img = [], []
    for it in range(reps + 1):
        ms = 0.0
        for pr, d in zip(preps, descs):
            r.upload(pr)
            r.render(*d)
            ms += r.stats().render_ms
            if it == reps:
                plain_img.append(r.image(d[0], d[1]))
        if it:
            plain.append(ms)
    batch = api.Batch(preps)
    r.upload_batch(batch)
    batched = []
    for it in range(reps + 1):
        r.render_batch(descs, graph=True)
        if it:
            batched.append(r.stats().render_ms)
    batch_img = []
    for k, d in enumerate(descs):
        f = r.batch_film(k, d[0], d[1])
        batch_img.append(f[..., :3] / np.maximum(f[..., 3:4], 1e-30))
    r.close()
    pm, bm = statistics.median(plain), statistics.median(batched)
    rp, rb = batched_rmse(plain_img), batched_rmse(batch_img)
    rmse = None
    if rp is not None:
        rmse = {"fp64_windows": "32x32 centre window per variant, FP64 restatement at 4096 spp",
                "plain_mean": statistics.mean(rp), "batched_mean": statistics.mean(rb),
                "plain_max": max(rp), "batched_max": max(rb),
                "max_abs_difference": max(abs(a - b) for a, b in zip(rp, rb)),
                "reference_cpu_mean": float(np.mean(_fp64["batched_ref_rmse"]))}
    return {"workload": f"64 Cornell variants, {paths:,} paths", "paths": paths,
            "plain_ms": pm, "batched_graph_ms": bm,
            "plain_samples_per_s": paths / (pm / 1e3), "batched_samples_per_s": paths / (bm / 1e3),
            "speedup": pm / bm, "target_speedup": 20.0, "tuned_point": tuned, "rmse_vs_fp64": rmse}


def bench_frame(local, scene, reps=3, chunk_paths=0, fp64_name=None):
    """Device time of one frame of `scene` (median of reps after one warm-up),
    and its RMSE against the FP64 windows of `fp64_name`."""
    from anacapa_b200 import api
    r = api.Renderer(device=local, chunk_paths=chunk_paths)
    r.upload(api.Prepared(scene))
    times = []
    for it in range(reps + 1):
        r.render_scene(scene)
        if it:
            times.append(r.stats().render_ms)
    st = r.stats()
    img = r.image(scene.width, scene.height) if fp64_name else None
    r.close()
    ms = statistics.median(times)
    rays = st.extend_rays + st.shadow_rays + st.mis_rays
    out = {"paths": scene.num_paths, "ms": ms, "samples_per_s": scene.num_paths / (ms / 1e3),
           "rays_per_s": rays / (ms / 1e3)}
    if fp64_name:
        out["rmse_vs_fp64"] = rmse_vs_fp64(fp64_name, img)
    return out


def config_cpu(scene, seconds, port=False):
    """CPU baseline beside a configuration: the reference PathIntegrator on a
    stratified row sample (cpu_reference_sample), or for a mode the reference
    does not execute (port=True: Marschner hair) this repository's CPU
    restatement in float on a centre band of rows, one thread per core."""
    try:
        if not port:
            vals, _, _, desc, cores = cpu_reference_sample(scene, seconds)
            return {"value": vals[0], "unit": UNIT, "cores": cores, "kind": "reference", "sample": desc}
        from oracle import restatebind as P
        W, H = scene.width, scene.height
        po = P.PoScene(scene, 32)
        t0 = time.perf_counter()
        po.render(rect=(0, H // 2, W, H // 2 + 1))
        per_row = max(time.perf_counter() - t0, 1e-6)
        rows = int(max(1, min(H, seconds / per_row)))
        y0 = max(0, H // 2 - rows // 2)
        t0 = time.perf_counter()
        po.render(rect=(0, y0, W, y0 + rows))
        secs = time.perf_counter() - t0
        return {"value": W * rows * scene.spp / secs, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                "sample": f"rows {y0}..{y0 + rows - 1} of the {W}x{H} frame at {scene.spp} spp: the CPU "
                          "restatement (float) in Marschner mode, which the reference does not execute"}
    except Exception as e:  # a reported baseline, never required
        return {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port" if port else "reference",
                "sample": f"failed: {e}"}


def bench_configs(local, cpu_s=0.0):
    """The other single-frame configurations: Cornell 256x256x16 (depth 8),
    hair 200k strands 1280x720x32 (depth 10) in Kajiya-Kay mode (what the
    reference executes) and in Marschner mode, the throughput frame with 938
    spheres (about 1.2M triangles, the triangle count the throughput
    configuration states; its generator gives 5.24M with 4096 spheres), and
    the glass / alpha-mask and motion-blur scenes. With cpu_s > 0 each carries
    a CPU baseline of about cpu_s seconds."""
    from anacapa_b200 import scenes as S
    out = {}
    cases = [
        ("cornell_256x256x16", "Cornell box, 36 triangles, Lambert, area light; depth 8",
         S.cornell(256, 256, 16, 8), 0, "cornell", False),
        ("hair_1280x720x32", None, S.hair(1280, 720, 32, 10), 1 << 25, "hair", False),
        ("hair_marschner_1280x720x32", None, S.hair(1280, 720, 32, 10, hair_mode=1), 1 << 25, None, True),
        ("throughput_938_spheres", None, S.throughput(n_spheres=938), 1 << 27, None, False),
        ("glass_1280x720x16", "glass: smooth and rough dielectric spheres and panes, alpha-masked cards, "
         "directional + area light; depth 8", S.glass(1280, 720, 16, 8), 1 << 25, "glass", False),
        ("motion_1280x720x16", "motion blur: object-space meshes with 2-3 motion keys, shutter [0, 1]; depth 6",
         S.motion(1280, 720, 16, 6), 1 << 25, "motion", False),
    ]
    for key, what, sc, chunk, fp64, port in cases:
        if key.startswith("hair"):
            mode = "Marschner R/TT/TRT lobes" if port else "Kajiya-Kay as the reference executes it"
            what = f"hair: 200,000 strands, {sc.num_segments:,} cubic segments, {mode}, one area light; depth 10"
        elif key.startswith("throughput"):
            what = f"throughput scene with 938 spheres: {sc.num_triangles:,} triangles, 1920x1080x64, depth 12"
        out[key] = {"workload": what, **bench_frame(local, sc, chunk_paths=chunk, fp64_name=fp64)}
        if cpu_s > 0:
            out[key]["cpu_baseline"] = config_cpu(sc, cpu_s, port=port)
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
        grad = r.backward(2.0 * (img - target) / img.size)
        b = r.stats().render_ms
        if it:
            fwd.append(f)
            bwd.append(b)
    nm, nl = r.diff_counts()
    r.close()
    fm, bm = statistics.median(fwd), statistics.median(bwd)
    out = {"workload": "differentiable Cornell + icosphere 512x512x16, depth 8, L2 loss",
           "forward_ms": fm, "backward_ms": bm, "adjoint_over_forward": bm / fm, "target_ratio": 3.0,
           "forward_samples_per_s": W * H * spp / (fm / 1e3),
           "rmse_vs_fp64": rmse_vs_fp64("differentiable", img)}
    # the gradient against the FP64 adjoint of the same frame and loss
    # (tests/golden/adjoint_fp64_512.npz, made by tests/golden/make_adjoint_fp64.py)
    gp = os.path.join(ROOT, "tests", "golden", "adjoint_fp64_512.npz")
    if os.path.exists(gp):
        ref = np.load(gp)["grad"]
        g = np.zeros(8 * nm + 4 * nl)
        for i in range(nm):
            g[8 * i:8 * i + 3] = grad["albedo"][i]
            g[8 * i + 3] = grad["roughness"][i]
            g[8 * i + 4:8 * i + 7] = grad["emission"][i]
        for j in range(nl):
            g[8 * nm + 4 * j:8 * nm + 4 * j + 3] = grad["light_le"][j]
        big = np.abs(ref) > 1e-2 * np.abs(ref).max()
        out["grad_vs_fp64"] = {"rel_err_norm": float(np.linalg.norm(g - ref) / np.linalg.norm(ref)),
                               "max_rel_err_large_entries": float((np.abs(g - ref)[big] / np.abs(ref)[big]).max()),
                               "large_entries": int(big.sum()), "target": 1e-3}
    return out


def run_ours(a):
    ws, rank, local, pg = dist_setup(a)
    import torch
    from anacapa_b200 import api
    from anacapa_b200 import scenes as S
    if torch.cuda.is_available():
        torch.cuda.set_device(local)
    scene = make_scene(a)
    t_prep = time.perf_counter()
    prep = api.Prepared(scene, max_leaf_tris=a.leaf_tris, max_leaf_segments=a.leaf_segments)
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
    alg_bytes = (128 * work.node_fetches + 128 * work.curve_node_fetches + 48 * work.tri_tests + 80 * work.seg_tests
                 + (32 + 16) * work.extend_rays)
    peak, peak_kind = measured_peaks()
    achieved = (alg_bytes / ext_launches) / ((ext_ms / ext_launches) / 1e3) / 1e9 if ext_ms > 0 else None
    tpr = extend_profile_field("dram_bytes_per_ray") if a.scene == "throughput" else None  # measured on that scene
    traffic = (tpr * work.extend_rays / ext_launches) if tpr else None
    # the last timed frame against the FP64 windows of the configuration frame
    rmse = None
    if rank == 0 and a.scene == "throughput" and (W, H, spp, a.n_spheres) == (1920, 1080, 64, 4096):
        rmse = rmse_vs_fp64("throughput", r.image(W, H))
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
        extra["other_configs"] = bench_configs(local, cpu_s=0.0 if (a.no_cpu_baseline or ws > 1 or rank)
                                                else a.config_cpu_seconds)
        setup = bench_scene_setup(local, scene, t_prep)
        setup["same_bytes"] = setup.pop("digest") == prep.digest
        extra["scene_setup"] = setup
        extra["aov_film_io"] = bench_aov_film_io(r, scene, start)
    cpu = None
    if rank == 0 and ws == 1 and not a.no_cpu_baseline:
        try:
            vals, _, _, desc, cores = cpu_reference_sample(scene, a.cpu_seconds)
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
                         "launches_per_step": ext_launches,
                         # the roof that binds (ncu, profiles/extend_throughput.md): issue and
                         # the L1 data path, not HBM or L2
                         "binding": {"limiter": "instruction issue / L1 (node and triangle gathers)",
                                     "lanes_active_per_instruction_of_32":
                                         extend_profile_field("lanes_active_per_instruction"),
                                     "l2_throughput_pct_of_peak": extend_profile_field("l2_throughput_pct")}
                         if a.scene == "throughput" else None},
            "gpu_launches": launches,
            "rmse_vs_fp64": rmse,
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
