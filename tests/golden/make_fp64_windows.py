"""Generates the FP64 converged windows of the benchmark frames.

    python tests/golden/make_fp64_windows.py [name ...]

A full FP64 frame at 4096 samples per pixel is out of reach on a CPU for the
1920x1080 and 1280x720 frames, so each frame is pinned by named windows: the
same scene, camera and film size as the benchmark frame, rendered by the CPU
restatement in double precision (oracle/restate, precision 64) over the
window's pixels only, at 4096 samples per pixel with sampler seed 12345 (a
sample stream independent of the seed-0 streams the tests and the benchmark
render). For each window the file also records the RMSE, against the FP64
window, of the reference CPU integrator's own image (flags of record) at the
frame's samples per pixel, which the GPU image's RMSE is compared with.

Output: config_windows_fp64.npz, keys `<frame>_<k>_image` (h, w, 3),
`<frame>_<k>_rect` (x0, y0, x1, y1), `<frame>_<k>_ref_rmse`; the batched
frame stores one 32x32 centre window per variant (`batched_image` (64, 32,
32, 3), `batched_rect`, `batched_ref_rmse`).
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from anacapa_b200 import scenes as S  # noqa: E402
from oracle import refbind as R  # noqa: E402
from oracle import restatebind as P  # noqa: E402

CONV_SPP = 4096
SEED = 12345
OUT = os.path.join(HERE, "config_windows_fp64.npz")


def frames():
    """The benchmark frames (scene factories) and their windows."""
    return {
        "cornell": (lambda: S.cornell(256, 256, 16, 8), [(0, 0, 256, 256)]),
        "throughput": (lambda: S.throughput(1920, 1080, 64, 12),
                       [(936, 516, 984, 564), (1500, 750, 1548, 798)]),
        "hair": (lambda: S.hair(1280, 720, 32, 10), [(500, 350, 548, 398)]),
        "differentiable": (lambda: S.differentiable(512, 512, 16, 8), [(248, 184, 376, 312)]),
        "glass": (lambda: S.glass(1280, 720, 16, 8), [(540, 280, 588, 328)]),
        "motion": (lambda: S.motion(1280, 720, 16, 6), [(520, 250, 568, 298)]),
    }


def centre_window(sc, size=32):
    x0, y0 = sc.width // 2 - size // 2, sc.height // 2 - size // 2
    return (x0, y0, x0 + size, y0 + size)


def resolve(rgbw, rect):
    x0, y0, x1, y1 = rect
    w = rgbw[y0:y1, x0:x1]
    return (w[..., :3] / w[..., 3:4]).astype(np.float64)


def window(sc, rect):
    """FP64 converged window and the reference's RMSE at the frame's spp."""
    conv, _ = P.PoScene(sc, 64).render(spp=CONV_SPP, rect=rect, seed=SEED)
    conv = resolve(conv, rect)
    rgbw, _, _ = R.RefScene(sc, variant="record").render(rect=rect)
    ref = resolve(rgbw.astype(np.float64), rect)
    return conv.astype(np.float32), float(np.sqrt(np.mean((ref - conv) ** 2)))


def main(names):
    R.build()
    out = dict(np.load(OUT)) if os.path.exists(OUT) else {}
    for name, (make, rects) in frames().items():
        if names and name not in names:
            continue
        sc = make()
        for k, rect in enumerate(rects):
            t = time.time()
            img, rmse = window(sc, rect)
            out[f"{name}_{k}_image"] = img
            out[f"{name}_{k}_rect"] = np.array(rect, np.int32)
            out[f"{name}_{k}_ref_rmse"] = np.float64(rmse)
            print(f"{name} window {k} {rect}: {time.time() - t:.0f} s, reference RMSE {rmse:.5f}", flush=True)
    if not names or "batched" in names:
        t = time.time()
        imgs, rects, rmses = [], [], []
        for sc in S.batched_variants(64, seed=0):
            rect = centre_window(sc)
            img, rmse = window(sc, rect)
            imgs.append(img)
            rects.append(rect)
            rmses.append(rmse)
        out["batched_image"] = np.stack(imgs)
        out["batched_rect"] = np.array(rects, np.int32)
        out["batched_ref_rmse"] = np.array(rmses, np.float64)
        print(f"batched: {time.time() - t:.0f} s, reference RMSE mean {np.mean(rmses):.5f}", flush=True)
    out["conv_spp"] = np.int32(CONV_SPP)
    out["conv_seed"] = np.int32(SEED)
    np.savez_compressed(OUT, **out)
    print("wrote", OUT)


if __name__ == "__main__":
    main(sys.argv[1:])
