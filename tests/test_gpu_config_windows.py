"""The benchmark frames at their configuration sizes (full film, full spp,
the library's default chunking) against the FP64 converged windows
(tests/golden/config_windows_fp64.npz, made by
tests/golden/make_fp64_windows.py) and against the reference CPU integrator
on the same windows.

Per window:
  - RMSE of the GPU image against the FP64 window equals the reference CPU's
    RMSE at the same spp within 5 % (the same estimator and the same samples;
    both are stated per window);
  - a per-pixel 3-sigma z-test of the GPU window against the reference
    CPU's render of that window (live, oracle/_ref) passes for >= 99.5 % of
    pixels, and the window means agree within 1e-3.
The batched frame is checked per variant in both forms (one scene per launch
sequence, and the whole batch replayed from a CUDA graph)."""
import os

import numpy as np
import pytest

from anacapa_b200 import api
from anacapa_b200 import scenes as S

from test_gpu_render import z_test

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = dict(np.load(os.path.join(HERE, "golden", "config_windows_fp64.npz")))

FRAMES = {
    "cornell": lambda: S.cornell(256, 256, 16, 8),
    "throughput": lambda: S.throughput(1920, 1080, 64, 12),
    "hair": lambda: S.hair(1280, 720, 32, 10),
    "differentiable": lambda: S.differentiable(512, 512, 16, 8),
    "glass": lambda: S.glass(1280, 720, 16, 8),
    "motion": lambda: S.motion(1280, 720, 16, 6),
}


def windows(name):
    k = 0
    while f"{name}_{k}_image" in GOLD:
        yield k, tuple(int(v) for v in GOLD[f"{name}_{k}_rect"])
        k += 1


def rmse(a, b):
    return float(np.sqrt(np.mean((np.asarray(a, np.float64) - np.asarray(b, np.float64)) ** 2)))


def resolve(f):
    return f[..., :3] / np.maximum(f[..., 3:4], 1e-30)


def check_window(film, sc, rect, conv, ref_rmse, ref_built):
    x0, y0, x1, y1 = rect
    win = film[y0:y1, x0:x1]
    e = rmse(resolve(win), conv)
    assert abs(e - ref_rmse) <= 0.05 * ref_rmse + 1e-7, (e, ref_rmse)
    rgbw, lsq, _ = ref_built.RefScene(sc, variant="record").render(rect=rect)
    rgbw, lsq = rgbw[y0:y1, x0:x1], lsq[y0:y1, x0:x1]
    assert np.array_equal(win[..., 3], rgbw[..., 3])
    rate = z_test(win, rgbw, lsq)
    assert rate >= 0.995, rate
    a = win[..., :3].sum((0, 1)) / win[..., 3].sum()
    b = rgbw[..., :3].sum((0, 1)) / rgbw[..., 3].sum()
    assert np.all(np.abs(a - b) <= 1e-3 * np.maximum(b, 1e-3)), (a, b)
    return e


@pytest.mark.parametrize("name", list(FRAMES))
def test_config_frame_windows(gpu, ref_built, name):
    sc = FRAMES[name]()
    r = api.Renderer()
    try:
        r.upload(sc)
        r.render_scene(sc)
        film = r.film(sc.width, sc.height)
    finally:
        r.close()
    assert np.all(np.isfinite(film))
    for k, rect in windows(name):
        check_window(film, sc, rect, GOLD[f"{name}_{k}_image"], float(GOLD[f"{name}_{k}_ref_rmse"]), ref_built)


def test_batched_variants_both_forms(gpu, ref_built):
    scenes = S.batched_variants(64, seed=0)
    preps = [api.Prepared(sc, max_leaf_tris=2) for sc in scenes]
    descs = [(sc.width, sc.height, sc.spp, sc.max_depth) for sc in scenes]
    r = api.Renderer(chunk_paths=8 << 20)
    try:
        plain = []
        for pr, d in zip(preps, descs):
            r.upload(pr)
            r.render(*d)
            plain.append(r.film(d[0], d[1]))
        r.upload_batch(api.Batch(preps))
        r.render_batch(descs, graph=True)
        r.render_batch(descs, graph=True)  # replayed
        batched = [r.batch_film(k, d[0], d[1]) for k, d in enumerate(descs)]
    finally:
        r.close()
    for k, sc in enumerate(scenes):
        rect = tuple(int(v) for v in GOLD["batched_rect"][k])
        conv = GOLD["batched_image"][k]
        ref = float(GOLD["batched_ref_rmse"][k])
        ep = check_window(plain[k], sc, rect, conv, ref, ref_built)
        eb = check_window(batched[k], sc, rect, conv, ref, ref_built)
        assert ep == eb, (k, ep, eb)
