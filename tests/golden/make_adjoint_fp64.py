"""Generates the FP64 reference gradient of the differentiable configuration.

    python tests/golden/make_adjoint_fp64.py

The frame is the differentiable scene (Cornell box + 20,480-triangle
icosphere, 6 standard_surface materials, emissive quad + area light) at
512x512, 16 spp, depth 8, seed 0; the loss is the L2 distance to a target
rendered with perturbed parameters (albedo +-0.2, roughness +-0.15, seed 1).
dLoss/dimage = 2 (image - target) / N comes from the CPU restatement's float
renders (which equal the reference's); the gradient is the restatement's
forward-mode adjoint traced in double precision (oracle/restate, precision
64). The GPU's own dLoss/dimage differs from this one by its float rounding
(about 1e-6 of a pixel), far below the 1e-3 gradient bar.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from anacapa_b200 import scenes as S  # noqa: E402
from oracle import restatebind as P  # noqa: E402

W = H = 512
SPP, DEPTH = 16, 8


def main():
    sc = S.differentiable(W, H, SPP, DEPTH)
    tsc = S.differentiable(W, H, SPP, DEPTH, params=S.perturbed_diff_params(1))
    t = time.time()
    tg, _ = P.PoScene(tsc, 32).render()
    im, _ = P.PoScene(sc, 32).render()
    tg = tg[..., :3] / tg[..., 3:4]
    im = im[..., :3] / im[..., 3:4]
    d = (2.0 * (im - tg) / im.size).astype(np.float32)
    g64 = P.PoScene(sc, 64).adjoint(d)
    loss = float(np.mean((im - tg) ** 2))
    secs = time.time() - t
    np.savez_compressed(os.path.join(HERE, "adjoint_fp64_512.npz"), grad=g64, loss=loss, width=W, height=H,
                        spp=SPP, depth=DEPTH, seconds=secs)
    print(f"FP64 adjoint of the 512x512x16 frame: {secs:.0f} s, loss {loss:.6g}, |g| {np.linalg.norm(g64):.6g}")


if __name__ == "__main__":
    main()
