"""Generates the FP64 converged reference image used by the RMSE tests.

    python tests/golden/make_fp64.py

The image is rendered by the CPU restatement in double precision
(oracle/restate, precision 64) at 4096 samples per pixel with sampler seed
12345, so its sample stream is independent of the seed-0 streams the tests
render. Also records the RMSE of the reference CPU integrator's own 16-spp
image (flags of record) against it.
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


def main(res=128, spp=4096):
    sc = S.cornell(res, res, spp)
    t = time.time()
    rgbw, _ = P.PoScene(sc, 64).render(seed=12345)
    conv = (rgbw[..., :3] / rgbw[..., 3:4]).astype(np.float32)
    secs = time.time() - t
    R.build()
    sc16 = S.cornell(res, res, 16)
    r16, _, _ = R.RefScene(sc16, variant="record").render()
    ref16 = r16[..., :3] / r16[..., 3:4]
    rmse16 = float(np.sqrt(np.mean((ref16 - conv) ** 2)))
    np.savez_compressed(os.path.join(HERE, f"cornell{res}_fp64.npz"), image=conv, spp=spp, seed=12345,
                        ref_rmse_16spp=rmse16, seconds=secs)
    print(f"cornell {res}^2 fp64 at {spp} spp: {secs:.1f}s, reference 16-spp RMSE {rmse16:.5f}")


if __name__ == "__main__":
    main()
