"""Pins the FP64 reference adjoint of the oracle (forward-mode dL/d theta
along every path) before it is used to check the device's path-replay
adjoint: on a small differentiable Cornell frame its gradient must equal
central finite differences of the oracle's own renders wherever the image is
a smooth function of the parameter at fixed samples — the emission (linear)
and the albedos with Russian roulette out of reach (max depth 1: a
polynomial)."""
import numpy as np
import pytest

from anacapa_b200 import scenes as S

W = H = 24
SPP = 2
DEPTH = 1


@pytest.fixture(scope="module")
def setup(restate_built):
    RB = restate_built
    p0 = S.default_diff_params()
    wimg = np.random.default_rng(0).uniform(0.5, 1.5, (H, W, 3)).astype(np.float32)
    sc = S.differentiable(W, H, SPP, DEPTH, subdiv=2, params=p0)
    g = RB.PoScene(sc, precision=32).adjoint(wimg, spp=SPP, max_depth=DEPTH)
    return RB, p0, wimg, sc, g


def loss(RB, p, wimg):
    sc = S.differentiable(W, H, SPP, DEPTH, subdiv=2, params=p)
    rgbw, _ = RB.PoScene(sc, precision=32).render(spp=SPP, max_depth=DEPTH)
    return float((rgbw[..., :3] / rgbw[..., 3:4] * wimg).sum())


def perturbed(p0, key, idx, h):
    a = {k: np.array(v, copy=True) for k, v in p0.items()}
    a[key][idx] += h
    return a


def test_layout(setup):
    _, _, _, sc, g = setup
    assert len(g) == 8 * len(sc.materials) + 4 * len(sc.area_lights)


@pytest.mark.parametrize("ch", [0, 1, 2])
def test_emission_matches_fd(setup, ch):
    RB, p0, wimg, sc, g = setup
    h = 0.05
    fd = (loss(RB, perturbed(p0, "emission", ch, h), wimg) - loss(RB, perturbed(p0, "emission", ch, -h), wimg)) / (2 * h)
    nm = len(sc.materials)
    # the emission parameter drives both the emissive material (index 6) and the area light
    ad = g[8 * 6 + 4 + ch] + g[8 * nm + ch]
    assert ad == pytest.approx(fd, rel=1e-4)


@pytest.mark.parametrize("k", range(6))
def test_albedo_matches_fd(setup, k):
    RB, p0, wimg, sc, g = setup
    h = 0.01
    for ch in range(3):
        fd = (loss(RB, perturbed(p0, "albedo", (k, ch), h), wimg)
              - loss(RB, perturbed(p0, "albedo", (k, ch), -h), wimg)) / (2 * h)
        assert g[8 * k + ch] == pytest.approx(fd, rel=1e-4, abs=1e-6)
