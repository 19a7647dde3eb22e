"""Path-replay adjoint (ana_forward / ana_backward) on the differentiable
Cornell scene (6 standard_surface materials, an emissive quad and its area
light).

Bars:
  - against the oracle's FP64 forward-mode adjoint of the same estimator and
    samples: relative error <= 1e-3 (norm over all parameters, and per entry
    for every entry above 1% of the largest);
  - against central finite differences of ana_forward at common random
    numbers: tight where the image is smooth in the parameter at fixed
    samples (emission: linear; albedo without Russian roulette: polynomial);
    loose for roughness, whose finite differences also move the sampled
    directions and so agree only in expectation."""
import numpy as np
import pytest

from anacapa_b200 import api
from anacapa_b200 import scenes as S

pytestmark = pytest.mark.gpu

W = H = 64
SPP = 4
DEPTH = 6


def flat(g, nm, nl):
    v = np.zeros(8 * nm + 4 * nl)
    for i in range(nm):
        v[8 * i:8 * i + 3] = g["albedo"][i]
        v[8 * i + 3] = g["roughness"][i]
        v[8 * i + 4:8 * i + 7] = g["emission"][i]
    for l in range(nl):
        v[8 * nm + 4 * l:8 * nm + 4 * l + 3] = g["light_le"][l]
    return v


@pytest.fixture(scope="module")
def diff(gpu):
    sc = S.differentiable(W, H, SPP, DEPTH, subdiv=3)
    r = api.Renderer()
    r.upload(sc)
    wimg = np.random.default_rng(0).uniform(0.5, 1.5, (H, W, 3)).astype(np.float32)
    yield r, sc, wimg
    r.close()


def loss(r, p, wimg, w=W, h=H, spp=SPP, depth=DEPTH):
    return float((r.forward(w, h, spp, depth, params=p) * wimg).sum())


def perturbed(p0, key, idx, h):
    a = {k: np.array(v, copy=True) for k, v in p0.items()}
    a[key][idx] += h
    return a


def test_forward_is_the_render(diff):
    r, sc, _ = diff
    img = r.forward(W, H, SPP, DEPTH)
    r.render_scene(sc)
    assert np.array_equal(img, r.image(W, H))


def test_backward_matches_fp64_oracle(diff, restate_built):
    r, sc, wimg = diff
    nm, nl = r.diff_counts()
    r.forward(W, H, SPP, DEPTH, params=r.diff_params())
    g = flat(r.backward(wimg), nm, nl)
    ref = restate_built.PoScene(sc, precision=32).adjoint(wimg, spp=SPP, max_depth=DEPTH)
    assert np.linalg.norm(g - ref) <= 1e-3 * np.linalg.norm(ref)
    big = np.abs(ref) > 1e-2 * np.abs(ref).max()
    assert big.sum() >= 20
    assert (np.abs(g - ref)[big] <= 1e-3 * np.abs(ref)[big]).all()
    # entries with no dependence are exactly zero on both sides
    assert np.array_equal(g[ref == 0], ref[ref == 0])


def test_backward_twice(diff):
    r, _, wimg = diff
    nm, nl = r.diff_counts()
    r.forward(W, H, SPP, DEPTH)
    a = flat(r.backward(wimg), nm, nl)
    b = flat(r.backward(wimg), nm, nl)
    assert np.linalg.norm(a - b) <= 1e-5 * np.linalg.norm(a)  # atomics sum in any order


@pytest.mark.parametrize("ch", [0, 1, 2])
def test_emission_matches_fd(diff, ch):
    r, _, wimg = diff
    nm, nl = r.diff_counts()
    p0 = r.diff_params()
    r.forward(W, H, SPP, DEPTH, params=p0)
    g = flat(r.backward(wimg), nm, nl)
    h = 0.05
    fd = ((loss(r, perturbed(p0, "emission", (6, ch), h), wimg)
           - loss(r, perturbed(p0, "emission", (6, ch), -h), wimg))
          + (loss(r, perturbed(p0, "light_le", (0, ch), h), wimg)
             - loss(r, perturbed(p0, "light_le", (0, ch), -h), wimg))) / (2 * h)
    assert g[8 * 6 + 4 + ch] + g[8 * nm + ch] == pytest.approx(fd, rel=1e-3)
    r.forward(W, H, SPP, DEPTH, params=p0)


def test_albedo_matches_fd_without_roulette(diff):
    r, _, wimg = diff
    nm, nl = r.diff_counts()
    p0 = r.diff_params()
    r.forward(W, H, SPP, 1, params=p0)
    g = flat(r.backward(wimg), nm, nl)
    h = 0.01
    for k in range(6):
        for ch in range(3):
            fd = (loss(r, perturbed(p0, "albedo", (k, ch), h), wimg, depth=1)
                  - loss(r, perturbed(p0, "albedo", (k, ch), -h), wimg, depth=1)) / (2 * h)
            assert g[8 * k + ch] == pytest.approx(fd, rel=1e-3, abs=1e-3), (k, ch)
    r.forward(W, H, SPP, DEPTH, params=p0)


def test_roughness_agrees_with_fd_in_expectation(diff):
    r, _, _ = diff
    nm, nl = r.diff_counts()
    p0 = r.diff_params()
    w2 = h2 = 128
    spp2 = 64
    wi = np.random.default_rng(1).uniform(0.5, 1.5, (h2, w2, 3)).astype(np.float32)
    r.forward(w2, h2, spp2, DEPTH, params=p0)
    g = flat(r.backward(wi), nm, nl)[[8 * k + 3 for k in range(6)]]
    h = 0.02
    fd = np.array([(loss(r, perturbed(p0, "roughness", k, h), wi, w2, h2, spp2)
                    - loss(r, perturbed(p0, "roughness", k, -h), wi, w2, h2, spp2)) / (2 * h)
                   for k in range(6)])
    assert (np.sign(fd) == np.sign(g)).all()
    assert np.linalg.norm(fd - g) <= 0.25 * np.linalg.norm(g)
    r.forward(W, H, SPP, DEPTH, params=p0)


def test_autograd_function(diff):
    torch = pytest.importorskip("torch")
    from anacapa_b200 import diff as D
    r, _, wimg = diff
    nm, nl = r.diff_counts()
    p = D.initial_params(r)
    frame = D.Frame(W, H, SPP, DEPTH)
    img = D.render(r, frame, p["albedo"], p["roughness"], p["emission"], p["light_le"])
    (img * torch.from_numpy(wimg)).sum().backward()
    r.forward(W, H, SPP, DEPTH)
    want = r.backward(wimg)
    for k in D.KEYS:
        np.testing.assert_allclose(p[k].grad.numpy(), want[k], rtol=1e-5, atol=1e-6)


def test_backward_needs_a_forward(gpu):
    r = api.Renderer()
    try:
        r.upload(S.differentiable(16, 16, 1, 2, subdiv=1))
        with pytest.raises(api.AnaError) as e:
            r.backward(np.zeros((16, 16, 3), np.float32))
        assert e.value.code == api.ANA_ERR_STATE
    finally:
        r.close()


# ---- the differentiable configuration: 512x512, 16 spp, depth 8, 20,480-triangle sphere ----
CW = CH = 512
CSPP, CDEPTH = 16, 8


@pytest.fixture(scope="module")
def config(gpu):
    """The configuration's frame, its L2 loss against the target rendered with
    perturbed parameters (albedo +-0.2, roughness +-0.15, seed 1) and the
    target itself."""
    r = api.Renderer()
    r.upload(S.differentiable(CW, CH, CSPP, CDEPTH, params=S.perturbed_diff_params(1)))
    target = r.forward(CW, CH, CSPP, CDEPTH)
    sc = S.differentiable(CW, CH, CSPP, CDEPTH)
    r.upload(sc)
    yield r, sc, target
    r.close()


def l2(r, p, target, depth=CDEPTH, tgt=None):
    img = r.forward(CW, CH, CSPP, depth, params=p)
    t = target if tgt is None else tgt
    return float(np.mean((img.astype(np.float64) - t) ** 2)), img


def test_config_backward_matches_fp64_oracle(config, restate_built):
    """Relative error <= 1e-3 against the FP64 adjoint: the oracle traces the
    same paths in double precision (oracle/restate, precision 64) with the
    same dLoss/dimage."""
    r, sc, target = config
    nm, nl = r.diff_counts()
    _, img = l2(r, r.diff_params(), target)
    d = (2.0 * (img - target) / img.size).astype(np.float32)
    g = flat(r.backward(d), nm, nl)
    ref = restate_built.PoScene(sc, precision=64).adjoint(d)
    rel = np.linalg.norm(g - ref) / np.linalg.norm(ref)
    assert rel <= 1e-3, rel
    big = np.abs(ref) > 1e-2 * np.abs(ref).max()
    assert big.sum() >= 12
    assert (np.abs(g - ref)[big] <= 1e-3 * np.abs(ref)[big]).all(), (g[big], ref[big])


@pytest.mark.parametrize("ch", [0, 1, 2])
def test_config_emission_matches_central_fd(config, ch):
    """Central finite differences at h = 1e-3 of the L2 loss in the light's
    emission channel (the emissive quad and the area light share it): the
    image is linear in it at fixed samples, so the loss is quadratic and the
    difference quotient exact up to float rounding."""
    r, _, target = config
    nm, nl = r.diff_counts()
    p0 = r.diff_params()
    _, img = l2(r, p0, target)
    g = flat(r.backward(2.0 * (img - target) / img.size), nm, nl)
    h = 1e-3
    up = perturbed(perturbed(p0, "emission", (6, ch), h), "light_le", (0, ch), h)
    dn = perturbed(perturbed(p0, "emission", (6, ch), -h), "light_le", (0, ch), -h)
    fd = (l2(r, up, target)[0] - l2(r, dn, target)[0]) / (2 * h)
    assert g[8 * 6 + 4 + ch] + g[8 * nm + ch] == pytest.approx(fd, rel=1e-3)
    r.forward(CW, CH, CSPP, CDEPTH, params=p0)


def test_config_albedo_matches_central_fd_at_depth_1(config):
    """Central finite differences at h = 1e-3 of the L2 loss in every
    material's albedo, depth 1 (no Russian roulette, and standard_surface's
    lobe selection does not depend on the base colour, so the image is a
    polynomial in the albedo at fixed samples)."""
    r, _, target = config
    nm, nl = r.diff_counts()
    p0 = r.diff_params()
    tp = S.perturbed_diff_params(1)
    r2 = api.Renderer()
    try:
        r2.upload(S.differentiable(CW, CH, CSPP, 1, params=tp))
        t1 = r2.forward(CW, CH, CSPP, 1)
    finally:
        r2.close()
    _, img = l2(r, p0, None, depth=1, tgt=t1)
    g = flat(r.backward(2.0 * (img - t1) / img.size), nm, nl)
    h = 1e-3
    for k in range(6):
        for ch in range(3):
            fd = (l2(r, perturbed(p0, "albedo", (k, ch), h), None, depth=1, tgt=t1)[0]
                  - l2(r, perturbed(p0, "albedo", (k, ch), -h), None, depth=1, tgt=t1)[0]) / (2 * h)
            assert g[8 * k + ch] == pytest.approx(fd, rel=2e-3, abs=1e-3 * np.abs(g).max()), (k, ch, g[8 * k + ch], fd)
    r.forward(CW, CH, CSPP, CDEPTH, params=p0)
