"""Differentiable rendering: the C ABI's ana_forward / ana_backward pair as a
torch.autograd.Function over the scene's parameters.

    img = diff.render(renderer, frame, albedo, roughness, emission, light_le)
    loss = ((img - target) ** 2).mean()
    loss.backward()          # -> albedo.grad, roughness.grad, ...

`frame` is a Frame (width, height, spp, max_depth, seed, sample_start). The
parameter tensors are indexed like the uploaded scene's materials (albedo
(M,3), roughness (M,), emission (M,3)) and lights (light_le (L,3)); what a
material type does not use is ignored and receives a zero gradient. The
renderer keeps the state of its last forward pass only (the frame whose
paths the backward pass replays), so each backward must follow its own
forward on that renderer; a stale one raises.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import api

KEYS = ("albedo", "roughness", "emission", "light_le")


@dataclass(frozen=True)
class Frame:
    width: int
    height: int
    spp: int
    max_depth: int
    seed: int = 0
    sample_start: int = 0
    min_depth: int = 2


class PathReplayRender(torch.autograd.Function):
    @staticmethod
    def forward(ctx, renderer: api.Renderer, frame: Frame, albedo, roughness, emission, light_le):
        params = {k: t.detach().to("cpu", torch.float32).contiguous().numpy()
                  for k, t in zip(KEYS, (albedo, roughness, emission, light_le))}
        img = renderer.forward(frame.width, frame.height, frame.spp, frame.max_depth, params=params,
                               sample_start=frame.sample_start, min_depth=frame.min_depth,
                               seed=frame.seed)
        serial = getattr(renderer, "_diff_serial", 0) + 1
        renderer._diff_serial = serial
        ctx.renderer, ctx.serial, ctx.device = renderer, serial, albedo.device
        return torch.from_numpy(img).to(albedo.device)

    @staticmethod
    def backward(ctx, grad_image):
        r = ctx.renderer
        if getattr(r, "_diff_serial", None) != ctx.serial:
            raise RuntimeError("the renderer has run another forward pass since this one; "
                               "backward replays only the last frame")
        g = r.backward(grad_image.detach().to("cpu", torch.float32).contiguous().numpy())
        out = [torch.from_numpy(g[k]).to(ctx.device) for k in KEYS]
        return (None, None, *out)


def render(renderer: api.Renderer, frame: Frame, albedo, roughness, emission, light_le):
    return PathReplayRender.apply(renderer, frame, albedo, roughness, emission, light_le)


def initial_params(renderer: api.Renderer, requires_grad=True):
    """The uploaded scene's parameters as float32 tensors."""
    d = renderer.diff_params()
    return {k: torch.tensor(np.asarray(d[k]), dtype=torch.float32, requires_grad=requires_grad) for k in KEYS}
