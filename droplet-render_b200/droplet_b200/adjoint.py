"""Differentiable rendering: the path-replay adjoint behind torch.autograd.

`render(bricks, albedo, views)` renders every view of one scene with the brick
samples taken from a CUDA tensor and the single-scatter albedo from a scalar
tensor; backward runs the GPU adjoint (dr_adjoint_tile_async), which replays
each path from its random stream (no stored tape) and returns
dL/d(brick samples) and dL/d(albedo).  The extinction sigma_t of every view is
held fixed: sigma_s = albedo sigma_t, sigma_a = sigma_t - sigma_s.

Images are means over the samples (tile sums / spp), shape (views, h, w, 4)
for the sun and sky buffers; alpha carries no gradient.  Rendering uses
DR_KERNEL_FINITE_PATHS (a path sample whose sum is not finite, the
reference's sky 0/0 for rd.y == 0, adds nothing), and the adjoint leaves such
paths out the same way.  The leaf majorants
are recomputed from the bricks on each forward (majorant_scale x maximum,
floor 0.01) and held fixed through the backward pass.

Several GPUs (one process each): every rank renders its share of the views
(ranks.my_views), computes its part of the loss and calls backward, then
ranks.sum_gradients(bricks.grad, albedo.grad) sums the gradients over the ranks
before the optimizer step: the gradient of the loss summed over all views.
"""
from __future__ import annotations

from dataclasses import dataclass, replace

import numpy as np

from .renderer import Renderer, RenderSettings, stream_handle


@dataclass
class DiffView:
    settings: RenderSettings  # camera, sun, sky, phase, image size; sigma_s + sigma_a = this view's sigma_t
    spp: int
    seed: int = 0


def _with_albedo(s: RenderSettings, albedo: float) -> RenderSettings:
    st = np.float32(s.sigma_s) + np.float32(s.sigma_a)
    ss = np.float32(st * np.float32(albedo))
    return replace(s, sigma_s=float(ss), sigma_a=float(np.float32(st - ss)), finite_paths=True)


def _function():
    import torch

    class RenderFn(torch.autograd.Function):
        @staticmethod
        def forward(ctx, bricks, albedo, renderer, views, adjoint_seed_offset, majorant_scale):
            bricks = bricks.detach().contiguous()
            stream = torch.cuda.current_stream(bricks.device)
            sh = stream_handle(stream)
            renderer.set_bricks_dev(bricks.data_ptr(), bricks.shape[0], majorant_scale, sh)
            a = float(albedo.detach().cpu())
            h = max(v.settings.h for v in views)
            w = max(v.settings.w for v in views)
            sun = torch.zeros((len(views), h, w, 4), dtype=torch.float32, device=bricks.device)
            sky = torch.zeros_like(sun)
            for i, v in enumerate(views):
                renderer.set_params(_with_albedo(v.settings, a))
                vs = torch.empty((v.settings.h, v.settings.w, 4), dtype=torch.float32, device=bricks.device)
                vk = torch.empty_like(vs)
                renderer.render_tile_async(0, 0, v.settings.w, v.settings.h, v.spp, v.seed, 0, vs.data_ptr(),
                                           vk.data_ptr(), sh)
                sun[i, :v.settings.h, :v.settings.w] = vs / v.spp
                sky[i, :v.settings.h, :v.settings.w] = vk / v.spp
            ctx.renderer, ctx.views, ctx.albedo = renderer, views, a
            ctx.offset = adjoint_seed_offset
            ctx.shape = bricks.shape
            return sun, sky

        @staticmethod
        def backward(ctx, g_sun, g_sky):
            r, views = ctx.renderer, ctx.views
            dev = g_sun.device
            sh = stream_handle(torch.cuda.current_stream(dev))
            grad = torch.zeros(ctx.shape, dtype=torch.float32, device=dev)
            galb = torch.zeros(1, dtype=torch.float64, device=dev)
            for i, v in enumerate(views):
                hh, ww = v.settings.h, v.settings.w
                ds = (g_sun[i, :hh, :ww] / v.spp).contiguous().float()
                dk = (g_sky[i, :hh, :ww] / v.spp).contiguous().float()
                r.set_params(_with_albedo(v.settings, ctx.albedo))
                # ds / dk may be freed after this iteration: the caching allocator
                # reuses their memory only for work queued after the kernel on this stream
                r.adjoint_tile_async(0, 0, ww, hh, v.spp, v.seed + ctx.offset, 0, ds.data_ptr(), dk.data_ptr(),
                                     grad.data_ptr(), galb.data_ptr(), sh)
            return grad, galb.to(torch.float32).reshape(()), None, None, None, None

    return RenderFn


_FN = None


def render(bricks, albedo, renderer: Renderer, views: list, adjoint_seed_offset: int = 0x9E3779B9,
           majorant_scale: float = 1.0):
    """(sun, sky) mean images of all views, differentiable in bricks and albedo.

    adjoint_seed_offset: the backward pass replays paths drawn from seed +
    offset, independent of the forward samples (offset 0 replays the forward's
    own paths, which correlates the loss gradient with the image noise)."""
    global _FN
    if _FN is None:
        _FN = _function()
    return _FN.apply(bricks, albedo, renderer, views, adjoint_seed_offset, majorant_scale)
