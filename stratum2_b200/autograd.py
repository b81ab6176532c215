"""torch.autograd bridge for the differentiable renderer: textures in, image out, texel gradients
back through the adjoint path replay (s2_render_adjoint).  torch supplies the device tensors and the
autograd bookkeeping; the rendering and its adjoint are the library's CUDA kernels."""
from __future__ import annotations

import torch

from . import _abi


class _DiffRender(torch.autograd.Function):
    @staticmethod
    def forward(ctx, device, view, width, height, params, indices, *textures):
        for i, t in zip(indices, textures):
            device.update_image(i, t.detach().to(torch.float32).contiguous())
        out = torch.empty((height, width, 4), dtype=torch.float32, device="cuda")
        device.render_diff_device(view, params, out.data_ptr())
        ctx.device, ctx.view, ctx.params, ctx.indices = device, view, params, list(indices)
        ctx.save_for_backward(*textures)
        return out

    @staticmethod
    def backward(ctx, grad_out):
        textures = ctx.saved_tensors
        dev = ctx.device
        # the adjoint replays the forward's paths: make sure the scene holds the forward's textures
        for i, t in zip(ctx.indices, textures):
            dev.update_image(i, t.detach().to(torch.float32).contiguous())
        g = grad_out.detach().to(torch.float32).contiguous()
        n = len(dev.scene.images)
        bufs = {i: torch.zeros(t.shape[:2] + (4,), dtype=torch.float32, device="cuda") for i, t in zip(ctx.indices, textures)}
        ptrs = [bufs[k].data_ptr() if k in bufs else None for k in range(n)]
        dev.render_adjoint_device(ctx.view, ctx.params, g.data_ptr(), ptrs)
        grads = [bufs[i][..., :t.shape[2]].to(t.dtype) for i, t in zip(ctx.indices, textures)]
        return (None, None, None, None, None, None, *grads)


def render(device, view, width: int, height: int, params: _abi.S2RenderParams, textures: dict) -> torch.Tensor:
    """Differentiable render (s2_render_diff) of `view` with the scene images {index: (h, w, c) CUDA
    tensor} replaced by `textures`; returns the (height, width, 4) radiance image.  Gradients of any
    loss of the image flow back to the textures by adjoint path replay (base-colour textures,
    packed[2] roughness channel, environment image)."""
    idx = list(textures.keys())
    return _DiffRender.apply(device, view, width, height, params, idx, *[textures[k] for k in idx])
