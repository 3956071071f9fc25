"""torch.autograd wrapper of the differentiable form (aarbf_render_diff_forward / _backward).

The function renders expected-stochastic-marching images of particles with learnable positions,
radii, attributes and RGBA transfer function through the CUDA kernels behind the C ABI; its
backward is the hand-written adjoint (path replay). Every call rebuilds the context's Hilbert
order and BVH for the current positions and radii. The context's domain must hold the
attribute range the attributes are normalised by (set_domain).
"""
from __future__ import annotations

import torch

from . import Context, RenderParams


class ParticleVolumeRender(torch.autograd.Function):
    """images (nviews, H, W, 3) = render(pos (n, 3), radius (n,), attr (n,), tf (nc, 4) RGBA);
    float32 CUDA tensors."""

    @staticmethod
    def forward(fctx, pos, radius, attr, tf, rctx: Context, views, width: int, height: int, ppl: int = 8):
        dev = pos.device
        n = pos.shape[0]
        nc = tf.shape[0]
        ones = [1.0] * nc
        rctx.set_transfer_functions_f32(tf.detach().float().cpu().numpy(), ones, ones)
        xyzw = torch.cat([pos.detach().float(), attr.detach().float()[:, None]], 1).contiguous()
        rad = radius.detach().float().contiguous()
        rctx.set_particles(xyzw, rad)
        rctx.build(float(rad.max()) if n else 0.0, ppl)
        images = torch.empty((len(views), height, width, 4), dtype=torch.float32, device=dev)
        rctx.render_diff_forward(views, width, height, images)
        rctx.sync()
        fctx.rctx, fctx.views, fctx.size = rctx, views, (width, height, n, nc)
        return images[..., :3]

    @staticmethod
    def backward(fctx, grad_rgb):
        width, height, n, nc = fctx.size
        dev = grad_rgb.device
        g = torch.zeros((len(fctx.views), height, width, 4), dtype=torch.float32, device=dev)
        g[..., :3] = grad_rgb
        gp = torch.empty((n, 3), dtype=torch.float32, device=dev)
        gr = torch.empty(n, dtype=torch.float32, device=dev)
        ga = torch.empty(n, dtype=torch.float32, device=dev)
        gt = torch.empty((nc, 4), dtype=torch.float32, device=dev)
        fctx.rctx.render_diff_backward(fctx.views, width, height, g.contiguous(), gp, gr, ga, gt)
        fctx.rctx.sync()
        return gp, gr, ga, gt, None, None, None, None, None


def render(pos, radius, attr, tf, rctx: Context, views: list[RenderParams], width: int, height: int, ppl: int = 8):
    """Differentiable render of nviews images (nviews, H, W, 3)."""
    return ParticleVolumeRender.apply(pos, radius, attr, tf, rctx, views, width, height, ppl)
