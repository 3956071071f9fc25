"""Differentiable form on the GPU (aarbf_render_diff_forward / _backward) against the FP64 oracle
of the same model: images and every gradient (positions, radii, attributes, transfer function),
through the C ABI and through the torch.autograd wrapper."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

W, H = 16, 12


def _case(n=400, seed=5, dense=False):
    from aarbf import scenes
    rng = np.random.default_rng(seed)
    gt, init = scenes.config_differentiable(n, clusters=4, seed=seed, tf_size=16)
    if dense:  # every particle in one small ball: single steps exceed the staging buffer
        init.pos[:] = (0.5 + rng.normal(0.0, 0.01, (n, 3))).astype(np.float32)
        gt.pos[:] = (0.5 + rng.normal(0.0, 0.01, (n, 3))).astype(np.float32)
        init.radii[:] = 0.05
        gt.radii[:] = 0.05
    else:
        gt.radii[:] = rng.uniform(0.04, 0.08, n).astype(np.float32)
        init.radii[:] = rng.uniform(0.04, 0.08, n).astype(np.float32)
    dom = np.array([0, 0, 0, 1, 1, 1, 0, 1], np.float32)
    scale = 0.5 if dense else 10.0
    fov = 3.0 if dense else 60.0  # the dense ball fills the frame
    views = [scenes.native_params(cam, W, H, 0.08, 0.01, scale, dom, spp=2, frame_id=7 * k, marching=True)
             for k, cam in enumerate(scenes.orbit_views(2, fov_deg=fov))]
    return gt, init, views, dom


def _gpu(ctx, sc, views, dom, grad_images):
    import torch
    nc = len(sc.tf)
    ctx.set_domain(dom)
    ctx.set_transfer_functions_f32(sc.tf, np.ones(nc, np.float32), np.ones(nc, np.float32))
    xyzw = np.concatenate([sc.pos, sc.attr[:, None]], 1).astype(np.float32)
    ctx.set_particles(xyzw, sc.radii)
    ctx.build(float(sc.radii.max()), 4)
    img = torch.zeros((len(views), H, W, 4), dtype=torch.float32, device="cuda")
    ctx.render_diff_forward(views, W, H, img)
    ctx.sync()
    out = img[..., :3].double().cpu().numpy()
    g = torch.zeros((len(views), H, W, 4), dtype=torch.float32, device="cuda")
    g[..., :3] = torch.from_numpy(grad_images.astype(np.float32)).cuda()
    n = len(sc.radii)
    gp = torch.zeros((n, 3), device="cuda")
    gr = torch.zeros(n, device="cuda")
    ga = torch.zeros(n, device="cuda")
    gt = torch.zeros((nc, 4), device="cuda")
    ctx.render_diff_backward(views, W, H, g, gp, gr, ga, gt)
    ctx.sync()
    return out, [x.double().cpu().numpy() for x in (gp, gr, ga, gt)]


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.fixture(scope="module")
def ctx(aarbf_mod):
    c = aarbf_mod.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("dense", [False, True])
def test_diff_forward_and_adjoint_match_fp64(ctx, orc, dense):
    gt, init, views, dom = _case(dense=dense, n=400 if not dense else 600)
    ov = [orc.params_from(v) for v in views]
    target = orc.diff_forward(gt.pos, gt.radii, gt.attr, gt.tf, ov, W, H)
    ref = orc.diff_forward(init.pos, init.radii, init.attr, init.tf, ov, W, H)
    assert ref.max() > 0.05  # the views are not empty
    gimg = 2.0 * (ref - target)
    img, grads = _gpu(ctx, init, views, dom, gimg)
    # images: float kernels against the FP64 model, tolerance 1e-4 of the image range
    assert np.abs(img - ref).max() <= 1e-4 * ref.max() + 1e-6
    refg = orc.diff_backward(init.pos, init.radii, init.attr, init.tf, ov, W, H, gimg)
    for got, want, name in zip(grads, refg, ("position", "radius", "attribute", "transfer function")):
        assert np.linalg.norm(want) > 0, name
        assert _rel(got, want) < 2e-3, name  # float adjoint against the FP64 adjoint


def test_autograd_wrapper(ctx, orc):
    """ParticleVolumeRender: images and .grad of every input equal the FP64 reference's"""
    import torch
    from aarbf import autograd
    gt, init, views, dom = _case()
    ctx.set_domain(dom)
    ov = [orc.params_from(v) for v in views]
    target_np = orc.diff_forward(gt.pos, gt.radii, gt.attr, gt.tf, ov, W, H)
    target = torch.from_numpy(target_np).float().cuda()
    t = [torch.tensor(x, device="cuda", requires_grad=True) for x in (init.pos, init.radii, init.attr, init.tf)]
    img = autograd.render(*t, ctx, views, W, H, 4)
    loss = ((img - target) ** 2).sum()
    loss.backward()
    ref = orc.diff_forward(init.pos, init.radii, init.attr, init.tf, ov, W, H)
    refg = orc.diff_backward(init.pos, init.radii, init.attr, init.tf, ov, W, H,
                             2.0 * (ref - target.double().cpu().numpy()))
    assert np.abs(img.detach().double().cpu().numpy() - ref).max() <= 1e-4 * ref.max() + 1e-6
    for x, want in zip(t, refg):
        assert _rel(x.grad.double().cpu().numpy(), want) < 2e-3
