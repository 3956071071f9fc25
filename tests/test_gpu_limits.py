"""Device-side iteration bounds are reported, not truncated silently.

Every device loop without a natural end (the tracking and marching loops over bins and chunks,
the warp-wide BVH traversal, the splat slab loops, the differentiable form's chunk loop) has an
iteration bound. A launch that runs out of one leaves its pixel incomplete and ors a status bit
that the next aarbf_sync turns into AARBF_ERR_DEVICE_LIMIT; the kernels still return normally, so
the context stays usable. aarbf_params.loop_cap lowers every bound for one launch, which makes the
path reachable on small scenes. No test here faults, traps or hangs the GPU: the bounds are
ordinary loop exits.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DEVICE_LIMIT = 4


@pytest.fixture(scope="module")
def ctx(aarbf_mod):
    c = aarbf_mod.Context(0)
    yield c
    c.close()


def _scene(ctx, orc, aarbf_mod):
    from aarbf import scenes
    sc = scenes.config_clusters(30_000, clusters=8, seed=6)
    cm, rm, dm = scenes.tf_linear_ramp()
    dom = orc.domain([sc.xyzw])
    ctx.set_particles(sc.xyzw, sc.radii)
    ctx.set_domain(dom)
    ctx.set_opacity_floor(0.0)
    ctx.set_transfer_functions_f32(cm, rm, dm)
    ctx.build(float(sc.radii.max()), 4)
    ctx.set_noise_atlas(aarbf_mod.generate_noise_atlas())
    scene = orc.build_scene(sc.xyzw, sc.radii, dom, 4, float(sc.radii.max()), (cm, rm, dm), 0.0)[0]
    return sc, dom, scene


def _render(ctx, rp, w, h, splat=False):
    import torch
    acc = torch.zeros((h, w, 4), dtype=torch.float32, device="cuda")
    img = torch.zeros_like(acc)
    if splat:
        ctx.render_splat(rp, w, h, img)
    else:
        ctx.render(rp, w, h, acc, img)
    return img


@pytest.mark.parametrize("kind", ["majorant_warp", "majorant_thread", "march_warp", "splat_warp", "splat_thread"])
def test_loop_cap_reports_device_limit(ctx, orc, aarbf_mod, kind):
    import torch
    from aarbf import scenes
    sc, dom, scene = _scene(ctx, orc, aarbf_mod)
    w, h = 32, 24
    rmax = float(sc.radii.max())
    trav = {"majorant_warp": 0, "majorant_thread": 2, "march_warp": 0, "splat_warp": 0, "splat_thread": 2}[kind]
    rp = scenes.native_params(scenes.orbit_camera(), w, h, rmax, 0.002, 200.0, dom, spp=2,
                              majorant=kind.startswith("majorant"), marching=kind.startswith("march"),
                              bin_length=0.004, traversal=trav)
    splat = kind.startswith("splat")
    rp.loop_cap = 2
    _render(ctx, rp, w, h, splat)
    with pytest.raises(aarbf_mod.AarbfError) as ei:
        ctx.sync()
    assert ei.value.status == DEVICE_LIMIT
    # the status was reported and cleared; the context renders correctly afterwards
    rp.loop_cap = 0
    img = _render(ctx, rp, w, h, splat)
    ctx.sync()
    got = img.cpu().numpy()
    atlas = aarbf_mod.generate_noise_atlas()
    p = orc.params_from(rp, noise=atlas)
    want = scene.render_splat(p, w, h) if splat else scene.render(p, w, h)[1]
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert not torch.isnan(img).any()


def test_loop_cap_differentiable_form(ctx, aarbf_mod):
    import torch
    from aarbf import scenes
    gt, _ = scenes.config_differentiable(400, clusters=4, seed=5, tf_size=16)
    gt.radii[:] = 0.06
    dom = np.array([0, 0, 0, 1, 1, 1, 0, 1], np.float32)
    nc = len(gt.tf)
    ctx.set_domain(dom)
    ctx.set_transfer_functions_f32(gt.tf, np.ones(nc, np.float32), np.ones(nc, np.float32))
    ctx.set_particles(np.concatenate([gt.pos, gt.attr[:, None]], 1).astype(np.float32), gt.radii)
    ctx.build(0.06, 4)
    w, h = 16, 12
    views = [scenes.native_params(cam, w, h, 0.08, 0.002, 10.0, dom, spp=2, frame_id=3 * k, marching=True)
             for k, cam in enumerate(scenes.orbit_views(2))]
    img = torch.zeros((2, h, w, 4), dtype=torch.float32, device="cuda")
    ref = torch.zeros_like(img)
    ctx.render_diff_forward(views, w, h, ref)
    ctx.sync()
    for v in views:
        v.loop_cap = 2
    ctx.render_diff_forward(views, w, h, img)
    with pytest.raises(aarbf_mod.AarbfError) as ei:
        ctx.sync()
    assert ei.value.status == DEVICE_LIMIT
    for v in views:
        v.loop_cap = 0
    ctx.render_diff_forward(views, w, h, img)
    ctx.sync()
    assert torch.equal(img, ref)


def test_work_item_count_is_checked(ctx, orc, aarbf_mod):
    """a launch whose width x height x spp (pixels padded to 8 x 4 tiles) exceeds the persistent
    kernels' 32-bit work-item count is refused on the host, before any allocation or launch"""
    from aarbf import scenes
    sc, dom, scene = _scene(ctx, orc, aarbf_mod)
    rp = scenes.native_params(scenes.orbit_camera(), 64, 64, float(sc.radii.max()), 0.002, 200.0, dom, spp=2,
                              majorant=True, bin_length=0.004)
    small = ctx.device_alloc(1 << 16)
    try:
        with pytest.raises(aarbf_mod.AarbfError) as ei:
            ctx.render(rp, 65536, 65536, small, small)  # 2^33 samples
        assert ei.value.status == 1  # AARBF_ERR_INVALID_ARGUMENT
        ctx.sync()  # nothing was launched: no device status either
    finally:
        ctx.device_free(small)
