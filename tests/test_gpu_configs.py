"""The benchmarked configurations themselves, on the GPU through the C ABI, against the oracle.

* The small configuration (100k particles of 8 isotropic Gaussians, radius 0.01, 256-entry
  linear-ramp transfer function, density scale 50, the reference's delta tracker with the global
  majorant, 512x512, 1 spp, orbit camera at distance 2.5, 60-degree field of view): the full frame.
* The headline frame (10M particles of 64 anisotropic clusters plus background, four-peak
  transfer function, delta tracking with per-bin majorants of 16 units, 8 particles per leaf,
  opacity floor 1/255, 1920x1080): the GPU renders the whole frame at 2 spp, the oracle a
  128x96 region of the same frame (pixel seeds depend on the frame size, so the region is taken
  from the full-size frame rather than rendered as a smaller image).

Every float of accum and image is compared bit for bit (the stated per-pixel tolerance of 1e-4
relative is met with zero difference).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _gpu_frame(ctx, rp, w, h):
    import torch
    acc = torch.zeros((h, w, 4), dtype=torch.float32, device="cuda")
    img = torch.zeros_like(acc)
    ctx.render(rp, w, h, acc, img)
    ctx.sync()
    return acc.cpu().numpy(), img.cpu().numpy()


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def test_config_small_full_frame(aarbf_mod, orc):
    from aarbf import scenes
    sc = scenes.config_small()
    tf = scenes.tf_linear_ramp()
    dom = orc.domain([sc.xyzw])
    w = h = 512
    rp = scenes.config_small_params(dom, w, h)
    with aarbf_mod.Context(0) as ctx:
        ctx.set_particles(sc.xyzw, sc.radii)
        ctx.set_domain(dom)
        ctx.set_transfer_functions_f32(*tf)
        ctx.build(0.01, 1)
        ga, gi = _gpu_frame(ctx, rp, w, h)
    scene = orc.build_scene(sc.xyzw, sc.radii, dom, 1, 0.01, tf, 0.0)[0]
    oa, oi = scene.render(orc.params_from(rp), w, h)
    assert (oi[..., :3] > 0).mean() > 0.01  # the view is not empty
    assert np.array_equal(_bits(gi), _bits(oi)), int((_bits(gi) != _bits(oi)).sum())
    assert np.array_equal(_bits(ga), _bits(oa))


def test_headline_frame_region_10m(aarbf_mod, orc):
    from aarbf import scenes
    sc = scenes.config_clusters(10_000_000, seed=2)
    tf = scenes.tf_four_peaks()
    dom = orc.domain([sc.xyzw])
    W, H = 1920, 1080
    rmax = float(sc.radii.max())
    rp = scenes.native_params(scenes.orbit_camera(), W, H, rmax, 0.001, 50.0, dom, spp=2, majorant=True,
                              bin_length=16 * 0.001)
    with aarbf_mod.Context(0) as ctx:
        ctx.set_particles(sc.xyzw, sc.radii)
        ctx.set_domain(dom)
        ctx.set_transfer_functions_f32(*tf)
        ctx.set_opacity_floor(1 / 255)
        ctx.build(rmax, 8)
        assert aarbf_mod.uses_warp_kernel(rp)
        ga, gi = _gpu_frame(ctx, rp, W, H)
    scene = orc.build_scene(sc.xyzw, sc.radii, dom, 8, rmax, tf, 1 / 255)[0]
    x0, y0, cw, ch = W // 2 - 64, H // 2 - 48, 128, 96
    oa = np.zeros((H, W, 4), np.float32)
    oi = np.zeros((H, W, 4), np.float32)
    scene.render(orc.params_from(rp), W, H, accum=oa, image=oi, region=(x0, x0 + cw, y0, y0 + ch))
    sl = (slice(y0, y0 + ch), slice(x0, x0 + cw))
    assert (oi[sl][..., :3] > 0).mean() > 0.5  # the region shows the clusters
    diff = int((_bits(gi[sl]) != _bits(oi[sl])).sum())
    assert diff == 0, f"{diff} of {cw * ch * 4} image floats differ"
    assert np.array_equal(_bits(ga[sl]), _bits(oa[sl]))
