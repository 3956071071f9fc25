"""FP16 storage form (aarbf_set_storage): the GPU's rounded scene (sorted particles, prepass
records, BVH) and its renders with the packed records are bit-identical to the oracle's FP16
scene; the rounding changes the image only slightly against the fp32 form."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32 if a.dtype == np.float32 else a.dtype)


@pytest.fixture(scope="module")
def ctx(aarbf_mod):
    c = aarbf_mod.Context(0)
    yield c
    c.close()


def _setup(ctx, orc, sc, tf, ppl, fp16, floor=1 / 255):
    dom = orc.domain([sc.xyzw])
    ctx.set_storage(fp16)
    ctx.set_particles(sc.xyzw, sc.radii)
    ctx.set_domain(dom)
    ctx.set_opacity_floor(floor)
    ctx.set_transfer_functions_f32(*tf)
    ctx.build(float(sc.radii.max()), ppl)
    scene, _, _ = orc.build_scene(sc.xyzw, sc.radii, dom, ppl, float(sc.radii.max()), tf, floor, fp16=fp16)
    return scene, dom


def _render(ctx, rp, w, h):
    import torch
    acc = torch.zeros((h, w, 4), device="cuda")
    img = torch.zeros_like(acc)
    ctx.render(rp, w, h, acc, img)
    ctx.sync()
    return acc.cpu().numpy(), img.cpu().numpy()


def test_fp16_scene_bitexact(ctx, orc):
    from aarbf import scenes
    sc = scenes.config_clusters(50_000, clusters=8, seed=13)
    scene, _ = _setup(ctx, orc, sc, scenes.tf_four_peaks(), 4, True)
    got = ctx.sorted_particles()
    assert np.array_equal(_bits(got), _bits(scene.particles()))
    assert not np.array_equal(got, scene.xyzw)  # the positions were rounded
    for g, w in zip(ctx.prepass(), scene.prepass()):
        assert np.array_equal(_bits(g), _bits(w))
    for g, w in zip(ctx.bvh(), scene.bvh()):
        assert np.array_equal(_bits(np.asarray(g)), _bits(np.asarray(w)))


@pytest.mark.parametrize("mode", ["majorant_warp", "majorant_thread", "plain"])
def test_fp16_render_bitexact(ctx, orc, mode):
    from aarbf import scenes
    sc = scenes.config_clusters(100_000, clusters=8, seed=14)
    scene, dom = _setup(ctx, orc, sc, scenes.tf_four_peaks(), 8, True)
    w, h = 40, 30
    rp = scenes.native_params(scenes.orbit_camera(), w, h, float(sc.radii.max()), 0.002, 200.0, dom, spp=2,
                              majorant=mode != "plain", bin_length=0.016, traversal=2 if mode == "majorant_thread" else 0)
    ga, gi = _render(ctx, rp, w, h)
    oa, oi = scene.render(orc.params_from(rp), w, h)
    assert (oi[..., :3] > 0).mean() > 0.01
    assert np.array_equal(_bits(gi), _bits(oi))
    assert np.array_equal(_bits(ga), _bits(oa))


def test_fp16_close_to_fp32(ctx, orc):
    """same random streams: the FP16 form's image differs from the fp32 form's by a small RMSE"""
    from aarbf import scenes
    sc = scenes.config_clusters(200_000, clusters=16, seed=15)
    tf = scenes.tf_four_peaks()
    imgs = []
    for fp16 in (False, True):
        dom = orc.domain([sc.xyzw])
        ctx.set_storage(fp16)
        ctx.set_particles(sc.xyzw, sc.radii)
        ctx.set_domain(dom)
        ctx.set_opacity_floor(1 / 255)
        ctx.set_transfer_functions_f32(*tf)
        ctx.build(float(sc.radii.max()), 8)
        rp = scenes.native_params(scenes.orbit_camera(), 64, 48, float(sc.radii.max()), 0.001, 100.0, dom, spp=16,
                                  majorant=True, bin_length=0.016)
        imgs.append(_render(ctx, rp, 64, 48)[1][..., :3].astype(np.float64))
    ctx.set_storage(False)
    rmse = float(np.sqrt(((imgs[0] - imgs[1]) ** 2).mean()))
    assert imgs[0].mean() > 0.01
    assert 0.0 < rmse < 0.05
