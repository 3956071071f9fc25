"""Count mode (aarbf_render_count) of the ray-per-warp kernels: it runs its own kernel instance
(the timed instance carries no accounting code), renders the same bits as aarbf_render, and
its counters describe the work: stagings, traversal steps, particle tests and tracking steps."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("marching", [False, True])
def test_count_mode_renders_the_same_image(aarbf_mod, marching):
    import torch
    from aarbf import scenes
    sc = scenes.config_clusters(60_000, clusters=8, seed=41)
    cm, rm, dm = scenes.tf_four_peaks(64, seed=2)
    dom = np.concatenate([sc.xyzw[:, :3].min(0), sc.xyzw[:, :3].max(0),
                          [sc.xyzw[:, 3].min(), sc.xyzw[:, 3].max()]]).astype(np.float32)
    ctx = aarbf_mod.Context(0)
    try:
        ctx.set_domain(dom)
        ctx.set_transfer_functions_f32(cm, rm, dm)
        ctx.set_opacity_floor(1 / 255)
        ctx.set_particles(sc.xyzw, sc.radii)
        ctx.build(float(sc.radii.max()), 8)
        w, h = 48, 40
        rp = scenes.native_params(scenes.orbit_camera(), w, h, float(sc.radii.max()), 0.002, 300.0, dom, spp=3,
                                  frame_id=7, marching=marching, majorant=not marching, bin_length=0.016)
        assert aarbf_mod.uses_warp_kernel(rp.to_c())
        acc = torch.zeros((h, w, 4), device="cuda")
        img = torch.zeros_like(acc)
        ctx.render(rp, w, h, acc, img)
        ctx.sync()
        want = img.cpu().numpy()
        assert (want[..., :3] > 0).any()
        acc.zero_()
        img.zero_()
        c = ctx.render_count(rp, w, h, acc, img)
        ctx.sync()
        assert np.array_equal(img.cpu().numpy().view(np.uint32), want.view(np.uint32))
        # particles and nodes on the traversed ray segments (every warp kernel)
        assert c["segment_particles"] > 0 and c["segment_nodes"] > 0
        if not marching:  # the majorant tracker's own work counters
            assert c["stagings"] > 0 and c["traversal_iterations"] > 0 and c["particles_tested"] > 0
            assert c["steps"] > 0 and c["bins"] > 0 and c["candidates_staged"] > 0
    finally:
        ctx.close()
