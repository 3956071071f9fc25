"""Series playback with overlapped upload/build (aarbf.streaming.SeriesRenderer): the images of
every frame equal those of the reference's one-after-the-other order with a single context, and
both equal the oracle's render of that frame bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_series_overlap_matches_sequential(aarbf_mod, orc):
    import torch
    from aarbf import scenes, streaming
    base = scenes.config_clusters(40_000, clusters=6, seed=31)
    frames_np = []
    for k in range(4):
        x = base.xyzw.copy()
        x[:, 0] += np.float32(0.002 * k)
        frames_np.append((x, base.radii))
    allx = np.concatenate([f[0] for f in frames_np])
    dom = np.concatenate([allx[:, :3].min(0), allx[:, :3].max(0), [allx[:, 3].min(), allx[:, 3].max()]]).astype(np.float32)
    tf = scenes.tf_four_peaks()
    w, h = 48, 32
    rmax = float(base.radii.max())

    def params(k):
        return scenes.native_params(scenes.orbit_camera(), w, h, rmax, 0.002, 200.0, dom, spp=2, frame_id=2 * k,
                                    majorant=True, bin_length=0.016)

    frames = [(torch.from_numpy(x).pin_memory(), torch.from_numpy(r).pin_memory()) for x, r in frames_np]
    accum = torch.zeros((h, w, 4), device="cuda")
    imgs = [torch.zeros((h, w, 4), device="cuda") for _ in frames]
    sr = streaming.SeriesRenderer(0, dom, tf, rmax, ppl=4, alpha_floor=1 / 255)
    sr.render_series(frames, params, w, h, accum, imgs, overlap=True)
    sr.close()
    # the reference's order with one context
    ctx = aarbf_mod.Context(0)
    ctx.set_domain(dom)
    ctx.set_transfer_functions_f32(*tf)
    ctx.set_opacity_floor(1 / 255)
    for k, (x, r) in enumerate(frames_np):
        ctx.set_particles(x, r)
        ctx.build(rmax, 4)
        ref = torch.zeros((h, w, 4), device="cuda")
        ctx.render(params(k), w, h, accum, ref)
        ctx.sync()
        assert np.array_equal(ref.cpu().numpy().view(np.uint32), imgs[k].cpu().numpy().view(np.uint32))
        if k == 0:
            assert (ref[..., :3] > 0).float().mean() > 0.01
        # the oracle's render of the same frame
        scene = orc.build_scene(x, r, dom, 4, rmax, tf, 1 / 255)[0]
        _, want = scene.render(orc.params_from(params(k)), w, h)
        assert np.array_equal(imgs[k].cpu().numpy().view(np.uint32), want.view(np.uint32)), f"frame {k}"
    ctx.close()


def _frames(n=30_000, count=4, seed=33):
    """a drifting, jittering series: particle i of every frame is the same particle"""
    from aarbf import scenes
    base = scenes.config_clusters(n, clusters=6, seed=seed)
    rng = np.random.default_rng(seed)
    frames = []
    for k in range(count):
        x = base.xyzw.copy()
        x[:, 0] += np.float32(0.003 * k)
        x[:, :3] += rng.normal(0.0, 0.002, (n, 3)).astype(np.float32)
        frames.append(np.ascontiguousarray(x, np.float32))
    allx = np.concatenate(frames)
    dom = np.concatenate([allx[:, :3].min(0), allx[:, :3].max(0), [allx[:, 3].min(), allx[:, 3].max()]]).astype(
        np.float32)
    return frames, base.radii, dom


@pytest.mark.parametrize("keep_order", [False, True])
def test_refit_frame_matches_rebuild_and_oracle(aarbf_mod, orc, keep_order):
    """aarbf_refit_frame: frames after the first refit the first frame's BVH topology (the
    reference's gprtAccelUpdate path on a frame change); every frame renders the same bits as a full
    rebuild and as the oracle, with majorant tracking and with the reference's delta tracker"""
    import torch
    from aarbf import scenes
    frames, radii, dom = _frames()
    tf = scenes.tf_four_peaks()
    w, h = 40, 30
    rmax = float(radii.max())
    ctx, fresh = aarbf_mod.Context(0), aarbf_mod.Context(0)
    try:
        for c in (ctx, fresh):
            c.set_domain(dom)
            c.set_transfer_functions_f32(*tf)
            c.set_opacity_floor(1 / 255)
        for k, x in enumerate(frames):
            ctx.set_particles(x, radii)
            if k == 0:
                ctx.build(rmax, 4)
            else:
                ctx.refit_frame(keep_order)
            fresh.set_particles(x, radii)
            fresh.build(rmax, 4)
            scene = orc.build_scene(x, radii, dom, 4, rmax, tf, 1 / 255)[0]
            if not keep_order:  # the frame's own Hilbert order: the same leaves as a rebuild
                assert np.array_equal(ctx.sorted_particles().view(np.uint32), scene.xyzw.view(np.uint32))
                assert np.array_equal(ctx.bvh()[3].view(np.uint32), scene.bvh()[3].view(np.uint32))
            # every node box holds its children's boxes (the refit topology is consistent)
            left, right, nb, _, lb, _ = ctx.bvh()
            LEAF = np.uint32(0x80000000)
            for ch in (left, right):
                is_leaf = (ch & LEAF) != 0
                cb = np.where(is_leaf[:, None], lb[(ch & ~LEAF) % len(lb)], nb[ch % max(len(nb), 1)])
                ok = np.isnan(cb).all(1) | ((cb[:, :3] >= nb[:, :3]).all(1) & (cb[:, 3:] <= nb[:, 3:]).all(1))
                assert ok.all()
            for majorant in (True, False):
                rp = scenes.native_params(scenes.orbit_camera(), w, h, rmax, 0.002, 200.0, dom, spp=2, frame_id=3 * k,
                                          majorant=majorant, bin_length=0.016)
                imgs = []
                for c in (ctx, fresh):
                    acc = torch.zeros((h, w, 4), device="cuda")
                    img = torch.zeros_like(acc)
                    c.render(rp, w, h, acc, img)
                    c.sync()
                    imgs.append(img.cpu().numpy())
                _, want = scene.render(orc.params_from(rp), w, h)
                assert np.array_equal(imgs[0].view(np.uint32), imgs[1].view(np.uint32)), f"frame {k}: refit vs rebuild"
                assert np.array_equal(imgs[0].view(np.uint32), want.view(np.uint32)), f"frame {k}: vs oracle"
                assert (want[..., :3] > 0).mean() > 0.01
        # a frame of another particle count cannot refit
        ctx.set_particles(frames[0][:1000], radii[:1000])
        with pytest.raises(aarbf_mod.AarbfError):
            ctx.refit_frame(keep_order)
    finally:
        ctx.close()
        fresh.close()
