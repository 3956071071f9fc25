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
