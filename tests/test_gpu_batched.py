"""Batched rendering (aarbf_batch_create / aarbf_batch_render): several scenes of different
sizes, resolutions and spp in one persistent launch give the same bits as one aarbf_render per
scene and as the oracle's render of each scene, also when the launch is replayed from a CUDA
graph."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _scenes(aarbf_mod):
    from aarbf import scenes
    rng = np.random.default_rng(11)
    out = []
    for k, (n, w, h, spp) in enumerate([(3000, 24, 16, 1), (20000, 40, 30, 3), (8000, 16, 16, 2), (50000, 32, 24, 4)]):
        sc = scenes.config_clusters(n, clusters=4 + k, seed=20 + k)
        cm, rm, dm = scenes.tf_four_peaks(64, seed=k)
        dom = np.concatenate([sc.xyzw[:, :3].min(0), sc.xyzw[:, :3].max(0),
                              [sc.xyzw[:, 3].min(), sc.xyzw[:, 3].max()]]).astype(np.float32)
        ctx = aarbf_mod.Context(0)
        ctx.set_domain(dom)
        ctx.set_transfer_functions_f32(cm, rm, dm)
        ctx.set_opacity_floor(1 / 255)
        ctx.set_particles(sc.xyzw, sc.radii)
        ctx.build(float(sc.radii.max()), 4)
        cam = scenes.orbit_camera(azimuth_deg=float(rng.uniform(0, 360)), elevation_deg=float(rng.uniform(-30, 30)))
        rp = scenes.native_params(cam, w, h, float(sc.radii.max()), 0.002, 300.0, dom, spp=spp, frame_id=5 * k,
                                  majorant=True, bin_length=0.008)
        out.append((ctx, rp, (w, h), (sc, (cm, rm, dm), dom)))
    return out


def test_batched_matches_single_renders(aarbf_mod, orc):
    import torch
    items = _scenes(aarbf_mod)
    ref = []
    for ctx, rp, (w, h), (sc, tf, dom) in items:
        acc = torch.zeros((h, w, 4), device="cuda")
        img = torch.zeros_like(acc)
        ctx.render(rp, w, h, acc, img)
        ctx.sync()
        ref.append((acc.cpu().numpy(), img.cpu().numpy()))
        # every scene's single render equals the oracle's
        scene = orc.build_scene(sc.xyzw, sc.radii, dom, 4, float(sc.radii.max()), tf, 1 / 255)[0]
        oa, oi = scene.render(orc.params_from(rp), w, h)
        assert np.array_equal(ref[-1][1].view(np.uint32), oi.view(np.uint32))
        assert np.array_equal(ref[-1][0].view(np.uint32), oa.view(np.uint32))
    assert any((r[1][..., :3] > 0).mean() > 0.01 for r in ref)
    accs = [torch.zeros((h, w, 4), device="cuda") for _, _, (w, h), _ in items]
    imgs = [torch.zeros_like(a) for a in accs]
    b = aarbf_mod.Batch([c for c, _, _, _ in items], [p for _, p, _, _ in items], [s for _, _, s, _ in items], accs,
                        imgs)
    for cap, bps, smaj in ((0, 0, False), (512, 6, True), (1024, 7, False), (256, 1, True)):
        for a in accs:
            a.zero_()
        b.set_shape(bps, smaj)  # launch shape: speed only, the same bits
        b.render(cap)
        torch.cuda.synchronize()
        for (ra, ri), a, i in zip(ref, accs, imgs):
            assert np.array_equal(a.cpu().numpy().view(np.uint32), ra.view(np.uint32))
            assert np.array_equal(i.cpu().numpy().view(np.uint32), ri.view(np.uint32))
    with pytest.raises(aarbf_mod.AarbfError):
        b.set_shape(-1, False)
    b.set_shape(0, False)
    # the autotuner's plan (longest first, each scene's own first-staging length): the same bits
    import copy
    from aarbf import autotune
    order, bins, cost = autotune.scene_plan([c for c, _, _, _ in items], [p for _, p, _, _ in items],
                                            [s for _, _, s, _ in items], accs, imgs)
    assert sorted(order) == list(range(len(items))) and all(x in autotune.STAGE_BINS for x in bins)
    assert all(cost[order[k]] >= cost[order[k + 1]] for k in range(len(order) - 1))
    planned = []
    for i in order:
        q = copy.copy(items[i][1])
        q.stage_bins = bins[i]
        planned.append(q)
    for a in accs:
        a.zero_()
    bp = aarbf_mod.Batch([items[i][0] for i in order], planned, [items[i][2] for i in order],
                         [accs[i] for i in order], [imgs[i] for i in order])
    bp.render(0)
    torch.cuda.synchronize()
    for (ra, ri), i in zip(ref, imgs):
        assert np.array_equal(i.cpu().numpy().view(np.uint32), ri.view(np.uint32))
    bp.close()
    # the same launch replayed from a CUDA graph
    st = torch.cuda.Stream()
    with torch.cuda.stream(st):
        b.render(0, st)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=st):
        b.render(0, st)
    for a, i in zip(accs, imgs):
        a.zero_()
        i.zero_()
    torch.cuda.synchronize()
    g.replay()
    torch.cuda.synchronize()
    for (ra, ri), a, i in zip(ref, accs, imgs):
        assert np.array_equal(i.cpu().numpy().view(np.uint32), ri.view(np.uint32))
    del g
    b.close()
    for ctx, _, _, _ in items:
        ctx.close()


def test_batch_of_repeated_contexts_over_several_launches(aarbf_mod, orc):
    """70 views of three scenes (more than the 64 scenes of one launch, each context several
    times): every view equals its single render, which equals the oracle; a single render through
    a context between batch renders (which grows that context's own sample planes) leaves the
    batch's results unchanged"""
    import torch
    from aarbf import scenes
    rng = np.random.default_rng(31)
    ctxs, oracle_scenes = [], []
    for k, n in enumerate((3000, 6000, 4000)):
        sc = scenes.config_clusters(n, clusters=3 + k, seed=40 + k)
        cm, rm, dm = scenes.tf_four_peaks(64, seed=10 + k)
        dom = np.concatenate([sc.xyzw[:, :3].min(0), sc.xyzw[:, :3].max(0),
                              [sc.xyzw[:, 3].min(), sc.xyzw[:, 3].max()]]).astype(np.float32)
        ctx = aarbf_mod.Context(0)
        ctx.set_domain(dom)
        ctx.set_transfer_functions_f32(cm, rm, dm)
        ctx.set_opacity_floor(1 / 255)
        ctx.set_particles(sc.xyzw, sc.radii)
        ctx.build(float(sc.radii.max()), 4)
        ctxs.append((ctx, float(sc.radii.max()), dom))
        oracle_scenes.append(orc.build_scene(sc.xyzw, sc.radii, dom, 4, float(sc.radii.max()), (cm, rm, dm),
                                             1 / 255)[0])
    entries = []
    for j in range(70):
        k = j % 3
        ctx, rmax, dom = ctxs[k]
        w, h, spp = int(rng.choice([8, 16])), 8, int(rng.integers(1, 3))
        cam = scenes.orbit_camera(azimuth_deg=float(rng.uniform(0, 360)), elevation_deg=float(rng.uniform(-30, 30)))
        rp = scenes.native_params(cam, w, h, rmax, 0.002, 300.0, dom, spp=spp, frame_id=7 * j, majorant=True,
                                  bin_length=0.008)
        entries.append((k, rp, w, h))
    ref = []
    for j, (k, rp, w, h) in enumerate(entries):
        acc = torch.zeros((h, w, 4), device="cuda")
        img = torch.zeros_like(acc)
        ctxs[k][0].render(rp, w, h, acc, img)
        ctxs[k][0].sync()
        ref.append(img.cpu().numpy())
        if j < 3:  # the first view of each scene against the oracle
            want = oracle_scenes[k].render(orc.params_from(rp), w, h)[1]
            assert np.array_equal(ref[-1].view(np.uint32), want.view(np.uint32))
    assert any((r[..., :3] > 0).mean() > 0.01 for r in ref)
    accs = [torch.zeros((h, w, 4), device="cuda") for _, _, w, h in entries]
    imgs = [torch.zeros_like(a) for a in accs]
    b = aarbf_mod.Batch([ctxs[k][0] for k, _, _, _ in entries], [rp for _, rp, _, _ in entries],
                        [(w, h) for _, _, w, h in entries], accs, imgs)
    for step in range(2):
        for a in accs:
            a.zero_()
        b.render(0)
        torch.cuda.synchronize()
        for r, i in zip(ref, imgs):
            assert np.array_equal(i.cpu().numpy().view(np.uint32), r.view(np.uint32))
        if step == 0:  # a larger single render through the first context between batch renders
            k, rp, _, _ = entries[0]
            big = torch.zeros((64, 96, 4), device="cuda")
            ctxs[0][0].render(rp, 96, 64, big, torch.zeros_like(big))
            ctxs[0][0].sync()
    b.close()
    for ctx, _, _ in ctxs:
        ctx.close()
