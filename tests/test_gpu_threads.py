"""Launch configuration is cached per device under a lock (kernel shared-memory limits and grid
sizes): two host threads, each with its own context, render at the same time from a cold start
of a fresh process's first launches and both match the oracle bit for bit. With more than one
visible GPU the second thread uses the second device."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_two_threads_two_contexts(aarbf_mod, orc):
    import torch
    from aarbf import scenes
    ndev = torch.cuda.device_count()
    sc = scenes.config_clusters(20_000, clusters=6, seed=12)
    tf = scenes.tf_four_peaks()
    dom = orc.domain([sc.xyzw])
    w, h = 40, 30
    rmax = float(sc.radii.max())
    scene = orc.build_scene(sc.xyzw, sc.radii, dom, 4, rmax, tf, 1 / 255)[0]
    kinds = [dict(majorant=True, bin_length=0.016), dict(marching=True), dict()]
    results, errors = {}, []

    def work(slot):
        try:
            dev = slot % ndev
            ctx = aarbf_mod.Context(dev)
            try:
                ctx.set_particles(sc.xyzw, sc.radii)
                ctx.set_domain(dom)
                ctx.set_opacity_floor(1 / 255)
                ctx.set_transfer_functions_f32(*tf)
                ctx.build(rmax, 4)
                # candidate_cap 1024: the largest dynamic shared memory, which needs the per-device limit
                for j, kw in enumerate(kinds):
                    rp = scenes.native_params(scenes.orbit_camera(), w, h, rmax, 0.002, 200.0, dom, spp=2,
                                              frame_id=slot, **kw)
                    rp.candidate_cap = 1024
                    nb = w * h * 16
                    acc, img = ctx.device_alloc(nb), ctx.device_alloc(nb)
                    ctx.memset(acc, 0, nb)
                    ctx.render(rp, w, h, acc, img)
                    out = np.zeros((h, w, 4), np.float32)
                    ctx.memcpy(out, img, nb)
                    ctx.sync()
                    ctx.device_free(acc)
                    ctx.device_free(img)
                    results[(slot, j)] = (rp, out)
            finally:
                ctx.close()
        except Exception as e:  # reported by the main thread
            errors.append(repr(e))

    threads = [threading.Thread(target=work, args=(k,)) for k in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    atlas = aarbf_mod.generate_noise_atlas()
    for (slot, j), (rp, out) in results.items():
        _, want = scene.render(orc.params_from(rp, noise=atlas), w, h)
        assert np.array_equal(out.view(np.uint32), want.view(np.uint32)), (slot, j)
        assert (want[..., :3] > 0).mean() > 0.01
