"""World-size-2 gloo tests (CPU) of the multi-GPU host logic: the max-over-ranks timing
reduction, distinct frame ids per replica, and the interleaved-row image split whose all-gather
must reassemble exactly the frame a single process renders (rendered here with the oracle)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _scene():
    import oracle.oracle as orc
    from aarbf import scenes
    sc = scenes.config_clusters(3000, clusters=4, seed=9)
    tf = scenes.tf_linear_ramp(64)
    dom = orc.domain([sc.xyzw])
    scene, _, _ = orc.build_scene(sc.xyzw, sc.radii, dom, 2, float(sc.radii.max()), tf)
    rp = scenes.native_params(scenes.orbit_camera(), 24, 17, float(sc.radii.max()), 0.004, 400.0, dom,
                              majorant=True, bin_length=0.016)
    return orc, scene, rp


def _worker(rank, world, port, out_dir):
    import sys
    for p in (ROOT, os.path.join(ROOT, "attribute-aware-rbfs_b200")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import torch.distributed as dist
    from aarbf import replicas
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        # timing reduction and frame ids
        m = replicas.max_over_ranks(1.5 + rank)
        fids = [replicas.frame_id(rank, s, 16) for s in range(4)]
        # interleaved-row image split
        orc, scene, rp = _scene()
        W, H = 24, 17
        p = orc.params_from(rp)
        rows = replicas.rows_of(rank, world, H)
        accum = np.zeros((H, W, 4), np.float32)
        image = np.zeros((H, W, 4), np.float32)
        for y in rows:
            scene.render(p, W, H, accum=accum, image=image, region=(0, W, int(y), int(y) + 1), threads=1)
        frame = replicas.gather_rows(image[rows], rank, world, H, W)
        np.save(os.path.join(out_dir, f"frame{rank}.npy"), frame)
        np.save(os.path.join(out_dir, f"meta{rank}.npy"), np.array([m] + fids, np.float64))
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_and_image_split(tmp_path):
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
        assert p.exitcode == 0
    orc, scene, rp = _scene()
    _, full = scene.render(orc.params_from(rp), 24, 17, threads=1)
    for r in range(world):
        frame = np.load(tmp_path / f"frame{r}.npy")
        assert np.array_equal(frame.view(np.uint32), full.view(np.uint32))
        meta = np.load(tmp_path / f"meta{r}.npy")
        assert meta[0] == 2.5
    f0 = np.load(tmp_path / "meta0.npy")[1:]
    f1 = np.load(tmp_path / "meta1.npy")[1:]
    assert len(set(f0) & set(f1)) == 0
    assert (full[..., :3] > 0).any()
