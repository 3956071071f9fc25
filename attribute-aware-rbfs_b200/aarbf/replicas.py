"""Multi-GPU host logic: replicas and the image-space split.

The path does not shard the scene: every GPU holds the whole particle set and BVH (a few GB at
100M particles). Two ways to use N GPUs, one process per GPU over torch.distributed:

* replicas (what bench.py runs): each rank renders its own frames; ranks draw different frame ids
  so their samples are independent; throughput is the sum, time is the max over ranks;
* image split: pixels are independent given the scene, so rank r renders the rows
  r, r + N, r + 2N, ... (interleaved rows balance the cost of dense image regions) and one
  all-gather assembles the frame (W x H x 16 B, 33 MB at 1080p).
"""
from __future__ import annotations

import numpy as np


def frame_id(rank: int, step: int, spp: int, stride: int = 7919) -> int:
    """frame id (uint16 like the reference's PushConstants.frameID) of a rank's step: consecutive
    steps of one rank advance by spp, ranks are offset by a prime stride."""
    return (step * spp + rank * stride) & 0xFFFF


def rows_of(rank: int, world: int, height: int) -> np.ndarray:
    """rows rendered by `rank` in the interleaved image split"""
    return np.arange(rank, height, world, dtype=np.int64)


def max_over_ranks(value: float, device=None) -> float:
    """max of a per-rank float (e.g. a CUDA-event time) over the default process group"""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_rows(local_rows: np.ndarray, rank: int, world: int, height: int, width: int,
                device=None) -> np.ndarray:
    """Assemble a frame from every rank's interleaved rows (local_rows: len(rows_of(...)) x W x 4).
    Ranks with fewer rows pad their contribution so the collective sees equal shapes."""
    import torch
    import torch.distributed as dist
    per = (height + world - 1) // world
    buf = np.zeros((per, width, 4), np.float32)
    buf[: len(local_rows)] = local_rows
    t = torch.from_numpy(buf).to(device) if device is not None else torch.from_numpy(buf)
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t)
    out = np.zeros((height, width, 4), np.float32)
    for r in range(world):
        rows = rows_of(r, world, height)
        out[rows] = parts[r].cpu().numpy()[: len(rows)]
    return out
