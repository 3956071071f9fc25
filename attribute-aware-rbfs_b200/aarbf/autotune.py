"""Launch-shape autotuner of the batched renderer.

The staging-buffer depth of the ray-per-warp kernel (candidate_cap 256, 512 or 1024) and the
number of majorant bins its first staging covers (stage_bins) change only speed, never results.
The best pair depends on the scenes (particle density along the rays, resolution, spp), so the
tuner times every pair on the batch itself with CUDA events and keeps the fastest, cached per
batch signature.
"""
from __future__ import annotations

import copy

CAPS = (256, 512, 1024)
STAGE_BINS = (2, 4, 8)

_cache: dict = {}


def signature(contexts, params, sizes) -> tuple:
    return tuple((id(c), int(p.spp), int(w), int(h)) for c, p, (w, h) in zip(contexts, params, sizes))


def tune_batch(contexts, params, sizes, accums, images, stream=None, reps: int = 1):
    """(candidate_cap, stage_bins, {(cap, bins): ms}) of the fastest batched launch."""
    import torch

    from . import Batch
    key = signature(contexts, params, sizes)
    if key in _cache:
        return _cache[key]
    times = {}
    st = stream or torch.cuda.current_stream()
    for bins in STAGE_BINS:
        ps = []
        for p in params:
            q = copy.copy(p)
            q.stage_bins = bins
            ps.append(q)
        b = Batch(contexts, ps, sizes, accums, images)
        for cap in CAPS:
            b.render(cap, st)  # warm-up
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(reps):
                b.render(cap, st)
            e1.record(st)
            torch.cuda.synchronize()
            times[(cap, bins)] = e0.elapsed_time(e1) / reps
        b.close()
    best = min(times, key=times.get)
    _cache[key] = (best[0], best[1], times)
    return _cache[key]
