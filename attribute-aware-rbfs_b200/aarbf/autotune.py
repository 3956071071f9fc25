"""Launch-shape autotuner of the batched renderer.

Every knob changes only speed, never results:
  - candidate_cap: staging-buffer depth of the ray-per-warp kernel (256, 512 or 1024 candidates);
  - stage_bins: majorant bins covered by a ray's first staging (2, 4, 8, 16 or 32; later stagings adapt),
    per scene (scene_plan: each scene's 1-spp render timed with each length) or one for the whole
    batch (tune_batch);
  - blocks_per_sm: resident blocks of four warps per SM (6, 7 or the occupancy limit of 8), the
    block-level shape of the persistent launch;
  - sample_major: the ray order -- the work items of a batch run tile by tile with a tile's
    samples in sequence (rays of one 8 x 4 pixel tile together), or sample by sample over all
    tiles;
  - scene order: scenes are placed longest first (by their own timed 1-spp proxy render scaled
    by spp), so the persistent launch ends on short work instead of one long scene.
The best setting depends on the scenes (particle density along the rays, resolution, spp), so
the tuner times the batch itself with CUDA events, one knob after the other (the pair of staging
knobs jointly), and caches the result per batch signature.
"""
from __future__ import annotations

import copy

CAPS = (256, 512, 1024)
STAGE_BINS = (2, 4, 8, 16, 32)
BLOCKS_PER_SM = (6, 7, 0)
SAMPLE_MAJOR = (False, True)

_cache: dict = {}


def signature(contexts, params, sizes) -> tuple:
    return tuple((id(c), int(p.spp), int(w), int(h)) for c, p, (w, h) in zip(contexts, params, sizes))


def _events():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def scene_order(contexts, params, sizes, accums, images, stream=None):
    """indices of the scenes, longest first: each scene's 1-spp render timed on its own, times its spp"""
    import torch
    st = stream or torch.cuda.current_stream()
    cost = []
    for i, (c, p, (w, h), a, im) in enumerate(zip(contexts, params, sizes, accums, images)):
        q = copy.copy(p)
        q.spp = 1
        c.render(q, w, h, a, im, stream=st.cuda_stream)
        e0, e1 = _events()
        e0.record(st)
        c.render(q, w, h, a, im, stream=st.cuda_stream)
        e1.record(st)
        torch.cuda.synchronize()
        cost.append(e0.elapsed_time(e1) * max(int(p.spp), 1))
    return sorted(range(len(cost)), key=lambda i: -cost[i])


def scene_plan(contexts, params, sizes, accums, images, stream=None):
    """(order, stage_bins, cost): for every scene the first-staging length of STAGE_BINS whose 1-spp
    render, timed on its own, is fastest; the scene indices longest first by that time x spp; and
    the cost estimates (ms)"""
    import torch
    st = stream or torch.cuda.current_stream()
    bins_of, cost = [], []
    for c, p, (w, h), a, im in zip(contexts, params, sizes, accums, images):
        best = None
        for bins in STAGE_BINS:
            q = copy.copy(p)
            q.spp = 1
            q.stage_bins = bins
            c.render(q, w, h, a, im, stream=st.cuda_stream)  # warm-up
            e0, e1 = _events()
            e0.record(st)
            c.render(q, w, h, a, im, stream=st.cuda_stream)
            e1.record(st)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            if best is None or ms < best[0]:
                best = (ms, bins)
        bins_of.append(best[1])
        cost.append(best[0] * max(int(p.spp), 1))
    order = sorted(range(len(cost)), key=lambda i: -cost[i])
    return order, bins_of, cost


def tune_batch(contexts, params, sizes, accums, images, stream=None, reps: int = 1, stage_bins=STAGE_BINS):
    """(candidate_cap, stage_bins, {(cap, bins): ms}) of the fastest batched launch (tuned on these
    parameters; the caller usually passes 1-spp proxies of its scenes). stage_bins: the lengths
    tried for the whole batch, or None to keep each scene's own (then the returned stage_bins is
    None). The blocks-per-SM and ray-order choices are in tune_shape."""
    import torch

    from . import Batch
    key = (signature(contexts, params, sizes), stage_bins,
           tuple(int(p.stage_bins) for p in params) if stage_bins is None else None)
    if key in _cache:
        return _cache[key]
    times = {}
    st = stream or torch.cuda.current_stream()
    for bins in (stage_bins if stage_bins is not None else (None,)):
        ps = []
        for p in params:
            q = copy.copy(p)
            if bins is not None:
                q.stage_bins = bins
            ps.append(q)
        b = Batch(contexts, ps, sizes, accums, images)
        for cap in CAPS:
            b.render(cap, st)  # warm-up
            e0, e1 = _events()
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


def tune_shape(batch, candidate_cap, stream=None, reps: int = 1):
    """(blocks_per_sm, sample_major, {(blocks_per_sm, sample_major): ms}) of the fastest launch
    shape of an existing Batch; the batch is left set to it."""
    import torch
    st = stream or torch.cuda.current_stream()
    times = {}
    for bps in BLOCKS_PER_SM:
        for sm in SAMPLE_MAJOR:
            batch.set_shape(bps, sm)
            batch.render(candidate_cap, st)
            e0, e1 = _events()
            e0.record(st)
            for _ in range(reps):
                batch.render(candidate_cap, st)
            e1.record(st)
            torch.cuda.synchronize()
            times[(bps, sm)] = e0.elapsed_time(e1) / reps
    best = min(times, key=times.get)
    batch.set_shape(*best)
    return best[0], best[1], times
