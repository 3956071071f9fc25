"""Time-series playback with the upload and build of the next frame overlapped with the render
of the current one.

The reference's frame loop (hostCode.cpp:751-799) uploads a frame, regenerates the leaf bounds,
refits the acceleration structure (a rebuild only when the radius changes) and renders, one after
the other. Here two contexts alternate: while frame k renders on one stream with one context's
scene, frame k+1 is uploaded (from pinned host memory) and built or refit on a second stream into
the other context. The build synchronises its own stream on the host (tie check, root box
read-back), which does not wait for the render in flight.

update: "build" rebuilds every frame (Hilbert sort + LBVH); "refit" sorts the frame along the
curve and refits the topology of the context's first build (aarbf_refit_frame, the reference's
update path); "refit_keep_order" refits without sorting (particle i of every frame is the same
particle). All three render the same bits.
"""
from __future__ import annotations

from typing import Callable, Sequence

from . import Context, RenderParams


class SeriesRenderer:
    """Renders frames of a particle series into caller-owned framebuffers.

    dom: the space-time domain shared by every frame (aarbf_set_domain); tf: (colormap,
    radiusmap, densitymap) fp32 tables; alpha_floor, ppl and rbf_radius as for aarbf_build.
    fp16: build the scenes in the FP16 storage form."""

    def __init__(self, device: int, dom, tf, rbf_radius: float, ppl: int = 8, alpha_floor: float = 0.0,
                 fp16: bool = False, update: str = "build"):
        import torch
        self.ctx = [Context(device), Context(device)]
        for c in self.ctx:
            c.set_domain(dom)
            c.set_transfer_functions_f32(*tf)
            c.set_opacity_floor(alpha_floor)
            c.set_storage(fp16)
        if update not in ("build", "refit", "refit_keep_order"):
            raise ValueError(f"update must be build, refit or refit_keep_order, not {update!r}")
        self.update = update
        self.built = [False, False]
        self.rbf_radius, self.ppl = float(rbf_radius), int(ppl)
        dev = torch.device("cuda", device)
        self.streams = [torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)]

    def _build(self, k: int, frame):
        xyzw, radii = frame
        c, st = self.ctx[k % 2], self.streams[k % 2]
        c.set_particles(xyzw, radii, stream=st)
        if self.update == "build" or not self.built[k % 2]:
            c.build(self.rbf_radius, self.ppl, stream=st)
            self.built[k % 2] = True
        else:
            c.refit_frame(self.update == "refit_keep_order", stream=st)

    def render_series(self, frames: Sequence, params: Callable[[int], RenderParams], width: int, height: int,
                      accum, images, overlap: bool = True):
        """frames: sequence of (xyzw, radii) (pinned host tensors or device pointers);
        params(k): the render parameters of frame k; images[k]: device framebuffer of frame k
        (accum: one shared accumulation buffer). overlap=False runs the reference's order."""
        n = len(frames)
        if n == 0:
            return
        self._build(0, frames[0])
        for k in range(n):
            c, st = self.ctx[k % 2], self.streams[k % 2]
            if overlap and k + 1 < n:
                c.render(params(k), width, height, accum, images[k], stream=st)
                self._build(k + 1, frames[k + 1])  # overlaps the render in flight
            else:
                c.render(params(k), width, height, accum, images[k], stream=st)
                c.sync(st)
                if k + 1 < n:
                    self._build(k + 1, frames[k + 1])
            # the next frame's context renders only after this frame's render is done with accum
            self.streams[(k + 1) % 2].wait_stream(st)
        for c, st in zip(self.ctx, self.streams):
            c.sync(st)

    def close(self):
        for c in self.ctx:
            c.close()
