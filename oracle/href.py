"""TEST INFRASTRUCTURE ONLY: ctypes access to the reference's own device programs compiled for the
CPU (oracle/_ref/libaarbf_hlsl_ref.so, built by `make -C oracle hlsl REF=<reference tree>` from
the reference's HLSL through hlsl2cpp.py and the GPRT stand-in gprt.h).

Used by tests/golden/make_golden.py to write golden images and by the CPU tests to pin the oracle
against the reference itself where the reference tree exists. Nothing in the product loads it.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libaarbf_hlsl_ref.so")
_LIB = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _LIB
    if _LIB is None:
        from . import oracle  # the reference programs call the oracle's exp/log/pow and sampler
        oracle.lib()
        _LIB = ctypes.CDLL(LIB_PATH)
        for name in ("href_bounds", "href_rbf_render", "href_splat_render", "href_taa"):
            getattr(_LIB, name).restype = None
    return _LIB


def _p(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else ctypes.c_void_p(0)


def bounds(xyzw, ppl, rbf_radius, radiusmap):
    """GenRBFBounds (deviceCodeBounds.hlsl:29-82) over every leaf: (nleaves, 6) lo xyz, hi xyz."""
    xyzw = np.ascontiguousarray(xyzw, np.float32)
    rm = np.ascontiguousarray(radiusmap, np.float32)
    n = len(xyzw)
    nl = (n + ppl - 1) // ppl
    out = np.zeros((nl, 6), np.float32)
    lib().href_bounds(_p(xyzw), ctypes.c_uint32(n), ctypes.c_uint32(ppl), ctypes.c_float(rbf_radius), _p(rm),
                      len(rm), _p(out))
    return out


def _ip_fp(p, ppl, spp, reverse):
    """p: an aarbf.RenderParams-like object; flags decoded to PushConstants booleans"""
    blue, show, vis = (int(p.flags) >> 0) & 1, (int(p.flags) >> 1) & 1, (int(p.flags) >> 2) & 1
    ip = np.array([p.accum_id, p.frame_id, blue, show, vis, ppl, spp, int(reverse)], np.int32)
    fp = np.array([p.light_azimuth, p.light_elevation, p.light_ambient, *p.cam_pos, *p.cam_dir00, *p.cam_du,
                   *p.cam_dv, p.rbf_radius, p.unit, *p.aabb_min, *p.aabb_max], np.float32)
    return ip, fp


def render(xyzw, boxes, ppl, p, tf, w, h, accum=None, stbn=None, reverse=False, threads=0):
    """ParticleRBFRayGen (deviceCodeRBF.hlsl:206-336) for p.spp successive launches; returns
    (accum, image). tf = (colormap RGBA, radiusmap, densitymap) decoded tables; stbn: uint8 RGBA
    atlas or None."""
    xyzw = np.ascontiguousarray(xyzw, np.float32)
    boxes = np.ascontiguousarray(boxes, np.float32)
    cm, rm, dm = (np.ascontiguousarray(t, np.float32) for t in tf)
    ip, fp = _ip_fp(p, ppl, int(p.spp), reverse)
    acc = np.zeros((h, w, 4), np.float32) if accum is None else np.ascontiguousarray(accum, np.float32).copy()
    img = np.zeros((h, w, 4), np.float32)
    nf = None
    if stbn is not None:
        nf = (np.ascontiguousarray(stbn, np.uint8).astype(np.float32) / np.float32(255.0)).astype(np.float32)
    lib().href_rbf_render(_p(xyzw), ctypes.c_uint32(len(xyzw)), _p(boxes), ctypes.c_uint32(len(boxes)), _p(ip),
                          _p(fp), _p(cm), len(cm), _p(rm), len(rm), _p(dm), len(dm), _p(nf),
                          0 if nf is None else nf.shape[1], 0 if nf is None else nf.shape[0], w, h, _p(acc),
                          _p(img), threads)
    return acc, img


def render_splat(xyzw, boxes, ppl, p, tf, w, h, reverse=False, threads=0):
    """ParticleSplatRayGen (deviceCodeSplat.hlsl:58-154): the image."""
    xyzw = np.ascontiguousarray(xyzw, np.float32)
    boxes = np.ascontiguousarray(boxes, np.float32)
    cm, _, dm = (np.ascontiguousarray(t, np.float32) for t in tf)
    ip, fp = _ip_fp(p, ppl, 1, reverse)
    img = np.zeros((h, w, 4), np.float32)
    lib().href_splat_render(_p(xyzw), ctypes.c_uint32(len(xyzw)), _p(boxes), ctypes.c_uint32(len(boxes)), _p(ip),
                            _p(fp), _p(cm), len(cm), _p(dm), len(dm), w, h, _p(img), threads)
    return img


def taa(image, prev, disable=False):
    """CompositeGui (deviceCodeCommon.hlsl:67-115) with an empty GUI layer: (taa, bgra)."""
    image = np.ascontiguousarray(image, np.float32)
    prev = np.ascontiguousarray(prev, np.float32)
    h, w = image.shape[:2]
    out = np.zeros_like(image)
    bgra = np.zeros((h, w), np.uint32)
    lib().href_taa(_p(image), _p(prev), _p(out), _p(bgra), w, h, int(disable))
    return out, bgra
