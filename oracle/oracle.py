"""ctypes binding of the oracle (TEST INFRASTRUCTURE ONLY).

The oracle is the CPU restatement of the reference's particle-volume path in
oracle/aarbf_oracle.c. Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
reference arm use it, as the checker; the product library never loads it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libaarbf_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libaarbf_ref.so")

FLAG_BLUE_NOISE = 1 << 0
FLAG_SHOW_NOISE = 1 << 1
FLAG_VISUALIZE_ATTRIBUTES = 1 << 2
FLAG_TRACK_FROM_ENTRY = 1 << 3
FLAG_DENSITY_LINEAR = 1 << 4
FLAG_SPLAT_PARTICLE_RADIUS = 1 << 5


class OrcParams(ctypes.Structure):
    _fields_ = [
        ("accum_id", ctypes.c_uint32), ("frame_id", ctypes.c_uint32), ("spp", ctypes.c_uint32),
        ("flags", ctypes.c_uint32),
        ("light_azimuth", ctypes.c_float), ("light_elevation", ctypes.c_float),
        ("light_ambient", ctypes.c_float),
        ("cam_pos", ctypes.c_float * 3), ("cam_dir00", ctypes.c_float * 3),
        ("cam_du", ctypes.c_float * 3), ("cam_dv", ctypes.c_float * 3),
        ("rbf_radius", ctypes.c_float), ("unit", ctypes.c_float),
        ("aabb_min", ctypes.c_float * 3), ("aabb_max", ctypes.c_float * 3),
        ("density_gain", ctypes.c_float), ("jitter_x", ctypes.c_float), ("jitter_y", ctypes.c_float),
        ("density_scale", ctypes.c_float), ("bin_length", ctypes.c_float),
        ("noise", ctypes.c_void_p), ("noise_w", ctypes.c_int), ("noise_h", ctypes.c_int),
    ]


class OrcTF(ctypes.Structure):
    _fields_ = [("color", ctypes.c_void_p), ("nc", ctypes.c_int), ("radius", ctypes.c_void_p),
                ("nr", ctypes.c_int), ("density", ctypes.c_void_p), ("nd", ctypes.c_int),
                ("alpha_floor", ctypes.c_float), ("storage_fp16", ctypes.c_int)]


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        P, u64, u32, f32, i32 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_float, ctypes.c_int
        sigs = {
            "orc_logf": ([f32], f32), "orc_expf": ([f32], f32), "orc_powf": ([f32, f32], f32),
            "orc_hilbert_c2i": ([ctypes.c_uint, ctypes.c_uint, P], u64),
            "orc_hilbert_i2c": ([ctypes.c_uint, ctypes.c_uint, u64, P], None),
            "orc_murmur_mix": ([u32, u32], u32), "orc_murmur_finalize": ([u32], u32),
            "orc_get_rng": ([i32, u32, u32, u32], u32),
            "orc_lcg_next": ([ctypes.POINTER(u32)], u32),
            "orc_lcg_randomf": ([ctypes.POINTER(u32)], f32),
            "orc_domain_init": ([P], None), "orc_domain_accumulate": ([P, u64, P], None),
            "orc_hilbert_keys": ([P, u64, P, P], None),
            "orc_sort_perm": ([P, P, u64, P], None),
            "orc_gather_normalize": ([P, P, P, u64, f32, f32, P, P], None),
            "orc_decode_rgba8": ([P, i32, i32, P], None),
            "orc_tex_sample": ([P, i32, i32, i32, f32], f32),
            "orc_make_8bit": ([f32], ctypes.c_uint8),
            "orc_camera": ([P, P, P, f32, i32, i32, P, P, P, P], None),
            "orc_light_dir": ([f32, f32, P], None),
            "orc_scene_create": ([P, P, P, u64, u32, f32, ctypes.POINTER(OrcTF)], P),
            "orc_scene_destroy": ([P], None),
            "orc_scene_num_leaves": ([P], u32),
            "orc_scene_get_bvh": ([P, P, P, P, P, P, P], None),
            "orc_scene_get_prepass": ([P, P, P, P], None),
            "orc_scene_get_particles": ([P, P], None),
            "orc_point_query": ([P, P, P], i32),
            "orc_point_query_brute": ([P, P, P], i32),
            "orc_render": ([P, ctypes.POINTER(OrcParams), i32, i32, P, P, i32], None),
            "orc_render_region": ([P, ctypes.POINTER(OrcParams), i32, i32, i32, i32, i32, i32, P, P, i32], None),
            "orc_render_region_gaps": ([P, ctypes.POINTER(OrcParams), i32, i32, i32, i32, i32, i32, P, P, P, i32],
                                       None),
            "orc_render_splat": ([P, ctypes.POINTER(OrcParams), i32, i32, P, i32], None),
            "orc_taa": ([P, P, P, P, i32, i32, i32], None),
            "orc_set_threads": ([i32], None),
            "orc_f2h": ([f32], ctypes.c_uint16), "orc_h2f": ([ctypes.c_uint16], f32),
            "orc_diff_forward": ([P, P, i32, i32, i32, P, i32], ctypes.c_double),
            "orc_diff_backward": ([P, P, i32, i32, i32, P, P, P, P, P, i32], None),
            "orc_render_f64": ([P, ctypes.POINTER(OrcParams), i32, i32, i32, i32, i32, i32, i32, i32, u64, P, i32],
                               None),
        }
        for k, (a, r) in sigs.items():
            f = getattr(L, k)
            f.argtypes = a
            f.restype = r
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


# ---- preprocessing -----------------------------------------------------------------------

def domain(frames):
    d = np.zeros(8, np.float32)
    lib().orc_domain_init(_p(d))
    for f in frames:
        f = np.ascontiguousarray(f, np.float32)
        lib().orc_domain_accumulate(_p(f), len(f), _p(d))
    return d


def hilbert_keys(xyzw, dom):
    xyzw = np.ascontiguousarray(xyzw, np.float32)
    k = np.zeros(len(xyzw), np.uint64)
    lib().orc_hilbert_keys(_p(xyzw), len(xyzw), _p(np.ascontiguousarray(dom, np.float32)), _p(k))
    return k


def sort_perm(keys, xyzw):
    xyzw = np.ascontiguousarray(xyzw, np.float32)
    keys = np.ascontiguousarray(keys, np.uint64)
    perm = np.zeros(len(xyzw), np.uint32)
    lib().orc_sort_perm(_p(keys), _p(xyzw), len(xyzw), _p(perm))
    return perm


def gather_normalize(xyzw, radii, perm, amin, amax):
    xyzw = np.ascontiguousarray(xyzw, np.float32)
    out = np.zeros_like(xyzw)
    rout = None
    if radii is not None:
        radii = np.ascontiguousarray(radii, np.float32)
        rout = np.zeros_like(radii)
    lib().orc_gather_normalize(_p(xyzw), _p(radii), _p(np.ascontiguousarray(perm, np.uint32)), len(xyzw),
                               float(amin), float(amax), _p(out), _p(rout))
    return out, rout


def decode_rgba8(tex, srgb=True):
    tex = np.ascontiguousarray(tex, np.uint8).reshape(-1, 4)
    out = np.zeros((len(tex), 4), np.float32)
    lib().orc_decode_rgba8(_p(tex), len(tex), int(srgb), _p(out))
    return out


def tf_from_rgba8(cm, rm, dm):
    """float tables the reference's sRGB textures decode to (colormap RGBA, radius R, density R)."""
    return decode_rgba8(cm), decode_rgba8(rm)[:, 0].copy(), decode_rgba8(dm)[:, 0].copy()


# ---- scene -------------------------------------------------------------------------------

class Scene:
    """Prepass + leaf bounds + LBVH of Hilbert-sorted particles (as aarbf_build leaves them)."""

    def __init__(self, sorted_xyzw, sorted_radii, keys, ppl, rbf_radius, tf, alpha_floor=0.0, fp16=False):
        self.xyzw = np.ascontiguousarray(sorted_xyzw, np.float32)
        self.radii = None if sorted_radii is None else np.ascontiguousarray(sorted_radii, np.float32)
        self.keys = np.ascontiguousarray(keys, np.uint64)
        cm, rm, dm = tf
        self._tf_arrays = (np.ascontiguousarray(cm, np.float32).reshape(-1, 4),
                           np.ascontiguousarray(rm, np.float32).reshape(-1),
                           np.ascontiguousarray(dm, np.float32).reshape(-1))
        c, r, d = self._tf_arrays
        t = OrcTF(c.ctypes.data, len(c), r.ctypes.data, len(r), d.ctypes.data, len(d), float(alpha_floor),
                  int(bool(fp16)))
        self.n = len(self.xyzw)
        self.h = lib().orc_scene_create(_p(self.xyzw), _p(self.radii), _p(self.keys), self.n, int(ppl),
                                        float(rbf_radius), ctypes.byref(t))
        self.nleaves = lib().orc_scene_num_leaves(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_scene_destroy(self.h)
            self.h = None

    def bvh(self):
        ni = max(self.nleaves - 1, 0)
        left = np.zeros(ni, np.uint32)
        right = np.zeros(ni, np.uint32)
        nb = np.zeros((ni, 6), np.float32)
        lb = np.zeros((self.nleaves, 6), np.float32)
        le = np.zeros((self.nleaves, 6), np.float32)
        rb = np.zeros(6, np.float32)
        lib().orc_scene_get_bvh(self.h, _p(left), _p(right), _p(nb), _p(lb), _p(le), _p(rb))
        return left, right, nb, lb, le, rb

    def particles(self):
        out = np.zeros((self.n, 4), np.float32)
        if self.n:
            lib().orc_scene_get_particles(self.h, _p(out))
        return out

    def prepass(self):
        rec0 = np.zeros((self.n, 4), np.float32)
        w4 = np.zeros((self.n, 4), np.float32)
        rg = np.zeros(self.n, np.float32)
        lib().orc_scene_get_prepass(self.h, _p(rec0), _p(w4), _p(rg))
        return rec0, w4, rg

    def point_query(self, x, brute=False):
        x = np.ascontiguousarray(x, np.float32)
        acc = np.zeros(4, np.int64)
        f = lib().orc_point_query_brute if brute else lib().orc_point_query
        c = f(self.h, _p(x), _p(acc))
        return c, acc

    def render(self, params, w, h, accum=None, threads=0, region=None, image=None):
        if accum is None:
            accum = np.zeros((h, w, 4), np.float32)
        accum = np.ascontiguousarray(accum, np.float32)
        if image is None:
            image = np.zeros((h, w, 4), np.float32)
        if region is None:
            lib().orc_render(self.h, ctypes.byref(params), w, h, _p(accum), _p(image), threads)
        else:
            x0, x1, y0, y1 = region
            lib().orc_render_region(self.h, ctypes.byref(params), w, h, x0, x1, y0, y1, _p(accum),
                                    _p(image), threads)
        return accum, image

    def render_gaps(self, params, w, h, accum=None, threads=0):
        """render() of the whole frame plus, per pixel, the smallest relative gap between the two
        sides of any random decision its samples took (see orc_render_region_gaps)."""
        accum = np.zeros((h, w, 4), np.float32) if accum is None else np.ascontiguousarray(accum, np.float32)
        image = np.zeros((h, w, 4), np.float32)
        gaps = np.full((h, w), np.inf, np.float32)
        lib().orc_render_region_gaps(self.h, ctypes.byref(params), w, h, 0, w, 0, h, _p(accum), _p(image), _p(gaps),
                                     threads)
        return accum, image, gaps

    def render_f64(self, params, w, h, region, spp, clamp_plain=False, seed=1, threads=0):
        """FP64 twin of the native volume model: mean RGB over spp samples of the region
        (x0, x1, y0, y1) of a w x h frame, shape (y1 - y0, x1 - x0, 3)."""
        x0, x1, y0, y1 = region
        out = np.zeros((y1 - y0, x1 - x0, 3), np.float32)
        lib().orc_render_f64(self.h, ctypes.byref(params), w, h, x0, x1, y0, y1, int(spp), int(bool(clamp_plain)),
                             int(seed), _p(out), threads)
        return out

    def render_splat(self, params, w, h, threads=0):
        image = np.zeros((h, w, 4), np.float32)
        lib().orc_render_splat(self.h, ctypes.byref(params), w, h, _p(image), threads)
        return image


class OrcDiffScene(ctypes.Structure):
    _fields_ = [("pos", ctypes.c_void_p), ("radius", ctypes.c_void_p), ("attr", ctypes.c_void_p),
                ("tf", ctypes.c_void_p), ("n", ctypes.c_int), ("nc", ctypes.c_int)]


def _diff_args(pos, radius, attr, tf, views):
    arrs = [np.ascontiguousarray(a, np.float64) for a in (pos, radius, attr, tf)]
    sc = OrcDiffScene(arrs[0].ctypes.data, arrs[1].ctypes.data, arrs[2].ctypes.data, arrs[3].ctypes.data,
                      len(arrs[1]), len(arrs[3]))
    vs = (OrcParams * len(views))(*views)
    return arrs, sc, vs


def diff_forward(pos, radius, attr, tf, views, w, h, threads=0):
    """FP64 differentiable model (expected stochastic marching): images (nviews, h, w, 3)."""
    arrs, sc, vs = _diff_args(pos, radius, attr, tf, views)
    out = np.zeros((len(views), h, w, 3), np.float64)
    lib().orc_diff_forward(ctypes.byref(sc), vs, len(views), w, h, _p(out), threads)
    return out


def diff_backward(pos, radius, attr, tf, views, w, h, grad_images, threads=0):
    """FP64 adjoint: (dL/dpos (n,3), dL/dradius (n), dL/dattr (n), dL/dtf (nc,4)) for dL/dimages."""
    arrs, sc, vs = _diff_args(pos, radius, attr, tf, views)
    n, nc = len(arrs[1]), len(arrs[3])
    g = np.ascontiguousarray(grad_images, np.float64)
    gp, gr, ga, gt = np.zeros((n, 3)), np.zeros(n), np.zeros(n), np.zeros((nc, 4))
    lib().orc_diff_backward(ctypes.byref(sc), vs, len(views), w, h, _p(g), _p(gp), _p(gr), _p(ga), _p(gt), threads)
    return gp, gr, ga, gt


def build_scene(xyzw, radii, dom, ppl, rbf_radius, tf, alpha_floor=0.0, fp16=False):
    """The whole build pipeline on the CPU: keys, sort, gather/normalise, scene."""
    xyzw = np.ascontiguousarray(xyzw, np.float32)
    keys = hilbert_keys(xyzw, dom)
    perm = sort_perm(keys, xyzw)
    sx, sr = gather_normalize(xyzw, radii, perm, dom[6], dom[7])
    return Scene(sx, sr, keys[perm], ppl, rbf_radius, tf, alpha_floor, fp16), keys[perm], perm


def taa(image, prev, disable=False):
    image = np.ascontiguousarray(image, np.float32)
    prev = np.ascontiguousarray(prev, np.float32)
    h, w = image.shape[:2]
    out = np.zeros_like(image)
    bgra = np.zeros((h, w), np.uint32)
    lib().orc_taa(_p(image), _p(prev), _p(out), _p(bgra), w, h, int(disable))
    return out, bgra


def camera(look_from, look_at, look_up, cos_fovy, w, h):
    out = [np.zeros(3, np.float32) for _ in range(4)]
    args = [np.ascontiguousarray(v, np.float32) for v in (look_from, look_at, look_up)]
    lib().orc_camera(*[_p(a) for a in args], float(cos_fovy), w, h, *[_p(o) for o in out])
    return tuple(out)


def params_from(rp, noise=None):
    """OrcParams from an aarbf.RenderParams-like object (same field names)."""
    p = OrcParams()
    p.accum_id, p.frame_id, p.spp, p.flags = int(rp.accum_id), int(rp.frame_id), int(rp.spp), int(rp.flags)
    p.light_azimuth, p.light_elevation, p.light_ambient = rp.light_azimuth, rp.light_elevation, rp.light_ambient
    for name in ("cam_pos", "cam_dir00", "cam_du", "cam_dv", "aabb_min", "aabb_max"):
        getattr(p, name)[:] = [float(np.float32(v)) for v in getattr(rp, name)]
    p.rbf_radius, p.unit, p.density_gain = rp.rbf_radius, rp.unit, rp.density_gain
    p.jitter_x, p.jitter_y = rp.jitter_x, rp.jitter_y
    p.density_scale = getattr(rp, "density_scale", 0.0)
    p.bin_length = getattr(rp, "bin_length", 0.0)
    if noise is not None:
        noise = np.ascontiguousarray(noise, np.uint8)
        p.noise = noise.ctypes.data
        p.noise_h, p.noise_w = noise.shape[0], noise.shape[1]
        p._noise_keepalive = noise  # p.noise points into this array: it lives as long as p
    return p
