"""aarbf -- Python binding of the B200 attribute-aware Gaussian-RBF particle-volume renderer.

A thin ctypes layer over ``libaarbf.so`` (include/aarbf.h). It mirrors the reference's
host-side interface (gprt-org/attribute-aware-rbfs hostCode.cpp): upload a frame of particles
(``importParticles`` layout, float4 x/y/z/attribute), set the three transfer functions, build the
acceleration structure (replacing GenRBFBounds + gprtAccelBuild, hostCode.cpp:770-789), render
(gprtRayGenLaunch2D(ParticleRBFRayGen), hostCode.cpp:813) and resolve TAA (CompositeGui,
hostCode.cpp:822).

Device buffers are plain CUDA pointers; torch tensors are accepted wherever a device pointer is
(``tensor.data_ptr()``). The library must be built (``make -C attribute-aware-rbfs_b200``);
importing this module on a machine without the library raises immediately -- there is no CPU
fallback.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libaarbf.so")

FLAG_BLUE_NOISE = 1 << 0
FLAG_SHOW_NOISE = 1 << 1
FLAG_VISUALIZE_ATTRIBUTES = 1 << 2
FLAG_TRACK_FROM_ENTRY = 1 << 3
FLAG_DENSITY_LINEAR = 1 << 4
FLAG_SPLAT_PARTICLE_RADIUS = 1 << 5
FLAG_MAJORANT_TRACKING = 1 << 6

TRAVERSAL_AUTO = 0      # one warp per ray (warp-wide traversal, staged candidate lists) for every estimator
TRAVERSAL_STAGED = 0    # the same (staged candidates; kept name)
TRAVERSAL_POINT = 1     # one BVH point query per tracking step, one thread per sample
TRAVERSAL_THREAD = 2    # per-thread staged segments for every estimator

STORAGE_FP32 = 0
STORAGE_FP16 = 1        # FP16 positions (relative to 256-particle run origins), attributes, weights


def uses_warp_kernel(p) -> bool:
    """True when a render with these parameters runs a ray-per-warp kernel: every estimator (the
    reference's delta tracking, delta tracking with per-bin majorants, stochastic marching) with
    the default traversal."""
    return int(p.traversal) == TRAVERSAL_AUTO

STATUS = {
    0: "ok", 1: "invalid argument", 2: "out of memory", 3: "CUDA error",
    4: "device-side limit exceeded", 5: "not ready", 6: "I/O error", 7: "unsupported",
}

#: every symbol include/aarbf.h declares
EXPORTED_SYMBOLS = (
    "aarbf_create", "aarbf_destroy", "aarbf_last_error", "aarbf_status_string", "aarbf_get_version",
    "aarbf_sync", "aarbf_set_particles", "aarbf_set_domain", "aarbf_domain_init",
    "aarbf_domain_accumulate", "aarbf_set_transfer_functions_rgba8",
    "aarbf_set_transfer_functions_f32", "aarbf_marks_to_rgba8", "aarbf_build", "aarbf_refit",
    "aarbf_refit_frame", "aarbf_render", "aarbf_render_splat", "aarbf_taa_resolve", "aarbf_get_framebuffers",
    "aarbf_set_noise_atlas", "aarbf_generate_noise_atlas", "aarbf_camera", "aarbf_series_load",
    "aarbf_series_num_frames", "aarbf_series_frame", "aarbf_series_free", "aarbf_series_save",
    "aarbf_get_num_particles", "aarbf_get_hilbert_keys", "aarbf_get_sorted_particles",
    "aarbf_get_prepass", "aarbf_get_bvh", "aarbf_device_alloc", "aarbf_device_free",
    "aarbf_memcpy", "aarbf_memset", "aarbf_render_count", "aarbf_set_opacity_floor",
    "aarbf_hilbert_sort_noalloc", "aarbf_set_kernel_timing", "aarbf_get_kernel_times",
    "aarbf_render_diff_forward", "aarbf_render_diff_backward", "aarbf_batch_create", "aarbf_batch_render",
    "aarbf_batch_destroy", "aarbf_batch_last_error", "aarbf_set_storage", "aarbf_batch_set_shape",
)


class AarbfError(RuntimeError):
    def __init__(self, status: int, msg: str = ""):
        super().__init__(f"aarbf: {STATUS.get(status, status)}" + (f": {msg}" if msg else ""))
        self.status = status


class Params(ctypes.Structure):
    """aarbf_params (include/aarbf.h) == PushConstants + RayGenData of sharedCode.h:33-117."""

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
        ("traversal", ctypes.c_int32), ("density_scale", ctypes.c_float), ("bin_length", ctypes.c_float),
        ("candidate_cap", ctypes.c_int32), ("stage_bins", ctypes.c_int32), ("loop_cap", ctypes.c_uint32),
    ]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libaarbf.so not built at {LIB_PATH} (run make -C attribute-aware-rbfs_b200)")
    lib = ctypes.CDLL(LIB_PATH)
    P = ctypes.c_void_p
    u64, u32, i32, f32 = ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int, ctypes.c_float
    sig = {
        "aarbf_create": [ctypes.POINTER(P), i32],
        "aarbf_destroy": [P],
        "aarbf_sync": [P, P],
        "aarbf_set_particles": [P, P, u64, P, P],
        "aarbf_set_domain": [P, P],
        "aarbf_domain_init": [P],
        "aarbf_domain_accumulate": [P, P, u64, P, P],
        "aarbf_set_transfer_functions_rgba8": [P, P, i32, P, i32, P, i32],
        "aarbf_set_transfer_functions_f32": [P, P, i32, P, i32, P, i32],
        "aarbf_marks_to_rgba8": [P, P, i32, i32, P, i32],
        "aarbf_build": [P, f32, u32, P],
        "aarbf_refit": [P, f32, P],
        "aarbf_refit_frame": [P, i32, P],
        "aarbf_render": [P, ctypes.POINTER(Params), i32, i32, P, P, P],
        "aarbf_render_splat": [P, ctypes.POINTER(Params), i32, i32, P, P],
        "aarbf_taa_resolve": [P, P, P, P, P, i32, i32, i32, P],
        "aarbf_get_framebuffers": [P, i32, i32, ctypes.POINTER(P), ctypes.POINTER(P)],
        "aarbf_set_noise_atlas": [P, P, i32, i32],
        "aarbf_generate_noise_atlas": [P, i32, i32],
        "aarbf_camera": [P, P, P, f32, i32, i32, P, P, P, P],
        "aarbf_series_load": [ctypes.c_char_p, ctypes.POINTER(P)],
        "aarbf_series_num_frames": [P, ctypes.POINTER(u64)],
        "aarbf_series_frame": [P, u64, ctypes.POINTER(P), ctypes.POINTER(u64)],
        "aarbf_series_free": [P],
        "aarbf_series_save": [ctypes.c_char_p, P, P, u64],
        "aarbf_get_num_particles": [P, ctypes.POINTER(u64), ctypes.POINTER(u32)],
        "aarbf_get_hilbert_keys": [P, P, P],
        "aarbf_get_sorted_particles": [P, P],
        "aarbf_get_prepass": [P, P, P, P],
        "aarbf_get_bvh": [P, P, P, P, P, P, P],
        "aarbf_set_opacity_floor": [P, f32],
        "aarbf_hilbert_sort_noalloc": [P, u64, P, P, P, P],
        "aarbf_get_version": [ctypes.POINTER(i32), ctypes.POINTER(i32)],
        "aarbf_device_alloc": [P, ctypes.c_size_t, ctypes.POINTER(P)],
        "aarbf_device_free": [P, P],
        "aarbf_memcpy": [P, P, P, ctypes.c_size_t, P],
        "aarbf_memset": [P, P, i32, ctypes.c_size_t, P],
        "aarbf_render_count": [P, ctypes.POINTER(Params), i32, i32, P, P, P, P],
        "aarbf_set_kernel_timing": [P, i32],
        "aarbf_set_storage": [P, i32],
        "aarbf_batch_create": [ctypes.POINTER(P), P, ctypes.POINTER(Params), i32, P, P, P, P],
        "aarbf_batch_render": [P, i32, P],
        "aarbf_batch_set_shape": [P, i32, i32],
        "aarbf_batch_destroy": [P],
        "aarbf_render_diff_forward": [P, ctypes.POINTER(Params), i32, i32, i32, P, P],
        "aarbf_render_diff_backward": [P, ctypes.POINTER(Params), i32, i32, i32, P, P, P, P, P, P],
        "aarbf_get_kernel_times": [P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(u32)],
    }
    for name, args in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int
    lib.aarbf_last_error.argtypes = [P]
    lib.aarbf_last_error.restype = ctypes.c_char_p
    lib.aarbf_batch_last_error.argtypes = [P]
    lib.aarbf_batch_last_error.restype = ctypes.c_char_p
    lib.aarbf_status_string.argtypes = [ctypes.c_int]
    lib.aarbf_status_string.restype = ctypes.c_char_p
    return lib


_lib = None


def lib():
    """The loaded libaarbf.so (raises ImportError when it was not built)."""
    global _lib
    if _lib is None:
        _lib = _load()
    return _lib


def _ptr(a) -> Optional[int]:
    """Device or host address of a torch tensor / numpy array / int (None passes through)."""
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("array must be C-contiguous")
        return a.ctypes.data
    raise TypeError(f"cannot take the address of {type(a)}")


def _stream_ptr(stream) -> Optional[int]:
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream  # torch.cuda.Stream


def marks_to_rgba8(pos: Sequence[float], rgba: Sequence[Sequence[float]], gamma: bool,
                   ntexels: int = 64) -> np.ndarray:
    """Gradient marks -> RGBA8 texture as hostCode.cpp:528-572 uploads it."""
    p = np.ascontiguousarray(pos, np.float32)
    c = np.ascontiguousarray(rgba, np.float32).reshape(-1, 4)
    out = np.zeros((ntexels, 4), np.uint8)
    st = lib().aarbf_marks_to_rgba8(_ptr(p), _ptr(c), len(p), int(bool(gamma)), _ptr(out), ntexels)
    if st:
        raise AarbfError(st)
    return out


def default_transfer_functions_rgba8():
    """The reference's startup transfer functions (hostCode.cpp:416-436) as 64-texel RGBA8."""
    cm = marks_to_rgba8([0.0, 0.25, 0.5, 0.75, 1.0],
                        [[0, 0, 1, 1], [0, 0.972549, 1, 1], [0, 1, 0.00784314, 1],
                         [0.996078, 1, 0, 1], [1, 0, 0, 1]], gamma=True)
    rm = marks_to_rgba8([0.0, 1.0], [[1, 1, 1, 1], [1, 1, 1, 1]], gamma=False)
    dm = marks_to_rgba8([0.0, 1.0], [[0, 0, 0, 0], [1, 1, 1, 1]], gamma=False)
    return cm, rm, dm


def camera(look_from, look_at, look_up, cos_fovy: float, width: int, height: int):
    """Camera basis (pos, dir00, du, dv) of hostCode.cpp:669-676."""
    f = np.ascontiguousarray(look_from, np.float32)
    a = np.ascontiguousarray(look_at, np.float32)
    u = np.ascontiguousarray(look_up, np.float32)
    out = [np.zeros(3, np.float32) for _ in range(4)]
    st = lib().aarbf_camera(_ptr(f), _ptr(a), _ptr(u), float(cos_fovy), int(width), int(height),
                            *[_ptr(o) for o in out])
    if st:
        raise AarbfError(st)
    return tuple(out)


def generate_noise_atlas(width: int = 2048, height: int = 4096) -> np.ndarray:
    out = np.zeros((height, width, 4), np.uint8)
    st = lib().aarbf_generate_noise_atlas(_ptr(out), width, height)
    if st:
        raise AarbfError(st)
    return out


#: largest particle count aarbf_hilbert_sort_noalloc accepts (include/aarbf.h)
NOALLOC_MAX_PARTICLES = 1 << 20


def hilbert_sort_noalloc(xyzw_dev: int, n: int, dom, keys_dev: int, perm_dev: int, stream=None):
    """aarbf_hilbert_sort_noalloc: Hilbert keys and sort permutation of n device-resident
    particles into caller-provided device outputs, without allocating device memory."""
    d = np.ascontiguousarray(dom, np.float32)
    st = lib().aarbf_hilbert_sort_noalloc(_ptr(xyzw_dev), int(n), _ptr(d), _ptr(keys_dev), _ptr(perm_dev),
                                          _stream_ptr(stream))
    if st:
        raise AarbfError(st, "aarbf_hilbert_sort_noalloc")


def domain_init() -> np.ndarray:
    d = np.zeros(8, np.float32)
    lib().aarbf_domain_init(_ptr(d))
    return d


@dataclass
class RenderParams:
    """Per-launch parameters (aarbf_params)."""

    cam_pos: Sequence[float] = (0.0, 0.0, 0.0)
    cam_dir00: Sequence[float] = (0.0, 0.0, 1.0)
    cam_du: Sequence[float] = (1.0, 0.0, 0.0)
    cam_dv: Sequence[float] = (0.0, 1.0, 0.0)
    aabb_min: Sequence[float] = (0.0, 0.0, 0.0)
    aabb_max: Sequence[float] = (1.0, 1.0, 1.0)
    rbf_radius: float = 0.01
    unit: float = 0.001
    accum_id: int = 1
    frame_id: int = 0
    spp: int = 1
    flags: int = FLAG_VISUALIZE_ATTRIBUTES
    light_azimuth: float = 0.0
    light_elevation: float = 0.0
    light_ambient: float = 0.5
    density_gain: float = 1.0
    jitter_x: float = 0.0
    jitter_y: float = 0.0
    traversal: int = TRAVERSAL_STAGED
    density_scale: float = 0.0
    bin_length: float = 0.0
    candidate_cap: int = 0
    stage_bins: int = 0
    loop_cap: int = 0  # 0: built-in device loop bounds; > 0 lowers them (exercises AARBF_ERR_DEVICE_LIMIT)

    def to_c(self) -> Params:
        p = Params()
        p.accum_id, p.frame_id, p.spp, p.flags = (int(self.accum_id), int(self.frame_id),
                                                   int(self.spp), int(self.flags))
        p.light_azimuth, p.light_elevation, p.light_ambient = (
            self.light_azimuth, self.light_elevation, self.light_ambient)
        for name in ("cam_pos", "cam_dir00", "cam_du", "cam_dv", "aabb_min", "aabb_max"):
            getattr(p, name)[:] = [float(np.float32(v)) for v in getattr(self, name)]
        p.rbf_radius, p.unit = self.rbf_radius, self.unit
        p.density_gain, p.jitter_x, p.jitter_y = self.density_gain, self.jitter_x, self.jitter_y
        p.traversal = int(self.traversal)
        p.density_scale, p.bin_length = self.density_scale, self.bin_length
        p.candidate_cap = int(self.candidate_cap)
        p.stage_bins = int(self.stage_bins)
        p.loop_cap = int(self.loop_cap)
        return p


class Context:
    """One device context (include/aarbf.h aarbf_ctx); not thread safe, like the reference's."""

    def __init__(self, device: int = 0):
        self._lib = lib()
        h = ctypes.c_void_p()
        st = self._lib.aarbf_create(ctypes.byref(h), int(device))
        if st:
            raise AarbfError(st, f"aarbf_create(device={device})")
        self._h = h

    # -- plumbing ------------------------------------------------------------------------
    def _check(self, st: int):
        if st:
            raise AarbfError(st, self._lib.aarbf_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            self._lib.aarbf_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def sync(self, stream=None):
        self._check(self._lib.aarbf_sync(self._h, _stream_ptr(stream)))

    # -- scene ---------------------------------------------------------------------------
    def set_particles(self, xyzw, radii=None, n: Optional[int] = None, stream=None):
        """xyzw: float32 (n, 4) numpy array or device tensor; radii: optional (n,) float32."""
        if n is None:
            n = int(xyzw.shape[0])
        self._keep = (xyzw, radii)
        self._check(self._lib.aarbf_set_particles(self._h, _ptr(xyzw), int(n), _ptr(radii),
                                                  _stream_ptr(stream)))

    def set_domain(self, dom):
        d = np.ascontiguousarray(dom, np.float32)
        self._check(self._lib.aarbf_set_domain(self._h, _ptr(d)))

    def domain_accumulate(self, xyzw, dom: np.ndarray, n: Optional[int] = None, stream=None):
        if n is None:
            n = int(xyzw.shape[0])
        self._check(self._lib.aarbf_domain_accumulate(self._h, _ptr(xyzw), int(n), _ptr(dom),
                                                      _stream_ptr(stream)))
        return dom

    def set_transfer_functions_rgba8(self, colormap, radiusmap, densitymap):
        c = np.ascontiguousarray(colormap, np.uint8).reshape(-1, 4)
        r = np.ascontiguousarray(radiusmap, np.uint8).reshape(-1, 4)
        d = np.ascontiguousarray(densitymap, np.uint8).reshape(-1, 4)
        self._check(self._lib.aarbf_set_transfer_functions_rgba8(
            self._h, _ptr(c), len(c), _ptr(r), len(r), _ptr(d), len(d)))

    def set_transfer_functions_f32(self, colormap, radiusmap, densitymap):
        c = np.ascontiguousarray(colormap, np.float32).reshape(-1, 4)
        r = np.ascontiguousarray(radiusmap, np.float32).reshape(-1)
        d = np.ascontiguousarray(densitymap, np.float32).reshape(-1)
        self._check(self._lib.aarbf_set_transfer_functions_f32(
            self._h, _ptr(c), len(c), _ptr(r), len(r), _ptr(d), len(d)))

    def set_noise_atlas(self, rgba8: Optional[np.ndarray] = None):
        if rgba8 is None:
            self._check(self._lib.aarbf_set_noise_atlas(self._h, None, 0, 0))
        else:
            a = np.ascontiguousarray(rgba8, np.uint8)
            self._check(self._lib.aarbf_set_noise_atlas(self._h, _ptr(a), a.shape[1], a.shape[0]))

    def build(self, rbf_radius: float, particles_per_leaf: int = 1, stream=None):
        self._check(self._lib.aarbf_build(self._h, float(rbf_radius), int(particles_per_leaf),
                                          _stream_ptr(stream)))

    def refit(self, rbf_radius: float, stream=None):
        self._check(self._lib.aarbf_refit(self._h, float(rbf_radius), _stream_ptr(stream)))

    def refit_frame(self, keep_order: bool = False, stream=None):
        """aarbf_refit_frame: the frame set by set_particles refits the last build's BVH topology
        (the reference's update on a frame change)."""
        self._check(self._lib.aarbf_refit_frame(self._h, int(bool(keep_order)), _stream_ptr(stream)))

    # -- launches ------------------------------------------------------------------------
    def render(self, params: RenderParams, width: int, height: int, accum=None, image=None,
               stream=None):
        p = params.to_c() if isinstance(params, RenderParams) else params
        self._check(self._lib.aarbf_render(self._h, ctypes.byref(p), int(width), int(height),
                                           _ptr(accum), _ptr(image), _stream_ptr(stream)))

    def render_count(self, params: RenderParams, width: int, height: int, accum=None, image=None,
                     stream=None):
        """render + accounting: dict of the AARBF_COUNT_SLOTS counters (include/aarbf.h)"""
        p = params.to_c() if isinstance(params, RenderParams) else params
        c = np.zeros(10, np.uint64)
        self._check(self._lib.aarbf_render_count(self._h, ctypes.byref(p), int(width), int(height),
                                                 _ptr(accum), _ptr(image), _ptr(c), _stream_ptr(stream)))
        if uses_warp_kernel(p):
            names = ("segment_particles", "segment_nodes", "steps", "stagings", "staging_overflows",
                     "direct_bin_sums", "candidates_staged", "bins", "traversal_iterations",
                     "particles_tested")
        else:
            names = ("segment_particles", "segment_nodes", "steps", "stagings", "staging_overflows",
                     "point_queries", "candidate_checks", "particle_evals", "staging_nodes", "point_nodes")
        return {k: int(v) for k, v in zip(names, c)}

    @staticmethod
    def _views(views):
        vs = [v.to_c() if isinstance(v, RenderParams) else v for v in views]
        return (Params * len(vs))(*vs), len(vs)

    def render_diff_forward(self, views, width: int, height: int, images, stream=None):
        """Differentiable form, forward: images (device float32, nviews x height x width x 4)."""
        arr, nv = self._views(views)
        self._check(self._lib.aarbf_render_diff_forward(self._h, arr, nv, int(width), int(height), _ptr(images),
                                                        _stream_ptr(stream)))

    def render_diff_backward(self, views, width: int, height: int, grad_images, grad_xyz, grad_radius, grad_attr,
                             grad_tf, stream=None):
        """Adjoint of the last render_diff_forward: gradients in the caller's particle order."""
        arr, nv = self._views(views)
        self._check(self._lib.aarbf_render_diff_backward(self._h, arr, nv, int(width), int(height),
                                                         _ptr(grad_images), _ptr(grad_xyz), _ptr(grad_radius),
                                                         _ptr(grad_attr), _ptr(grad_tf), _stream_ptr(stream)))

    def set_kernel_timing(self, enable: bool = True):
        """Record CUDA events around the kernels of every render (include/aarbf.h)."""
        self._check(self._lib.aarbf_set_kernel_timing(self._h, int(bool(enable))))

    def kernel_times(self):
        """(tracking-kernel ms, accumulation-pass ms, renders) summed since the last call."""
        r, a, k = ctypes.c_double(), ctypes.c_double(), ctypes.c_uint32()
        self._check(self._lib.aarbf_get_kernel_times(self._h, ctypes.byref(r), ctypes.byref(a),
                                                     ctypes.byref(k)))
        return r.value, a.value, k.value

    def render_splat(self, params: RenderParams, width: int, height: int, image=None, stream=None):
        p = params.to_c() if isinstance(params, RenderParams) else params
        self._check(self._lib.aarbf_render_splat(self._h, ctypes.byref(p), int(width), int(height),
                                                 _ptr(image), _stream_ptr(stream)))

    def taa_resolve(self, image, prev, taa, bgra=None, width: int = 0, height: int = 0,
                    disable: bool = False, stream=None):
        self._check(self._lib.aarbf_taa_resolve(self._h, _ptr(image), _ptr(prev), _ptr(taa),
                                                _ptr(bgra), int(width), int(height), int(disable),
                                                _stream_ptr(stream)))

    def device_alloc(self, nbytes: int) -> int:
        p = ctypes.c_void_p()
        self._check(self._lib.aarbf_device_alloc(self._h, int(nbytes), ctypes.byref(p)))
        return p.value

    def device_free(self, ptr: int):
        self._check(self._lib.aarbf_device_free(self._h, ptr))

    def memcpy(self, dst, src, nbytes: int, stream=None):
        self._check(self._lib.aarbf_memcpy(self._h, _ptr(dst), _ptr(src), int(nbytes), _stream_ptr(stream)))

    def memset(self, dst, value: int, nbytes: int, stream=None):
        self._check(self._lib.aarbf_memset(self._h, _ptr(dst), int(value), int(nbytes), _stream_ptr(stream)))

    def framebuffers(self, width: int, height: int):
        a, i = ctypes.c_void_p(), ctypes.c_void_p()
        self._check(self._lib.aarbf_get_framebuffers(self._h, width, height, ctypes.byref(a),
                                                     ctypes.byref(i)))
        return a.value, i.value

    # -- debug getters -------------------------------------------------------------------
    def counts(self):
        n, nl = ctypes.c_uint64(), ctypes.c_uint32()
        self._check(self._lib.aarbf_get_num_particles(self._h, ctypes.byref(n), ctypes.byref(nl)))
        return n.value, nl.value

    def hilbert_keys(self):
        n, _ = self.counts()
        k = np.zeros(n, np.uint64)
        p = np.zeros(n, np.uint32)
        self._check(self._lib.aarbf_get_hilbert_keys(self._h, _ptr(k), _ptr(p)))
        return k, p

    def sorted_particles(self):
        n, _ = self.counts()
        out = np.zeros((n, 4), np.float32)
        self._check(self._lib.aarbf_get_sorted_particles(self._h, _ptr(out)))
        return out

    def prepass(self):
        n, _ = self.counts()
        rec0 = np.zeros((n, 4), np.float32)
        w4 = np.zeros((n, 4), np.float32)
        rg = np.zeros(n, np.float32)
        self._check(self._lib.aarbf_get_prepass(self._h, _ptr(rec0), _ptr(w4), _ptr(rg)))
        return rec0, w4, rg

    def bvh(self):
        _, nl = self.counts()
        ni = max(nl - 1, 0)
        left = np.zeros(ni, np.uint32)
        right = np.zeros(ni, np.uint32)
        nb = np.zeros((ni, 6), np.float32)
        lb = np.zeros((nl, 6), np.float32)
        le = np.zeros((nl, 6), np.float32)
        rb = np.zeros(6, np.float32)
        self._check(self._lib.aarbf_get_bvh(self._h, _ptr(left), _ptr(right), _ptr(nb), _ptr(lb),
                                            _ptr(le), _ptr(rb)))
        return left, right, nb, lb, le, rb

    def set_storage(self, fp16: bool):
        """FP16 storage form of the scene the next build makes (aarbf_set_storage)."""
        self._check(self._lib.aarbf_set_storage(self._h, STORAGE_FP16 if fp16 else STORAGE_FP32))

    def set_opacity_floor(self, alpha_floor: float):
        self._check(self._lib.aarbf_set_opacity_floor(self._h, float(alpha_floor)))


def load_series(path: str):
    """importParticles (importParticles.h:8-31): list of float32 (n, 4) frames."""
    L = lib()
    h = ctypes.c_void_p()
    st = L.aarbf_series_load(path.encode(), ctypes.byref(h))
    if st:
        raise AarbfError(st, path)
    try:
        nf = ctypes.c_uint64()
        L.aarbf_series_num_frames(h, ctypes.byref(nf))
        frames = []
        for k in range(nf.value):
            p, n = ctypes.c_void_p(), ctypes.c_uint64()
            L.aarbf_series_frame(h, k, ctypes.byref(p), ctypes.byref(n))
            if n.value:
                buf = (ctypes.c_float * (4 * n.value)).from_address(p.value)
                frames.append(np.frombuffer(buf, np.float32).reshape(-1, 4).copy())
            else:
                frames.append(np.zeros((0, 4), np.float32))
        return frames
    finally:
        L.aarbf_series_free(h)


def save_series(path: str, frames):
    L = lib()
    arrs = [np.ascontiguousarray(f, np.float32).reshape(-1, 4) for f in frames]
    ptrs = (ctypes.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
    counts = (ctypes.c_uint64 * len(arrs))(*[len(a) for a in arrs])
    st = L.aarbf_series_save(path.encode(), ptrs, counts, len(arrs))
    if st:
        raise AarbfError(st, path)


class Batch:
    """Several scenes rendered by one persistent launch (aarbf_batch_create / aarbf_batch_render).

    contexts: built Contexts on one device; params: one RenderParams per scene (majorant
    tracking); sizes: (width, height) per scene; accums / images: per-scene device framebuffers
    (float32 H x W x 4). render() only enqueues kernels: it can be captured in a CUDA graph."""

    def __init__(self, contexts, params, sizes, accums, images):
        self._lib = lib()
        n = len(contexts)
        P = ctypes.c_void_p
        hs = (P * n)(*[c._h for c in contexts])
        ps = (Params * n)(*[p.to_c() if isinstance(p, RenderParams) else p for p in params])
        ws = (ctypes.c_int * n)(*[int(w) for w, _ in sizes])
        hh = (ctypes.c_int * n)(*[int(h) for _, h in sizes])
        ac = (P * n)(*[_ptr(a) for a in accums])
        im = (P * n)(*[_ptr(a) for a in images])
        self._keep = (contexts, accums, images)
        self._h = P()
        st = self._lib.aarbf_batch_create(ctypes.byref(self._h), hs, ps, n, ws, hh, ac, im)
        if st != 0:
            msg = self._lib.aarbf_last_error(contexts[0]._h).decode()
            raise AarbfError(st, msg)

    def render(self, candidate_cap: int = 0, stream=None):
        st = self._lib.aarbf_batch_render(self._h, int(candidate_cap), _stream_ptr(stream))
        if st != 0:
            raise AarbfError(st, self._lib.aarbf_batch_last_error(self._h).decode())

    def set_shape(self, blocks_per_sm: int = 0, sample_major: bool = False):
        """aarbf_batch_set_shape: resident blocks per SM (0 = occupancy limit) and work-item order."""
        st = self._lib.aarbf_batch_set_shape(self._h, int(blocks_per_sm), int(bool(sample_major)))
        if st != 0:
            raise AarbfError(st, self._lib.aarbf_batch_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            self._lib.aarbf_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
