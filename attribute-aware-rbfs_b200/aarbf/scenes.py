"""Seeded synthetic particle scenes and transfer functions.

* ``reference_synthetic`` -- the reference's built-in dataset (hostCode.cpp:147-168): 500 frames
  of a 10^3 grid whose scale pulses over time, attribute = y / 10.
* ``gaussian_mixture`` -- the benchmark scenes: isotropic or anisotropic Gaussian clusters
  (optionally with a uniform background), per-particle radii and attributes.

No dataset ships with the reference (no ``*.particles`` files), so every benchmark scene is one of
these generators at the sizes and value distributions of the benchmark configurations.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import (FLAG_DENSITY_LINEAR, FLAG_TRACK_FROM_ENTRY, FLAG_VISUALIZE_ATTRIBUTES,
               FLAG_SPLAT_PARTICLE_RADIUS, RenderParams)


def reference_synthetic(frames: int = 500) -> list:
    """hostCode.cpp:147-168, float32 like the reference (sin in double, as C++ sin(double))."""
    out = []
    z, y, x = np.meshgrid(np.arange(10), np.arange(10), np.arange(10), indexing="ij")
    x = x.reshape(-1).astype(np.float32)
    y = y.reshape(-1).astype(np.float32)
    z = z.reshape(-1).astype(np.float32)
    t1 = (y / np.float32(10.0)).astype(np.float32)
    for f in range(frames):
        t2 = np.float32(f) / np.float32(frames)
        s = np.float32(math.sin(float(t2) * 2.0 * 3.14) + 1.5)
        p = np.stack([s * ((x - np.float32(5)) / np.float32(10)),
                      s * ((y - np.float32(5)) / np.float32(10)),
                      s * ((z - np.float32(5)) / np.float32(10)), t1], axis=1).astype(np.float32)
        out.append(np.ascontiguousarray(p))
    return out


def _random_rotations(rng, k):
    q = rng.normal(size=(k, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1)], 1)


@dataclass
class Scene:
    xyzw: np.ndarray    # (n, 4) float32
    radii: np.ndarray   # (n,) float32 or None
    name: str


def config_small(n: int = 100_000, seed: int = 1) -> Scene:
    """100k particles: mixture of 8 isotropic Gaussians (sigma 0.08) clipped to the unit cube;
    radius 0.01; attribute = 0.5 + 0.5 sin(6x) cos(6y) sin(6z)."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.2, 0.8, size=(8, 3))
    lab = rng.integers(0, 8, size=n)
    p = centres[lab] + rng.normal(0.0, 0.08, size=(n, 3))
    p = np.clip(p, 0.0, 1.0)
    a = 0.5 + 0.5 * np.sin(6 * p[:, 0]) * np.cos(6 * p[:, 1]) * np.sin(6 * p[:, 2])
    xyzw = np.concatenate([p, a[:, None]], 1).astype(np.float32)
    return Scene(np.ascontiguousarray(xyzw), np.full(n, 0.01, np.float32), f"gauss8_iso_{n}")


def config_clusters(n: int = 10_000_000, clusters: int = 64, background: float = 0.05,
                    seed: int = 2) -> Scene:
    """n particles: 64 anisotropic Gaussian clusters (random rotation, axis sigma U[0.01, 0.1])
    plus a uniform background in [0,1]^3; radius log-uniform [0.002, 0.02]; attribute =
    cluster / 64 + N(0, 0.05) (background: U[0, 1])."""
    rng = np.random.default_rng(seed)
    nb = int(round(n * background))
    nc = n - nb
    centres = rng.uniform(0.15, 0.85, size=(clusters, 3))
    sig = rng.uniform(0.01, 0.1, size=(clusters, 3))
    rot = _random_rotations(rng, clusters)
    lab = rng.integers(0, clusters, size=nc)
    xyzw = np.empty((n, 4), np.float32)
    chunk = 1 << 22
    for s in range(0, nc, chunk):
        e = min(nc, s + chunk)
        l = lab[s:e]
        g = rng.normal(size=(e - s, 3)) * sig[l]
        g = np.einsum("nij,nj->ni", rot[l], g) + centres[l]
        xyzw[s:e, :3] = g
        xyzw[s:e, 3] = l / clusters + rng.normal(0.0, 0.05, size=e - s)
    xyzw[nc:, :3] = rng.uniform(0.0, 1.0, size=(nb, 3))
    xyzw[nc:, 3] = rng.uniform(0.0, 1.0, size=nb)
    u = rng.uniform(size=n)
    radii = np.exp(np.log(0.002) + u * (np.log(0.02) - np.log(0.002))).astype(np.float32)
    return Scene(xyzw, radii, f"gauss{clusters}_aniso_{n}")


def tf_linear_ramp(n: int = 256):
    """n-entry RGBA fp32 linear ramp (blue -> red, alpha 0 -> 1), unit radius and density maps."""
    u = np.linspace(0.0, 1.0, n, dtype=np.float32)
    cm = np.stack([u, 0.25 + 0.5 * u * (1 - u) * 2, 1 - u, u], 1).astype(np.float32)
    return cm, np.ones(n, np.float32), u.copy()


def tf_four_peaks(n: int = 256, seed: int = 3):
    """n-entry RGBA fp32 transfer function with 4 Gaussian opacity peaks."""
    rng = np.random.default_rng(seed)
    u = np.linspace(0.0, 1.0, n)
    mus = np.sort(rng.uniform(0.1, 0.9, size=4))
    amps = rng.uniform(0.5, 1.0, size=4)
    a = np.zeros(n)
    for m, s in zip(mus, amps):
        a += s * np.exp(-0.5 * ((u - m) / 0.05) ** 2)
    a = np.clip(a, 0.0, 1.0)
    cm = np.stack([np.clip(1.5 - np.abs(4 * u - 3), 0, 1), np.clip(1.5 - np.abs(4 * u - 2), 0, 1),
                   np.clip(1.5 - np.abs(4 * u - 1), 0, 1), a], 1).astype(np.float32)
    return cm, np.ones(n, np.float32), u.astype(np.float32)


def orbit_camera(center=(0.5, 0.5, 0.5), distance: float = 2.5, azimuth_deg: float = 30.0,
                 elevation_deg: float = 20.0, fov_deg: float = 60.0):
    """(look_from, look_at, look_up, scale) for an orbit camera. The reference's 10th --camera
    value is used as a plain scale of the image plane (hostCode.cpp:672-674); a vertical field of
    view of fov_deg corresponds to scale 2 tan(fov/2)."""
    az, el = math.radians(azimuth_deg), math.radians(elevation_deg)
    c = np.asarray(center, np.float64)
    f = c + distance * np.array([math.cos(el) * math.sin(az), math.sin(el), math.cos(el) * math.cos(az)])
    return (f.astype(np.float32), c.astype(np.float32), np.array([0, 1, 0], np.float32),
            float(2.0 * math.tan(math.radians(fov_deg) / 2.0)))


@dataclass
class DiffScene:
    """Particles of the differentiable form: positions (n, 3), radii (n,), attributes in [0, 1]
    (n,) and an RGBA transfer function (nc, 4), all float32."""
    pos: np.ndarray
    radii: np.ndarray
    attr: np.ndarray
    tf: np.ndarray


def config_differentiable(n: int = 1_000_000, clusters: int = 16, seed: int = 4, tf_size: int = 64):
    """(ground truth, initial guess) of the differentiable configuration: a seeded mixture of
    `clusters` anisotropic Gaussian clusters; ground-truth radii log-uniform in [0.005, 0.02],
    attribute cluster/clusters + N(0, 0.05); the initial guess has radii 0.01, positions jittered
    by U(-0.005, 0.005) per axis, attributes perturbed by N(0, 0.05) and a linear-ramp transfer
    function in place of the ground truth's four peaks."""
    rng = np.random.default_rng(seed)
    sc = config_clusters(n, clusters=clusters, background=0.0, seed=seed)
    r_gt = np.exp(rng.uniform(np.log(0.005), np.log(0.02), n)).astype(np.float32)
    attr = np.clip(sc.xyzw[:, 3], 0.0, 1.0).astype(np.float32)
    cm, _, _ = tf_four_peaks(tf_size)
    gt = DiffScene(np.ascontiguousarray(sc.xyzw[:, :3]), r_gt, attr, cm.astype(np.float32))
    pos0 = (gt.pos + rng.uniform(-0.005, 0.005, gt.pos.shape)).astype(np.float32)
    attr0 = np.clip(attr + rng.normal(0.0, 0.05, n), 0.0, 1.0).astype(np.float32)
    ramp, _, _ = tf_linear_ramp(tf_size)
    init = DiffScene(pos0, np.full(n, 0.01, np.float32), attr0, ramp.astype(np.float32))
    return gt, init


def orbit_views(count: int = 32, distance: float = 2.5, fov_deg: float = 60.0):
    """`count` orbit cameras around the unit cube's centre: azimuths evenly spread, elevations
    alternating between +20 and -20 degrees."""
    return [orbit_camera(distance=distance, azimuth_deg=360.0 * k / count,
                         elevation_deg=20.0 if k % 2 == 0 else -20.0, fov_deg=fov_deg) for k in range(count)]


def halton(index: int, base: int) -> float:
    """Radical inverse of index in base (the Halton sequence, index >= 1)."""
    f, r = 1.0, 0.0
    while index > 0:
        f /= base
        r += f * (index % base)
        index //= base
    return r


def halton_jitter(frame: int):
    """Subpixel jitter of frame k of a TAA sequence: Halton(2, 3) point k + 1, centred on the
    pixel (offsets in [-0.5, 0.5) pixels)."""
    return halton(frame + 1, 2) - 0.5, halton(frame + 1, 3) - 0.5


def native_params(cam, width: int, height: int, rbf_radius: float, unit: float, density_scale: float,
                  dom, spp: int = 1, frame_id: int = 0, traversal: int = 0, marching: bool = False,
                  majorant: bool = False, bin_length: float = None, camera_fn=None):
    """Render parameters of the benchmark configurations (native mode: per-particle radii, fp32
    transfer function). Plain form: delta tracking with the global majorant 1/unit, density
    min(density_scale * D * unit, 1) per unit step, from the volume entry. Majorant form: delta
    tracking of extinction density_scale * D with per-bin majorants (bins of bin_length, default
    4 units). camera_fn(look_from, look_at, look_up, scale, width, height) computes the camera
    basis (default: the library's aarbf_camera; any function with the same results will do)."""
    from . import camera, FLAG_BLUE_NOISE, FLAG_MAJORANT_TRACKING
    pos, d00, du, dv = (camera_fn or camera)(cam[0], cam[1], cam[2], cam[3], width, height)
    flags = FLAG_VISUALIZE_ATTRIBUTES | FLAG_DENSITY_LINEAR | FLAG_TRACK_FROM_ENTRY | FLAG_SPLAT_PARTICLE_RADIUS
    if marching:
        flags |= FLAG_BLUE_NOISE
    if majorant:
        flags |= FLAG_MAJORANT_TRACKING
    return RenderParams(cam_pos=pos, cam_dir00=d00, cam_du=du, cam_dv=dv, aabb_min=dom[0:3],
                        aabb_max=dom[3:6], rbf_radius=rbf_radius, unit=unit, accum_id=1,
                        frame_id=frame_id, spp=spp, flags=flags, light_ambient=0.5,
                        density_gain=float(np.float32(density_scale) * np.float32(unit)),
                        traversal=traversal, density_scale=float(density_scale),
                        bin_length=float(np.float32(bin_length if bin_length else 4.0 * unit)))


def config_small_params(dom, width: int = 512, height: int = 512, spp: int = 1, frame_id: int = 0,
                        camera_fn=None):
    """Render parameters of the small configuration (100k particles of config_small): delta
    tracking with the global majorant 1/unit (the reference's tracker in native mode), step unit
    0.005 (half the particle radius), density scale 50, orbit camera at distance 2.5 around the
    unit cube's centre with a 60-degree field of view, 512x512, 1 spp."""
    return native_params(orbit_camera(distance=2.5, fov_deg=60.0), width, height, 0.01, 0.005, 50.0, dom,
                         spp=spp, frame_id=frame_id, camera_fn=camera_fn)
