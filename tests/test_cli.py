"""The headless CLI (attribute-aware-rbfs_b200/bin/aarbf), the consumer that keeps the reference's
argparse interface (hostCode.cpp:103-131): argument errors on the host, and on the GPU a saved
.particles series rendered frame by frame (build on the first frame, refit on a frame change of the
same count, rebuild on a new count) in every mode, each PFM compared with the oracle bit for bit."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "attribute-aware-rbfs_b200", "bin", "aarbf")

pytestmark = pytest.mark.skipif(not os.path.exists(CLI), reason="CLI not built (make -C attribute-aware-rbfs_b200)")


def run(*args, timeout=600):
    return subprocess.run([CLI, *map(str, args)], capture_output=True, text=True, timeout=timeout)


def test_cli_arguments():
    r = run("--help")
    assert r.returncode == 0 and "--particles" in r.stderr and "--camera" in r.stderr
    r = run("--no-such-flag")
    assert r.returncode == 1 and "unknown argument" in r.stderr
    r = run("--camera", 1, 2, 3)
    assert r.returncode == 1 and "expected 10" in r.stderr
    r = run("--particles", os.path.join(ROOT, "no", "such", "series"))
    assert r.returncode == 1 and "cannot load" in r.stderr


def read_pfm(path):
    with open(path, "rb") as f:
        assert f.readline().strip() == b"PF"
        w, h = (int(v) for v in f.readline().split())
        assert float(f.readline()) < 0  # little endian
        data = np.frombuffer(f.read(), dtype="<f4").reshape(h, w, 3)
    return data[::-1]  # rows run bottom to top


def series(tmp_path, aarbf_mod):
    """three frames: a cluster scene, the same particles moved (same count: refit), and a frame
    with fewer particles (a new count: rebuild)"""
    rng = np.random.default_rng(17)
    n = 3000
    p = np.clip(rng.normal(0.5, 0.15, (n, 3)), 0, 1)
    f0 = np.concatenate([p, rng.uniform(0, 1, (n, 1))], 1).astype(np.float32)
    f1 = f0.copy()
    f1[:, :3] += rng.normal(0.0, 0.01, (n, 3)).astype(np.float32)
    f2 = f0[: 2 * n // 3].copy()
    path = str(tmp_path / "cloud")
    aarbf_mod.save_series(path, [f0, f1, f2])
    return path, [f0, f1, f2]


def expected(orc, aarbf_mod, frames, mode, w, h, spp, taa):
    """what the CLI computes, through the oracle: space-time domain over all frames, radius 1 % of
    its diagonal, unit 0.1 radius, the startup camera, default transfer functions"""
    dom = orc.domain(frames)
    f32 = np.float32
    d = dom[3:6] - dom[0:3]
    diag = np.sqrt(f32(f32(d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]))
    radius = f32(f32(0.01) * diag)
    unit = max(f32(radius * f32(0.1)), f32(0.0001))
    cam = orc.camera(dom[3:6], (dom[3:6] + dom[0:3]) * f32(0.5), (0, -1, 0), 0.66, w, h)
    tf = orc.tf_from_rgba8(*aarbf_mod.default_transfer_functions_rgba8())
    flags = aarbf_mod.FLAG_VISUALIZE_ATTRIBUTES | (aarbf_mod.FLAG_BLUE_NOISE if mode == "march" else 0)
    atlas = aarbf_mod.generate_noise_atlas() if mode == "march" else None
    out, prev = [], np.zeros((h, w, 4), np.float32)
    for k, f in enumerate(frames):
        scene = orc.build_scene(f, None, dom, 1, float(radius), tf)[0]
        rp = aarbf_mod.RenderParams(cam_pos=cam[0], cam_dir00=cam[1], cam_du=cam[2], cam_dv=cam[3],
                                    aabb_min=dom[0:3], aabb_max=dom[3:6], rbf_radius=float(radius), unit=float(unit),
                                    accum_id=1, frame_id=k * spp, spp=spp, flags=flags, light_ambient=0.5)
        p = orc.params_from(rp, noise=atlas)
        img = scene.render_splat(p, w, h) if mode == "splat" else scene.render(p, w, h)[1]
        if taa:
            img, _ = orc.taa(img, prev)
            prev = img
        out.append(img[..., :3])
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("mode,taa,rebuild", [("track", False, False), ("track", False, True), ("march", False, False),
                                              ("splat", False, False), ("track", True, False)])
def test_cli_series_matches_oracle(tmp_path, orc, aarbf_mod, mode, taa, rebuild):
    path, frames = series(tmp_path, aarbf_mod)
    w, h, spp = 40, 30, 2
    out = str(tmp_path / "img")
    args = ["--particles", path, "--frames", 3, "--width", w, "--height", h, "--spp", spp, "--mode", mode,
            "--out", out] + (["--taa"] if taa else []) + (["--rebuild"] if rebuild else [])
    r = run(*args)
    assert r.returncode == 0, r.stderr
    want = expected(orc, aarbf_mod, frames, mode, w, h, spp, taa)
    for k in range(3):
        got = read_pfm(f"{out}_{k:04d}.pfm")
        assert (want[k] > 0).mean() > 0.01  # the view is not empty
        diff = int((got.view(np.uint32) != np.ascontiguousarray(want[k]).view(np.uint32)).sum())
        assert diff == 0, f"frame {k}: {diff} values differ from the oracle"
