"""CPU-side checks of the product library: it loads, exports every entry point include/aarbf.h
declares, and its host logic (camera, transfer-function marks, importParticles-format I/O, noise
atlas, argument errors) behaves as the reference's host code does. No kernels run here."""
import os
import re
import struct

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    src = open(os.path.join(ROOT, "include", "aarbf.h")).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\**\s*(aarbf_[a-z_0-9]+)\s*\(", src, re.M)))


def test_library_exports_every_declared_symbol(aarbf_mod):
    L = aarbf_mod.lib()
    syms = header_symbols()
    assert len(syms) >= 30
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing
    assert set(syms) == set(aarbf_mod.EXPORTED_SYMBOLS)


def test_version_and_status_strings(aarbf_mod):
    import ctypes
    L = aarbf_mod.lib()
    a, b = ctypes.c_int(), ctypes.c_int()
    assert L.aarbf_get_version(ctypes.byref(a), ctypes.byref(b)) == 0
    assert (a.value, b.value) == (0, 1)
    assert L.aarbf_status_string(4) == b"device-side limit exceeded"


def test_create_without_gpu_fails_cleanly(aarbf_mod):
    from conftest import gpu_available
    if gpu_available():
        pytest.skip("a GPU is present")
    with pytest.raises(aarbf_mod.AarbfError):
        aarbf_mod.Context(0)


def test_camera_matches_oracle(aarbf_mod, orc):
    rng = np.random.default_rng(0)
    for _ in range(200):
        f, a = rng.normal(size=3) * 3, rng.normal(size=3)
        up = rng.normal(size=3)
        s = float(np.float32(rng.uniform(0.2, 2.0)))
        w, h = int(rng.integers(16, 2000)), int(rng.integers(16, 2000))
        got = aarbf_mod.camera(f, a, up, s, w, h)
        want = orc.camera(f, a, up, s, w, h)
        for g, e in zip(got, want):
            assert np.array_equal(g.view(np.uint32), e.view(np.uint32))


def test_default_transfer_functions(aarbf_mod, orc):
    cm, rm, dm = aarbf_mod.default_transfer_functions_rgba8()
    # hostCode.cpp:428-436: radius map constant 1 -> make_8bit(1) = 255; density ramp 0 -> 1
    assert (rm[:, 0] == 255).all()
    assert dm[0, 0] == 0 and dm[-1, 0] == 255
    assert all(int(dm[i, 0]) == orc.lib().orc_make_8bit(np.float32(i / 63.0)) for i in range(64))
    # colormap: first mark pure blue, last pure red, alpha 1 everywhere
    assert list(cm[0]) == [0, 0, 255, 255] and list(cm[-1]) == [255, 0, 0, 255]
    assert (cm[:, 3] == 255).all()
    # sRGB decode of the 255 radius texel is exactly 1 (so r = rbfRadius, hostCode.cpp:350-351)
    c, r, d = orc.tf_from_rgba8(cm, rm, dm)
    assert (r == 1.0).all() and d[0] == 0.0 and d[-1] == 1.0


def test_series_roundtrip_and_errors(aarbf_mod, tmp_path):
    rng = np.random.default_rng(1)
    frames = [rng.normal(size=(n, 4)).astype(np.float32) for n in (5, 0, 17)]
    path = str(tmp_path / "test.particles")
    aarbf_mod.save_series(path, frames)
    got = aarbf_mod.load_series(path)
    assert len(got) == 3
    for a, b in zip(frames, got):
        assert np.array_equal(a, b)
    # byte layout of importParticles.h:14-29: u64 count then float4s
    raw = open(path + "_2", "rb").read()
    assert struct.unpack("<Q", raw[:8])[0] == 17 and len(raw) == 8 + 17 * 16
    # truncated file: count larger than the data present
    with open(path + "_2", "wb") as f:
        f.write(struct.pack("<Q", 100) + b"\0" * 64)
    with pytest.raises(aarbf_mod.AarbfError):
        aarbf_mod.load_series(path)
    # missing timestep file
    os.remove(path + "_1")
    with pytest.raises(aarbf_mod.AarbfError):
        aarbf_mod.load_series(path)
    with pytest.raises(aarbf_mod.AarbfError):
        aarbf_mod.load_series(str(tmp_path / "nope.particles"))


def test_noise_atlas_layout(aarbf_mod):
    a = aarbf_mod.generate_noise_atlas(2048, 4096)
    assert a.shape == (4096, 2048, 4) and (a[..., 3] == 255).all()
    # each 256x256 tile is close to uniform over [0, 255]
    t = a[:256, :256, 0].astype(np.float64)
    assert abs(t.mean() - 127.5) < 3 and abs(np.histogram(t, 8, (0, 256))[0] - 8192).max() < 400


def test_reference_synthetic_dataset():
    from aarbf import scenes
    fr = scenes.reference_synthetic(3)
    assert len(fr) == 3 and fr[0].shape == (1000, 4)
    # attribute = y / 10 and frame 0 scale = sin(0) + 1.5 (hostCode.cpp:157-163)
    assert np.isclose(fr[0][999, 3], 0.9) and np.isclose(fr[0][0, 0], 1.5 * -0.5)


def test_noise_atlas_is_spatiotemporal_blue_noise(aarbf_mod):
    """aarbf_generate_noise_atlas (host code, no GPU): 8 x 16 tiles of 256 x 256 in the reference's
    stbn.png layout (hostCode.cpp:337-352); each tile holds every 8-bit value exactly 256 times;
    tile 0 is void-and-cluster blue noise (almost no energy at low spatial frequencies, where white
    noise keeps its area share), the other frames are its golden-ratio shifts (still far below
    white noise at low frequencies), and a texel's values over successive frames advance by the
    golden-ratio conjugate modulo 1."""
    a = aarbf_mod.generate_noise_atlas()
    assert a.shape == (4096, 2048, 4) and (a[..., 3] == 255).all()
    assert np.array_equal(a, aarbf_mod.generate_noise_atlas())  # deterministic
    k = np.fft.fftfreq(256) * 256
    low = np.sqrt(k[:, None] ** 2 + k[None, :] ** 2) < 32  # 4.9 % of the spectrum

    def low_share(t):
        f = np.abs(np.fft.fft2(t - t.mean())) ** 2
        return f[low].sum() / f.sum()

    tiles = [a[256 * (f // 8):256 * (f // 8 + 1), 256 * (f % 8):256 * (f % 8 + 1), 0].astype(np.float64)
             for f in range(128)]
    for f in (0, 1, 37, 127):
        assert (np.bincount(tiles[f].astype(np.int64).ravel(), minlength=256) == 256).all()
    assert low_share(tiles[0]) < 1e-3
    assert max(low_share(tiles[f]) for f in (1, 2, 37, 127)) < 1e-2
    white = np.random.default_rng(0).integers(0, 256, (256, 256)).astype(np.float64)
    assert low_share(white) > 0.03
    step = (tiles[1].astype(np.int64) - tiles[0].astype(np.int64)) % 256
    assert np.isin(step, [157, 158, 159]).all()  # 0.618 x 256 = 158.2
