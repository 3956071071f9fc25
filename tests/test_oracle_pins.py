"""The oracle is pinned before it is trusted: Hilbert encoder and RNG against golden vectors made
by the reference's own hilbert.h / rng.h (and live against that library when it is present),
the deterministic exp/log/pow against float64, and the renderer restatement against closed-form
known answers (single particle densities, empty scene, fixed points)."""
import ctypes
import json
import math
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = json.load(open(os.path.join(ROOT, "tests", "golden", "hilbert_rng.json")))


def test_hilbert_c2i_golden(orc):
    L = orc.lib()
    bad = 0
    for nd, nb, x, y, z, idx in GOLD["hilbert_c2i"]:
        c = np.array([x, y, z], np.uint64)
        bad += L.orc_hilbert_c2i(nd, nb, c.ctypes.data) != idx
    assert bad == 0
    assert len(GOLD["hilbert_c2i"]) >= 4096 + 4000


def test_hilbert_i2c_golden_and_roundtrip(orc):
    L = orc.lib()
    for nd, nb, idx, x, y, z in GOLD["hilbert_i2c"]:
        c = np.zeros(3, np.uint64)
        L.orc_hilbert_i2c(nd, nb, idx, c.ctypes.data)
        assert list(c) == [x, y, z]
        assert L.orc_hilbert_c2i(nd, nb, c.ctypes.data) == idx


def test_hilbert_is_a_curve(orc):
    """consecutive indices map to unit-distance neighbours over the whole 2^12 grid"""
    L = orc.lib()
    prev = None
    seen = set()
    for i in range(4096):
        c = np.zeros(3, np.uint64)
        L.orc_hilbert_i2c(3, 4, i, c.ctypes.data)
        t = tuple(int(v) for v in c)
        seen.add(t)
        if prev is not None:
            assert sum(abs(a - b) for a, b in zip(t, prev)) == 1
        prev = t
    assert len(seen) == 4096


def test_rng_golden(orc):
    L = orc.lib()
    for e in GOLD["rng"]:
        s = L.orc_get_rng(e["frame"], e["pixel"][0], e["pixel"][1], e["width"])
        assert s == e["seed"]
        st = ctypes.c_uint32(s)
        for want_state, want_f in zip(e["states"], e["floats"]):
            f = L.orc_lcg_randomf(ctypes.byref(st))
            assert st.value == want_state
            assert float(np.float32(f)).hex() == want_f
    for h, k, m, fin in GOLD["murmur"]:
        assert L.orc_murmur_mix(h, k) == m
        assert L.orc_murmur_finalize(h) == fin


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libaarbf_ref.so")),
                    reason="reference tree not present (golden vectors still pin the oracle)")
def test_hilbert_live_reference(orc):
    R = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libaarbf_ref.so"))
    R.ref_hilbert_c2i.restype = ctypes.c_ulonglong
    L = orc.lib()
    rng = np.random.default_rng(5)
    for nd, nb in [(3, 16), (2, 8), (4, 5), (3, 21), (2, 32), (3, 1)]:
        for _ in range(500):
            c = rng.integers(0, 2 ** nb, size=nd).astype(np.uint64)
            assert L.orc_hilbert_c2i(nd, nb, c.ctypes.data) == R.ref_hilbert_c2i(nd, nb, ctypes.c_void_p(c.ctypes.data))


def test_det_math_accuracy(orc):
    L = orc.lib()
    rng = np.random.default_rng(0)
    xs = rng.uniform(1e-30, 10.0, 5000).astype(np.float32)
    for x in xs:
        g = L.orc_logf(float(x))
        r = math.log(float(x))
        assert abs(g - r) <= 3 * np.spacing(np.float32(abs(r))) + 1e-12
    for x in rng.uniform(-100, 80, 5000).astype(np.float32):
        g = L.orc_expf(float(x))
        r = math.exp(float(x))
        if r > 1.2e-38:
            assert abs(g - r) <= 1.5 * float(np.spacing(np.float32(r)))
    assert L.orc_expf(0.0) == 1.0 and L.orc_logf(1.0) == 0.0
    assert L.orc_expf(-200.0) == 0.0 and math.isinf(L.orc_expf(100.0))
    assert math.isinf(L.orc_logf(0.0)) and L.orc_powf(0.0, 2.2) == 0.0


def _one_particle_scene(orc, p=(0.5, 0.5, 0.5, 0.5), r=0.1, alpha=1.0):
    cm = np.tile(np.array([[0.2, 0.4, 0.8, alpha]], np.float32), (4, 1))
    tf = (cm, np.ones(4, np.float32), np.linspace(0, 1, 4).astype(np.float32))
    xyzw = np.array([p], np.float32)
    return orc.Scene(xyzw, None, np.zeros(1, np.uint64), 1, r, tf)


def test_single_particle_density_kat(orc):
    """D(p) = alpha^3; D at distance d = alpha^3 exp(-4.5 (d/r)^2); D = 0 at and beyond r
    (evaluate_rbf with sigma 3, sharedCode.h:137-140; any-hit sum deviceCodeRBF.hlsl:375)"""
    for alpha in (1.0, 0.5):
        s = _one_particle_scene(orc, alpha=alpha)
        c, acc = s.point_query([0.5, 0.5, 0.5])
        assert c == 1
        assert abs(acc[0] * 2.0 ** -40 - alpha ** 3) < 1e-6
        for d in (0.03, 0.07, 0.0999):
            c, acc = s.point_query([0.5 + d, 0.5, 0.5])
            want = alpha ** 3 * math.exp(-4.5 * (d / 0.1) ** 2)
            assert c == 1 and abs(acc[0] * 2.0 ** -40 - want) < 2e-6 * max(1, want)
        for d in (0.1, 0.2):
            c, acc = s.point_query([0.5 + d, 0.5, 0.5])
            assert c == 0 and acc[0] == 0
    # a transparent particle is never counted (deviceCodeRBF.hlsl:369-372)
    s = _one_particle_scene(orc, alpha=0.0)
    assert s.point_query([0.5, 0.5, 0.5])[0] == 0


def test_point_query_bvh_matches_brute_force(orc):
    rng = np.random.default_rng(3)
    n = 3000
    xyzw = np.concatenate([rng.uniform(0, 1, (n, 3)), rng.uniform(0, 1, (n, 1))], 1).astype(np.float32)
    dom = orc.domain([xyzw])
    cm = np.stack([np.linspace(0, 1, 64)] * 3 + [np.linspace(0.1, 1, 64)], 1).astype(np.float32)
    tf = (cm, np.linspace(0.5, 1, 64).astype(np.float32), np.linspace(0, 1, 64).astype(np.float32))
    for ppl in (1, 3, 8):
        s, _, _ = orc.build_scene(xyzw, None, dom, ppl, 0.05, tf)
        for q in rng.uniform(-0.05, 1.05, (300, 3)).astype(np.float32):
            a = s.point_query(q)
            b = s.point_query(q, brute=True)
            assert a[0] == b[0] and np.array_equal(a[1], b[1])


def _tf_default(orc):
    import aarbf
    return orc.tf_from_rgba8(*aarbf.default_transfer_functions_rgba8())


def test_empty_scene_renders_background(orc):
    s = orc.Scene(np.zeros((0, 4), np.float32), None, np.zeros(0, np.uint64), 1, 0.1, _tf_default(orc))
    from aarbf import RenderParams
    rp = RenderParams(cam_pos=(0.5, 0.5, -2), cam_dir00=(-0.5, -0.5, 1), cam_du=(1, 0, 0), cam_dv=(0, 1, 0),
                      unit=0.01, rbf_radius=0.1)
    acc, img = s.render(orc.params_from(rp), 16, 16)
    assert np.array_equal(img, np.tile(np.array([0, 0, 0, 1], np.float32), (16, 16, 1)))


def test_taa_constant_image_is_fixed_point(orc):
    img = np.tile(np.array([0.3, 0.6, 0.2, 1.0], np.float32), (8, 8, 1))
    out, bgra = orc.taa(img, img.copy())
    assert np.allclose(out, img, atol=1e-6)
    assert (bgra == ((255 << 24) | (int(0.3 * 255 + .5) << 16) | (int(0.6 * 255 + .5) << 8) | int(0.2 * 255 + .5))).all()


def test_majorant_estimator_is_unbiased(orc):
    """delta tracking with per-bin majorants converges to the plain estimator's image where the
    plain estimator's global majorant (1 per unit) bounds the extinction (no clamping)"""
    from aarbf import scenes
    sc = scenes.config_clusters(20_000, clusters=8, seed=6)
    tf = scenes.tf_linear_ramp()
    dom = orc.domain([sc.xyzw])
    scene, _, _ = orc.build_scene(sc.xyzw, sc.radii, dom, 1, float(sc.radii.max()), tf)
    means = []
    for majorant in (False, True):
        rp = scenes.native_params(scenes.orbit_camera(), 32, 24, float(sc.radii.max()), 0.001, 20.0, dom,
                                  spp=192, majorant=majorant, bin_length=0.008)
        _, img = scene.render(orc.params_from(rp), 32, 24)
        means.append(img[..., :3].astype(np.float64).mean())
    assert means[0] > 0
    assert abs(means[1] - means[0]) < 0.03 * means[0]


@pytest.mark.parametrize("majorant", [True, False])
def test_fp32_estimators_converge_to_fp64_twin(orc, majorant):
    """the float estimators (bit-identical to the GPU) agree with the FP64 twin of the volume
    model up to Monte-Carlo noise: their RMSE against one FP64 image is about that of a second,
    independent FP64 image of the same spp, and their mean shows no bias"""
    from aarbf import scenes
    sc = scenes.config_clusters(50_000, clusters=8, seed=6)
    tf = scenes.tf_four_peaks()
    dom = orc.domain([sc.xyzw])
    w, h, spp = 32, 24, 256
    rp = scenes.native_params(scenes.orbit_camera(), w, h, float(sc.radii.max()), 0.002, 500.0, dom, spp=spp,
                              majorant=majorant, bin_length=0.008)
    scene, _, _ = orc.build_scene(sc.xyzw, sc.radii, dom, 4, rp.rbf_radius, tf, 1 / 255)
    p = orc.params_from(rp)
    _, img = scene.render(p, w, h)
    f32 = img[..., :3].astype(np.float64)
    ref_a = scene.render_f64(p, w, h, (0, w, 0, h), spp, clamp_plain=not majorant, seed=11).astype(np.float64)
    ref_b = scene.render_f64(p, w, h, (0, w, 0, h), spp, clamp_plain=not majorant, seed=12).astype(np.float64)
    assert ref_a.mean() > 0.01  # the view is not empty
    rmse_f32 = math.sqrt(((f32 - ref_a) ** 2).mean())
    rmse_f64 = math.sqrt(((ref_b - ref_a) ** 2).mean())
    assert rmse_f32 < 1.5 * rmse_f64  # heavy-tailed per-pixel noise: a loose factor
    assert abs(f32.mean() - ref_b.mean()) < 0.03 * ref_b.mean()


def test_sort_tie_break(orc):
    """equal Hilbert keys are ordered by (x, y, z, w) then input index"""
    xyzw = np.array([[0.5, 0.5, 0.5, 0.9], [0.5, 0.5, 0.5, 0.1], [0.0, 0.0, 0.0, 0.0], [1, 1, 1, 1],
                     [0.5, 0.5, 0.5, 0.1]], np.float32)
    dom = orc.domain([xyzw])
    k = orc.hilbert_keys(xyzw, dom)
    perm = orc.sort_perm(k, xyzw)
    order = [int(i) for i in perm]
    pos = {i: order.index(i) for i in range(5)}
    assert pos[1] < pos[4] < pos[0]


def _diff_case(n=400, w=12, h=12, seed=5):
    from aarbf import scenes
    rng = np.random.default_rng(seed)
    gt, init = scenes.config_differentiable(n, clusters=4, seed=seed, tf_size=16)
    gt.radii[:] = rng.uniform(0.04, 0.08, n).astype(np.float32)
    init.radii[:] = 0.06
    dom = np.array([0, 0, 0, 1, 1, 1, 0, 1], np.float32)
    views = [scenes.native_params(cam, w, h, 0.08, 0.01, 10.0, dom, spp=2, frame_id=7 * k, marching=True)
             for k, cam in enumerate(scenes.orbit_views(2))]
    return gt, init, views


def test_diff_adjoint_matches_finite_differences(orc):
    """the FP64 adjoint of the differentiable form against central differences (h = 1e-3) of the
    FP64 forward on 48 parameters with non-zero gradient: positions, radii, attributes and
    transfer-function entries"""
    gt, init, rviews = _diff_case()
    w = h = 12
    views = [orc.params_from(v) for v in rviews]
    P = [init.pos.astype(np.float64), init.radii.astype(np.float64), init.attr.astype(np.float64),
         init.tf.astype(np.float64)]
    target = orc.diff_forward(gt.pos, gt.radii, gt.attr, gt.tf, views, w, h)

    def loss(p):
        return float(((orc.diff_forward(*p, views, w, h) - target) ** 2).sum())

    img = orc.diff_forward(*P, views, w, h)
    grads = orc.diff_backward(*P, views, w, h, 2.0 * (img - target))
    rng = np.random.default_rng(2)
    an, fd = [], []
    for kind in range(4):
        nz = np.argwhere(np.abs(grads[kind]) > 1e-6 * np.abs(grads[kind]).max())
        for j in rng.choice(len(nz), size=min(12, len(nz)), replace=False):
            idx = tuple(nz[j])
            pp = [x.copy() for x in P]
            pm = [x.copy() for x in P]
            pp[kind][idx] += 1e-3
            pm[kind][idx] -= 1e-3
            fd.append((loss(pp) - loss(pm)) / 2e-3)
            an.append(grads[kind][idx])
    an, fd = np.array(an), np.array(fd)
    assert len(an) == 48
    cos = an @ fd / (np.linalg.norm(an) * np.linalg.norm(fd))
    assert cos > 0.999
    assert np.linalg.norm(an - fd) < 0.03 * np.linalg.norm(fd)


def test_fp16_conversion_matches_ieee(orc):
    """the oracle's float -> half rounding (nearest, ties to even) and widening agree with IEEE
    binary16 (numpy's float16) on every half value, random floats over 13 decades, values next
    to halfway points, overflow, underflow and the specials"""
    L = orc.lib()
    for h in range(0, 65536, 7):
        ref = np.array([h], np.uint16).view(np.float16)[0]
        f = L.orc_h2f(h)
        assert (np.isnan(ref) and math.isnan(f)) or np.float32(ref) == np.float32(f)
    rng = np.random.default_rng(4)
    xs = np.concatenate([rng.normal(0, s, 4000) for s in (1e-8, 1e-6, 1e-4, 1e-2, 1, 100, 1e4, 1e5)])
    hw = (np.float16(rng.normal(0, 1, 500)).astype(np.float32) + np.float16(rng.normal(0, 1, 500)).astype(np.float32)) / 2
    xs = np.concatenate([xs, hw, np.nextafter(hw, np.float32(9)), np.nextafter(hw, np.float32(-9)),
                         [65504, 65519.99, 65520, 2 ** -25, 2 ** -24, 3 * 2 ** -26, 0.0, -0.0, np.inf, -np.inf]])
    xs = xs.astype(np.float32)
    with np.errstate(over="ignore"):
        want = xs.astype(np.float16).view(np.uint16)
    got = np.array([L.orc_f2h(float(x)) for x in xs], np.uint16)
    assert np.array_equal(got, want)
