"""GPU parity: the CUDA path through the C ABI against the oracle on the same seeded inputs.

Integer/index work (Hilbert keys, sort permutation, BVH topology) and every float the kernels
produce (prepass records, boxes, radiance) are compared bit for bit: the library and the oracle
evaluate the same operation sequence, and the per-sample density is an exact fixed-point sum, so
the stated 1e-4 relative tolerance of the per-pixel radiance check is met with zero difference.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BVH_PARTS = ("left", "right", "node boxes", "bounds-program leaf boxes", "traversal leaf boxes", "root box")


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32) if a.dtype == np.float32 else a


def assert_bitexact(got, want, what=""):
    g, w = bits(got), bits(want)
    assert g.shape == w.shape, (what, g.shape, w.shape)
    diff = np.argwhere(g != w)
    assert len(diff) == 0, f"{what}: {len(diff)} differing entries, first {diff[:5].tolist()}"


def assert_radiance(got, want, what=""):
    """per-pixel radiance within 1e-4 relative (and report exact equality)"""
    err = np.abs(got.astype(np.float64) - want) / np.maximum(np.abs(want), 1e-6)
    bad = np.argwhere(err > 1e-4)
    assert len(bad) == 0, f"{what}: {len(bad)} pixels beyond 1e-4 rel, first {bad[:5].tolist()}"
    assert_bitexact(got, want, what)


@pytest.fixture(scope="module")
def ctx(aarbf_mod):
    c = aarbf_mod.Context(0)
    yield c
    c.close()


def gpu_render(ctx, params, w, h, accum0=None, splat=False):
    nb = w * h * 16
    acc = ctx.device_alloc(nb)
    img = ctx.device_alloc(nb)
    try:
        if accum0 is None:
            ctx.memset(acc, 0, nb)
        else:
            ctx.memcpy(acc, np.ascontiguousarray(accum0, np.float32), nb)
        ctx.memset(img, 0, nb)
        if splat:
            ctx.render_splat(params, w, h, img)
        else:
            ctx.render(params, w, h, acc, img)
        ctx.sync()
        oa = np.zeros((h, w, 4), np.float32)
        oi = np.zeros((h, w, 4), np.float32)
        ctx.memcpy(oa, acc, nb)
        ctx.memcpy(oi, img, nb)
        ctx.sync()
        return oa, oi
    finally:
        ctx.device_free(acc)
        ctx.device_free(img)


def random_scene(n, seed, dup=0, radii=False):
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.2, 0.8, (6, 3))
    lab = rng.integers(0, 6, n)
    p = np.clip(centres[lab] + rng.normal(0, 0.08, (n, 3)), 0, 1)
    a = rng.uniform(0, 1, (n, 1))
    xyzw = np.concatenate([p, a], 1).astype(np.float32)
    if dup and n > 2:
        idx = rng.integers(0, n, dup)
        xyzw[idx[: dup // 2]] = xyzw[0]           # exact duplicates (same key, same position)
        xyzw[idx[dup // 2:], :3] = xyzw[1, :3]    # same position, different attribute
    r = np.exp(rng.uniform(np.log(0.004), np.log(0.03), n)).astype(np.float32) if radii else None
    return xyzw, r


def setup_both(ctx, orc, aarbf_mod, xyzw, radii, ppl, rbf, tf8=None, tf32=None, alpha_floor=0.0):
    dom = orc.domain([xyzw])
    ctx.set_particles(xyzw, radii)
    ctx.set_domain(dom)
    ctx.set_opacity_floor(alpha_floor)
    if tf32 is not None:
        ctx.set_transfer_functions_f32(*tf32)
        tf = tf32
    else:
        tf8 = tf8 if tf8 is not None else aarbf_mod.default_transfer_functions_rgba8()
        ctx.set_transfer_functions_rgba8(*tf8)
        tf = orc.tf_from_rgba8(*tf8)
    ctx.build(rbf, ppl)
    scene, keys, perm = orc.build_scene(xyzw, radii, dom, ppl, rbf, tf, alpha_floor)
    return scene, keys, perm, dom


@pytest.mark.parametrize("n,ppl,dup", [(1, 1, 0), (2, 1, 0), (7, 4, 0), (1000, 1, 0), (1000, 16, 40),
                                       (50_000, 1, 0), (50_000, 8, 500), (3, 8, 0),
                                       (200_000, 1, 60)])
def test_build_bitexact(ctx, orc, aarbf_mod, n, ppl, dup):
    xyzw, radii = random_scene(n, seed=n + ppl, dup=dup, radii=(ppl == 8))
    scene, keys, perm, dom = setup_both(ctx, orc, aarbf_mod, xyzw, radii, ppl, 0.02)
    gk, gp = ctx.hilbert_keys()
    assert_bitexact(gk, keys, "hilbert keys")
    assert_bitexact(gp, perm, "sort permutation")
    assert_bitexact(ctx.sorted_particles(), scene.xyzw, "sorted particles")
    for g, w, name in zip(ctx.prepass(), scene.prepass(), ("rec0", "w4", "rgeom")):
        assert_bitexact(g, w, name)
    for g, w, name in zip(ctx.bvh(), scene.bvh(), BVH_PARTS):
        assert_bitexact(g, w, name)


def test_domain_reduce_matches_oracle(ctx, orc):
    xyzw, _ = random_scene(100_000, 9)
    d = ctx.domain_accumulate(xyzw, __import__("aarbf").domain_init())
    assert_bitexact(d, orc.domain([xyzw]), "domain")
    bad = xyzw.copy()
    bad[17, 1] = np.nan
    with pytest.raises(Exception):
        ctx.domain_accumulate(bad, __import__("aarbf").domain_init())


def test_series_domain_matches_oracle(ctx, orc, aarbf_mod):
    """the space-time box and attribute range of a whole series (hostCode.cpp:183-193, :227-240):
    frames of different sizes that move, grow and shift their attributes, reduced frame by frame
    on the device into one running domain; then the series' Hilbert keys of the last frame"""
    frames = []
    for k, n in enumerate((50_000, 20_000, 80_000)):
        xyzw, _ = random_scene(n, 40 + k)
        xyzw[:, :3] = xyzw[:, :3] * np.float32(1.0 + 0.5 * k) + np.float32(0.3 * k - 0.2)
        xyzw[:, 3] = xyzw[:, 3] * np.float32(2.0) - np.float32(k)
        frames.append(xyzw)
    dom = aarbf_mod.domain_init()
    for f in frames:
        dom = ctx.domain_accumulate(f, dom)
    want = orc.domain(frames)
    assert_bitexact(dom, want, "series domain")
    # no frame alone spans it
    assert all(not np.array_equal(orc.domain([f]), want) for f in frames)
    # the last frame quantised in the series' domain (not its own): keys and order as the oracle's
    scene, keys, perm, _ = setup_both(ctx, orc, aarbf_mod, frames[-1], None, 1, 0.02)
    ctx.set_domain(want)
    ctx.build(0.02, 1)
    scene, keys, perm = orc.build_scene(frames[-1], None, want, 1, 0.02,
                                        orc.tf_from_rgba8(*aarbf_mod.default_transfer_functions_rgba8()))
    gk, gp = ctx.hilbert_keys()
    assert_bitexact(gk, keys, "hilbert keys in the series domain")
    assert_bitexact(gp, perm, "sort permutation in the series domain")
    assert_bitexact(ctx.sorted_particles(), scene.xyzw, "normalised attributes in the series domain")


def reference_params(aarbf_mod, dom, w, h, **kw):
    """the reference's startup state: radius 0.01 diag, unit 0.1 radius, ambient 0.5, light 0/0,
    visualizeAttributes on, camera from the domain max looking at the centre (hostCode.cpp:252-271)"""
    diag = float(np.linalg.norm(dom[3:6] - dom[0:3]))
    r = float(np.float32(0.01 * diag))
    cam = aarbf_mod.camera(dom[3:6] + np.float32(0.3), (dom[3:6] + dom[0:3]) * 0.5, (0, -1, 0), 0.66, w, h)
    base = dict(cam_pos=cam[0], cam_dir00=cam[1], cam_du=cam[2], cam_dv=cam[3], aabb_min=dom[0:3],
                aabb_max=dom[3:6], rbf_radius=r, unit=float(np.float32(r * 0.1)), accum_id=1, frame_id=0,
                spp=1, flags=aarbf_mod.FLAG_VISUALIZE_ATTRIBUTES, light_ambient=0.5)
    base.update(kw)
    return aarbf_mod.RenderParams(**base), r


@pytest.mark.parametrize("traversal", [0, 1, 2])  # one warp per ray / point queries / one thread per ray
@pytest.mark.parametrize("ppl", [1, 4])
def test_render_tracking_reference_mode(ctx, orc, aarbf_mod, traversal, ppl):
    xyzw, _ = random_scene(20_000, 11)
    dom = orc.domain([xyzw])
    w, h = 40, 32
    rp, r = reference_params(aarbf_mod, dom, w, h, spp=2, traversal=traversal)
    scene, *_ = setup_both(ctx, orc, aarbf_mod, xyzw, None, ppl, r)
    ga, gi = gpu_render(ctx, rp, w, h)
    oa, oi = scene.render(orc.params_from(rp), w, h)
    assert_radiance(gi, oi, "image")
    assert_radiance(ga, oa, "accum")
    assert (oi[..., :3] > 0).mean() > 0.05  # the view is not empty


def test_render_accumulation_continues(ctx, orc, aarbf_mod):
    xyzw, _ = random_scene(5_000, 12)
    dom = orc.domain([xyzw])
    w, h = 24, 24
    rp, r = reference_params(aarbf_mod, dom, w, h, accum_id=5, frame_id=4, spp=3)
    scene, *_ = setup_both(ctx, orc, aarbf_mod, xyzw, None, 1, r)
    prev = np.random.default_rng(1).uniform(0, 1, (h, w, 4)).astype(np.float32)
    ga, gi = gpu_render(ctx, rp, w, h, accum0=prev)
    oa, oi = scene.render(orc.params_from(rp), w, h, accum=prev.copy())
    assert_radiance(ga, oa, "accum")
    assert_radiance(gi, oi, "image")
    # three launches of one sample == one launch of three
    acc = prev.copy()
    for k in range(3):
        rp1, _ = reference_params(aarbf_mod, dom, w, h, accum_id=5 + k, frame_id=4 + k, spp=1)
        acc, img = gpu_render(ctx, rp1, w, h, accum0=acc)
    assert_bitexact(acc, ga, "spp loop vs launches")


@pytest.mark.parametrize("flags_extra,kw", [
    (0, dict(light_ambient=1.0)),
    (0, dict(light_azimuth=0.3, light_elevation=0.7, light_ambient=0.2)),
    ("no_vis", {}),
    ("noise", {}),
    (0, dict(jitter_x=0.25, jitter_y=-0.4)),
])
def test_render_flags(ctx, orc, aarbf_mod, flags_extra, kw):
    xyzw, _ = random_scene(8_000, 13)
    dom = orc.domain([xyzw])
    w, h = 32, 24
    rp, r = reference_params(aarbf_mod, dom, w, h, **kw)
    if flags_extra == "no_vis":
        rp.flags = 0
    elif flags_extra == "noise":
        rp.flags |= aarbf_mod.FLAG_SHOW_NOISE
    scene, *_ = setup_both(ctx, orc, aarbf_mod, xyzw, None, 2, r)
    ga, gi = gpu_render(ctx, rp, w, h)
    oa, oi = scene.render(orc.params_from(rp), w, h)
    assert_radiance(gi, oi, "image")
    assert_radiance(ga, oa, "accum")


@pytest.mark.parametrize("traversal,unit_scale", [(0, 0.1), (1, 0.1), (2, 0.1), (0, 0.004)])
def test_render_marching_blue_noise(ctx, orc, aarbf_mod, traversal, unit_scale):
    """stochastic marching: one warp per ray (0), point queries (1), one thread per ray (2); the
    tiny unit makes rays run out of the 10000-step budget"""
    xyzw, _ = random_scene(10_000, 14)
    dom = orc.domain([xyzw])
    w, h = 40, 24
    rp, r = reference_params(aarbf_mod, dom, w, h, spp=2, traversal=traversal,
                             flags=aarbf_mod.FLAG_VISUALIZE_ATTRIBUTES | aarbf_mod.FLAG_BLUE_NOISE)
    rp.unit = float(np.float32(r * unit_scale))
    scene, *_ = setup_both(ctx, orc, aarbf_mod, xyzw, None, 1, r)
    atlas = aarbf_mod.generate_noise_atlas()
    ctx.set_noise_atlas(atlas)
    ga, gi = gpu_render(ctx, rp, w, h)
    oa, oi = scene.render(orc.params_from(rp, noise=atlas), w, h)
    assert_radiance(gi, oi, "image")
    assert (oi[..., :3] > 0).mean() > 0.01


@pytest.mark.parametrize("traversal", [0, 2])
def test_render_marching_native_dense(ctx, orc, aarbf_mod, traversal):
    """native-mode marching (per-particle radii, linear density) through dense clusters: the warp
    tracker's staging overflows and falls back to shorter chunks and direct steps"""
    from aarbf import scenes
    sc = scenes.config_clusters(60_000, clusters=8, seed=19)
    cm, rm, dm = scenes.tf_linear_ramp()
    dom = orc.domain([sc.xyzw])
    w, h = 32, 24
    rp = scenes.native_params(scenes.orbit_camera(), w, h, float(sc.radii.max()), 0.002, 400.0, dom, spp=2,
                              marching=True, traversal=traversal)
    scene, *_ = setup_both(ctx, orc, aarbf_mod, sc.xyzw, sc.radii, 4, rp.rbf_radius, tf32=(cm, rm, dm))
    atlas = aarbf_mod.generate_noise_atlas()
    ctx.set_noise_atlas(atlas)
    ga, gi = gpu_render(ctx, rp, w, h)
    oa, oi = scene.render(orc.params_from(rp, noise=atlas), w, h)
    assert_radiance(gi, oi, "image")
    assert_radiance(ga, oa, "accum")
    assert (oi[..., :3] > 0).mean() > 0.01


@pytest.mark.parametrize("traversal", [0, 2])
@pytest.mark.parametrize("cap,bins", [(256, 0), (1024, 64), (256, 5), (512, 48)])
def test_render_delta_native_dense(ctx, orc, aarbf_mod, traversal, cap, bins):
    """the reference's delta tracking (global majorant 1/unit, native density) through dense
    clusters: the warp tracker's stagings overflow and fall back to shorter runs and direct warp
    point queries; every buffer depth and first staging length gives the same bits"""
    from aarbf import scenes
    sc = scenes.config_clusters(60_000, clusters=8, seed=19)
    cm, rm, dm = scenes.tf_linear_ramp()
    dom = orc.domain([sc.xyzw])
    w, h = 32, 24
    rp = scenes.native_params(scenes.orbit_camera(), w, h, float(sc.radii.max()), 0.002, 400.0, dom, spp=2,
                              traversal=traversal, bin_length=0.032)
    if traversal == 0:
        rp.candidate_cap, rp.stage_bins = cap, bins
    scene, *_ = setup_both(ctx, orc, aarbf_mod, sc.xyzw, sc.radii, 4, rp.rbf_radius, tf32=(cm, rm, dm))
    ga, gi = gpu_render(ctx, rp, w, h)
    oa, oi = scene.render(orc.params_from(rp), w, h)
    assert_radiance(gi, oi, "image")
    assert_radiance(ga, oa, "accum")
    assert (oi[..., :3] > 0).mean() > 0.01


@pytest.mark.parametrize("traversal", [0, 1, 2])
def test_render_native_mode(ctx, orc, aarbf_mod, traversal):
    from aarbf import scenes
    sc = scenes.config_clusters(30_000, clusters=8, seed=5)
    cm, rm, dm = scenes.tf_linear_ramp()
    dom = orc.domain([sc.xyzw])
    w, h = 40, 30
    cam = scenes.orbit_camera()
    rp = scenes.native_params(cam, w, h, float(sc.radii.max()), 0.002, 2000.0, dom, spp=2, traversal=traversal)
    scene, *_ = setup_both(ctx, orc, aarbf_mod, sc.xyzw, sc.radii, 1, rp.rbf_radius, tf32=(cm, rm, dm))
    ga, gi = gpu_render(ctx, rp, w, h)
    oa, oi = scene.render(orc.params_from(rp), w, h)
    assert_radiance(gi, oi, "image")
    assert (oi[..., :3] > 0).mean() > 0.01  # the view is not empty


@pytest.mark.parametrize("n,ppl,bins,scale,floor", [(30_000, 1, 4.0, 200.0, 0.0), (30_000, 4, 1.0, 200.0, 0.0),
                                                    (200_000, 1, 8.0, 200.0, 1 / 255),
                                                    (200_000, 8, 32.0, 5000.0, 1 / 255)])
@pytest.mark.parametrize("traversal", [0, 2])  # one warp per ray / one thread per ray
def test_render_majorant_tracking(ctx, orc, aarbf_mod, n, ppl, bins, scale, floor, traversal):
    """delta tracking with per-bin majorants (native extinction density_scale * D); the dense
    case exercises the bin refinement and the direct (unstaged) bins"""
    from aarbf import scenes
    sc = scenes.config_clusters(n, clusters=8, seed=6)
    cm, rm, dm = scenes.tf_linear_ramp()
    dom = orc.domain([sc.xyzw])
    w, h = 40, 30
    rp = scenes.native_params(scenes.orbit_camera(), w, h, float(sc.radii.max()), 0.002, scale, dom, spp=2,
                              majorant=True, bin_length=bins * 0.002, traversal=traversal)
    scene, *_ = setup_both(ctx, orc, aarbf_mod, sc.xyzw, sc.radii, ppl, rp.rbf_radius, tf32=(cm, rm, dm),
                           alpha_floor=floor)
    ga, gi = gpu_render(ctx, rp, w, h)
    oa, oi = scene.render(orc.params_from(rp), w, h)
    assert_radiance(gi, oi, "image")
    assert_radiance(ga, oa, "accum")
    assert (oi[..., :3] > 0).mean() > 0.01  # the view is not empty


@pytest.mark.parametrize("stage_bins", [1, 3, 48, 64])
def test_render_majorant_stage_lengths(ctx, orc, aarbf_mod, stage_bins):
    """the warp tracker's first staging length (any of 1..64; later stagings adapt to the staged
    candidate density and never exceed the 64-bin lists) changes no bit"""
    from aarbf import scenes
    sc = scenes.config_clusters(200_000, clusters=8, seed=6)
    cm, rm, dm = scenes.tf_linear_ramp()
    dom = orc.domain([sc.xyzw])
    w, h = 40, 30
    rp = scenes.native_params(scenes.orbit_camera(), w, h, float(sc.radii.max()), 0.002, 200.0, dom, spp=2,
                              majorant=True, bin_length=8 * 0.002)
    rp.stage_bins = stage_bins
    scene, *_ = setup_both(ctx, orc, aarbf_mod, sc.xyzw, sc.radii, 1, rp.rbf_radius, tf32=(cm, rm, dm),
                           alpha_floor=1 / 255)
    ga, gi = gpu_render(ctx, rp, w, h)
    oa, oi = scene.render(orc.params_from(rp), w, h)
    assert_radiance(gi, oi, "image")
    assert_radiance(ga, oa, "accum")
    assert (oi[..., :3] > 0).mean() > 0.01


def test_kernel_timing(ctx, orc, aarbf_mod):
    """event timing around the render's kernels leaves the result unchanged and reports one
    positive duration per kernel for each timed render"""
    from aarbf import scenes
    sc = scenes.config_clusters(20_000, clusters=4, seed=9)
    cm, rm, dm = scenes.tf_linear_ramp()
    dom = orc.domain([sc.xyzw])
    w, h = 24, 16
    rp = scenes.native_params(scenes.orbit_camera(), w, h, float(sc.radii.max()), 0.002, 200.0, dom, spp=2,
                              majorant=True, bin_length=0.008)
    scene, *_ = setup_both(ctx, orc, aarbf_mod, sc.xyzw, sc.radii, 4, rp.rbf_radius, tf32=(cm, rm, dm))
    ctx.set_kernel_timing(True)
    try:
        ga, gi = gpu_render(ctx, rp, w, h)
        ga2, gi2 = gpu_render(ctx, rp, w, h)
        r_ms, a_ms, k = ctx.kernel_times()
    finally:
        ctx.set_kernel_timing(False)
    assert k == 2 and r_ms > 0 and a_ms > 0
    assert ctx.kernel_times() == (0.0, 0.0, 0)
    oa, oi = scene.render(orc.params_from(rp), w, h)
    assert_radiance(gi, oi, "image")
    assert_bitexact(gi2, gi, "image (second timed render)")


@pytest.mark.parametrize("traversal", [0, 2])  # one warp per pixel / one thread per pixel
@pytest.mark.parametrize("native", [False, True])
def test_splat_parity(ctx, orc, aarbf_mod, native, traversal):
    w, h = 32, 24
    if native:
        from aarbf import scenes
        sc = scenes.config_clusters(20_000, clusters=8, seed=6)
        dom = orc.domain([sc.xyzw])
        cm, rm, dm = scenes.tf_four_peaks()
        rp = scenes.native_params(scenes.orbit_camera(), w, h, float(sc.radii.max()), 0.004, 50.0, dom)
        scene, *_ = setup_both(ctx, orc, aarbf_mod, sc.xyzw, sc.radii, 2, rp.rbf_radius, tf32=(cm, rm, dm))
    else:
        xyzw, _ = random_scene(10_000, 15)
        dom = orc.domain([xyzw])
        rp, r = reference_params(aarbf_mod, dom, w, h)
        rp.unit = float(np.float32(r * 0.5))
        scene, *_ = setup_both(ctx, orc, aarbf_mod, xyzw, None, 1, r)
    rp.traversal = traversal
    _, gi = gpu_render(ctx, rp, w, h, splat=True)
    oi = scene.render_splat(orc.params_from(rp), w, h)
    assert_radiance(gi, oi, "splat image")
    assert (oi[..., :3] > 0).mean() > 0.01  # the view is not empty


def test_splat_crowded_slab(ctx, orc, aarbf_mod):
    """thousands of samples in one slab (particles on a sphere around the camera): the warp
    kernel's staging overflows even for a single slab and takes the 15 smallest (t, index) by
    repeated minimum traversals"""
    from aarbf import scenes
    rng = np.random.default_rng(8)
    n = 3000
    cam = scenes.orbit_camera(distance=2.5)
    c, o = np.asarray(cam[1], np.float64), np.asarray(cam[0], np.float64)
    fwd = (c - o) / np.linalg.norm(c - o)
    side = np.cross(fwd, [0.0, 1.0, 0.0])
    side /= np.linalg.norm(side)
    up = np.cross(side, fwd)
    ang = rng.uniform(-0.004, 0.004, (n, 2))
    dirs = fwd[None] + ang[:, :1] * side[None] + ang[:, 1:] * up[None]
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    pos = o[None] + 2.5 * dirs
    xyzw = np.concatenate([pos, rng.uniform(0, 1, (n, 1))], 1).astype(np.float32)
    radii = np.full(n, 0.05, np.float32)
    dom = orc.domain([xyzw])
    cm, rm, dm = scenes.tf_linear_ramp()
    w, h = 8, 8
    cam_narrow = (cam[0], cam[1], cam[2], 0.004)
    rp = scenes.native_params(cam_narrow, w, h, 0.05, 0.001, 50.0, dom)
    scene, *_ = setup_both(ctx, orc, aarbf_mod, xyzw, radii, 1, 0.05, tf32=(cm, rm, dm))
    _, gi = gpu_render(ctx, rp, w, h, splat=True)
    oi = scene.render_splat(orc.params_from(rp), w, h)
    assert (oi[..., 3] > 0).all()
    assert_radiance(gi, oi, "splat image")


def test_taa_parity(ctx, orc):
    rng = np.random.default_rng(3)
    w, h = 37, 29
    img = rng.uniform(0, 1, (h, w, 4)).astype(np.float32)
    prev = rng.uniform(0, 1, (h, w, 4)).astype(np.float32)
    nb = w * h * 16
    bufs = [ctx.device_alloc(nb) for _ in range(3)]
    bg = ctx.device_alloc(w * h * 4)
    try:
        ctx.memcpy(bufs[0], img, nb)
        ctx.memcpy(bufs[1], prev, nb)
        for disable in (0, 1):
            ctx.taa_resolve(bufs[0], bufs[1], bufs[2], bg, w, h, disable=bool(disable))
            ctx.sync()
            out = np.zeros((h, w, 4), np.float32)
            bgra = np.zeros((h, w), np.uint32)
            ctx.memcpy(out, bufs[2], nb)
            ctx.memcpy(bgra, bg, w * h * 4)
            ctx.sync()
            want, wbgra = orc.taa(img, prev, disable=bool(disable))
            if not disable:
                assert_bitexact(out, want, "taa")
            assert_bitexact(bgra, wbgra, "bgra")
    finally:
        for b in bufs + [bg]:
            ctx.device_free(b)


@pytest.mark.parametrize("case", ["empty", "one", "ppl_gt_n", "identical", "radius_zero", "alpha_zero"])
def test_edge_cases(ctx, orc, aarbf_mod, case):
    rng = np.random.default_rng(21)
    xyzw, _ = random_scene(3_000, 22)
    ppl = 1
    tf8 = None
    if case == "empty":
        xyzw = np.zeros((0, 4), np.float32)
    elif case == "one":
        xyzw = np.array([[0.5, 0.5, 0.5, 0.5]], np.float32)
    elif case == "ppl_gt_n":
        xyzw = xyzw[:5]
        ppl = 16
    elif case == "identical":
        xyzw = np.tile(np.array([[0.5, 0.5, 0.5, 0.3]], np.float32), (500, 1))
        xyzw[::3, 3] = 0.7
    elif case in ("radius_zero", "alpha_zero"):
        cm, rm, dm = aarbf_mod.default_transfer_functions_rgba8()
        if case == "radius_zero":
            rm = rm.copy()
            rm[20:40, 0] = 0   # radiusmap 0 -> skipped by the bounds program, never hit
        else:
            cm = cm.copy()
            cm[10:30, 3] = 0   # transparent -> ignored by the any-hit program
        tf8 = (cm, rm, dm)
        ppl = 4
    dom = orc.domain([xyzw]) if len(xyzw) else np.array([0, 0, 0, 1, 1, 1, 0, 1], np.float32)
    w, h = 24, 20
    rp, r = reference_params(aarbf_mod, dom, w, h)
    if case in ("one", "identical"):
        r = 0.2
        rp.rbf_radius, rp.unit = r, 0.02
        rp.cam_pos = np.array([0.5, 0.5, -1.5], np.float32)
        cam = aarbf_mod.camera((0.5, 0.5, -1.5), (0.5, 0.5, 0.5), (0, 1, 0), 0.5, w, h)
        rp.cam_pos, rp.cam_dir00, rp.cam_du, rp.cam_dv = cam
    if case == "empty":
        ctx.set_particles(xyzw)
        ctx.set_domain(dom)
        ctx.set_transfer_functions_rgba8(*aarbf_mod.default_transfer_functions_rgba8())
        ctx.build(r, 1)
        _, gi = gpu_render(ctx, rp, w, h)
        assert np.array_equal(gi, np.tile(np.array([0, 0, 0, 1], np.float32), (h, w, 1)))
        return
    ctx.set_domain(dom)
    scene, keys, perm, _ = setup_both(ctx, orc, aarbf_mod, xyzw, None, ppl, r, tf8=tf8)
    for g, wv, name in zip(ctx.bvh(), scene.bvh(), BVH_PARTS):
        assert_bitexact(g, wv, name)
    for trav in (0, 1):
        rp.traversal = trav
        ga, gi = gpu_render(ctx, rp, w, h)
        oa, oi = scene.render(orc.params_from(rp), w, h)
        assert_radiance(gi, oi, f"{case} image traversal {trav}")


def test_refit_after_transfer_function_change(ctx, orc, aarbf_mod):
    xyzw, _ = random_scene(4_000, 30)
    dom = orc.domain([xyzw])
    w, h = 24, 24
    rp, r = reference_params(aarbf_mod, dom, w, h)
    setup_both(ctx, orc, aarbf_mod, xyzw, None, 2, r)
    cm, rm, dm = aarbf_mod.default_transfer_functions_rgba8()
    rm = rm.copy()
    rm[:, 0] = np.linspace(80, 255, 64).astype(np.uint8)
    ctx.set_transfer_functions_rgba8(cm, rm, dm)
    with pytest.raises(aarbf_mod.AarbfError):
        ctx.render(rp, w, h)          # prepass is stale until refit
    ctx.refit(r * 1.5)
    scene, *_ = orc.build_scene(xyzw, None, dom, 2, r * 1.5, orc.tf_from_rgba8(cm, rm, dm))
    for g, wv, name in zip(ctx.bvh(), scene.bvh(), BVH_PARTS):
        assert_bitexact(g, wv, name)
    rp.rbf_radius = r * 1.5
    ga, gi = gpu_render(ctx, rp, w, h)
    oa, oi = scene.render(orc.params_from(rp), w, h)
    assert_radiance(gi, oi, "image after refit")


def test_full_size_properties(ctx, orc, aarbf_mod):
    """the 10M-particle benchmark scene: sort order, permutation, BVH containment, and the two
    traversal strategies agreeing bit for bit on a crop; plus oracle pixels on a small crop"""
    from aarbf import scenes
    sc = scenes.config_clusters(10_000_000, seed=2)
    cm, rm, dm = scenes.tf_four_peaks()
    dom = orc.domain([sc.xyzw])
    ctx.set_particles(sc.xyzw, sc.radii)
    ctx.set_domain(dom)
    ctx.set_transfer_functions_f32(cm, rm, dm)
    ctx.build(float(sc.radii.max()), 1)
    k, p = ctx.hilbert_keys()
    assert (np.diff(k.astype(np.int64)) >= 0).all()
    assert np.array_equal(np.sort(p), np.arange(len(p), dtype=np.uint32))
    left, right, nb, _, lb, rb = ctx.bvh()
    # every child box lies inside its parent's box
    LEAF = np.uint32(0x80000000)
    for ch in (left, right):
        is_leaf = (ch & LEAF) != 0
        cb = np.where(is_leaf[:, None], lb[(ch & ~LEAF) % len(lb)], nb[ch % max(len(nb), 1)])
        ok = np.isnan(cb).all(1) | ((cb[:, :3] >= nb[:, :3]).all(1) & (cb[:, 3:] <= nb[:, 3:]).all(1))
        assert ok.all()
    # the two traversal strategies agree bit for bit on the full-size scene
    w, h = 96, 64
    rp = scenes.native_params(scenes.orbit_camera(), w, h, float(sc.radii.max()), 0.001, 50.0, dom)
    imgs = []
    for trav in (0, 1):
        rp.traversal = trav
        imgs.append(gpu_render(ctx, rp, w, h)[1])
    assert_bitexact(imgs[0], imgs[1], "staged vs point at 10M")
    assert (imgs[0][..., :3] > 0).mean() > 0.01


def test_oracle_parity_1m(ctx, orc, aarbf_mod):
    """1M particles of the benchmark distribution, native mode, against the oracle on a crop"""
    from aarbf import scenes
    sc = scenes.config_clusters(1_000_000, seed=4)
    cm, rm, dm = scenes.tf_four_peaks()
    w, h = 48, 32
    dom = orc.domain([sc.xyzw])
    rp = scenes.native_params(scenes.orbit_camera(), w, h, float(sc.radii.max()), 0.001, 50.0, dom, spp=1)
    scene, *_ = setup_both(ctx, orc, aarbf_mod, sc.xyzw, sc.radii, 8, rp.rbf_radius, tf32=(cm, rm, dm),
                           alpha_floor=1 / 255)
    ga, gi = gpu_render(ctx, rp, w, h)
    oa, oi = scene.render(orc.params_from(rp), w, h)
    assert_radiance(gi, oi, "1M image")
    rpm = scenes.native_params(scenes.orbit_camera(), w, h, float(sc.radii.max()), 0.001, 50.0, dom, spp=2,
                               majorant=True, bin_length=0.016)
    ga, gi = gpu_render(ctx, rpm, w, h)
    oa, oi = scene.render(orc.params_from(rpm), w, h)
    assert_radiance(gi, oi, "1M image, majorant tracking")
