"""Cases of the reference-pinning fixtures (tests/golden/hlsl_ref.npz): small seeded scenes,
transfer functions and views on which the reference's own device programs (compiled for the CPU
from its HLSL, oracle/href.py) and the oracle are compared. Shared by make_golden.py, which writes
the reference's outputs, and tests/test_reference_pin.py, which checks the oracle against them.
Every input is rebuilt here from seeds; the fixtures hold only the reference's outputs."""
import numpy as np

W = H = 24


def scene(n, seed):
    """n particles in six Gaussian blobs (sigma 0.08) clipped to the unit cube, attribute U[0,1]."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.2, 0.8, (6, 3))
    lab = rng.integers(0, 6, n)
    p = np.clip(centres[lab] + rng.normal(0, 0.08, (n, 3)), 0, 1)
    a = rng.uniform(0, 1, (n, 1))
    return np.concatenate([p, a], 1).astype(np.float32)


def transfer_functions(kind):
    """(colormap, radiusmap, densitymap) as 64-texel RGBA8 textures: the reference's startup maps
    (hostCode.cpp:416-436 through :524-572), or variations with transparent texels and a steep
    density map, with a radius map of zero and partial texels ("variant") or of full texels
    ("variant_r1"). Splatting is compared on full radius maps only: there the reference's splat
    candidates (particles of leaves whose bounds-program box the slab meets, tested with the global
    radius) are exactly the particles whose sphere holds an accepted sample, which is the oracle's
    model; with partial radii the hardware's box test of leaves smaller than the splat spheres
    decides."""
    import aarbf
    cm, rm, dm = (t.copy() for t in aarbf.default_transfer_functions_rgba8())
    if kind in ("variant", "variant_r1"):
        cm[5:12, 3] = 0                                        # transparent attributes
        dm[:, 0] = np.clip(np.linspace(0, 600, 64), 0, 255).astype(np.uint8)
    if kind == "variant":
        rm[:, 0] = np.linspace(40, 255, 64).astype(np.uint8)   # radius 16 % .. 100 %
        rm[30:34, 0] = 0                                       # skipped by the bounds program
    return cm, rm, dm


def params(orc, dom, flags, spp=2, accum_id=1, frame_id=0, unit_scale=0.1, light=(0.0, 0.0, 0.5)):
    """the reference's startup view (hostCode.cpp:252-271): radius 1 % of the box diagonal, unit
    unit_scale x radius, camera from the box max + 0.3 looking at the centre, up (0, -1, 0)"""
    import aarbf
    diag = float(np.linalg.norm(dom[3:6] - dom[0:3]))
    r = float(np.float32(0.01 * diag))
    cam = orc.camera(dom[3:6] + np.float32(0.3), (dom[3:6] + dom[0:3]) * 0.5, (0, -1, 0), 0.66, W, H)
    return aarbf.RenderParams(cam_pos=cam[0], cam_dir00=cam[1], cam_du=cam[2], cam_dv=cam[3], aabb_min=dom[0:3],
                              aabb_max=dom[3:6], rbf_radius=r, unit=float(np.float32(r * unit_scale)),
                              accum_id=accum_id, frame_id=frame_id, spp=spp, flags=flags,
                              light_azimuth=light[0], light_elevation=light[1], light_ambient=light[2]), r


def stbn_atlas(seed=9):
    """a seeded stand-in for the reference's 2048 x 4096 RGBA8 blue-noise atlas (input only)"""
    return np.random.default_rng(seed).integers(0, 256, (4096, 2048, 4), dtype=np.uint8)


def cases():
    """name -> dict(kind, n, seed, ppl, tf, flags, spp, accum_id, frame_id, unit_scale, light)"""
    vis, blue, show = 1 << 2, 1 << 0, 1 << 1
    out = {}
    for n, seed, ppl in [(1500, 1, 1), (2000, 2, 4)]:
        for tfk in ("default", "variant"):
            base = dict(n=n, seed=seed, ppl=ppl, tf=tfk)
            out[f"bounds_{n}_{ppl}_{tfk}"] = dict(base, kind="bounds")
            out[f"track_{n}_{ppl}_{tfk}"] = dict(base, kind="render", flags=vis, spp=2)
            out[f"track_novis_{n}_{ppl}_{tfk}"] = dict(base, kind="render", flags=0, spp=2)
            out[f"march_{n}_{ppl}_{tfk}"] = dict(base, kind="render", flags=vis | blue, spp=2)
            sbase = dict(base, tf="default" if tfk == "default" else "variant_r1")
            out[f"splat_{n}_{ppl}_{tfk}"] = dict(sbase, kind="splat", flags=vis, unit_scale=0.5)
            out[f"splat_novis_{n}_{ppl}_{tfk}"] = dict(sbase, kind="splat", flags=0, unit_scale=0.5)
    base = dict(n=1500, seed=1, ppl=1, tf="default")
    out["track_light"] = dict(base, kind="render", flags=vis, spp=2, light=(0.3, 0.7, 0.2))
    out["track_accumulate"] = dict(base, kind="render", flags=vis, spp=3, accum_id=5, frame_id=4)
    out["track_shownoise"] = dict(base, kind="render", flags=vis | show, spp=1)
    out["march_light"] = dict(base, kind="render", flags=vis | blue, spp=2, frame_id=9, light=(0.6, 0.2, 0.0))
    out["march_budget"] = dict(base, kind="render", flags=vis | blue, spp=1, unit_scale=0.004)
    out["taa"] = dict(kind="taa", seed=3)
    return out


def inputs(orc, case):
    """(scene, tf decoded, params, accum0, atlas) of a render/splat/bounds case"""
    xyzw = scene(case["n"], case["seed"])
    dom = orc.domain([xyzw])
    tf8 = transfer_functions(case["tf"])
    tf = orc.tf_from_rgba8(*tf8)
    flags = case.get("flags", 0)
    p, r = params(orc, dom, flags, spp=case.get("spp", 1), accum_id=case.get("accum_id", 1),
                  frame_id=case.get("frame_id", 0), unit_scale=case.get("unit_scale", 0.1),
                  light=case.get("light", (0.0, 0.0, 0.5)))
    sc = orc.build_scene(xyzw, None, dom, case["ppl"], r, tf)[0]
    accum0 = None
    if case.get("accum_id", 1) > 1:
        accum0 = np.random.default_rng(case["seed"] + 100).uniform(0, 1, (H, W, 4)).astype(np.float32)
    atlas = stbn_atlas() if flags & 1 else None
    return sc, tf, p, r, accum0, atlas


def taa_inputs(seed):
    rng = np.random.default_rng(seed)
    w, h = 37, 29
    return rng.uniform(0, 1, (h, w, 4)).astype(np.float32), rng.uniform(0, 1, (h, w, 4)).astype(np.float32)
