"""The oracle's restatement of the renderer pinned to the reference itself.

The reference's own device programs -- GenRBFBounds, ParticleRBFRayGen with its intersection and
any-hit programs (delta tracking and stochastic marching), ParticleSplatRayGen with its programs,
and the CompositeGui TAA pass -- were compiled for the CPU from its HLSL (oracle/hlsl: a syntactic
rewrite plus a stand-in for the GPRT runtime that fixes what the GPU would decide by the same
documented model the oracle uses) and run on the seeded cases of tests/golden/hlsl_cases.py;
tests/golden/hlsl_ref.npz holds their outputs. Here the oracle runs the same cases:

  - leaf boxes of the bounds program, splat images and the TAA resolve (float and BGRA8) must be
    bit-identical;
  - tracking and marching images must agree per channel within 1e-4 relative plus 1e-6 absolute:
    the reference sums the any-hit contributions in float in hardware order, the oracle exactly
    in 2^-40 fixed point, so a channel built from very small weights keeps only about 1e-6 of
    absolute resolution. A pixel beyond that is allowed only if one of its random decisions came
    within 1e-4 (relative) of going the other way, which the rounding of the reference's float
    sums can decide, and at most 1 % of the pixels of a case may be such.

Where the reference tree exists (oracle/_ref built by make), the fixtures are also checked to be
the live reference's current outputs.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
import hlsl_cases as hc  # noqa: E402

GOLD = np.load(os.path.join(ROOT, "tests", "golden", "hlsl_ref.npz"))
CASES = hc.cases()


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def same(a, b):
    """bit-identical floats; a NaN (an inactive leaf box) matches any NaN"""
    a, b = np.ascontiguousarray(a, np.float32), np.ascontiguousarray(b, np.float32)
    return bool(((bits(a) == bits(b)) | (np.isnan(a) & np.isnan(b))).all())


def within(got, want):
    """per pixel: every channel within 1e-4 relative + 1e-6 absolute"""
    g, w = got.astype(np.float64), want.astype(np.float64)
    return (np.abs(g - w) <= 1e-4 * np.abs(w) + 1e-6).all(-1)


def oracle_outputs(orc, name):
    case = CASES[name]
    if case["kind"] == "taa":
        img, prev = hc.taa_inputs(case["seed"])
        return {"taa": orc.taa(img, prev, False), "taa_off": orc.taa(img, prev, True)}
    sc, tf, p, r, accum0, atlas = hc.inputs(orc, case)
    if case["kind"] == "bounds":
        return {"boxes": sc.bvh()[3]}
    if case["kind"] == "splat":
        return {"image": sc.render_splat(orc.params_from(p), hc.W, hc.H)}
    acc, img, gaps = sc.render_gaps(orc.params_from(p, noise=atlas), hc.W, hc.H, accum=accum0)
    return {"accum": acc, "image": img, "gaps": gaps}


@pytest.mark.parametrize("name", sorted(n for n, c in CASES.items() if c["kind"] in ("bounds", "splat", "taa")))
def test_bitexact_programs(orc, name):
    kind = CASES[name]["kind"]
    out = oracle_outputs(orc, name)
    if kind == "bounds":
        assert same(out["boxes"], GOLD[name])
        if CASES[name]["ppl"] == 1:  # one particle per leaf: a zero radius makes an inactive (NaN) box
            assert np.isnan(GOLD[name]).any() == (CASES[name]["tf"] == "variant")
    elif kind == "splat":
        want = GOLD[f"{name}_image"]
        assert (want[..., :3] > 0).mean() > 0.05  # the view shows particles
        assert np.array_equal(bits(out["image"]), bits(want))
    else:
        taa, bgra = out["taa"]
        assert np.array_equal(bits(taa), bits(GOLD[f"{name}_taa"]))
        assert np.array_equal(bgra, GOLD[f"{name}_bgra0"])
        assert np.array_equal(out["taa_off"][1], GOLD[f"{name}_bgra1"])


@pytest.mark.parametrize("name", sorted(n for n, c in CASES.items() if c["kind"] == "render"))
def test_tracking_and_marching(orc, name):
    out = oracle_outputs(orc, name)
    want_img, want_acc = GOLD[f"{name}_image"], GOLD[f"{name}_accum"]
    assert (want_img[..., :3] > 0).mean() > 0.05 or CASES[name]["flags"] & 2  # not an empty view
    ok = within(out["image"], want_img) & within(out["accum"], want_acc)
    bad = ~ok
    # every pixel outside the tolerance took a decision within 1e-4 of its threshold
    assert (out["gaps"][bad] < 1e-4).all(), np.argwhere(bad & (out["gaps"] >= 1e-4))[:5].tolist()
    assert bad.mean() <= 0.01, f"{int(bad.sum())} pixels differ"
    # most pixels are bit-identical: the models agree operation by operation
    assert (bits(out["image"]) == bits(want_img)).all(-1).mean() > 0.9


def test_reference_order_dependence_is_rare():
    """the reference itself: visiting the leaves in reverse order changes few pixels"""
    for name, c in CASES.items():
        if c["kind"] != "render":
            continue
        a, b = GOLD[f"{name}_image"], GOLD[f"{name}_image_reverse"]
        assert (~within(a, b)).mean() <= 0.01, name


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libaarbf_hlsl_ref.so")),
                    reason="reference tree not present (the fixtures still pin the oracle)")
def test_fixtures_are_the_live_reference(orc):
    import oracle.href as href
    for name in ("bounds_2000_4_variant", "track_1500_1_default", "march_2000_4_variant", "splat_2000_4_variant"):
        case = CASES[name]
        sc, tf, p, r, accum0, atlas = hc.inputs(orc, case)
        boxes = href.bounds(sc.xyzw, case["ppl"], r, tf[1])
        if case["kind"] == "bounds":
            assert same(boxes, GOLD[name])
        elif case["kind"] == "splat":
            assert np.array_equal(bits(href.render_splat(sc.xyzw, boxes, case["ppl"], p, tf, hc.W, hc.H)),
                                  bits(GOLD[f"{name}_image"]))
        else:
            _, img = href.render(sc.xyzw, boxes, case["ppl"], p, tf, hc.W, hc.H, accum=accum0, stbn=atlas)
            assert np.array_equal(bits(img), bits(GOLD[f"{name}_image"]))
