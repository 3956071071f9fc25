"""Generate the golden vectors in tests/golden/ from the reference's own code.

Runs in a container that has the reference tree ($AARBF_REFERENCE, else the read-only tree this
build environment mounts): oracle/Makefile compiles the reference's hilbert.h and rng.h unchanged
into oracle/_ref/libaarbf_ref.so, and its HLSL device programs (rewritten to C++ by
oracle/hlsl/hlsl2cpp.py, run on the GPRT stand-in oracle/hlsl/gprt.h) into
oracle/_ref/libaarbf_hlsl_ref.so. This script calls them and writes hilbert_rng.json and
hlsl_ref.npz (the reference programs' outputs on the cases of hlsl_cases.py). The CPU tests pin
the oracle's restatements against these fixtures (on machines without the reference tree) and
against the live reference libraries (where they exist).

    python tests/golden/make_golden.py
"""
import ctypes
import json
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
REF = os.path.join(ROOT, "oracle", "_ref", "libaarbf_ref.so")


def reference_tree():
    for cand in (os.environ.get("AARBF_REFERENCE"), "/root/reference"):
        if cand and os.path.isfile(os.path.join(cand, "hilbert.h")):
            return cand
    raise SystemExit("reference tree not found (set AARBF_REFERENCE)")


def write_hlsl_golden():
    """the reference's device programs on every case of hlsl_cases.py -> hlsl_ref.npz"""
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "attribute-aware-rbfs_b200"))
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import hlsl_cases as hc
    import oracle.href as href
    import oracle.oracle as orc
    out = {}
    for name, case in hc.cases().items():
        if case["kind"] == "taa":
            img, prev = hc.taa_inputs(case["seed"])
            for d in (0, 1):
                taa, bgra = href.taa(img, prev, disable=bool(d))
                if not d:
                    out[f"{name}_taa"] = taa
                out[f"{name}_bgra{d}"] = bgra
            continue
        sc, tf, p, r, accum0, atlas = hc.inputs(orc, case)
        boxes = href.bounds(sc.xyzw, case["ppl"], r, tf[1])
        if case["kind"] == "bounds":
            out[name] = boxes
        elif case["kind"] == "render":
            acc, img = href.render(sc.xyzw, boxes, case["ppl"], p, tf, hc.W, hc.H, accum=accum0, stbn=atlas)
            out[f"{name}_accum"], out[f"{name}_image"] = acc, img
            # the same launches with the leaves visited in reverse order: pixels that differ
            # depend on the hardware's (unspecified) any-hit order
            _, img_rev = href.render(sc.xyzw, boxes, case["ppl"], p, tf, hc.W, hc.H, accum=accum0, stbn=atlas,
                                     reverse=True)
            out[f"{name}_image_reverse"] = img_rev
        else:
            out[f"{name}_image"] = href.render_splat(sc.xyzw, boxes, case["ppl"], p, tf, hc.W, hc.H)
    path = os.path.join(ROOT, "tests", "golden", "hlsl_ref.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, len(out), "arrays")


def main():
    ref = reference_tree()
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), f"REF={ref}"], check=True)
    write_hlsl_golden()
    L = ctypes.CDLL(REF)
    ull = ctypes.c_ulonglong
    L.ref_hilbert_c2i.restype = ull
    L.ref_hilbert_c2i.argtypes = [ctypes.c_uint, ctypes.c_uint, ctypes.POINTER(ull)]
    L.ref_hilbert_i2c.argtypes = [ctypes.c_uint, ctypes.c_uint, ull, ctypes.POINTER(ull)]
    L.ref_get_rng.restype = ctypes.c_uint32
    L.ref_get_rng.argtypes = [ctypes.c_int] + [ctypes.c_uint32] * 4
    L.ref_lcg_step.restype = ctypes.c_uint32
    L.ref_lcg_step.argtypes = [ctypes.c_uint32, ctypes.POINTER(ctypes.c_float)]
    L.ref_murmur_mix.restype = ctypes.c_uint32
    L.ref_murmur_mix.argtypes = [ctypes.c_uint32, ctypes.c_uint32]
    L.ref_murmur_finalize.restype = ctypes.c_uint32
    L.ref_murmur_finalize.argtypes = [ctypes.c_uint32]

    rng = np.random.default_rng(20240607)
    out = {"source": "reference hilbert.h / rng.h compiled unchanged (oracle/ref_shim.cpp)"}

    # every 4-bit 3-D coordinate (the whole 2^12 grid) and random 16-bit coordinates,
    # including the coordinate-equals-2^16 overflow the reference produces at the domain max
    c2i = []
    for x in range(16):
        for y in range(16):
            for z in range(16):
                c = (ull * 3)(x, y, z)
                c2i.append([3, 4, x, y, z, int(L.ref_hilbert_c2i(3, 4, c))])
    for _ in range(4000):
        c = [int(v) for v in rng.integers(0, 65536, size=3)]
        if rng.random() < 0.15:
            c[int(rng.integers(0, 3))] = 65536
        a = (ull * 3)(*c)
        c2i.append([3, 16] + c + [int(L.ref_hilbert_c2i(3, 16, a))])
    for c in ([0, 0, 0], [65535, 65535, 65535], [65536, 65536, 65536], [65536, 0, 0], [0, 65536, 0],
              [0, 0, 65536], [32768, 32768, 32768]):
        a = (ull * 3)(*c)
        c2i.append([3, 16] + c + [int(L.ref_hilbert_c2i(3, 16, a))])
    out["hilbert_c2i"] = c2i

    i2c = []
    for _ in range(1000):
        idx = int(rng.integers(0, 2 ** 48, dtype=np.uint64))
        a = (ull * 3)()
        L.ref_hilbert_i2c(3, 16, idx, a)
        i2c.append([3, 16, idx, int(a[0]), int(a[1]), int(a[2])])
    out["hilbert_i2c"] = i2c

    seeds = []
    for (px, py, w, frame) in [(0, 0, 512, 0), (511, 511, 512, 0), (0, 0, 512, 1), (511, 511, 512, 1),
                               (1919, 1079, 1920, 65535), (123, 45, 1920, 7), (0, 0, 1, 0)]:
        s = int(L.ref_get_rng(frame, px, py, w, 1))
        st = s
        seq, fl = [], []
        for _ in range(8):
            f = ctypes.c_float()
            st = int(L.ref_lcg_step(st, ctypes.byref(f)))
            seq.append(st)
            fl.append(float(f.value))
        seeds.append({"pixel": [px, py], "width": w, "frame": frame, "seed": s, "states": seq,
                      "floats": [float(np.float32(v)).hex() for v in fl]})
    out["rng"] = seeds
    mix = []
    for _ in range(200):
        h, k = (int(v) for v in rng.integers(0, 2 ** 32, size=2, dtype=np.uint64))
        mix.append([h, k, int(L.ref_murmur_mix(h, k)), int(L.ref_murmur_finalize(h))])
    out["murmur"] = mix
    path = os.path.join(ROOT, "tests", "golden", "hilbert_rng.json")
    with open(path, "w") as f:
        json.dump(out, f)
    print("wrote", path)


if __name__ == "__main__":
    main()
