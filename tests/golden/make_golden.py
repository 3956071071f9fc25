"""Generate the golden vectors in tests/golden/ from the reference's own code.

Runs in a container that has the reference tree: oracle/Makefile compiles the reference's
hilbert.h and rng.h unchanged into oracle/_ref/libaarbf_ref.so; this script calls it and writes
hilbert_rng.json. The CPU tests pin the oracle's restatements against these vectors (on machines
without the reference tree) and against the live reference library (where it exists).

    python tests/golden/make_golden.py
"""
import ctypes
import json
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
REF = os.path.join(ROOT, "oracle", "_ref", "libaarbf_ref.so")


def main():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
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
