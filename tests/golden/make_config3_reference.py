"""The converged reference of the precision configuration: the FP64 oracle (the native volume model
in double precision, an independent random stream) at 1024 samples per pixel on the 256 x 256
centre crop of the 1920 x 1080 frame of the 100M-particle scene (64 anisotropic clusters + 5 %
background, radii log-uniform [0.002, 0.02], four-peak transfer function, density scale 50, the
benchmark's orbit camera). bench.py's precision measurement reports the RMSE of the fp32 and FP16
storage forms' 4-spp renders against it.

    python tests/golden/make_config3_reference.py [--particles N] [--spp S] [--threads T]

Writes tests/golden/config3_fp64_crop.npz (float32 RGB and the settings). CPU only; with 8 threads
the default settings take about 40 minutes.
"""
import argparse
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
for p in (ROOT, os.path.join(ROOT, "attribute-aware-rbfs_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

W, H, CROP = 1920, 1080, 256


def crop_region():
    x0, y0 = W // 2 - CROP // 2, H // 2 - CROP // 2
    return x0, x0 + CROP, y0, y0 + CROP


def main():
    import oracle.oracle as orc
    from aarbf import scenes
    ap = argparse.ArgumentParser()
    ap.add_argument("--particles", type=int, default=100_000_000)
    ap.add_argument("--spp", type=int, default=1024)
    ap.add_argument("--threads", type=int, default=0)
    args = ap.parse_args()
    t0 = time.time()
    sc = scenes.config_clusters(args.particles, seed=2)
    tf = scenes.tf_four_peaks()
    dom = np.empty(8, np.float32)
    dom[0:3], dom[3:6] = sc.xyzw[:, :3].min(0), sc.xyzw[:, :3].max(0)
    dom[6], dom[7] = sc.xyzw[:, 3].min(), sc.xyzw[:, 3].max()
    rmax = float(sc.radii.max())
    scene = orc.build_scene(sc.xyzw, sc.radii, dom, 8, rmax, tf, 1.0 / 255.0)[0]
    del sc
    t1 = time.time()
    rp = scenes.native_params(scenes.orbit_camera(), W, H, rmax, 0.001, 50.0, dom, spp=4, majorant=True,
                              bin_length=16 * 0.001, camera_fn=orc.camera)
    ref = scene.render_f64(orc.params_from(rp), W, H, crop_region(), args.spp, threads=args.threads)
    t2 = time.time()
    path = os.path.join(ROOT, "tests", "golden", "config3_fp64_crop.npz")
    np.savez_compressed(path, rgb=ref.astype(np.float32), particles=args.particles, spp=args.spp,
                        region=np.array(crop_region()), width=W, height=H)
    print(f"wrote {path}: build {t1 - t0:.0f} s, FP64 {args.spp} spp {t2 - t1:.0f} s, mean {ref.mean():.5f}")


if __name__ == "__main__":
    main()
