#!/usr/bin/env python
"""Benchmark: Mrays/s of attribute-aware Gaussian-RBF particle-volume rendering on B200.

Workload (one step): the 10M-particle scene of the benchmark configuration (64 anisotropic
Gaussian clusters + 5% uniform background, radii log-uniform [0.002, 0.02], 256-entry RGBA fp32
transfer function with 4 opacity peaks), delta tracking with one shadow ray per sample,
1920x1080, 16 samples per pixel, step unit 0.001 (0.5 x min radius), density scale 50.
A ray is one primary camera sample including its shadow ray. Inputs are larger than L2 (the
particle records and BVH nodes alone exceed 1 GB), so no L2 flush is inserted between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value      : rays of all ranks / max-over-ranks device time of the K timed steps (scene resident)
e2e        : the same metric through the public C ABI with host buffers: per step the particle
             upload (pinned host -> device), the build (Hilbert sort + LBVH), the render and the
             image read-back are inside the timed region
roofline   : algorithmic bytes of one render launch / measured launch time, against the measured
             HBM copy bandwidth. Algorithmic bytes: 20 B per particle whose sphere meets a
             traversed ray segment (16 B record + 4 B radius) + 32 B per BVH node visit of those
             segment queries + 48 B per sample of framebuffer traffic (accum read and write, image
             write: spp x W x H x 48 B). The same figure with this library's own 64-byte nodes and
             per-pixel framebuffer traffic is reported beside it.
cpu_baseline: the oracle (C restatement of the reference's device code, OpenMP over pixels) on a
             bounded, evenly spread sample of the same frame's pixels, on this host's cores; the
             GPU renders the same frame at the same spp and its pixels in the sampled tiles are
             compared bit for bit with the oracle's ("parity")
Multi-GPU: replicas (each rank renders its own frames of the replicated scene; weak scaling).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "attribute-aware-rbfs_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "Mrays/s at 10M particles 1080p vs plain & CPU at equal RMSE; fwd+bwd ms/iter"
UNIT = "Mrays/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--particles", type=int, default=10_000_000)
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--spp", type=int, default=16)
    ap.add_argument("--unit", type=float, default=0.001)
    ap.add_argument("--density-scale", type=float, default=50.0)
    ap.add_argument("--traversal", type=int, default=0, help="0 staged, 1 point query")
    ap.add_argument("--ppl", type=int, default=8, help="particles per BVH leaf")
    ap.add_argument("--estimator", default="majorant", choices=["majorant", "plain"],
                    help="delta tracking with per-bin majorants, or with the global majorant 1/unit")
    ap.add_argument("--bin", type=float, default=16.0, help="majorant bin length in units")
    ap.add_argument("--alpha-floor", type=float, default=1.0 / 255.0,
                    help="opacity below this is transparent (1/255: the 8-bit transfer-function resolution)")
    ap.add_argument("--cap", type=int, default=0,
                    help="staged candidates per ray: 256/512/1024 per warp (majorant), 0 = default")
    ap.add_argument("--stage-bins", type=int, default=0,
                    help="bins covered by a ray's first staging (1..64), 0 = default; tuning only")
    ap.add_argument("--plain-spp", type=int, default=1, help="spp of the plain-estimator comparison (0: skip)")
    ap.add_argument("--marching-spp", type=int, default=1, help="spp of the stochastic-marching variant")
    ap.add_argument("--taa-frames", type=int, default=64, help="frames of the jittered splat + TAA sequence")
    ap.add_argument("--no-variants", action="store_true", help="skip the marching / splat / TAA lines")
    ap.add_argument("--rmse-crop", type=int, default=32, help="side of the centre crop of the RMSE study (0: skip)")
    ap.add_argument("--rmse-ref-spp", type=int, default=256, help="spp of the FP64 oracle reference of the crop")
    ap.add_argument("--diff-views", type=int, default=32,
                    help="views of the differentiable-form measurement (1M particles, 512x512, 8 spp; 0: skip)")
    ap.add_argument("--batch-scenes", type=int, default=64,
                    help="scenes of the batched-rendering measurement (0: skip)")
    ap.add_argument("--precision-particles", type=int, default=100_000_000,
                    help="particles of the fp32/FP16 storage comparison (0: skip)")
    ap.add_argument("--series-frames", type=int, default=6, help="frames of the series-playback measurement (0: skip)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU-baseline sample time")
    return ap.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")),
            int(os.environ.get("WORLD_SIZE", "1")))


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_figures(args):
    """ncu figures of the render kernel from the committed summary (profiles/render_traffic.txt):
    DRAM bytes of one full launch of the default workload, L2 bytes per ray and the L2 throughput
    of the small-case capture. Empty for any other workload."""
    default = (args.particles, args.width, args.height, args.spp, args.estimator) == (
        10_000_000, 1920, 1080, 16, "majorant")
    out = {}
    if not default:
        return out
    try:
        with open(os.path.join(ROOT, "profiles", "render_traffic.txt")) as f:
            for line in f:
                if ":" in line and not line.startswith("#"):
                    k, v = line.split(":", 1)
                    out[k.strip()] = float(v)
    except Exception:
        pass
    return out


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.idx)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for k, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(k)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_scene(args):
    from aarbf import scenes
    sc = scenes.config_clusters(args.particles, seed=2)
    cm, rm, dm = scenes.tf_four_peaks()
    return sc, (cm, rm, dm)


def domain_of(xyzw):
    d = np.empty(8, np.float32)
    d[0:3] = xyzw[:, :3].min(0)
    d[3:6] = xyzw[:, :3].max(0)
    d[6] = xyzw[:, 3].min()
    d[7] = xyzw[:, 3].max()
    return d


def params_for(args, dom, rmax, frame_id=0, estimator=None, spp=None, camera_fn=None):
    from aarbf import scenes
    est = estimator or args.estimator
    rp = scenes.native_params(scenes.orbit_camera(), args.width, args.height, rmax, args.unit,
                              args.density_scale, dom, spp=spp or args.spp, frame_id=frame_id,
                              traversal=args.traversal, majorant=(est == "majorant"),
                              bin_length=args.bin * args.unit, camera_fn=camera_fn)
    rp.candidate_cap = args.cap if est == "majorant" else 0
    rp.stage_bins = args.stage_bins
    return rp


def cpu_scene(args, sc, tf, dom, rbf_radius):
    import oracle.oracle as orc
    return orc.build_scene(sc.xyzw, sc.radii, dom, args.ppl, rbf_radius, tf, args.alpha_floor)[0]


def cpu_sample(args, scene, rp, target_s, threads, out=None):
    """Render an evenly spread sample of the frame's pixels with the oracle at 1 spp; returns
    (Mrays/s, rays, seconds, description). out (optional dict) receives the oracle's image and
    the sampled tiles (x0, y0, size) of the last, timed pass."""
    import oracle.oracle as orc
    p = orc.params_from(rp)
    p.spp = 1
    W, H = args.width, args.height
    tile = 8
    accum = np.zeros((H, W, 4), np.float32)
    image = np.zeros((H, W, 4), np.float32)

    def run(ntiles_side):
        xs = np.linspace(0, W - tile, ntiles_side).astype(int)
        ys = np.linspace(0, H - tile, ntiles_side).astype(int)
        accum[:] = 0.0
        t0 = time.perf_counter()
        for y in ys:
            for x in xs:
                scene.render(p, W, H, accum=accum, threads=threads, image=image,
                             region=(int(x), int(x) + tile, int(y), int(y) + tile))
        dt = time.perf_counter() - t0
        return len(xs) * len(ys) * tile * tile, dt, [(int(x), int(y), tile) for y in ys for x in xs]

    rays, dt, tiles = run(4)
    side = 4
    while dt < target_s * 0.4 and side < 64:
        side = min(64, int(side * max(1.5, (target_s / max(dt, 1e-3)) ** 0.5)))
        rays, dt, tiles = run(side)
    desc = (f"{side}x{side} tiles of {tile}x{tile} pixels spread evenly over the {W}x{H} frame, 1 spp "
            f"({rays} rays) of the same scene, camera and estimator")
    if out is not None:
        out["image"], out["tiles"] = image, tiles
    return rays / dt / 1e6, rays, dt, desc


def tile_parity(gpu_image, cpu):
    """Bit-for-bit comparison of the GPU frame with the oracle on the oracle's sampled tiles."""
    g = np.ascontiguousarray(gpu_image).view(np.uint32)
    o = np.ascontiguousarray(cpu["image"]).view(np.uint32)
    pixels = mism = 0
    for x, y, t in cpu["tiles"]:
        a, b = g[y:y + t, x:x + t], o[y:y + t, x:x + t]
        pixels += t * t
        mism += int((a != b).any(axis=-1).sum())
    return {"pixels": pixels, "mismatches": mism, "spp": 1,
            "compared": "every float of the image in the CPU baseline's tiles, GPU frame vs oracle, bit for bit"}


def run_reference(args):
    """--impl reference: the oracle port of the reference's device code on the host cores."""
    rank, _, world = dist_env()
    if world > 1 and rank != 0:
        return
    import oracle.oracle as orc
    threads = os.cpu_count() or 1
    sc, tf = make_scene(args)
    dom = domain_of(sc.xyzw)
    rp = params_for(args, dom, float(sc.radii.max()), camera_fn=orc.camera)  # no product library here
    scene = cpu_scene(args, sc, tf, dom, rp.rbf_radius)
    vals = []
    for k in range(args.warmup + args.steps):
        v, rays, dt, desc = cpu_sample(args, scene, rp, max(2.0, args.cpu_seconds / 2), threads)
        if k >= args.warmup:
            vals.append(v)
    value = statistics.median(vals)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "dtype": "f32",
        "data": "synthetic (seeded generator at the benchmark configuration's sizes and distributions)",
        "config": config_dict(args),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": desc},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "vs_baseline": None,
    }
    print(json.dumps(line), flush=True)


def traversal_label(args):
    if args.traversal == 1:
        return "point queries per step (thread per sample)"
    if args.traversal == 2:
        return "staged segments (thread per sample)"
    return "ray per warp (warp-wide BVH frontier, shared candidate lists)"


def config_dict(args):
    return {"workload": f"clusters_{args.particles // 1_000_000}M_{args.width}x{args.height}_{args.spp}spp_delta_tracking",
            "particles": args.particles, "width": args.width, "height": args.height, "spp": args.spp,
            "estimator": ("delta tracking with per-bin majorants (bin %g units) + shadow ray" % args.bin
                          if args.estimator == "majorant" else
                          "delta tracking with the global majorant 1/unit + shadow ray"),
            "unit": args.unit, "density_scale": args.density_scale,
            "traversal": traversal_label(args), "particles_per_leaf": args.ppl,
            "alpha_floor": args.alpha_floor, "candidate_cap": args.cap, "stage_bins": args.stage_bins,
            "l2": "inputs_larger_than_l2", "parallelism": f"replicas{args.gpus}"}


def crop_params(rp, W, H, x0, y0, cw, ch):
    """Parameters whose cw x ch frame shows pixels [x0, x0+cw) x [y0, y0+ch) of the W x H frame."""
    import copy
    q = copy.copy(rp)
    d00, du, dv = (np.asarray(v, np.float64) for v in (rp.cam_dir00, rp.cam_du, rp.cam_dv))
    q.cam_dir00 = tuple(float(x) for x in np.float32(d00 + (x0 / W) * du + (y0 / H) * dv))
    q.cam_du = tuple(float(x) for x in np.float32(du * (cw / W)))
    q.cam_dv = tuple(float(x) for x in np.float32(dv * (ch / H)))
    return q


def rmse_study(ctx, args, scene, dom, rmax, threads, stream):
    """RMSE on the centre crop against the FP64 oracle (the same volume model in double precision,
    an independent random stream, rmse_ref_spp samples): the majorant and the plain GPU estimators
    at the benchmark's spp."""
    import torch
    import oracle.oracle as orc
    W, H, c = args.width, args.height, args.rmse_crop
    x0, y0 = W // 2 - c // 2, H // 2 - c // 2
    p64 = orc.params_from(params_for(args, dom, rmax))
    t0 = time.perf_counter()
    ref = scene.render_f64(p64, W, H, (x0, x0 + c, y0, y0 + c), args.rmse_ref_spp, threads=threads)
    t_ref = time.perf_counter() - t0
    out = {"crop": [x0, y0, c, c], "spp": args.spp,
           "reference": f"FP64 oracle, {args.rmse_ref_spp} spp, {threads} threads, {t_ref:.1f} s",
           "reference_mean": float(ref.mean()), "rmse": {}}
    imgs = {}
    for est in ("majorant", "plain", "majorant_fp16"):
        if est == "majorant_fp16":  # the same scene in the FP16 storage form
            ctx.set_storage(True)
            ctx.build(rmax, args.ppl, stream=stream.cuda_stream)
        q = crop_params(params_for(args, dom, rmax, estimator=est.split("_")[0], spp=args.spp), W, H, x0, y0, c, c)
        acc = torch.zeros((c, c, 4), dtype=torch.float32, device="cuda")
        img = torch.zeros_like(acc)
        ctx.render(q, c, c, acc, img, stream=stream.cuda_stream)
        ctx.sync(stream.cuda_stream)
        g = img[..., :3].cpu().numpy().astype(np.float64)
        imgs[est] = g
        out["rmse"][est + "_gpu"] = float(np.sqrt(((g - ref) ** 2).mean()))
    ctx.set_storage(False)
    ctx.build(rmax, args.ppl, stream=stream.cuda_stream)
    # storage rounding alone: FP16 against fp32 form with the same random streams
    out["rmse_fp16_vs_fp32_same_stream"] = float(np.sqrt(((imgs["majorant_fp16"] - imgs["majorant"]) ** 2).mean()))
    return out


def precision_timing(args, dev, stream):
    """The precision configuration: precision_particles particles of the benchmark distribution,
    1920x1080, 4 spp, majorant tracking, in the fp32 and the FP16 storage form (same random
    streams); CUDA events on the stream, one untimed render first, then the mean of two. Reports
    Mrays/s of each form and the RMSE between their images."""
    import torch
    import aarbf
    from aarbf import scenes
    sc = scenes.config_clusters(args.precision_particles, seed=2)
    cm, rm, dm = scenes.tf_four_peaks()
    dom = domain_of(sc.xyzw)
    rmax = float(sc.radii.max())
    W, H, S = args.width, args.height, 4
    ctx = aarbf.Context(dev.index or 0)
    sp = stream.cuda_stream
    ctx.set_domain(dom)
    ctx.set_transfer_functions_f32(cm, rm, dm)
    ctx.set_opacity_floor(args.alpha_floor)
    xyzw = torch.from_numpy(sc.xyzw).pin_memory()
    radii = torch.from_numpy(sc.radii).pin_memory()
    del sc
    out = {"particles": args.precision_particles, "width": W, "height": H, "spp": S}
    imgs = {}
    for form in ("fp32", "fp16"):
        ctx.set_storage(form == "fp16")
        ctx.set_particles(xyzw, radii, stream=sp)
        ctx.build(rmax, args.ppl, stream=sp)
        acc = torch.zeros((H, W, 4), dtype=torch.float32, device=dev)
        img = torch.zeros_like(acc)
        rp = params_for(args, dom, rmax, spp=S)
        ctx.render(rp, W, H, acc, img, stream=sp)
        ctx.sync(sp)
        ctx.set_kernel_timing(True)
        for _ in range(2):
            ctx.render(rp, W, H, acc, img, stream=sp)
        r_ms, _, k = ctx.kernel_times()
        ctx.set_kernel_timing(False)
        ms = r_ms / k
        out[form] = {"kernel_ms": ms, "mrays_s": W * H * S / ms / 1e3}
        imgs[form] = img[..., :3].double()
    out["rmse_fp16_vs_fp32_same_stream"] = float(((imgs["fp16"] - imgs["fp32"]) ** 2).mean().sqrt())
    out["speedup_fp16"] = out["fp16"]["mrays_s"] / out["fp32"]["mrays_s"]
    # per image against the converged FP64 oracle of the 256 x 256 centre crop (committed fixture
    # made by tests/golden/make_config3_reference.py for this scene)
    fx = os.path.join(ROOT, "tests", "golden", "config3_fp64_crop.npz")
    if os.path.exists(fx):
        ref = np.load(fx)
        if int(ref["particles"]) == args.precision_particles and (int(ref["width"]), int(ref["height"])) == (W, H):
            x0, x1, y0, y1 = (int(v) for v in ref["region"])
            r64 = torch.from_numpy(ref["rgb"].astype(np.float64)).to(dev)
            out["fp64_reference"] = {"spp": int(ref["spp"]), "crop": [x0, y0, x1 - x0, y1 - y0],
                                     "source": "FP64 oracle (CPU), tests/golden/config3_fp64_crop.npz"}
            for form in ("fp32", "fp16"):
                out[form]["rmse_vs_fp64"] = float(((imgs[form][y0:y1, x0:x1] - r64) ** 2).mean().sqrt())
    ctx.close()
    return out


def differentiable_timing(args, dev, stream):
    """The differentiable configuration: 1M particles in 16 clusters, learnable positions, radii,
    attributes and 64-entry RGBA transfer function, diff_views target views of 512x512 at 8 spp,
    expected stochastic marching (unit 0.005 = half the initial radius, density scale 50), L2
    image loss. One iteration = forward of every view + the adjoint; CUDA events on the stream,
    one untimed iteration first, then the mean of two."""
    import torch
    import aarbf
    from aarbf import scenes
    W = H = 512
    n = 1_000_000
    gt, init = scenes.config_differentiable(n)
    dom = np.array([0, 0, 0, 1, 1, 1, 0, 1], np.float32)
    views = [scenes.native_params(cam, W, H, 0.02, 0.005, 50.0, dom, spp=8, frame_id=8 * k, marching=True)
             for k, cam in enumerate(scenes.orbit_views(32)[:args.diff_views])]
    nv = len(views)
    ctx = aarbf.Context(dev.index or 0)
    sp = stream.cuda_stream
    ctx.set_domain(dom)

    def setup(sc):
        nc = len(sc.tf)
        ctx.set_transfer_functions_f32(sc.tf, np.ones(nc, np.float32), np.ones(nc, np.float32))
        ctx.set_particles(np.concatenate([sc.pos, sc.attr[:, None]], 1).astype(np.float32), sc.radii, stream=sp)
        ctx.build(float(sc.radii.max()), 8, stream=sp)

    img = torch.zeros((nv, H, W, 4), dtype=torch.float32, device=dev)
    setup(gt)
    ctx.render_diff_forward(views, W, H, img, stream=sp)
    ctx.sync(sp)
    target = img.clone()
    setup(init)
    g = torch.zeros_like(img)
    gp = torch.zeros((n, 3), device=dev)
    gr = torch.zeros(n, device=dev)
    ga = torch.zeros(n, device=dev)
    gtf = torch.zeros((64, 4), device=dev)
    fwd, tot = [], []
    with torch.cuda.stream(stream):
        for it in range(3):
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record(stream)
            ctx.render_diff_forward(views, W, H, img, stream=sp)
            e1.record(stream)
            torch.sub(img, target, out=g)
            g.mul_(2.0)
            g[..., 3] = 0.0
            ctx.render_diff_backward(views, W, H, g, gp, gr, ga, gtf, stream=sp)
            e2.record(stream)
            torch.cuda.synchronize()
            ctx.sync(sp)
            if it > 0:
                fwd.append(e0.elapsed_time(e1))
                tot.append(e0.elapsed_time(e2))
    ctx.close()
    f, t = sum(fwd) / len(fwd), sum(tot) / len(tot)
    return {"config": f"1M particles, 16 clusters, {nv} views 512x512, 8 spp, expected stochastic marching "
                      "(unit 0.005, density scale 50), L2 image loss; gradients for positions, radii, attributes "
                      "and the 64-entry RGBA transfer function",
            "fwd_ms": f, "fwd_bwd_ms_per_iter": t, "bwd_over_fwd": (t - f) / f, "fwd_bwd_over_fwd": t / f,
            "rays_per_iter": nv * W * H * 8}


def batched_timing(args, dev, stream):
    """The batched configuration: batch_scenes independent scenes, particle counts log-uniform in
    [10k, 5M] from seeded Gaussian-cluster mixtures (8-64 clusters) with their own four-peak
    transfer functions, orbit cameras at random azimuth/elevation, resolutions from
    {256^2, 512^2, 1024^2}, 1-16 spp, majorant tracking. Timed with CUDA events: every scene
    rendered by its own launch in sequence, and all scenes in one persistent launch replayed
    from a CUDA graph with the launch shape the autotuner picked (tuned on a 1-spp copy of the
    batch). The plain estimator (global majorant 1/unit, ray per warp) is timed on the first
    eight scenes at 1 spp."""
    import torch
    import aarbf
    from aarbf import autotune, scenes
    rng = np.random.default_rng(55)
    sp = stream.cuda_stream
    ctxs, params, sizes, accs, imgs = [], [], [], [], []
    particles = 0
    for k in range(args.batch_scenes):
        n = int(np.exp(rng.uniform(np.log(1e4), np.log(5e6))))
        sc = scenes.config_clusters(n, clusters=int(rng.integers(8, 65)), seed=100 + k)
        cm, rm, dm = scenes.tf_four_peaks(256, seed=200 + k)
        dom = domain_of(sc.xyzw)
        c = aarbf.Context(dev.index or 0)
        c.set_domain(dom)
        c.set_transfer_functions_f32(cm, rm, dm)
        c.set_opacity_floor(1.0 / 255.0)
        c.set_particles(sc.xyzw, sc.radii, stream=sp)
        c.build(float(sc.radii.max()), 8, stream=sp)
        res = int(rng.choice([256, 512, 1024]))
        spp = int(rng.integers(1, 17))
        cam = scenes.orbit_camera(azimuth_deg=float(rng.uniform(0, 360)), elevation_deg=float(rng.uniform(-40, 40)))
        params.append(scenes.native_params(cam, res, res, float(sc.radii.max()), args.unit, args.density_scale, dom,
                                           spp=spp, frame_id=k * 16, majorant=True, bin_length=args.bin * args.unit))
        ctxs.append(c)
        sizes.append((res, res))
        accs.append(torch.zeros((res, res, 4), dtype=torch.float32, device=dev))
        imgs.append(torch.zeros((res, res, 4), dtype=torch.float32, device=dev))
        particles += n
    rays = sum(w * h * int(p.spp) for p, (w, h) in zip(params, sizes))
    torch.cuda.synchronize()

    def events():
        return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    # every scene by its own launch, in sequence
    for c, p, (w, h), a, i in zip(ctxs, params, sizes, accs, imgs):
        c.render(p, w, h, a, i, stream=sp)
    torch.cuda.synchronize()
    e0, e1 = events()
    e0.record(stream)
    for c, p, (w, h), a, i in zip(ctxs, params, sizes, accs, imgs):
        c.render(p, w, h, a, i, stream=sp)
    e1.record(stream)
    torch.cuda.synchronize()
    t_seq = e0.elapsed_time(e1)
    ref = [i.clone() for i in imgs]
    # autotune on a 1-spp copy, then one launch in a CUDA graph
    import copy
    proxy = []
    for p in params:
        q = copy.copy(p)
        q.spp = 1
        proxy.append(q)
    # longest first, and each scene's own best first-staging length
    order, scene_bins, _ = autotune.scene_plan(ctxs, params, sizes, accs, imgs, stream)
    o = lambda seq: [seq[i] for i in order]  # noqa: E731

    def with_bins(ps, bins):
        out = []
        for p, b_ in zip(ps, bins):
            q = copy.copy(p)
            q.stage_bins = b_
            out.append(q)
        return out

    # one staging length for the whole batch, or each scene's own: whichever runs the proxy faster
    cap, bins, table = autotune.tune_batch(o(ctxs), o(proxy), o(sizes), o(accs), o(imgs), stream)
    own = o(scene_bins)
    cap_s, _, table_s = autotune.tune_batch(o(ctxs), with_bins(o(proxy), own), o(sizes), o(accs), o(imgs), stream,
                                            stage_bins=None)
    if min(table_s.values()) < min(table.values()):
        cap, bins_list, bins = cap_s, own, "per scene"
        table.update({(c_, "own"): v for (c_, _), v in table_s.items()})
    else:
        bins_list = [bins] * len(own)
    tuned = with_bins(o(params), bins_list)
    proxy_tuned = with_bins(o(proxy), bins_list)
    pb = aarbf.Batch(o(ctxs), proxy_tuned, o(sizes), o(accs), o(imgs))
    bps, smaj, shape_table = autotune.tune_shape(pb, cap, stream)
    pb.close()
    b = aarbf.Batch(o(ctxs), tuned, o(sizes), o(accs), o(imgs))
    b.set_shape(bps, smaj)
    with torch.cuda.stream(stream):
        b.render(cap, stream)
        torch.cuda.synchronize()
        e0, e1 = events()
        e0.record(stream)
        b.render(cap, stream)
        e1.record(stream)
        torch.cuda.synchronize()
        t_direct = e0.elapsed_time(e1)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=stream):
        b.render(cap, stream)
    for i in imgs:
        i.zero_()
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):  # replay on the timed stream
        g.replay()
        torch.cuda.synchronize()
        for i in imgs:
            i.zero_()
        torch.cuda.synchronize()
        e0, e1 = events()
        e0.record(stream)
        g.replay()
        e1.record(stream)
        torch.cuda.synchronize()
    t_graph = e0.elapsed_time(e1)
    same = all(torch.equal(r, i) for r, i in zip(ref, imgs))
    del g
    b.close()
    # the plain estimator on the first eight scenes at 1 spp
    pr = 0
    e0, e1 = events()
    e0.record(stream)
    for c, p, (w, h), a, i in list(zip(ctxs, params, sizes, accs, imgs))[:8]:
        q = copy.copy(p)
        q.spp = 1
        q.flags &= ~aarbf.FLAG_MAJORANT_TRACKING
        c.render(q, w, h, a, i, stream=sp)
        pr += w * h
    e1.record(stream)
    torch.cuda.synchronize()
    t_plain = e0.elapsed_time(e1)
    for c in ctxs:
        c.close()
    return {"scenes": len(ctxs), "particles": particles, "rays": rays,
            "sequential_ms": t_seq, "sequential_mrays_s": rays / t_seq / 1e3,
            "batched_direct_ms": t_direct, "batched_graph_ms": t_graph, "batched_mrays_s": rays / t_graph / 1e3,
            "speedup_vs_sequential": t_seq / t_graph, "images_identical": bool(same),
            "autotuned": {"candidate_cap": cap, "stage_bins": bins,
                          "scene_stage_bins": {str(b_): bins_list.count(b_) for b_ in sorted(set(bins_list))},
                          "blocks_per_sm": bps or "occupancy limit",
                          "ray_order": "sample-major" if smaj else "tile-major",
                          "scene_order": "longest first (1-spp proxy time at the scene's best staging length x spp)",
                          "proxy_ms": {f"{k[0]}/{k[1]}": round(v, 3) for k, v in table.items()},
                          "shape_proxy_ms": {f"{k[0]}/{int(k[1])}": round(v, 3) for k, v in shape_table.items()}},
            "plain_estimator_mrays_s": pr / t_plain / 1e3, "plain_sample": "first 8 scenes, 1 spp",
            "speedup_vs_plain": (rays / t_graph) / (pr / t_plain)}


def build_timing(ctx, args, rmax, n, stream, reps=3):
    """Steady-state rebuild of the benchmark scene (particles already on the device, buffers
    reserved): Hilbert keys, 48-bit radix sort, ordering of equal-key runs, gather + attribute
    normalisation, Karras LBVH, refit, wide-node collapse and the largest-radius reduction.
    Device time between CUDA events on the build's stream (the build's one host read-back of the
    tie flag sits inside it). Algorithmic bytes: n * (20 B record + 8 B key) + 6 radix passes *
    2 * (8 B key + 4 B index) * n + 2 * ceil(n / ppl) nodes * 32 B."""
    import torch
    peak, kind = measured_peak()
    ms = []
    for _ in range(reps + 1):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.build(rmax, args.ppl, stream=stream.cuda_stream)
        e1.record(stream)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    ms = ms[1:]
    nl = -(-n // args.ppl)
    b_alg = n * (20 + 8) + 6 * 2 * 12 * n + 2 * nl * 32
    t = sum(ms) / len(ms)
    ach = b_alg / (t * 1e-3) / 1e9
    return {"ms": t, "ms_runs": ms, "particles": n, "algorithmic_bytes": b_alg, "achieved_gbs": ach,
            "frac": ach / peak, "peak": peak, "peak_kind": kind}


def series_timing(args, sc, xyzw_pin, radii_pin, tf, dom, rmax, dev):
    """Playback of a series of series_frames frames (the benchmark scene drifting by 0.001 per
    frame along x) at 1 spp per frame: the reference's order (upload, build, render, one after
    the other) against the overlapped pipeline of aarbf.streaming (upload and build of frame k+1
    during the render of frame k). Device-event time over the whole series."""
    import torch
    from aarbf import streaming
    W, H = args.width, args.height
    frames = [(xyzw_pin, radii_pin)]
    for k in range(1, args.series_frames):
        x = sc.xyzw.copy()
        x[:, 0] += np.float32(0.001 * k)
        frames.append((torch.from_numpy(x).pin_memory(), radii_pin))
    accum = torch.zeros((H, W, 4), dtype=torch.float32, device=dev)
    imgs = [torch.zeros((H, W, 4), dtype=torch.float32, device=dev) for _ in frames]

    def params(k):
        return params_for(args, dom, rmax, frame_id=k, spp=1)

    out = {"frames": len(frames), "spp": 1}
    ref_imgs = None
    for update in ("build", "refit", "refit_keep_order"):
        sr = streaming.SeriesRenderer(dev.index or 0, dom, tf, rmax, ppl=args.ppl, alpha_floor=args.alpha_floor,
                                      update=update)
        sr.render_series(frames[:2], params, W, H, accum, imgs[:2])  # warm-up (allocations, first builds)
        for overlap in (False, True):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            sr.render_series(frames, params, W, H, accum, imgs, overlap=overlap)
            torch.cuda.synchronize()
            dt = time.perf_counter() - t0
            key = ("overlapped" if overlap else "sequential") + ("" if update == "build" else "_" + update)
            out[key] = {"ms_per_frame": dt / len(frames) * 1e3, "frames_s": len(frames) / dt}
        sr.close()
        if ref_imgs is None:
            ref_imgs = [i.clone() for i in imgs]
        else:
            out[f"images_identical_{update}"] = all(torch.equal(a, b) for a, b in zip(ref_imgs, imgs))
    out["speedup"] = out["overlapped"]["frames_s"] / out["sequential"]["frames_s"]
    out["speedup_refit"] = out["sequential_refit"]["frames_s"] / out["sequential"]["frames_s"]
    out["timing"] = ("host wall clock around the whole series (uploads, builds or refits and renders of every "
                     "frame); refit: the frame is sorted along the curve and refits the first build's topology "
                     "(the reference's update path); refit_keep_order: no sort")
    return out


def variant_timings(ctx, args, dom, rmax, accum, image, stream):
    """The other estimators of the benchmark configuration's frame, each timed with CUDA events
    on the launching stream after one warm-up launch (untimed by the headline figure):
    stochastic marching (blue-noise thresholds), splatting, and a jittered splat + TAA sequence."""
    import torch
    from aarbf import scenes
    W, H = args.width, args.height
    sp = stream.cuda_stream

    def timed(fn, reps):
        fn(-1)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for k in range(reps):
            fn(k)
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    out = {}
    if args.marching_spp > 0:
        def march(k):
            rp = scenes.native_params(scenes.orbit_camera(), W, H, rmax, args.unit, args.density_scale, dom,
                                      spp=args.marching_spp, frame_id=max(k, 0) * args.marching_spp,
                                      traversal=args.traversal, marching=True)
            ctx.render(rp, W, H, accum, image, stream=sp)
        ms = timed(march, 1)
        out["marching"] = {"value": W * H * args.marching_spp / ms / 1e3, "unit": UNIT, "ms": ms,
                           "spp": args.marching_spp,
                           "estimator": "stochastic marching, step 1 unit, blue-noise thresholds + shadow ray"}

    def splat_params(k):
        rp = params_for(args, dom, rmax, frame_id=max(k, 0))
        if k >= 0:
            rp.jitter_x, rp.jitter_y = scenes.halton_jitter(k)
        return rp

    ms = timed(lambda k: ctx.render_splat(splat_params(k), W, H, image, stream=sp), 3)
    out["splat"] = {"value": W * H / ms / 1e3, "unit": "Mpixels/s", "ms_per_frame": ms,
                    "method": "slabs of 1 unit, 15 nearest particles per slab, over-composited"}
    if args.taa_frames > 0:
        prev = torch.zeros_like(image)
        taa = torch.zeros_like(image)
        bgra = torch.zeros((H, W), dtype=torch.int32, device=image.device)
        state = {"prev": prev, "taa": taa}

        def frame(k):
            ctx.render_splat(splat_params(k), W, H, image, stream=sp)
            ctx.taa_resolve(image, state["prev"], state["taa"], bgra, W, H, stream=sp)
            state["prev"], state["taa"] = state["taa"], state["prev"]

        ms = timed(frame, args.taa_frames)
        ms_taa = timed(lambda k: ctx.taa_resolve(image, state["prev"], state["taa"], bgra, W, H, stream=sp),
                       args.taa_frames)
        out["taa_sequence"] = {"frames": args.taa_frames, "ms_per_frame": ms, "value": 1e3 / ms, "unit": "frames/s",
                               "taa_resolve_ms": ms_taa, "taa_resolve_gbs": 52 * W * H / ms_taa / 1e6,
                               "jitter": "Halton(2,3)"}
    return out


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    import torch
    import torch.distributed as dist

    import aarbf
    from aarbf import replicas

    rank, local_rank, world = dist_env()
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    sc, tf = make_scene(args)
    dom = domain_of(sc.xyzw)
    rmax = float(sc.radii.max())
    ctx = aarbf.Context(local_rank)
    stream = torch.cuda.Stream(device=dev)
    sp = stream.cuda_stream
    xyzw_pin = torch.from_numpy(sc.xyzw).pin_memory()
    radii_pin = torch.from_numpy(sc.radii).pin_memory()
    ctx.set_domain(dom)
    ctx.set_transfer_functions_f32(*tf)
    ctx.set_opacity_floor(args.alpha_floor)
    ctx.set_particles(xyzw_pin, radii_pin, stream=sp)
    t_b0 = time.perf_counter()
    ctx.build(rmax, args.ppl, stream=sp)
    build_s = time.perf_counter() - t_b0
    W, H, S = args.width, args.height, args.spp
    accum = torch.zeros((H, W, 4), dtype=torch.float32, device=dev)
    image = torch.zeros((H, W, 4), dtype=torch.float32, device=dev)

    def step(k):
        rp = params_for(args, dom, rmax, frame_id=replicas.frame_id(rank, k, S))
        ctx.render(rp, W, H, accum, image, stream=sp)

    for k in range(args.warmup):
        step(k)
    ctx.sync(sp)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(local_rank)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ctx.set_kernel_timing(True)
    e0.record(stream)
    for k in range(args.steps):
        step(args.warmup + k)
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ctx.sync(sp)
    render_ms, accumulate_ms, timed_renders = ctx.kernel_times()
    ctx.set_kernel_timing(False)
    t = e0.elapsed_time(e1) / 1e3
    tt = torch.tensor([t], device=dev)
    if world > 1:
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        dist.barrier()
    t = float(tt.item())
    rays = W * H * S * args.steps * world
    value = rays / t / 1e6
    ms_per_step = t / args.steps * 1e3

    # roofline accounting: one counted launch (untimed)
    rp = params_for(args, dom, rmax, frame_id=0)
    counts = ctx.render_count(rp, W, H, accum, image, stream=sp)
    parts, visits = counts["segment_particles"], counts["segment_nodes"]
    # 20 B per particle on a traversed segment, 32 B per node visit, 48 B per sample
    alg_bytes = 20 * parts + 32 * visits + 48 * W * H * S
    # the same with this library's 64-byte nodes and per-pixel framebuffer traffic
    alg_bytes_own = 20 * parts + 64 * visits + 48 * W * H
    launch_s = render_ms / 1e3 / max(timed_renders, 1)
    achieved = alg_bytes / launch_s / 1e9
    peak, peak_kind = measured_peak()
    prof = profiled_figures(args)
    traffic = int(prof["dram_bytes_per_launch"]) if "dram_bytes_per_launch" in prof else None
    l2_bytes = int(prof["l2_bytes_per_ray"] * W * H * S) if "l2_bytes_per_ray" in prof else None
    l2_frac = prof["lts_throughput_pct"] / 100 if "lts_throughput_pct" in prof else None

    # the plain estimator (global majorant 1/unit, the reference's tracking loop) on the same frame
    plain = None
    if args.plain_spp > 0 and args.estimator == "majorant":
        rpp = params_for(args, dom, rmax, frame_id=0, estimator="plain", spp=args.plain_spp)
        ctx.render(rpp, W, H, accum, image, stream=sp)
        torch.cuda.synchronize()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        ctx.render(rpp, W, H, accum, image, stream=sp)
        g1.record(stream)
        torch.cuda.synchronize()
        tp = g0.elapsed_time(g1) / 1e3
        plain = {"value": W * H * args.plain_spp / tp / 1e6, "unit": UNIT, "spp": args.plain_spp,
                 "ms": tp * 1e3}

    # end to end through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        host_img = torch.empty((H, W, 4), dtype=torch.float32).pin_memory()
        k_e2e = max(1, min(args.steps, 3))
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for k in range(k_e2e):
            ctx.set_particles(xyzw_pin, radii_pin, stream=sp)
            ctx.build(rmax, args.ppl, stream=sp)
            rpk = params_for(args, dom, rmax, frame_id=(k * S) & 0xFFFF)
            ctx.render(rpk, W, H, accum, image, stream=sp)
            ctx.memcpy(host_img, image, H * W * 16, stream=sp)
        f1.record(stream)
        torch.cuda.synchronize()
        te = f0.elapsed_time(f1) / 1e3
        te_t = torch.tensor([te], device=dev)
        if world > 1:
            dist.all_reduce(te_t, op=dist.ReduceOp.MAX)
        te = float(te_t.item())
        e2e = {"value": W * H * S * k_e2e * world / te / 1e6, "unit": UNIT,
               "h2d_bytes_per_step": int(sc.xyzw.nbytes + sc.radii.nbytes), "d2h_bytes_per_step": H * W * 16,
               "steps": k_e2e, "ms_per_step": te / k_e2e * 1e3}

    variants = None if args.no_variants else variant_timings(ctx, args, dom, rmax, accum, image, stream)
    build = build_timing(ctx, args, rmax, int(sc.xyzw.shape[0]), stream) if world == 1 else None
    series = (series_timing(args, sc, xyzw_pin, radii_pin, tf, dom, rmax, dev)
              if args.series_frames > 1 and world == 1 else None)
    diff = differentiable_timing(args, dev, stream) if args.diff_views > 0 and world == 1 else None
    batched = batched_timing(args, dev, stream) if args.batch_scenes > 0 and world == 1 else None
    precision = precision_timing(args, dev, stream) if args.precision_particles > 0 and world == 1 else None

    cpu = None
    rmse = None
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        scene = cpu_scene(args, sc, tf, dom, rp.rbf_radius)
        sampled = {}
        v, r_cpu, dt, desc = cpu_sample(args, scene, rp, args.cpu_seconds, threads, out=sampled)
        cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": desc,
               "seconds": round(dt, 2)}
        # the GPU's render of the same frame at 1 spp, compared with the oracle on the sampled tiles
        rp1 = params_for(args, dom, rmax, frame_id=0, spp=1)
        accum.zero_()
        ctx.render(rp1, W, H, accum, image, stream=sp)
        ctx.sync(sp)
        parity = tile_parity(image.cpu().numpy(), sampled)
        if args.rmse_crop > 0 and args.rmse_ref_spp > 0:
            rmse = rmse_study(ctx, args, scene, dom, rmax, threads, stream)
            plain_v = plain["value"] if plain else None
            ms = rmse["rmse"]
            if plain_v and ms["majorant_gpu"] > 0:
                rmse["speedup_vs_plain_gpu"] = (value / plain_v) * (ms["plain_gpu"] / ms["majorant_gpu"]) ** 2
            if parity and parity["mismatches"] == 0:
                rmse["speedup_vs_cpu"] = value / v  # same images (parity record): equal RMSE

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded generator at the benchmark configuration's sizes and distributions)",
            "config": config_dict(args),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "l2_bytes_per_launch": l2_bytes, "l2_throughput_frac_small_case": l2_frac,
                         "l2_note": "L2 bytes scaled by rays from the 480x270 2-spp capture of the same "
                                    "kernel; the L2 throughput fraction is that capture's",
                         "algorithmic_bytes_per_launch": alg_bytes,
                         "bytes_rule": "20 B x particles on traversed segments + 32 B x node visits + "
                                       "48 B x spp x W x H",
                         "achieved_own_layout": alg_bytes_own / launch_s / 1e9,
                         "algorithmic_bytes_own_layout": alg_bytes_own,
                         "own_layout_rule": "20 B x particles + 64 B x node visits (this library's node "
                                            "size) + 48 B x W x H",
                         "particles_on_segments": parts,
                         "node_visits": visits, "kernel": "k_render_warp" if aarbf.uses_warp_kernel(rp)
                         else "k_render", "kernel_ms": launch_s * 1e3,
                         "accumulate_ms": accumulate_ms / max(timed_renders, 1), "kernel_counters": counts},
            "cpu_baseline": cpu, "parity": parity, "e2e": e2e, "clocks": clk, "gpu_launches": 2 * timed_renders,
            "build_ms": build_s * 1e3, "build": build, "plain_estimator": plain, "variants": variants, "equal_rmse": rmse,
            "differentiable": diff, "batched": batched, "precision": precision, "series": series,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
