#!/usr/bin/env python
"""F3D registrations/s on the brain-MR-sized workload.

Workload: one plain single-pair F3D registration of a 182x218x182 float32, 1 mm 3-class
phantom pair (floating = reference warped by a seeded 5 mm FFD with N(0, 3 mm) control
displacements), 3 pyramid levels, 300 counted iterations at the finest level (the reference's
budget doubling per coarser level: 300/600/1200), NMI with 64 bins, bending energy 0.005, 5 mm
control spacing, linear interpolation, NaN padding. A "step" is one whole registration.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
  python bench.py --mode batched   # many uneven pairs at once vs the same pairs one by one
  python bench.py --mode served    # open-loop Poisson requests: p50/p95/p99 latency

On one GPU the default line also carries the metric's batched and served figures (a 64-pair
--mode batched run of config 3, a 128-pair run of 64^3 pairs and a two-rate --mode served run,
keys "batched", "batched_speedup_vs_plain", "batched_64cubed" and "served"), and one
registration of the workload by NiftyReg's own reg_f3d on the B200 platform ("platform_plugin");
--no-extras skips them.

Under torchrun every rank registers its own pair (replicas: registrations are independent) and
rank 0 prints one JSON line with the whole-job rate and the slowest rank's device time.
"""
from __future__ import annotations

import argparse
import contextlib
import gc
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "F3D registrations/s & p99 latency, batched/served vs plain GPU, |ΔNMI|≤1e-4"
SHAPE = (182, 218, 182)        # (nz, ny, nx)
LEVELS, MAXIT, BE, BINS, SPACING = 3, 300, 0.005, 64, -5.0
WORKLOAD = ("plain single-pair F3D, 182x218x182 float32 1 mm brain-MR-like 3-class phantom, "
            "3 levels, 300 counted iterations at the finest level (600/1200 coarser), NMI 64 bins, "
            "BE 0.005, 5 mm control spacing")
L2_FLUSH_BYTES = 256 << 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--floating-texture", type=int, default=1,
                    help="1: the registrations sample the floating image through its layered texture; 0: loads")
    ap.add_argument("--no-extras", action="store_true",
                    help="plain mode: skip the shortened batched and served runs attached to the line")
    ap.add_argument("--mode", choices=["plain", "batched", "served", "warp", "f3d2", "ct"], default="plain")
    ap.add_argument("--reference-platform", choices=["cpu", "cuda"], default="cpu",
                    help="--impl reference: the reference's CPU path (default) or its own CUDA platform")
    ap.add_argument("--pairs", type=int, default=64, help="batched: number of pairs")
    ap.add_argument("--ct-group", type=int, default=4, help="ct: pairs registered together at most in the batch of 4")
    ap.add_argument("--concurrency", type=int, default=16, help="batched/served: concurrent registrations")
    ap.add_argument("--grad-percent", type=int, default=50,
                    help="batched: run a level's gradient stage once this share of the active pairs waits for it")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--batch-only", action="store_true", help="batched: skip the one-by-one run (profiling)")
    ap.add_argument("--kernel-timing", action="store_true",
                    help="batched: run the batch once more driven from the host with per-kernel CUDA events")
    ap.add_argument("--requests", type=int, default=2000,
                    help="served: requests over the whole sweep, split across the rates in proportion to "
                         "the rate (every rate runs for about the same time)")
    ap.add_argument("--rates", default="1,2,5,10,20,30,40,50", help="served: Poisson arrival rates (requests/s)")
    ap.add_argument("--slots", type=int, default=2, help="served: workers (groups registered at once)")
    ap.add_argument("--max-group", type=int, default=16,
                    help="served: requests registered together at most during the rate sweep")
    ap.add_argument("--full-reference", action="store_true",
                    help="f3d2: time one full-budget reference registration instead of a 1/10 sample")
    ap.add_argument("--burst", type=int, default=300,
                    help="served: requests of the capacity run, submitted at once after the rate sweep")
    ap.add_argument("--burst-group", type=int, default=64, help="served: requests registered together at most "
                    "in the capacity run")
    ap.add_argument("--shape", default=None, help="kernel-only mode: nz,ny,nx of the volume (default: the workload's)")
    ap.add_argument("--group-mb", type=int, default=None,
                    help="batched/served: finest-level image MB a group of pairs may hold (default: the library's)")
    ap.add_argument("--batch-shapes", default=None,
                    help="batched: sizes to draw from, 'nz,ny,nx;nz,ny,nx;...' (default: config 3's four sizes)")
    ap.add_argument("--kernel", choices=["objective", "gradient", "velocity", "compose", "ops"], default=None,
                    help="profiling mode: run only `--steps` fused evaluations at the finest level "
                         "of the workload (for ncu captures); prints per-launch device times")
    return ap.parse_args()


def run_velocity_only(args, shape):
    """`--steps` exponentiations of a velocity grid (F3D2: flow, scaling, 6 squarings) or
    `--steps` single compositions, on a field of the workload's shape: a 5 mm velocity grid with
    N(0, 3 mm) node displacements over the volume (one node of margin). Per-launch device times."""
    import torch
    import niftyreg_b200 as nrb

    nz, ny, nx = shape
    dim, pix = (nx, ny, nz), (1.0, 1.0, 1.0)
    eye = nrb.identity_header(pix)
    cdim = [int(np.ceil(v / 5.0 + 3)) + 1 for v in dim]
    cxyz = nrb.identity_header((5.0, 5.0, 5.0), (-5.5, -5.5, -5.5))
    rng = np.random.default_rng(args.seed)
    cx, cy, cz = cdim
    zz, yy, xx = np.meshgrid(np.arange(cz), np.arange(cy), np.arange(cx), indexing="ij")
    ident = np.concatenate([(5.0 * v - 5.5).ravel() for v in (xx, yy, zz)]).astype(np.float32)
    vel = torch.from_numpy(ident + rng.normal(0, 3.0, ident.size).astype(np.float32)).cuda()
    g = nrb.make_geometry(dim, pix, eye, dim, pix, eye, cdim, (5.0, 5.0, 5.0), cxyz)
    n = nx * ny * nz
    d = torch.empty(3 * n, dtype=torch.float32, device="cuda")
    nrb.get_def_field_from_velocity_grid(g, vel, 6, d)
    torch.cuda.synchronize()
    pos = d.clone()
    nrb.timing_enable(True)
    for _ in range(args.steps):
        if args.kernel == "velocity":
            nrb.get_def_field_from_velocity_grid(g, vel, 6, d)
        else:
            pos.copy_(d)
            nrb.def_field_compose(dim, eye, d, pos)
    torch.cuda.synchronize()
    out = {k: nrb.timing_read(k) for k in ("f3d2_velocity", "f3d2_compose")}
    nrb.timing_enable(False)
    print(json.dumps({"mode": f"kernel-only {args.kernel}", "voxels": n, "nodes": int(np.prod(cdim)),
                      "timing": {k: {"launches": v[0], "avg_us": (v[1] / v[0] * 1e3) if v[0] else None,
                                     "GBps": (v[2] / (v[1] / 1e3) / 1e9) if v[1] and v[2] else None}
                                 for k, v in out.items()}}))
    return 0


def run_kernel_only(args):
    """A short, deterministic launch sequence of one fused evaluation on the finest level of the
    workload (rescaled images, 5 mm grid with N(0, 3 mm) displacements)."""
    import torch
    import niftyreg_b200 as nrb
    from niftyreg_b200 import phantom

    torch.cuda.set_device(0)
    nrb.build()
    shape = tuple(int(v) for v in args.shape.split(",")) if args.shape else SHAPE
    if args.kernel in ("velocity", "compose"):
        return run_velocity_only(args, shape)
    if args.kernel == "ops":
        return run_ops_only(args, shape)
    pair = phantom.brain_pair(shape, seed=args.seed)
    nz, ny, nx = shape
    dim, pix = (nx, ny, nz), (1.0, 1.0, 1.0)
    cdim, cpix, cxyz = nrb.control_grid_header(dim, pix, (5.0, 5.0, 5.0))
    rng = np.random.default_rng(args.seed)
    cx, cy, cz = cdim
    zz, yy, xx = np.meshgrid(np.arange(cz), np.arange(cy), np.arange(cx), indexing="ij")
    ident = np.concatenate([(5.0 * v - 5.0).ravel() for v in (xx, yy, zz)]).astype(np.float32)
    cpp = ident + rng.normal(0, 3.0, ident.size).astype(np.float32)
    g = nrb.make_geometry(dim, pix, nrb.identity_header(pix), dim, pix, nrb.identity_header(pix), cdim, cpix, cxyz)
    ref = torch.from_numpy(pair.reference.ravel().copy()).cuda()
    flo = torch.from_numpy(pair.floating.ravel().copy()).cuda()
    n = nx * ny * nz
    nrb.intensity_rescale(ref, n, 2.0, BINS + 1.0)
    nrb.intensity_rescale(flo, n, 2.0, BINS + 1.0)
    cppd = torch.from_numpy(cpp).cuda()
    ws, nmi = nrb.Workspace(g), nrb.Nmi(BINS + 4, BINS + 4)
    vg = torch.empty(3 * n, dtype=torch.float32, device="cuda")
    node = torch.empty(ident.size, dtype=torch.float32, device="cuda")
    nrb.timing_enable(True)
    for _ in range(args.steps):
        if args.kernel == "objective":
            nrb.f3d_objective(ws, nmi, ref, flo, cppd, 1 - BE, BE)
        else:
            nrb.f3d_gradient(ws, nmi, ref, flo, cppd, vg, node, 1 - BE, BE)
    torch.cuda.synchronize()
    out = {k: nrb.timing_read(k) for k in ("objective", "gradient", "finalize", "conv", "be_value", "be_gradient")}
    nrb.timing_enable(False)
    print(json.dumps({"mode": f"kernel-only {args.kernel}", "voxels": n, "nodes": int(np.prod(cdim)),
                      "timing": {k: {"launches": v[0], "avg_us": (v[1] / v[0] * 1e3) if v[0] else None,
                                     "GBps": (v[2] / (v[1] / 1e3) / 1e9) if v[1] else None}
                                 for k, v in out.items()}}))
    return 0


def run_ops_only(args, shape):
    """Each standalone entry point of the hot path (the staged, per-`Compute`-call kernels a
    platform binding calls; the fused evaluation is --kernel objective / gradient) once per
    repetition on the workload's finest level: rescaled brain-like pair, 5 mm grid with
    N(0, 3 mm) displacements. CUDA events on the launching stream around each call, a 256 MiB
    buffer written between calls (inputs larger than L2 or flushed), median of --steps calls
    after --warmup; achieved = the op's algorithmic bytes / its device time."""
    import torch
    import ctypes
    import niftyreg_b200 as nrb
    from niftyreg_b200 import phantom

    pair = phantom.brain_pair(shape, seed=args.seed)
    nz, ny, nx = shape
    dim, pix = (nx, ny, nz), (1.0, 1.0, 1.0)
    cdim, cpix, cxyz = nrb.control_grid_header(dim, pix, (5.0, 5.0, 5.0))
    rng = np.random.default_rng(args.seed)
    cx, cy, cz = cdim
    zz, yy, xx = np.meshgrid(np.arange(cz), np.arange(cy), np.arange(cx), indexing="ij")
    ident = np.concatenate([(5.0 * v - 5.0).ravel() for v in (xx, yy, zz)]).astype(np.float32)
    cpp = ident + rng.normal(0, 3.0, ident.size).astype(np.float32)
    g = nrb.make_geometry(dim, pix, nrb.identity_header(pix), dim, pix, nrb.identity_header(pix), cdim, cpix, cxyz)
    n, c = nx * ny * nz, int(np.prod(cdim))
    ref = torch.from_numpy(pair.reference.ravel().copy()).cuda()
    flo = torch.from_numpy(pair.floating.ravel().copy()).cuda()
    raw = flo.clone()
    nrb.intensity_rescale(ref, n, 2.0, BINS + 1.0)
    nrb.intensity_rescale(flo, n, 2.0, BINS + 1.0)
    cppd = torch.from_numpy(cpp).cuda()
    ws, nmi = nrb.Workspace(g), nrb.Nmi(BINS + 4, BINS + 4)
    d = torch.empty(3 * n, dtype=torch.float32, device="cuda")
    w = torch.empty(n, dtype=torch.float32, device="cuda")
    wg = torch.empty(3 * n, dtype=torch.float32, device="cuda")
    vg = torch.empty(3 * n, dtype=torch.float32, device="cuda")
    node = torch.empty(3 * c, dtype=torch.float32, device="cuda")
    field = torch.empty(3 * n, dtype=torch.float32, device="cuda")
    img = torch.empty(n, dtype=torch.float32, device="cuda")
    obj = torch.empty(16, dtype=torch.float64, device="cuda")  # an nrb_objective on the device
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    st = torch.cuda.current_stream()
    sp = ctypes.c_void_p(st.cuda_stream)
    L = nrb.lib()
    nrb.get_deformation_field(g, cppd, d, stream=st)
    nrb.resample_image(g, flo, d, w, stream=st)
    nrb.get_image_gradient(g, flo, d, wg, stream=st)
    ops = [
        ("deformation_field (a1)", 12.0 * n + 12.0 * c, lambda: nrb.get_deformation_field(g, cppd, d, stream=st)),
        ("resample_linear (a2)", 20.0 * n, lambda: nrb.resample_image(g, flo, d, w, stream=st)),
        ("image_gradient (a3)", 28.0 * n, lambda: nrb.get_image_gradient(g, flo, d, wg, stream=st)),
        ("intensity_rescale (a4)", 12.0 * n, lambda: nrb.intensity_rescale(img, n, 2.0, BINS + 1.0, stream=st)),
        ("nmi_value (a5)", 8.0 * n,
         lambda: nrb.check(L.nrb_nmi_value(nmi.h, ctypes.byref(g), nrb._p(ref), nrb._p(w), None, nrb._p(obj), None,
                                           sp))),
        ("nmi_voxel_gradient (a6)", 32.0 * n, lambda: nrb.nmi_voxel_gradient(nmi, g, ref, w, wg, vg, stream=st)),
        ("node_convolution (a7 + a8)", 12.0 * n + 12.0 * c,
         lambda: nrb.convolve_voxel_based_gradient(ws, vg, node, 1.0, stream=st)),
        ("kernel_convolution_x (a7, whole volume)", 24.0 * n,
         lambda: nrb.kernel_convolution_cubic(field, 3, dim, pix, 5.0, 0, stream=st)),
        ("bending_energy (a9)", 12.0 * c,
         lambda: nrb.check(L.nrb_approx_bending_energy(ws.h, ctypes.byref(ws.g), nrb._p(cppd), nrb._p(obj), None,
                                                       sp))),
        ("bending_energy_gradient (a10)", 36.0 * c,
         lambda: nrb.approx_bending_energy_gradient(ws, cppd, node, 0.005, stream=st)),
        ("resample_cubic (f2)", 20.0 * n, lambda: nrb.resample_image_order(g, flo, d, w, 3, stream=st)),
    ]
    peak, peak_src = peaks()
    out = {}
    launches0 = nrb.kernel_launch_count()
    for name, nbytes, fn in ops:
        times = []
        for k in range(args.warmup + args.steps):
            # in-place ops start from the same input every call (outside the timed region)
            if name.startswith("kernel_convolution"):
                field.copy_(vg)
            if name.startswith("intensity_rescale"):
                img.copy_(raw)
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            fn()
            e1.record(st)
            torch.cuda.synchronize()
            if k >= args.warmup:
                times.append(e0.elapsed_time(e1))
        ms = float(np.median(times))
        gbs = nbytes / (ms / 1e3) / 1e9
        out[name] = {"median_us": round(ms * 1e3, 2), "algorithmic_mb": round(nbytes / 1e6, 2),
                     "GBps": round(gbs, 1), "frac_of_" + peak_src + "_hbm": round(gbs / peak, 4)}
    print(json.dumps({"mode": "kernel-only ops", "voxels": n, "nodes": c, "peak_gbs": peak,
                      "l2": "256 MiB buffer written before every call", "steps": args.steps, "warmup": args.warmup,
                      "gpu_launches": nrb.kernel_launch_count() - launches0, "ops": out}))
    return 0


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


@contextlib.contextmanager
def collector_paused():
    """Python's cyclic garbage collector off inside a timed region (as timeit does): a full
    collection in a process holding torch's objects takes tens of milliseconds, and one that
    falls between a registration's return and its closing event would be counted as GPU time."""
    gc.collect()
    gc.disable()
    try:
        yield
    finally:
        gc.enable()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.idx = device_index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
            return
        # the timed region starts once nvidia-smi has its first sample: its start-up (NVML
        # initialisation) then lies before the region instead of inside one of its steps
        t0 = time.perf_counter()
        while time.perf_counter() - t0 < 5.0 and self.p.poll() is None:
            if os.path.getsize(self.f.name) > 0:
                break
            time.sleep(0.02)

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except (ValueError, IndexError):
                continue
            for name, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def traffic_per_launch(kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu summary (profiles/*.md line
    'dram_bytes_per_voxel_<kernel>: X', bytes per reference voxel of one launch), or None."""
    d = os.path.join(ROOT, "profiles")
    if not os.path.isdir(d):
        return None
    for name in sorted(os.listdir(d)):
        if not name.endswith(".md"):
            continue
        for line in open(os.path.join(d, name)):
            if line.strip().startswith(f"dram_bytes_per_voxel_{kernel}:"):
                try:
                    return float(line.split(":", 1)[1].split()[0])
                except ValueError:
                    return None
    return None


def reference_registration(pair, threads):
    """One full-budget registration of the workload by the reference NiftyReg CPU library
    (reg_f3d<float>::Run from oracle/_ref, -O3 -msse3 OpenMP, all host threads given), timed with
    the host clock around Run (in-memory images, no file I/O, as reg-apps/reg_benchmark.cpp
    times it). Returns None when the library is not built."""
    import oracle
    if not oracle.ref_available():
        return None
    R = oracle.Ref()
    cores = R.set_threads(threads)
    eye = np.eye(4, dtype=np.float32)
    _, _, st = R.f3d_register(pair.reference.ravel(), pair.floating.ravel(), pair.dim, pair.pixdim, eye, LEVELS,
                              MAXIT, BE, 0.0, BINS, SPACING)
    sec = float(st[4])
    n_obj, n_grad = int(st[2]), int(st[3])
    return {"seconds": sec, "cores": int(cores), "final_nmi": float(st[0]), "objective_evaluations": n_obj,
            "gradient_evaluations": n_grad, "evaluations_per_s": (n_obj + n_grad) / sec,
            "per_level_seconds": [float(st[7 + 3 * l]) for l in range(LEVELS)]}


def reference_baseline(pair, threads):
    """cpu_baseline of the b200 line: one full-budget reference registration (the bounded sample
    is one registration of the workload)."""
    r = reference_registration(pair, threads)
    if r is None:
        return None
    return {"value": 1.0 / r["seconds"], "unit": "registrations/s", "cores": r["cores"], "kind": "reference",
            "sample": (f"one full-budget reference reg_f3d<float> registration (oracle/_ref, -O3 -msse3 OpenMP, "
                       f"{r['cores']} threads) of the same pair: {r['seconds']:.1f} s, "
                       f"{r['objective_evaluations']} objective + {r['gradient_evaluations']} gradient "
                       f"evaluations, final NMI {r['final_nmi']:.7f}"),
            "final_nmi": r["final_nmi"], "objective_evaluations": r["objective_evaluations"],
            "gradient_evaluations": r["gradient_evaluations"], "evaluations_per_s": r["evaluations_per_s"]}


REF_ARM_BUDGET_S = 150.0       # reference arm: registrations are timed while they fit in this


def run_reference(args):
    """The reference arm: whole reference registrations of the workload on the host cores, each
    one timed (a step = one full-budget registration). At least one registration runs whatever
    --steps is; further ones run while --steps and REF_ARM_BUDGET_S allow, and the line states
    how many were timed. No warm-up is needed on the CPU (--warmup is recorded, not run)."""
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from niftyreg_b200 import phantom
    import oracle
    pair = phantom.brain_pair(SHAPE, seed=args.seed)
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libnrref.so not built (needs the "
                          "reference sources: make -C oracle ref)"}))
        return 0
    threads = os.cpu_count() or 1
    runs = []
    t_start = time.perf_counter()
    while True:
        runs.append(reference_registration(pair, threads))
        elapsed = time.perf_counter() - t_start
        mean = elapsed / len(runs)
        if len(runs) >= max(1, args.steps) or elapsed + mean > REF_ARM_BUDGET_S:
            break
    sec = float(np.mean([r["seconds"] for r in runs]))
    v = 1.0 / sec
    last = runs[-1]
    evals = float(np.mean([r["evaluations_per_s"] for r in runs]))
    sample = (f"{len(runs)} full-budget reference reg_f3d<float> registrations (oracle/_ref, -O3 -msse3 OpenMP, "
              f"{last['cores']} threads), each timed around Run: mean {sec:.1f} s; last: "
              f"{last['objective_evaluations']} objective + {last['gradient_evaluations']} gradient evaluations, "
              f"final NMI {last['final_nmi']:.7f}")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "registrations/s", "n_gpus": world,
            "steps": len(runs), "requested_steps": args.steps, "warmup": 0, "requested_warmup": args.warmup,
            "ms_per_step": sec * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "parallelism": "replicas", "host_threads": threads},
            "evaluations_per_s": evals,
            "registration": {"final_nmi": last["final_nmi"], "objective_evaluations": last["objective_evaluations"],
                             "gradient_evaluations": last["gradient_evaluations"],
                             "per_level_seconds": last["per_level_seconds"],
                             "step_s": [round(r["seconds"], 3) for r in runs]},
            "cpu_baseline": {"value": v, "unit": "registrations/s", "cores": last["cores"], "kind": "reference",
                             "sample": sample},
            "e2e": {"value": v, "unit": "registrations/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def max_over_ranks(x: float, world: int, device) -> float:
    """The slowest rank's value (every rank calls this at the same point)."""
    if world <= 1:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def replica_rate(world: int, per_rank_units: int, seconds_max: float) -> float:
    """Whole-job rate of independent replicas: every rank's units over the slowest rank's time."""
    return world * per_rank_units / seconds_max


def run_b200(args):
    import torch
    import niftyreg_b200 as nrb
    from niftyreg_b200 import phantom

    rank, world, local = dist_env()
    if not torch.cuda.is_available():
        raise SystemExit("bench.py: no CUDA device")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1 and not torch.distributed.is_initialized():
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                             device_id=dev)
    nrb.build()
    nrb.lib()
    pair = phantom.brain_pair(SHAPE, seed=args.seed + rank)
    nz, ny, nx = SHAPE
    dim, pix = (nx, ny, nz), pair.pixdim
    ref_h = torch.from_numpy(pair.reference.ravel().copy()).pin_memory()
    flo_h = torch.from_numpy(pair.floating.ravel().copy()).pin_memory()
    ref_d, flo_d = ref_h.to(dev), flo_h.to(dev)
    params = nrb.default_params(levels=LEVELS, max_iterations=MAXIT, bending_energy=BE, spacing=(SPACING,),
                                ref_bins=BINS, flo_bins=BINS, floating_texture=args.floating_texture)
    cdim = nrb.grid_dims(dim, pix, params)
    ncpp = 3 * int(np.prod(cdim))
    cpp_d = torch.empty(ncpp, dtype=torch.float32, device=dev)
    cpp_h = torch.empty(ncpp, dtype=torch.float32).pin_memory()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.Stream(dev)

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    def step():
        return nrb.register_device(ref_d, flo_d, dim, pix, params, cpp_d, ncpp, stream=stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()

    # ---- timed: device-resident inputs -------------------------------------------------------
    sampler = ClockSampler(torch.cuda.current_device())
    sampler.start()
    launches0 = nrb.kernel_launch_count()
    events, results = [], []
    with collector_paused():
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()  # L2 flush between timed steps, outside the events
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            results.append(step())
            e1.record(stream)
            events.append((e0, e1))
        torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    launches = nrb.kernel_launch_count() - launches0
    step_ms = [a.elapsed_time(b) for a, b in events]
    # one more registration with every fused launch bracketed by CUDA events on its own stream:
    # the per-kernel roofline (outside the headline timing, whose host time it would inflate)
    with torch.cuda.stream(stream):
        flush.zero_()
    nrb.timing_enable(True)
    step()
    torch.cuda.synchronize()
    timed = {k: nrb.timing_read(k) for k in ("objective", "gradient", "finalize", "conv", "be_value", "be_gradient")}
    nrb.timing_enable(False)
    total_max = max_over_ranks(float(sum(step_ms)), world, dev)
    value = replica_rate(world, args.steps, total_max / 1e3)

    # ---- e2e: host buffers through the C ABI, copies inside the timed region ------------------
    barrier()
    e2e_s = []
    with collector_paused():
        for _ in range(0 if args.no_e2e else args.steps):
            t0 = time.perf_counter()
            cpp_np, res = nrb.register_host(ref_h.numpy().reshape(SHAPE), flo_h.numpy().reshape(SHAPE), pix, params)
            e2e_s.append(time.perf_counter() - t0)
    e2e_max = max_over_ranks(float(sum(e2e_s)), world, dev)
    e2e_value = replica_rate(world, len(e2e_s), e2e_max) if e2e_s else None

    # ---- roofline of the dominant kernel ------------------------------------------------------
    dom = max(timed, key=lambda k: timed[k][1])
    n_l, ms_l, bytes_l = timed[dom]
    peak, peak_kind = peaks()
    achieved = (bytes_l / n_l) / (ms_l / n_l / 1e3) / 1e9 if n_l else 0.0
    per_voxel = traffic_per_launch(dom)
    voxels_per_launch = None
    traffic = None
    if per_voxel is not None and n_l:
        # units of one launch: the reference voxels of that launch (time-weighted mix of levels)
        voxels_per_launch = (bytes_l / n_l) / (8.0 if dom == "objective" else 20.0)
        traffic = per_voxel * voxels_per_launch
    share = {k: round(v[1] / sum(x[1] for x in timed.values()), 4) for k, v in timed.items()}

    if rank != 0:
        if world > 1:
            torch.distributed.destroy_process_group()
        return 0
    line = {
        "metric": METRIC, "value": value, "unit": "registrations/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "shape_zyx": list(SHAPE), "levels": LEVELS, "max_iterations": MAXIT,
                   "bins": BINS, "bending_energy": BE, "spacing_mm": 5.0, "parallelism": "replicas",
                   "l2": f"{L2_FLUSH_BYTES >> 20} MiB buffer written between timed steps"},
        "roofline": {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic,
                     "launches": n_l, "avg_launch_us": ms_l / n_l * 1e3 if n_l else None,
                     "algorithmic_bytes_per_launch": bytes_l / n_l if n_l else None,
                     "time_share": share},
        "e2e": {"value": e2e_value, "unit": "registrations/s", "h2d_bytes_per_step": 2 * 4 * nx * ny * nz,
                "d2h_bytes_per_step": 4 * ncpp, "step_ms": [round(1e3 * t, 2) for t in e2e_s]},
        "gpu_launches": int(launches),
        "evaluations_per_s": sum(r.objective_evaluations + r.gradient_evaluations for r in results)
                             / (sum(step_ms) / 1e3),
        "clocks": clocks,
        "registration": {"final_nmi": results[-1].final_nmi, "objective_evaluations": results[-1].objective_evaluations,
                         "gradient_evaluations": results[-1].gradient_evaluations,
                         "step_ms": [round(s, 3) for s in step_ms]},
    }
    if world == 1 and not args.no_extras:
        # the metric's batched and served figures (shortened runs of --mode batched / --mode served)
        import copy
        ba = copy.copy(args)
        ba.batch_only, ba.kernel_timing, ba.verbose = False, False, False
        # groups of up to 32: two groups, whose host work and device work overlap
        ba.pairs, ba.concurrency = 64, 32
        b = run_batched(ba, emit=False)
        line["batched"] = {k: b[k] for k in ("value", "plain_value", "speedup_vs_plain", "max_abs_dnmi_vs_plain",
                                             "bitwise_identical_to_plain")}
        line["batched"]["workload"] = b["config"]["workload"] + f", groups of up to {ba.concurrency}"
        line["batched_speedup_vs_plain"] = b["speedup_vs_plain"]
        # the same on small volumes, where a plain registration leaves the device waiting on
        # dependent launches: 128 pairs of 64^3
        ba.pairs, ba.batch_shapes, ba.concurrency = 128, "64,64,64", 64
        b64 = run_batched(ba, emit=False)
        line["batched_64cubed"] = {k: b64[k] for k in ("value", "plain_value", "speedup_vs_plain",
                                                       "max_abs_dnmi_vs_plain", "bitwise_identical_to_plain")}
        line["batched_64cubed"]["workload"] = b64["config"]["workload"] + f", groups of up to {ba.concurrency}"
        sa = copy.copy(args)
        sa.rates, sa.requests, sa.burst = "20,50", 350, 200
        sv = run_served(sa, emit=False)
        line["served"] = {"value": sv["value"], "plain_value": sv["plain_value"],
                          "served_vs_plain_at_saturation": sv["served_vs_plain_at_saturation"],
                          "capacity": sv["capacity"],
                          "sweep": [{k: r[k] for k in ("rate_req_s", "requests", "achieved_req_s", "p50_ms", "p95_ms",
                                                       "p99_ms", "peak_group")} for r in sv["sweep"]],
                          "workload": sv["config"]["workload"]}
    if world == 1 and not args.no_extras and nrb.platform_available():
        # NiftyReg's own reg_f3d<float>::Run on the B200 platform (niftyreg_b200/platform): the
        # reference driver and optimiser with every step one C-ABI call, host images in
        t0 = time.perf_counter()
        _, pr = nrb.platform_register(pair.reference, pair.floating, pix, levels=LEVELS, max_iterations=MAXIT,
                                      bending_energy=BE, spacing=SPACING, bins=BINS)
        wall = time.perf_counter() - t0
        ev = pr.objective_evaluations + pr.gradient_evaluations
        line["platform_plugin"] = {
            "value": 1.0 / wall, "unit": "registrations/s", "seconds_run": pr.seconds, "seconds_wall": wall,
            "final_nmi": pr.final_nmi, "objective_evaluations": pr.objective_evaluations,
            "gradient_evaluations": pr.gradient_evaluations, "evaluations_per_s": ev / pr.seconds,
            "abs_dnmi_vs_b200": abs(pr.final_nmi - results[-1].final_nmi),
            "what": "reg_f3d<float>::Run of the reference's own code (pyramid, CG optimiser) on the B200 Platform "
                    "classes, host images in, grid out, host wall clock"}
    if world == 1 and not args.no_cpu_baseline:
        cb = reference_baseline(pair, os.cpu_count() or 1)
        if cb is not None:
            line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
            line["reference_registration"] = {k: cb[k] for k in ("final_nmi", "objective_evaluations",
                                                                 "gradient_evaluations", "evaluations_per_s")}
            line["abs_dnmi_vs_reference"] = abs(results[-1].final_nmi - cb["final_nmi"])
    print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


# ---- batched and served modes --------------------------------------------------------------
BATCH_SHAPES = [(96, 96, 96), (96, 128, 128), (160, 192, 160), (182, 218, 182)]  # (nz, ny, nx)
BATCH_LEVELS, BATCH_MAXIT = 2, 150
SERVE_MIX = [((64, 64, 64), 0.30), ((128, 128, 128), 0.40), ((182, 218, 182), 0.25), ((256, 256, 256), 0.05)]
SERVE_LEVELS, SERVE_MAXIT = 2, 100


def _phantom_pool(shapes, per_shape, seed, spacing_vox=5.0, disp_vox=3.0):
    """Seeded blob phantoms (floating = reference warped by a 5-voxel FFD), `per_shape` distinct
    pairs per size; requests draw from this pool (the device work per request is the same as
    for a fresh pair of that size)."""
    from niftyreg_b200 import phantom
    pool = {}
    for k, shp in enumerate(shapes):
        pool[shp] = [phantom.blobs_pair(shp, seed=seed + 100 * k + j, spacing_vox=spacing_vox,
                                        disp_sigma_vox=disp_vox) for j in range(per_shape)]
    return pool


def _gpu_clock_sampler():
    import torch
    return ClockSampler(torch.cuda.current_device())


def run_batched(args, emit=True):
    """`--pairs` registrations with sizes drawn uniformly from BATCH_SHAPES: first one by one
    through the plain path (nrb_f3d_register_host), then all at once through
    nrb_f3d_register_batch with `--concurrency` registrations in flight. Reports both rates and
    the largest |dNMI| between a pair's plain and batched results."""
    import torch
    import niftyreg_b200 as nrb
    torch.cuda.set_device(0)
    nrb.build()
    rng = np.random.default_rng(args.seed)
    shapes = ([tuple(int(v) for v in t.split(",")) for t in args.batch_shapes.split(";")] if args.batch_shapes
              else BATCH_SHAPES)
    pool = _phantom_pool(shapes, 2, args.seed)
    picks = [shapes[i] for i in rng.integers(0, len(shapes), args.pairs)]
    pairs = [pool[s][int(rng.integers(0, 2))] for s in picks]
    params = nrb.default_params(levels=BATCH_LEVELS, max_iterations=BATCH_MAXIT, bending_energy=BE,
                                spacing=(SPACING,), ref_bins=BINS, flo_bins=BINS,
                                floating_texture=args.floating_texture)
    # warm-up: one registration of every size
    for s in shapes:
        p = pool[s][0]
        nrb.register_host(p.reference, p.floating, p.pixdim, params)
    sampler = _gpu_clock_sampler()
    sampler.start()
    with collector_paused():
        t0 = time.perf_counter()
        plain = [] if args.batch_only else [nrb.register_host(p.reference, p.floating, p.pixdim, params) for p in pairs]
        t_plain = time.perf_counter() - t0
    bparams = nrb.default_params(levels=BATCH_LEVELS, max_iterations=BATCH_MAXIT, bending_energy=BE,
                                 spacing=(SPACING,), ref_bins=BINS, flo_bins=BINS,
                                 batch_gradient_percent=args.grad_percent, verbose=int(args.verbose),
                                 floating_texture=args.floating_texture)
    if args.group_mb is not None:
        bparams.batch_group_mb = args.group_mb
    # warm-up of the batched path as the plain one had: the same batch once, untimed (device
    # memory pools and texture arrays grown to the groups' footprint, as in a running server)
    nrb.register_batch([(p.reference, p.floating, p.pixdim) for p in pairs], bparams, args.concurrency)
    with collector_paused():
        t0 = time.perf_counter()
        batched = nrb.register_batch([(p.reference, p.floating, p.pixdim) for p in pairs], bparams, args.concurrency)
        t_batch = time.perf_counter() - t0
    clocks = sampler.stop()
    kt = None
    if args.kernel_timing:
        # the same batch once more, driven from the host with every launch bracketed by events
        nrb.timing_enable(True)
        nrb.register_batch([(p.reference, p.floating, p.pixdim) for p in pairs], bparams, args.concurrency)
        torch.cuda.synchronize()
        raw = {k: nrb.timing_read(k) for k in ("objective", "gradient", "finalize", "conv", "be_value", "be_gradient")}
        nrb.timing_enable(False)
        peak, _ = peaks()
        tot = sum(v[1] for v in raw.values())
        kt = {k: {"launches": v[0], "ms": round(v[1], 3), "share": round(v[1] / tot, 4) if tot else None,
                  "avg_us": round(v[1] / v[0] * 1e3, 2) if v[0] else None,
                  "GBps": round(v[2] / (v[1] / 1e3) / 1e9, 1) if v[1] and v[2] else None,
                  "frac_of_measured_hbm": round(v[2] / (v[1] / 1e3) / 1e9 / peak, 4) if v[1] and v[2] else None}
              for k, v in raw.items()}
    if args.batch_only:
        print(json.dumps({"mode": "batched", "batch_only": True, "value": args.pairs / t_batch, "seconds": t_batch,
                          "kernel_timing": kt}))
        return 0
    dnmi = max(abs(a[1].final_nmi - b[1].final_nmi) for a, b in zip(plain, batched))
    identical = all(np.array_equal(a[0], b[0]) for a, b in zip(plain, batched))
    line = {"mode": "batched", "metric": METRIC, "value": args.pairs / t_batch, "unit": "registrations/s",
            "plain_value": args.pairs / t_plain, "speedup_vs_plain": t_plain / t_batch, "n_gpus": 1,
            "higher_is_better": True, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{args.pairs} pairs, sizes uniform over {shapes} (nz, ny, nx), blob "
                                   f"phantoms (2 distinct pairs per size), {BATCH_LEVELS} levels, {BATCH_MAXIT} "
                                   f"counted iterations at the finest level, NMI {BINS} bins, BE {BE}, 5-voxel grid",
                       "concurrency": args.concurrency, "timing": "host wall clock, host images, copies included"},
            "max_abs_dnmi_vs_plain": dnmi, "bitwise_identical_to_plain": identical, "clocks": clocks}
    if emit:
        print(json.dumps(line))
        return 0
    return line


def run_served(args, emit=True):
    """Open-loop Poisson request streams at each rate of `--rates` (`--requests` in total, split in
    proportion to the rates): sizes drawn from SERVE_MIX, admitted by a server with `--slots`
    workers grouping up to `--max-group` similar requests under 80% of free HBM. Reports latency
    percentiles (submit -> result) and the achieved rate per rate; the plain rate is the same
    request mix registered one by one."""
    import queue
    import threading
    import torch
    import niftyreg_b200 as nrb
    torch.cuda.set_device(0)
    nrb.build()
    rng = np.random.default_rng(args.seed)
    shapes = [s for s, _ in SERVE_MIX]
    probs = np.array([w for _, w in SERVE_MIX])
    pool = _phantom_pool(shapes, 2, args.seed)
    params = nrb.default_params(levels=SERVE_LEVELS, max_iterations=SERVE_MAXIT, bending_energy=BE,
                                spacing=(SPACING,), ref_bins=BINS, flo_bins=BINS,
                                floating_texture=args.floating_texture)
    if args.group_mb is not None:
        params.batch_group_mb = args.group_mb
    for s in shapes:
        p = pool[s][0]
        nrb.register_host(p.reference, p.floating, p.pixdim, params)
    # plain reference rate of the mix, one by one
    n_plain = 40
    mix = [pool[shapes[int(i)]][int(rng.integers(0, 2))] for i in rng.choice(len(shapes), n_plain, p=probs)]
    t0 = time.perf_counter()
    alone = {}
    for p in mix:
        _, r = nrb.register_host(p.reference, p.floating, p.pixdim, params)
        alone[id(p)] = r.final_nmi
    plain_rate = n_plain / (time.perf_counter() - t0)
    results = []
    sampler = _gpu_clock_sampler()
    sampler.start()
    rates = [float(x) for x in args.rates.split(",")]
    counts = [max(1, int(round(args.requests * r / sum(rates)))) for r in rates]
    for rate, n_req in zip(rates, counts):
        reqs = [pool[shapes[int(i)]][int(rng.integers(0, 2))]
                for i in rng.choice(len(shapes), n_req, p=probs)]
        gaps = rng.exponential(1.0 / rate, n_req)
        lat, dn = [], []
        with nrb.Server(slots=args.slots, max_group=args.max_group) as srv:
            tq = queue.Queue()

            def drain():
                # waits in submission order; latency is measured by the server (submit -> result)
                while True:
                    item = tq.get()
                    if item is None:
                        return
                    t, p = item
                    _, r, _, l = srv.wait(t)
                    lat.append(l)
                    if id(p) in alone:
                        dn.append(abs(r.final_nmi - alone[id(p)]))

            th = threading.Thread(target=drain)
            th.start()
            t_start = time.perf_counter()
            due = t_start
            for p, g in zip(reqs, gaps):
                due += g
                now = time.perf_counter()
                if due > now:
                    time.sleep(due - now)
                tq.put((srv.submit(p.reference, p.floating, p.pixdim, params), p))
            tq.put(None)
            th.join()
            t_end = time.perf_counter()
            peak_bytes, peak_active = srv.stats()
            peak_group = srv.peak_group()
        lat_ms = np.array(lat) * 1e3
        results.append({"rate_req_s": rate, "requests": n_req, "peak_group": peak_group,
                        "achieved_req_s": n_req / (t_end - t_start),
                        "p50_ms": float(np.percentile(lat_ms, 50)), "p95_ms": float(np.percentile(lat_ms, 95)),
                        "p99_ms": float(np.percentile(lat_ms, 99)), "peak_concurrent": peak_active,
                        "peak_admitted_gb": peak_bytes / 1e9,
                        "max_abs_dnmi_vs_alone": float(max(dn)) if dn else None})
    # capacity: a burst of requests submitted at once (the offered rates above stay below what the
    # server can take, so their achieved rate is the offered one)
    n_burst = max(1, args.burst)
    reqs = [pool[shapes[int(i)]][int(rng.integers(0, 2))] for i in rng.choice(len(shapes), n_burst, p=probs)]
    with nrb.Server(slots=args.slots, max_group=args.burst_group) as srv:
        # the first burst grows the device memory pool and the texture arrays to groups of
        # burst_group requests (a one-off cost of a server's first large groups); the second, on
        # the same server, is the steady-state capacity
        t_first = time.perf_counter()
        tickets = [srv.submit(p.reference, p.floating, p.pixdim, params) for p in reqs]
        for t in tickets:
            srv.wait(t)
        first_s = time.perf_counter() - t_first
        t_start = time.perf_counter()
        tickets = [srv.submit(p.reference, p.floating, p.pixdim, params) for p in reqs]
        outs = [srv.wait(t) for t in tickets]
        t_end = time.perf_counter()
        peak_group = srv.peak_group()
    lat_ms = np.array([o[3] for o in outs]) * 1e3
    capacity = {"requests": n_burst, "max_group": args.burst_group,
                "achieved_req_s": n_burst / (t_end - t_start), "peak_group": peak_group,
                "p50_ms": float(np.percentile(lat_ms, 50)), "p99_ms": float(np.percentile(lat_ms, 99)),
                "first_burst_req_s": n_burst / first_s}
    capacity["vs_plain"] = capacity["achieved_req_s"] / plain_rate
    clocks = sampler.stop()
    best = max(results, key=lambda r: r["achieved_req_s"])
    line = {"mode": "served", "metric": METRIC, "value": best["achieved_req_s"], "unit": "registrations/s",
            "p99_ms": best["p99_ms"], "plain_value": plain_rate, "capacity": capacity,
            "n_gpus": 1, "higher_is_better": True,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"open-loop Poisson requests, sizes {SERVE_MIX} ((nz, ny, nx), probability), "
                                   f"blob phantoms (2 distinct pairs per size), {SERVE_LEVELS} levels, {SERVE_MAXIT} "
                                   f"counted iterations at the finest level, NMI {BINS} bins, BE {BE}, 5-voxel grid",
                       "slots": args.slots, "max_group": args.max_group,
                       "admission": "FIFO against 80% of free HBM; a free worker takes the head and the queued "
                                    "requests of similar size (within 2x voxels) into one batched registration"},
            "served_vs_plain_at_best_offered_rate": best["achieved_req_s"] / plain_rate,
            "served_vs_plain_at_saturation": capacity["vs_plain"],
            "sweep": results, "clocks": clocks}
    if emit:
        print(json.dumps(line))
        return 0
    return line


CT_SHAPE, CT_PIX = (320, 512, 512), (0.8, 0.8, 1.5)   # (nz, ny, nx), (dx, dy, dz) mm
CT_LEVELS, CT_MAXIT, CT_BE, CT_BINS, CT_SPACING = 3, 200, 0.001, 128, 10.0


def run_ct(args):
    """The large CT-like pair: 512x512x320 float32 at 0.8x0.8x1.5 mm, HU phantom, floating warped by a
    seeded 10 mm FFD with N(0, 4 mm) displacements; 3 levels, 200 counted iterations at the finest
    level, NMI 128 bins, BE 0.001, 10 mm grid. Four registrations (two seeded phantoms, each
    twice) one by one through the plain path (host images in, grids out), then the same four in
    one batch; the batch must give the plain results bit for bit."""
    import torch
    import niftyreg_b200 as nrb
    from niftyreg_b200 import phantom

    torch.cuda.set_device(0)
    nrb.build()
    two = [phantom.ct_pair(CT_SHAPE, seed=args.seed + i, pixdim=CT_PIX, spacing_mm=CT_SPACING, disp_sigma_mm=4.0)
           for i in range(2)]
    pairs = two + two
    params = nrb.default_params(levels=CT_LEVELS, max_iterations=CT_MAXIT, bending_energy=CT_BE,
                                spacing=(CT_SPACING,), ref_bins=CT_BINS, flo_bins=CT_BINS,
                                floating_texture=args.floating_texture)
    # warm-up: one registration
    p0 = pairs[0]
    nrb.register_host(p0.reference, p0.floating, p0.pixdim, params)
    sampler = _gpu_clock_sampler()
    sampler.start()
    times, plain = [], []
    for p in pairs:
        t0 = time.perf_counter()
        plain.append(nrb.register_host(p.reference, p.floating, p.pixdim, params))
        times.append(time.perf_counter() - t0)
    # the batched path warmed as the plain one was (memory pool and texture arrays grown to the
    # groups' footprint), then timed
    items = [(p.reference, p.floating, p.pixdim) for p in pairs]
    nrb.register_batch(items, params, concurrency=args.ct_group)
    t0 = time.perf_counter()
    batched = nrb.register_batch(items, params, concurrency=args.ct_group)
    t_batch = time.perf_counter() - t0
    clocks = sampler.stop()
    identical = all(np.array_equal(a[0], b[0]) for a, b in zip(plain, batched))
    line = {"mode": "ct", "metric": METRIC, "value": 1.0 / float(np.mean(times)), "unit": "registrations/s",
            "plain_seconds": [round(t, 3) for t in times], "batch_of_4_value": 4 / t_batch,
            "batch_of_4_speedup_vs_plain": sum(times) / t_batch, "batch_group": args.ct_group,
            "bitwise_identical_to_plain": identical,
            "max_abs_dnmi_vs_plain": max(abs(a[1].final_nmi - b[1].final_nmi) for a, b in zip(plain, batched)),
            "registration": [{"final_nmi": r.final_nmi, "objective_evaluations": r.objective_evaluations,
                              "gradient_evaluations": r.gradient_evaluations} for _, r in plain],
            "n_gpus": 1, "higher_is_better": True, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "512x512x320 float32 at 0.8x0.8x1.5 mm CT-like HU phantom (air, lungs, soft "
                                   "tissue, bone ellipsoids), 10 mm FFD N(0, 4 mm); 3 levels, 200 counted iterations "
                                   "at the finest level, NMI 128 bins, BE 0.001, 10 mm grid",
                       "timing": "host wall clock, host images in and grids out (copies included)"},
            "clocks": clocks}
    print(json.dumps(line))
    return 0


def run_reference_cuda(args):
    """The reference arm on the reference's own CUDA platform (--impl reference
    --reference-platform cuda): reg-lib/cuda built for sm_100a into oracle/_refcuda,
    reg_f3d<float>::Run with PlatformType::Cuda on this GPU. One registration of the 64^3
    one-level workload (1 level, 100 counted iterations, BE 0.005, 64 bins, 5-voxel grid) and,
    unless --shape picks another size, --steps registrations of the brain-like workload, each
    timed with the host clock around Run (host images in, grid out: the reference's CUDA content
    copies the images to the device at every level). The library makes its own CUDA context, so
    this arm runs no other GPU work in the process; under torchrun only rank 0 runs it."""
    rank, _, _ = dist_env()
    if rank != 0:
        return 0
    import oracle
    from niftyreg_b200 import phantom
    if not oracle.refcuda_available():
        print(json.dumps({"impl": "reference", "reference_platform": "cuda",
                          "unavailable": "oracle/_refcuda/libnrref_cuda.so not built (make -C oracle refcuda, "
                                         "needs the reference sources)"}))
        return 0
    eye = np.eye(4, dtype=np.float32)
    sampler = ClockSampler(0)
    sampler.start()
    out = {}
    small = phantom.blobs_pair((64, 64, 64), seed=1)
    _, _, st = oracle.refcuda_register(small.reference.ravel(), small.floating.ravel(), small.dim, small.pixdim, eye,
                                       1, 100, 0.005, 0.0, 64, -5.0)
    out["blobs_64"] = {"seconds": float(st[4]), "final_nmi": float(st[0]), "objective_evaluations": int(st[2]),
                       "gradient_evaluations": int(st[3])}
    shape = tuple(int(v) for v in args.shape.split(",")) if args.shape else SHAPE
    pair = phantom.brain_pair(shape, seed=args.seed)
    runs = []
    for _ in range(max(1, args.steps)):
        _, _, st = oracle.refcuda_register(pair.reference.ravel(), pair.floating.ravel(), pair.dim, pair.pixdim, eye,
                                           LEVELS, MAXIT, BE, 0.0, BINS, SPACING)
        n_obj, n_grad = int(st[2]), int(st[3])
        runs.append({"seconds": float(st[4]), "final_nmi": float(st[0]), "objective_evaluations": n_obj,
                     "gradient_evaluations": n_grad, "evaluations_per_s": (n_obj + n_grad) / float(st[4]),
                     "per_level_seconds": [float(st[7 + 3 * l]) for l in range(LEVELS)]})
    clocks = sampler.stop()
    sec = float(np.mean([r["seconds"] for r in runs]))
    line = {"impl": "reference", "reference_platform": "cuda", "metric": METRIC, "value": 1.0 / sec,
            "unit": "registrations/s", "n_gpus": 1, "steps": len(runs), "warmup": 0, "ms_per_step": sec * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "evaluations_per_s": float(np.mean([r["evaluations_per_s"] for r in runs])),
            "registrations": runs, "blobs_64": out["blobs_64"],
            "config": {"workload": WORKLOAD if shape == SHAPE else f"brain-like phantom {shape}",
                       "parallelism": "replicas",
                       "timing": "host wall clock around reg_f3d<float>::Run on the reference CUDA platform"},
            "e2e": {"value": 1.0 / sec, "unit": "registrations/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "clocks": clocks}
    print(json.dumps(line))
    return 0


def run_warp(args):
    """The final warped image of a registration of the workload's volume (reg_f3d::GetWarpedImage:
    deformation field of the grid, cubic-spline resample of the floating image), on the device
    with inputs resident (CUDA events, L2 flushed between steps) and end to end from host
    buffers (copies included), against the reference's own CPU path (oracle/_ref:
    reg_spline_getDeformationField + reg_resampleImage order 3, all host threads)."""
    import torch
    import niftyreg_b200 as nrb
    from niftyreg_b200 import phantom

    torch.cuda.set_device(0)
    nrb.build()
    pair = phantom.brain_pair(SHAPE, seed=args.seed)
    nz, ny, nx = SHAPE
    dim, pix = (nx, ny, nz), (1.0, 1.0, 1.0)
    cdim, cpix, cxyz = nrb.control_grid_header(dim, pix, (5.0, 5.0, 5.0))
    rng = np.random.default_rng(args.seed)
    cx, cy, cz = cdim
    zz, yy, xx = np.meshgrid(np.arange(cz), np.arange(cy), np.arange(cx), indexing="ij")
    ident = np.concatenate([(5.0 * v - 5.0).ravel() for v in (xx, yy, zz)]).astype(np.float32)
    cpp = ident + rng.normal(0, 2.0, ident.size).astype(np.float32)
    g = nrb.make_geometry(dim, pix, nrb.identity_header(pix), dim, pix, nrb.identity_header(pix), cdim, cpix, cxyz)
    n = nx * ny * nz
    flo_h = torch.from_numpy(pair.floating.ravel().copy()).pin_memory()
    cpp_h = torch.from_numpy(cpp).pin_memory()
    out_h = torch.empty(n, dtype=torch.float32).pin_memory()
    flo_d, cpp_d = flo_h.cuda(), cpp_h.cuda()
    out_d = torch.empty(n, dtype=torch.float32, device="cuda")
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.Stream()
    for _ in range(args.warmup):
        nrb.f3d_warped_image(g, flo_d, cpp_d, out_d, order=3, padding=0.0, stream=stream)
    torch.cuda.synchronize()
    sampler = ClockSampler(torch.cuda.current_device())
    sampler.start()
    ms = []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        nrb.f3d_warped_image(g, flo_d, cpp_d, out_d, order=3, padding=0.0, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    clocks = sampler.stop()
    e2e = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        with torch.cuda.stream(stream):
            flo_d.copy_(flo_h, non_blocking=True)
            cpp_d.copy_(cpp_h, non_blocking=True)
            nrb.f3d_warped_image(g, flo_d, cpp_d, out_d, order=3, padding=0.0, stream=stream)
            out_h.copy_(out_d, non_blocking=True)
        stream.synchronize()
        e2e.append(time.perf_counter() - t0)
    warped = out_h.numpy().copy()
    t = sum(ms) / len(ms) / 1e3
    peak, peak_kind = peaks()
    alg = 8.0 * n + 12.0 * ident.size  # floating read + warped written + grid read
    line = {"mode": "warp", "metric": "final warped image (reg_f3d::GetWarpedImage, cubic spline) per second",
            "value": 1.0 / t, "unit": "warps/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t * 1e3, "higher_is_better": True, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "182x218x182 float32 brain-MR-like floating image, 5 mm grid with N(0, 2 mm) "
                                   "control-point displacements, cubic spline, padding 0",
                       "l2": f"{L2_FLUSH_BYTES >> 20} MiB buffer written between timed steps"},
            "roofline": {"bound": "hbm", "achieved": alg / t / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": alg / t / 1e9 / peak, "peak_source": peak_kind,
                         "algorithmic_bytes_per_launch": alg},
            "e2e": {"value": len(e2e) / sum(e2e), "unit": "warps/s", "h2d_bytes_per_step": 4 * (n + ident.size),
                    "d2h_bytes_per_step": 4 * n},
            "clocks": clocks}
    if not args.no_cpu_baseline:
        import oracle
        REF_SAMPLE_MAXIT = 30  # F3D2 reference: 1/10 of the finest level's budget, extrapolated
        if oracle.ref_available():
            R = oracle.Ref()
            cores = R.set_threads(os.cpu_count() or 1)
            eye = nrb.identity_header(pix)
            t0 = time.perf_counter()
            d = R.deformation_field(cpp, cdim, cpix, cxyz, dim, pix, eye)
            ref = R.resample_order(pair.floating.ravel(), dim, pix, eye, d, dim, pix, eye, 3, pad=0.0)
            wall = time.perf_counter() - t0
            line["cpu_baseline"] = {"value": 1.0 / wall, "unit": "warps/s", "cores": int(cores), "kind": "reference",
                                    "sample": "reference reg_spline_getDeformationField + reg_resampleImage order 3 "
                                              f"(oracle/_ref, OpenMP) on the same volume and grid, {wall:.2f} s"}
            ok = np.isfinite(ref)
            line["max_abs_diff_vs_reference"] = float(np.abs(warped[ok] - ref[ok]).max())
    print(json.dumps(line))
    return 0


def run_f3d2(args):
    """The symmetric registration (reg_f3d2, the -vel / -sym variant) of the workload's pair with
    the workload's schedule, through nrb_f3d2_register_images (host images in, both grids and the
    warped images out: copies included), against the reference's reg_f3d2<float> on the box's
    host cores (a 1/10 iteration budget, extrapolated x10). Also the roofline of the composition
    kernel (the squaring step, the most launched F3D2 kernel) timed alone on a full-size field."""
    import torch
    import niftyreg_b200 as nrb
    from niftyreg_b200 import phantom

    torch.cuda.set_device(0)
    nrb.build()
    pair = phantom.brain_pair(SHAPE, seed=args.seed)
    pix = tuple(float(p) for p in pair.pixdim)
    eye = nrb.identity_header(pix)
    params = nrb.default_params(levels=LEVELS, max_iterations=MAXIT, bending_energy=BE, spacing=(SPACING,),
                                ref_bins=BINS, flo_bins=BINS)
    for _ in range(args.warmup):
        nrb.f3d2_register_images(pair.reference, pix, eye, pair.floating, pix, eye, params)
    sampler = ClockSampler(torch.cuda.current_device())
    sampler.start()
    secs, res = [], None
    for _ in range(args.steps):
        t0 = time.perf_counter()
        gf, gb, _, steps, wf, wb, res = nrb.f3d2_register_images(pair.reference, pix, eye, pair.floating, pix, eye,
                                                                 params)
        secs.append(time.perf_counter() - t0)
    clocks = sampler.stop()
    t = float(np.mean(secs))
    # one more registration with every F3D2 stage bracketed by CUDA events: where the time goes,
    # and the composition kernel's launches inside a real registration
    stages = ("f3d2_velocity", "f3d2_gradient_exp", "f3d2_warp", "f3d2_nmi", "f3d2_voxel_gradient", "f3d2_nodes",
              "f3d2_be", "f3d2_update")
    nrb.timing_enable(True)
    t0 = time.perf_counter()
    nrb.f3d2_register_images(pair.reference, pix, eye, pair.floating, pix, eye, params, warped=False)
    t_timed = time.perf_counter() - t0
    timed = {k: nrb.timing_read(k) for k in stages + ("f3d2_compose",)}
    nrb.timing_enable(False)
    stage_ms = {k: timed[k][1] for k in stages}
    comp_n, comp_ms, comp_bytes = timed["f3d2_compose"]
    # composition kernel alone: one squaring of a full-size smooth field (a few mm of displacement,
    # as the fields of a registration are smooth)
    nz, ny, nx = SHAPE
    n = nx * ny * nz
    k, j, i = np.meshgrid(np.arange(nz, dtype=np.float32), np.arange(ny, dtype=np.float32),
                          np.arange(nx, dtype=np.float32), indexing="ij")
    disp = 2.0 * np.sin(2 * np.pi * i / 61.0) * np.cos(2 * np.pi * j / 47.0) * np.sin(2 * np.pi * k / 53.0)
    field = np.concatenate([(i + disp).ravel(), (j - disp).ravel(), (k + 0.5 * disp).ravel()])
    apply_d = torch.from_numpy(field.astype(np.float32)).cuda()
    pos_d = apply_d.clone()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.Stream()
    for _ in range(3):
        nrb.def_field_compose((nx, ny, nz), eye, apply_d, pos_d, stream=stream)
    ms = []
    for _ in range(10):
        with torch.cuda.stream(stream):
            pos_d.copy_(apply_d)
            flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        nrb.def_field_compose((nx, ny, nz), eye, apply_d, pos_d, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    tc = float(np.mean(ms)) / 1e3
    alg = 36.0 * n  # positions read, the applied field read once, the result written (3 x 4 B each)
    # (inside the registration every composition is a squaring: the field applied to itself, 24 B)
    peak, peak_kind = peaks()
    line = {"mode": "f3d2", "metric": "symmetric F3D2 registrations/s (reg_f3d2, velocity grids)",
            "value": 1.0 / t, "unit": "registrations/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": WORKLOAD.replace("single-pair F3D", "single-pair F3D2 (symmetric, velocity grids)"),
                       "api": "nrb_f3d2_register_images, host images in and out (copies inside the timed region)"},
            "registration": {"final_symmetric_nmi": res.final_nmi, "objective_evaluations": res.objective_evaluations,
                             "gradient_evaluations": res.gradient_evaluations, "squaring_steps": steps,
                             "seconds": secs},
            "roofline": {"kernel": "k_compose", "bound": "hbm",
                         "achieved": comp_bytes / (comp_ms / 1e3) / 1e9 if comp_ms else None, "peak": peak,
                         "unit": "GB/s", "frac": comp_bytes / (comp_ms / 1e3) / 1e9 / peak if comp_ms else None,
                         "peak_source": peak_kind, "launches": comp_n,
                         "avg_launch_us": comp_ms / max(comp_n, 1) * 1e3,
                         "algorithmic_bytes_per_launch": comp_bytes / max(comp_n, 1),
                         "alone_full_size": {"achieved": alg / tc / 1e9, "frac": alg / tc / 1e9 / peak,
                                             "avg_launch_us": tc * 1e6, "algorithmic_bytes_per_launch": alg,
                                             "field": "182x218x182, smooth displacement up to 2 mm, L2 flushed"}},
            "stage_ms": {k: round(v, 3) for k, v in stage_ms.items()},
            "stage_share_of_wall": {k: round(v / 1e3 / t_timed, 4) for k, v in stage_ms.items()},
            "e2e": {"value": 1.0 / t, "unit": "registrations/s",
                    "h2d_bytes_per_step": int(pair.reference.nbytes + pair.floating.nbytes),
                    "d2h_bytes_per_step": int(gf.nbytes + gb.nbytes + wf.nbytes + wb.nbytes)},
            "clocks": clocks}
    if not args.no_cpu_baseline:
        import oracle
        # F3D2 reference: 1/10 of the finest level's budget, extrapolated (a full-budget
        # registration takes minutes on the host cores); --full-reference times the whole budget
        ref_maxit = MAXIT if args.full_reference else 30
        if oracle.ref_available():
            R = oracle.Ref()
            cores = R.set_threads(os.cpu_count() or 1)
            dim = pair.dim
            t0 = time.perf_counter()
            _, _, _, _, _, st = R.f3d2_register(pair.reference.ravel(), dim, pix, eye, pair.floating.ravel(), dim,
                                                pix, eye, LEVELS, ref_maxit, BE, 0.0, BINS, SPACING)
            wall = time.perf_counter() - t0
            est = wall * MAXIT / ref_maxit
            sample = (f"one full-budget reference reg_f3d2<float> registration (oracle/_ref, OpenMP) of the same "
                      f"pair, timed: {wall:.1f} s" if args.full_reference else
                      f"reference reg_f3d2<float> (oracle/_ref, OpenMP) on the same pair with a 1/10 iteration "
                      f"budget ({ref_maxit} at the finest level): {wall:.1f} s, x10 = {est:.1f} s per registration")
            line["cpu_baseline"] = {"value": 1.0 / est, "unit": "registrations/s", "cores": int(cores),
                                    "kind": "reference", "sample": sample,
                                    "sample_final_symmetric_nmi": float(st[0]),
                                    "sample_evaluations": [int(st[2]), int(st[3])]}
    print(json.dumps(line))
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference_cuda(args) if args.reference_platform == "cuda" else run_reference(args)
    if args.kernel:
        return run_kernel_only(args)
    if args.mode == "batched":
        return run_batched(args)
    if args.mode == "served":
        return run_served(args)
    if args.mode == "f3d2":
        return run_f3d2(args)
    if args.mode == "warp":
        return run_warp(args)
    if args.mode == "ct":
        return run_ct(args)

    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
