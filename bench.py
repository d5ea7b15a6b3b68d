"""Benchmark: B-spline MSE score + gradient throughput (Gvox/s) on B200.

Workload (one "step" = one complete cost-function evaluation, coefficients
in -> score + gradient out):
    fixed/moving 256x256x128 CT-like volumes (int16 HU converted to float,
    0.98x0.98x2.5 mm), vox_per_rgn 5x5x5 (70,304 tiles, 263,175
    coefficients), coefficients N(0, 3 mm), MSE with the reference's
    nearest-voxel gradient semantics.  Synthetic, seeded (no dataset).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--form tc|fp32]
    python bench.py --impl reference      # the reference's CPU flavour g

value   device-resident throughput: inputs already in HBM, coefficients and
        outputs in device memory, CUDA events on the evaluation stream, L2
        flushed (256 MiB write) before every timed step and excluded.
e2e     the same evaluation through the public C ABI with host (pinned)
        buffers: coefficient upload, kernels, gradient + score download.
N > 1   independent replicas, one per GPU (weak scaling, no collective on
        the data path); max device time over ranks.
fp32_form / tc_over_fp32
        the other device form (plain FP32 SIMT) timed the same way in the
        same run, its fraction of the FP32 FMA peak, and the tensor-core
        form's speed-up over it (device and end to end).
accuracy
        score and gradient relative error of the timed form's evaluation
        against the double-precision oracle and the reference's own float
        flavour g on the same inputs (after the timed region).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "B-spline score+grad Gvox/s: BF16-TC vs FP32 form, one B200, grad err<=1e-3"
WORKLOAD = {"workload": "mse_score_grad_256x256x128_vpr5",
            "dims": [256, 256, 128], "spacing_mm": [0.98, 0.98, 2.5],
            "vox_per_rgn": [5, 5, 5], "coeff_sigma_mm": 3.0,
            "content": "CT-like int16 phantom (body/lung/bone ellipsoids + N(0,20))",
            "gradient": "nearest-voxel moving gradient (reference flavour g)"}
ALGO_BYTES_PER_VOXEL = 20   # fixed f32 + moving f32 + moving gradient 3xf32
# forward field 2*64*3 + adjoint 2*64*3 + trilinear, difference and dc/dv
ALGO_FLOP_PER_VOXEL = 808


def make_workload(seed=20261205):
    from plastimatch_b200 import synth
    from plastimatch_b200.geometry import BsplineGrid, Volume
    fixed = synth.ct_phantom((256, 256, 128), spacing=(0.98, 0.98, 2.5),
                             seed=seed)
    mov = synth.ct_phantom((256, 256, 128), spacing=(0.98, 0.98, 2.5),
                           seed=seed + 1)
    # shift the moving phantom by a fraction of a voxel so every sample is
    # a genuine trilinear blend
    moving = Volume(mov.img, origin=(0.37, -0.21, 0.55), spacing=mov.spacing)
    grid = BsplineGrid.for_volume(fixed, 5)
    coeff = synth.random_coeff(grid, 3.0, seed + 2)
    return fixed, moving, grid, coeff


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(kernel):
    """ncu DRAM bytes per launch of the kernel that ran ("tile", "xlane" or
    "fp32", as b200bsp_mse_kernel names it)."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f).get(kernel)
    return None


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device),
                 f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "20"], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # the first sample marks the sampler as live before timing starts
            t0 = time.time()
            while not self.lines and time.time() - t0 < 10:
                time.sleep(0.01)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 6:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for n, v in zip(names, parts[2:6]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [],
                    "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_reference_time(fixed, moving, grid, coeff, evals, threads,
                       warmup=1):
    """Seconds per evaluation of the reference's own OpenMP flavour g
    (oracle/_ref), or of the single-thread restatement when absent."""
    import oracle as O
    if O.ref_available():
        kind = "reference"
        fn = lambda: O.ref_metric(grid, fixed, moving, coeff, flavor="g",
                                  threads=threads)
    else:
        kind, threads = "port", 1
        mg = O.port_volume_grad(moving)
        fn = lambda: O.port_mse(grid, fixed, moving, coeff, moving_grad=mg)
    for _ in range(warmup):
        fn()
    ts = []
    for _ in range(evals):
        t0 = time.perf_counter()
        fn()
        ts.append(time.perf_counter() - t0)
    return float(np.median(ts)), kind, threads


def cpu_reference_others(fixed, moving, grid, coeff, threads):
    """One evaluation each, on the same workload, of the reference's other
    paths: MSE flavour h on one thread (the serial form), Mattes MI flavour
    g (PVI-8, 32 bins) and the analytic regulariser 'c' (curvature 0.005)
    on all host threads; seconds, with the device's Gvox/s beside them in
    also_measured."""
    import oracle as O
    if not O.ref_available():
        return None
    out = {"threads": threads}
    for name, fn in (
            ("mse_flavour_h_1_thread_s",
             lambda: O.ref_metric(grid, fixed, moving, coeff, flavor="h",
                                  threads=1)),
            ("mi_flavour_g_s",
             lambda: O.ref_metric(grid, fixed, moving, coeff, flavor="g",
                                  metric="mi", threads=threads)),
            ("regularizer_analytic_c_s",
             lambda: O.ref_regularize(grid, fixed, coeff, 0.005, impl="c",
                                      threads=threads))):
        t0 = time.perf_counter()
        fn()
        out[name] = time.perf_counter() - t0
    return out


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_reference_arm(args, rank, world):
    if rank != 0:
        return
    fixed, moving, grid, coeff = make_workload()
    import oracle as O
    threads = host_threads()
    if O.ref_available():
        kind = "reference"
        fn = lambda: O.ref_metric(grid, fixed, moving, coeff, flavor="g",
                                  threads=threads)
    else:
        kind, threads = "port", 1
        mg = O.port_volume_grad(moving)
        fn = lambda: O.port_mse(grid, fixed, moving, coeff, moving_grad=mg)
    for _ in range(args.warmup):
        fn()
    ts = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        fn()
        ts.append(time.perf_counter() - t0)
    sec = float(np.sum(ts)) / args.steps
    v = grid.num_roi_voxels / sec / 1e9
    out = {"metric": METRIC, "impl": "reference", "value": v,
           "unit": "Gvox/s", "n_gpus": args.gpus, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": sec * 1e3,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f32", "data": "synthetic",
           "config": dict(WORKLOAD, form="reference CPU flavour g (OpenMP)"),
           "cpu_baseline": {"value": v, "unit": "Gvox/s", "cores": threads,
                            "kind": kind,
                            "sample": "one full 256x256x128 evaluation per step"},
           "e2e": {"value": v, "unit": "Gvox/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def registration_c1(P, with_cpu):
    """The reference's CPU-runnable case: 64^3 blobs, moving = fixed under a
    seeded B-spline warp (8-voxel spacing, N(0, 2 mm)), vox_per_rgn 8, zero
    initial coefficients, MSE, 30 L-BFGS iterations (liblbfgs semantics,
    max_feval 100).  Wall time of the whole optimisation on the device, and
    of the reference's own bspline_optimize (liblbfgs) on the host cores."""
    from plastimatch_b200 import synth
    from plastimatch_b200.geometry import BsplineGrid
    fixed = synth.gaussian_blobs((64, 64, 64), spacing=(1, 1, 1),
                                 seed=20261204)
    g0 = BsplineGrid.for_volume(fixed, 8)
    moving = synth.warp_trilinear(fixed, fixed, g0,
                                  synth.random_coeff(g0, 2.0, 20261205))
    grid = BsplineGrid.for_volume(fixed, 8)
    x0 = np.zeros(grid.num_coeff, np.float32)
    out = {}
    with P.Context(fixed, moving, grid) as ctx:
        ctx.set_images()
        ctx.optimize_lbfgs(x0, max_its=2, max_feval=4)      # warm-up
        t0 = time.perf_counter()
        c, res = ctx.optimize_lbfgs(x0, max_its=30, max_feval=100)
        out["gpu_s"] = time.perf_counter() - t0
        out["fevals"] = res["fevals"]
        out["final_score"] = res["score"]
        s0, _, _ = ctx.score_mse(x0)
        out["initial_score"] = s0
    if with_cpu:
        import oracle as O
        if O.ref_available():
            t0 = time.perf_counter()
            _, sref, _, fe = O.ref_optimize(grid, fixed, moving, x0,
                                            max_its=30, max_feval=100,
                                            threads=host_threads())
            out["cpu_reference_s"] = time.perf_counter() - t0
            out["cpu_reference_fevals"] = fe
            out["cpu_reference_final_score"] = sref
    return out


def batched_c5(P, n_regs=16, its=40):
    """Batched multi-atlas registration: n_regs MSE registrations of seeded
    uneven sizes (U{128..320} x U{128..320} x U{64..160} voxels, in-plane and
    slice spacing U[1, 2.5] mm, Gaussian-blob content, moving = fixed under
    a seeded B-spline warp with 10 mm spacing and N(0, 2 mm) coefficients),
    a 10 mm control grid (vox_per_rgn = round(10 mm / spacing), at least
    4), zero initial coefficients, `its` L-BFGS iterations each (max_feval
    100).  Wall time with all registrations advancing together (one graph
    launch per round of evaluations), for the tensor-core and the FP32
    forms, and of the same registrations run one after another."""
    from plastimatch_b200 import synth
    from plastimatch_b200.geometry import BsplineGrid, Volume
    g = synth.rng(20261207)
    cases = []
    for k in range(n_regs):
        dim = (int(g.integers(128, 321)), int(g.integers(128, 321)),
               int(g.integers(64, 161)))
        sxy, sz = float(g.uniform(1.0, 2.5)), float(g.uniform(1.0, 2.5))
        fixed = synth.gaussian_blobs(dim, spacing=(sxy, sxy, sz),
                                     seed=20261207 + 100 * k)
        vpr = tuple(max(4, int(round(10.0 / s))) for s in (sxy, sxy, sz))
        g0 = BsplineGrid.for_volume(fixed, vpr)
        with P.Context(fixed, fixed, g0) as wctx:       # the moving image
            wctx.set_images()
            mimg = wctx.warp(synth.random_coeff(g0, 2.0,
                                                20261207 + 100 * k + 1))
        moving = Volume(mimg.reshape(fixed.img.shape), origin=fixed.origin,
                        spacing=fixed.spacing)
        cases.append((fixed, moving, BsplineGrid.for_volume(fixed, vpr)))
    nvox = [c[2].num_roi_voxels for c in cases]
    out = {"registrations": n_regs, "iterations": its,
           "voxels_total": int(sum(nvox))}

    def run(form, batched):
        ctxs = [P.Context(f, m, gr, form=form).set_images()
                for f, m, gr in cases]
        try:
            x = [np.zeros(gr.num_coeff, np.float32) for _, _, gr in cases]
            tiles = [c.autotune(xi, evals=2) for c, xi in zip(ctxs, x)]
            if batched:
                with P.Batch(ctxs) as b:
                    b.optimize_lbfgs([xi.copy() for xi in x], max_its=2,
                                     max_feval=4)                # warm-up
                    t0 = time.perf_counter()
                    res = b.optimize_lbfgs(x, max_its=its, max_feval=100)
                    dt = time.perf_counter() - t0
            else:
                for c, xi in zip(ctxs, x):
                    c.optimize_lbfgs(xi.copy(), max_its=2, max_feval=4)
                t0 = time.perf_counter()
                res = [c.optimize_lbfgs(xi, max_its=its, max_feval=100)[1]
                       for c, xi in zip(ctxs, x)]
                dt = time.perf_counter() - t0
        finally:
            for c in ctxs:
                c.close()
        fe = [r["fevals"] for r in res]
        return {"wall_s": dt, "fevals": int(sum(fe)),
                "autotuned_tiles_per_batch": tiles,
                "gvox_per_s": float(sum(f * n for f, n in zip(fe, nvox))
                                    / dt / 1e9),
                "final_scores": [round(float(r["score"]), 4) for r in res]}

    out["tc_batched"] = run("tc", True)
    out["tc_one_after_another"] = run("tc", False)
    out["fp32_batched"] = run("fp32", True)
    return out


def mi_registration_c4(P, its=50):
    """Multi-resolution Mattes MI registration: 512x512x160 CT-like fixed
    image (0.98 x 0.98 x 2.5 mm), moving = fixed under a smooth random
    B-spline warp (20 mm grid, N(0, 3 mm)) and a monotone intensity remap
    (gamma U[0.5, 2]) + N(0, 30); 32 x 32 joint histogram with cubic
    B-spline Parzen windows; subsampling 4, 2, 1; 10 mm grid; `its` L-BFGS
    iterations per level.  Wall time per level and in all, and the
    full-resolution MI before and after."""
    from plastimatch_b200 import synth
    from plastimatch_b200.geometry import BsplineGrid, Volume
    from plastimatch_b200.pipeline import register_pyramid
    seed = 20261206
    fixed = synth.ct_phantom((512, 512, 160), spacing=(0.98, 0.98, 2.5),
                             seed=seed)
    gw = BsplineGrid.for_grid_spacing(fixed, 20.0)
    with P.Context(fixed, fixed, gw, form="fp32") as ctx:
        ctx.set_images()
        warped = ctx.warp(synth.random_coeff(gw, 3.0, seed + 1),
                          default_value=-1000.0)
    gamma = float(synth.rng(seed + 2).uniform(0.5, 2.0))
    moving = synth.intensity_remap(
        Volume(warped, origin=fixed.origin, spacing=fixed.spacing), gamma,
        30.0, seed + 3)
    t0 = time.perf_counter()
    coeff, grid, hist = register_pyramid(fixed, moving, levels=(4, 2, 1),
                                         grid_mm=10.0, metric="mi",
                                         mi_window="parzen", its=its)
    total = time.perf_counter() - t0
    with P.Context(fixed, moving, grid, mi_window="parzen") as ctx:
        ctx.set_images()
        s_id = ctx.score_mi(np.zeros(grid.num_coeff, np.float32))[0]
        s_reg = ctx.score_mi(coeff)[0]
    return {"levels": [{k: (round(v, 4) if isinstance(v, float) else v)
                        for k, v in h.items()} for h in hist],
            "total_s": total, "gamma": gamma,
            "mi_identity": s_id, "mi_registered": s_reg}


def extra_metrics(P, ctx, stream, flush, d_coeff, d_grad, nvox, warmup,
                  evals=50, which=("mse_reg", "mi")):
    """The same workload with the curvature regulariser added (lambda 0.005)
    and with Mattes MI (PVI-8, 32 bins) instead of MSE: device time per
    evaluation (CUDA events on the context stream, L2 flushed before each),
    reported beside the headline MSE number."""
    import ctypes as C
    import torch
    lib = P.lib()
    reg = P.reg_parms(curvature=0.005)
    s_c, n_c = C.c_float(), C.c_int64()

    d_total = torch.zeros(4, device=d_grad.device)

    def mse_reg():
        # bspline_score with device outputs: the regulariser overlaps the
        # tile kernel on the context's second stream
        rc = lib.b200bsp_score(ctx._h, d_coeff.data_ptr(), 0, C.c_float(1.0),
                               C.byref(reg), d_total.data_ptr(),
                               d_grad.data_ptr(), d_total[1:].data_ptr(),
                               None)
        if rc:
            raise RuntimeError(lib.b200bsp_last_error(ctx._h))

    def mi():
        rc = lib.b200bsp_score_mi(ctx._h, d_coeff.data_ptr(), C.addressof(s_c),
                                  d_grad.data_ptr(), C.addressof(n_c), None,
                                  None, None)
        if rc:
            raise RuntimeError(lib.b200bsp_last_error(ctx._h))

    out = {}
    for key, name, fn in (("mse_reg", "mse_plus_curvature_regularizer", mse_reg),
                          ("mi", "mattes_mi_pvi8_32bins", mi)):
        if key not in which:
            continue
        ts = []
        for i in range(warmup + evals):
            with torch.cuda.stream(stream):
                flush.fill_(1)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            if i >= warmup:
                ts.append(a.elapsed_time(b))
        ms = float(np.median(ts))
        out[name] = {"value": nvox / (ms * 1e-3) / 1e9, "unit": "Gvox/s",
                     "ms_per_eval": ms, "evals": evals}
    return out


def measure_form(P, form, args, workload, local_rank, dist, flush,
                 tc_kernel="auto"):
    """Device and end-to-end throughput of one form on the workload.

    Returns a dict: device ms per evaluation (CUDA events on the context's
    stream, L2 flushed before every step and excluded, max over ranks),
    end-to-end ms through the C ABI with pinned host buffers, the tile
    kernel's own ms (the library's events, median of three probes), the
    launches per evaluation, the autotuned tiles per batch, and the last
    evaluation's score, gradient and voxel count (host copies)."""
    import ctypes as C
    import torch
    fixed, moving, grid, coeff = workload
    dev = f"cuda:{local_rank}"
    ctx = P.Context(fixed, moving, grid, form=form, device=local_rank,
                    tc_kernel=tc_kernel if form == "tc" else "auto")
    stream = torch.cuda.Stream(device=local_rank)
    ctx.set_stream(stream.cuda_stream)
    ctx.set_images()
    # the library's batch-split autotuner (setup, like a GEMM heuristic),
    # before any timing
    tiles = ctx.autotune(coeff, evals=3) if form == "tc" else None
    d_coeff = torch.from_numpy(coeff).to(dev)
    d_grad = torch.zeros(grid.num_coeff, device=dev)
    d_score = torch.zeros(1, device=dev)
    d_nvox = torch.zeros(1, dtype=torch.int64, device=dev)
    torch.cuda.synchronize()

    def step():
        ctx.score_mse(d_coeff, grad_out=d_grad, score_out=d_score,
                      nvox_out=d_nvox)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            flush.fill_(1)
            step()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        with torch.cuda.stream(stream):
            for i in range(args.steps):
                flush.fill_(1)
                ev[i][0].record(stream)
                step()
                ev[i][1].record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    dev_ms = sum(a.elapsed_time(b) for a, b in ev) / args.steps
    t = torch.tensor([dev_ms], device=dev)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dev_ms = float(t.item())

    # per-evaluation main-kernel time (library events on the same stream;
    # the instrumentation is on for these probes only)
    main_ms = []
    ctx.enable_timing(True)
    for _ in range(3):
        flush.fill_(1)
        stream.synchronize()
        s_h, g_h, n_h = ctx.score_mse(d_coeff)
        _, m_ms, launches = ctx.last_timing()
        main_ms.append(m_ms)
    ctx.enable_timing(False)

    # end to end through the C ABI with pinned host buffers
    h_coeff = torch.from_numpy(coeff).pin_memory()
    h_grad = torch.zeros(grid.num_coeff).pin_memory()
    lib = P.lib()
    s_c = C.c_float()
    n_c = C.c_int64()
    e2e = []
    for i in range(args.warmup + args.steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        rc = lib.b200bsp_score_mse(ctx._h, h_coeff.data_ptr(),
                                   C.addressof(s_c), h_grad.data_ptr(),
                                   C.addressof(n_c))
        b.record(stream)
        b.synchronize()
        if rc:
            raise RuntimeError(lib.b200bsp_last_error(ctx._h))
        if i >= args.warmup:
            e2e.append(a.elapsed_time(b))
    e2e_ms = float(np.mean(e2e))
    t = torch.tensor([e2e_ms], device=dev)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_ms = float(t.item())
    return {"ctx": ctx, "stream": stream, "d_coeff": d_coeff,
            "d_grad": d_grad, "dev_ms": dev_ms, "e2e_ms": e2e_ms,
            "kernel_ms": float(np.median(main_ms)), "launches": launches,
            "tiles": tiles, "kernel": ctx.mse_kernel(), "score": s_h,
            "grad": g_h, "num_vox": n_h, "clocks": clk.summary()}


def tc_kernel_probe(P, workload, local_rank, flush, probes=5):
    """Each tensor-core MSE kernel pinned in turn on the workload (x-lane:
    voxel x on the TMEM lanes; tile: one tile's 125 voxels on the lanes),
    autotuned over its batch splits: its own kernel time (the library's
    events, L2 flushed before each probe, median)."""
    import torch
    fixed, moving, grid, coeff = workload
    out = {}
    for k in ("xlane", "tile"):
        try:
            ctx = P.Context(fixed, moving, grid, form="tc", device=local_rank,
                            tc_kernel=k)
        except P.B200Error as e:
            out[k] = {"unsupported": str(e)}
            continue
        with ctx:
            ctx.set_images()
            ctx.autotune(coeff, evals=3)
            d_coeff = torch.from_numpy(coeff).to(f"cuda:{local_rank}")
            ctx.enable_timing(True)
            ms = []
            for _ in range(probes):
                flush.fill_(1)
                torch.cuda.synchronize()
                ctx.score_mse(d_coeff)
                ms.append(ctx.last_timing()[1])
            name, tiles, batches = ctx.mse_kernel()
            out[k] = {"kernel_ms": float(np.median(ms)), "tiles": tiles,
                      "batches": batches}
    return out


def accuracy_block(workload, score, grad, num_vox, threads):
    """Score and gradient relative error of a device evaluation against the
    double-precision oracle and against the reference's own float flavour
    g on the same inputs (computed after the timed region)."""
    import oracle as O
    fixed, moving, grid, coeff = workload
    mg = O.port_volume_grad(moving)
    f64 = O.port_mse(grid, fixed, moving, coeff, moving_grad=mg,
                     precision="f64")

    def rel(a, b):
        a = np.asarray(a, np.float64)
        b = np.asarray(b, np.float64)
        return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))

    out = {"vs_fp64_oracle": {
               "score_rel": abs(score - f64.score) / abs(f64.score),
               "grad_rel_l2": rel(grad, f64.grad),
               "num_vox": int(f64.num_vox)},
           "bars": {"score_rel": 1e-5,
                    "grad_rel_l2_vs_reference": 1e-3,
                    "grad_rel_l2_vs_fp64": "the reference float flavour's "
                                           "own error + 1e-4"}}
    r = (O.ref_metric(grid, fixed, moving, coeff, flavor="g",
                      threads=threads) if O.ref_available()
         else O.port_mse(grid, fixed, moving, coeff, moving_grad=mg))
    out["vs_reference_flavour_g"] = {
        "score_rel": abs(score - r.score) / abs(r.score),
        "grad_rel_l2": rel(grad, r.grad),
        "num_vox": int(r.num_vox)}
    # the reference's own float evaluation against double precision on
    # the same inputs (the floor any float implementation shares)
    out["reference_float_vs_fp64"] = {
        "score_rel": abs(r.score - f64.score) / abs(f64.score),
        "grad_rel_l2": rel(r.grad, f64.grad)}
    out["device_num_vox"] = int(num_vox)
    return out


def run_slab(args, rank, world, local_rank):
    """--mode slab: one 256x256x128 volume sharded by z-slab over the
    process group (plastimatch_b200.shard.SlabScorer): each rank evaluates
    its slab through a context on its GPU, then one NCCL all-reduce of the
    raw sums (FP64) assembles the global score and gradient on every rank.
    Strong scaling (the volume is fixed); one step = one global evaluation
    from host coefficients to the host gradient, so value and e2e are the
    same measurement."""
    import torch
    import plastimatch_b200 as P
    from plastimatch_b200 import shard
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    fixed, moving, grid, coeff = make_workload()
    dev = torch.device("cuda", local_rank)
    mg = P.volume_grad(moving)
    evaluate = shard.context_evaluator(fixed, moving, form=args.form,
                                       device=local_rank, moving_grad=mg)
    if world > 1:
        scorer = shard.SlabScorer(grid, evaluate, device=dev)
        step = lambda: scorer.score_mse(coeff)
    else:
        # one rank: the whole grid is the one slab, no collective
        def step():
            s, g, nv = evaluate(grid, coeff)
            return (float(np.float32(s / nv)),
                    (2.0 * g / nv).astype(np.float32), nv)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    for _ in range(args.warmup):
        flush.fill_(1)
        step()
    ev = [(torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        for i in range(args.steps):
            flush.fill_(1)
            ev[i][0].record(stream)
            res = step()
            ev[i][1].record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = sum(a.elapsed_time(b) for a, b in ev) / args.steps
    t = torch.tensor([ms], device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    nvox = grid.num_roi_voxels
    value = nvox / (ms * 1e-3) / 1e9
    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": "Gvox/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": dict(WORKLOAD, form=args.form, mode="slab",
                           l2="256 MiB flush write before every timed step",
                           parallelism=f"z-slabs x{world}, NCCL all-reduce "
                                       "of the raw sums (FP64)"),
            "e2e": {"value": value, "unit": "Gvox/s",
                    "h2d_bytes_per_step": 4 * grid.num_coeff,
                    "d2h_bytes_per_step": 8 * grid.num_coeff},
            # per step and rank: the slab's MSE kernel and finish kernel
            "gpu_launches": 2 * args.steps,
            "clocks": clk.summary(),
            "score": res[0], "num_vox": res[2],
        }
        print(json.dumps(out), flush=True)
    for c in evaluate.contexts.values():
        c.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--form", default="tc", choices=["tc", "fp32"])
    ap.add_argument("--tc-kernel", default="auto",
                    choices=["auto", "xlane", "tile"])
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--mode", default="replicas", choices=["replicas", "slab"],
                    help="replicas: one evaluation stream per GPU (the "
                         "headline); slab: one volume sharded by z-slab "
                         "with an NCCL all-reduce")
    ap.add_argument("--cpu-evals", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip also_measured (regulariser, MI, the "
                         "registration workloads)")
    ap.add_argument("--extras", default="all",
                    help="comma-separated also_measured entries to run: "
                         "kernels (both tensor-core kernels pinned), "
                         "mse_reg, mi, batched, mi_pyramid, registration "
                         "(default all)")
    args = ap.parse_args()
    extras = ({"kernels", "mse_reg", "mi", "batched", "mi_pyramid",
               "registration"} if args.extras == "all"
              else set(args.extras.split(",")))
    if args.no_extra:
        extras = set()
    if args.warmup < 3:
        args.warmup = 3

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return
    if args.mode == "slab":
        run_slab(args, rank, world, local_rank)
        return

    import torch
    import plastimatch_b200 as P
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))

    workload = make_workload()
    fixed, moving, grid, coeff = workload
    flush = torch.empty(256 << 20, dtype=torch.uint8,
                        device=f"cuda:{local_rank}")
    m = measure_form(P, args.form, args, workload, local_rank, dist, flush,
                     args.tc_kernel)
    ctx, stream = m["ctx"], m["stream"]
    # the other form, timed the same way in the same run (the metric's
    # comparison); replicas time it too so every rank takes the same
    # collective steps
    other = "fp32" if args.form == "tc" else "tc"
    mo = measure_form(P, other, args, workload, local_rank, dist, flush)
    mo["ctx"].close()

    extra = {}
    if "kernels" in extras:
        extra["tc_kernels"] = tc_kernel_probe(P, workload, local_rank, flush)
    extra.update(extra_metrics(P, ctx, stream, flush, m["d_coeff"],
                               m["d_grad"], grid.num_roi_voxels, args.warmup,
                               which=extras))
    if rank == 0 and world == 1:
        # one-GPU workloads, measured at N = 1 only (the other ranks would
        # idle meanwhile); the device-only ones first: the reference's
        # OpenMP threads (registration_c1's CPU leg) keep host cores busy
        # for a while after they finish, which would slow the host-side
        # line searches
        if "batched" in extras:
            extra["batched_16_registrations_40_lbfgs_its"] = batched_c5(P)
        if "mi_pyramid" in extras:
            extra["mi_parzen_registration_512x512x160_pyramid_4_2_1"] = \
                mi_registration_c4(P)
        if "registration" in extras:
            extra["registration_64cubed_vpr8_30_lbfgs_its"] = \
                registration_c1(P, not args.no_cpu_baseline and world == 1)

    nvox = grid.num_roi_voxels
    peak, peak_kind = measured_peaks()

    def summary(r, form):
        value = world * nvox / (r["dev_ms"] * 1e-3) / 1e9
        e2e_value = world * nvox / (r["e2e_ms"] * 1e-3) / 1e9
        achieved = ALGO_BYTES_PER_VOXEL * nvox / (r["kernel_ms"] * 1e-3) / 1e9
        return value, e2e_value, {
            "bound": "hbm", "achieved": achieved, "peak": peak,
            "unit": "GB/s", "frac": achieved / peak,
            "traffic": profile_traffic(r["kernel"][0]),
            "traffic_kernel": r["kernel"][0], "peak_source": peak_kind,
            "kernel_ms": r["kernel_ms"],
            "algorithmic_bytes_per_launch": ALGO_BYTES_PER_VOXEL * nvox}

    value, e2e_value, roofline = summary(m, args.form)
    o_value, o_e2e, o_roof = summary(mo, other)
    props = torch.cuda.get_device_properties(local_rank)
    clk = m["clocks"]
    sm_mhz = clk.get("sm_max_mhz") or 1965.0
    # FP32 FMA peak at the sampled maximum SM clock: SMs x 128 lanes x 2
    fp32_peak = props.multi_processor_count * 128 * 2 * sm_mhz * 1e6 / 1e12
    fp32_r = m if args.form == "fp32" else mo
    fp32_tflops = ALGO_FLOP_PER_VOXEL * nvox / (fp32_r["kernel_ms"] * 1e-3) / 1e12
    other_block = {"form": other, "value": o_value, "unit": "Gvox/s",
                   "ms_per_step": mo["dev_ms"],
                   "e2e": {"value": o_e2e, "unit": "Gvox/s"},
                   "kernel_ms": mo["kernel_ms"], "roofline": o_roof}
    if other == "fp32":
        other_block["fma"] = {
            "achieved_tflops": fp32_tflops, "peak_tflops": fp32_peak,
            "frac": fp32_tflops / fp32_peak,
            "flop_per_voxel": ALGO_FLOP_PER_VOXEL,
            "peak_source": "nominal: SMs x 128 FP32 lanes x 2 x max SM clock"}
    tc_v, fp_v = (value, o_value) if args.form == "tc" else (o_value, value)
    tc_e, fp_e = ((e2e_value, o_e2e) if args.form == "tc"
                  else (o_e2e, e2e_value))
    out = None
    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline and world == 1:
            sec, kind, th = cpu_reference_time(fixed, moving, grid, coeff,
                                               args.cpu_evals, host_threads())
            cpu = {"value": nvox / sec / 1e9, "unit": "Gvox/s", "cores": th,
                   "kind": kind,
                   "sample": f"{args.cpu_evals} full evaluations of the same "
                             "256x256x128 workload (median)"}
            if extras and args.extras == "all":
                extra["cpu_reference_other_paths"] = cpu_reference_others(
                    fixed, moving, grid, coeff, host_threads())
        acc = accuracy_block(workload, m["score"], m["grad"], m["num_vox"],
                             host_threads())
        out = {
            "metric": METRIC, "value": value, "unit": "Gvox/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": m["dev_ms"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": dict(WORKLOAD, form=args.form,
                           arithmetic="voxel work f32; tensor-core products "
                                      "as 3-term bf16 splits with f32 "
                                      "accumulation" if args.form == "tc"
                                      else "f32 SIMT",
                           l2="inputs 167 MB > L2 and 256 MiB flush write "
                              "before every timed step (excluded)",
                           parallelism=f"replicas x{world}",
                           tc_kernel=m["kernel"][0] if args.form == "tc"
                           else None,
                           tiles_per_batch=m["kernel"][1],
                           batches=m["kernel"][2]),
            "e2e": {"value": e2e_value, "unit": "Gvox/s",
                    "h2d_bytes_per_step": 4 * grid.num_coeff,
                    "d2h_bytes_per_step": 4 * grid.num_coeff + 32},
            "roofline": roofline,
            "accuracy": acc,
            ("fp32_form" if other == "fp32" else "tc_form"): other_block,
            "tc_over_fp32": {"value": tc_v / fp_v, "e2e": tc_e / fp_e,
                             "target": 5.0},
            "cpu_baseline": cpu,
            "also_measured": extra,
            "gpu_launches": m["launches"] * args.steps,
            "clocks": clk,
            "score": m["score"], "num_vox": m["num_vox"],
        }
        print(json.dumps(out), flush=True)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
