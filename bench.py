#!/usr/bin/env python
"""ESP throughput benchmark: the 54-atom l<=3 synthetic system at 30000 vdW points.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision fp64|mixed] [--points 30000]

A step is one evaluation of the ESP at all points of the workload with the
pair table resident in HBM (``value``, points/s).  ``e2e`` is the same metric
through the public API from pinned host buffers: density and points copied to
the device, the table built, the ESP evaluated and copied back, every step.
The table-build time is reported separately.  Under torchrun every rank
evaluates its own 30000-point set of the same molecule (weak scaling, no
collective on the data path); times are the max over ranks.

``--impl reference`` times the reference's own CPU path on the host cores:
its OpenMP C++ table builder (oracle/_ref/build_pairs, compiled from the
reference's source) plus its NumPy evaluator (restated in oracle/) on a
bounded per-class sample of pairs, scaled by the class pair counts.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOAD = ("frag54: 54 atoms (30 C / 8 N / 8 O / 8 H), l<=3 TZ-like basis with diffuse "
            "functions (1658 Cartesian functions, 2088 primitives), 30000 points on the "
            "1.4x Bondi vdW surface, screening tol 1e-12")
METRIC = "ESP points/s, 54-atom l<=3 basis: mixed vs FP64 GPU path at <=1e-6 a.u. max err"
PUBLISHED = {"e2e_points_per_s": 30000 / 2.4564, "hardware": "RTX 5090",
             "source": "reference README.md:48 (table build + GPU solve, 30000 points)"}


from fastesp_b200.shard import rank_info, rank_points  # noqa: E402


# ---------------------------------------------------------------------------
# clocks sampling
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 6:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for n, v in zip(names, f[2:6]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def peak_flops(torch, kind):
    """Measured FMA throughput (FLOP/s) of this GPU: kind 0 scalar FP32, 1 FP64,
    2 packed FP32x2 (fe_peak_run: 8 independent FMA chains per thread)."""
    from fastesp_b200 import _lib
    dev = torch.cuda.current_device()
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    blocks = sms * 8
    out = torch.empty(blocks, dtype=torch.float64, device="cuda")
    iters = 1 << 14 if kind == 1 else 1 << 15
    per_iter = 32.0 if kind == 2 else 16.0
    for _ in range(2):
        _lib.check(_lib.lib().fe_peak_run(kind, iters, blocks, _lib.ptr(out), _lib.stream_ptr()))
    best = 0.0
    for _ in range(5):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        _lib.check(_lib.lib().fe_peak_run(kind, iters, blocks, _lib.ptr(out), _lib.stream_ptr()))
        b.record()
        b.synchronize()
        best = max(best, per_iter * iters * 256 * blocks / (a.elapsed_time(b) * 1e-3))
    return best


def build_flops(wfn):
    """Algorithmic FLOPs of one table build without the point screen: every
    primitive pair of every shell pair si <= sj (hermite.build_flops)."""
    from fastesp_b200 import hermite as H
    sh = wfn.shells
    tot = 0
    for i in range(len(sh)):
        for j in range(i, len(sh)):
            la, lb = sh[i].l, sh[j].l
            tot += len(sh[i].exps) * len(sh[j].exps) * H.build_flops(min(la, lb), max(la, lb))
    return float(tot)


def build_pairs_count(wfn):
    sh = wfn.shells
    n = [len(s.exps) for s in sh]
    return int(sum(n[i] * n[j] for i in range(len(sh)) for j in range(i, len(sh))))


def per_class_rates(torch, tab, pts_d, npts, flush, peak64, peak32, reps=5):
    """Time each class alone (fe_electron_classes) in both precisions: ms,
    algorithmic TFLOP/s and the fraction of the FP64 / FP32 peak."""
    from fastesp_b200 import _lib, hermite as H
    L_ = _lib.lib()
    out = torch.empty(npts, dtype=torch.float64, device=pts_d.device)
    ws = torch.empty(max(tab.ws_bytes(npts, "fp64"), tab.ws_bytes(npts, "mixed")),
                     dtype=torch.uint8, device=pts_d.device)
    rows = []
    for L, c in enumerate(tab.counts):
        if not c:
            continue
        fl = float(c) * H.eval_flops(L) * npts
        row = {"class": L, "pairs": int(c), "flops": fl}
        for prec, name, peak in ((0, "fp64", peak64), (1, "mixed", peak32)):
            def run():
                _lib.check(L_.fe_electron_classes(_lib.ptr(tab._buf), _lib.ptr(pts_d), npts,
                                                  _lib.ptr(out), _lib.ptr(ws), ws.numel(), prec,
                                                  0.0, L, L, None, _lib.stream_ptr()))
            ms = _median_ms(run, reps, warm=2, flush=flush)
            row[f"{name}_ms"] = ms
            row[f"{name}_tflops"] = fl / (ms * 1e-3) / 1e12
            row[f"{name}_frac"] = fl / (ms * 1e-3) / peak
        rows.append(row)
    return rows


def hbm_view(traffic, ms):
    """The memory side of the dominant kernel: its ncu DRAM bytes per launch over
    the step time, against the measured HBM copy bandwidth (MEASURED_PEAKS.json)."""
    if traffic is None:
        return None
    peaks = ROOT / "MEASURED_PEAKS.json"
    gbs = json.loads(peaks.read_text()).get("hbm_gbs") if peaks.exists() else None
    src = "MEASURED_PEAKS.json hbm_gbs (measured)"
    if not gbs:
        gbs, src = 6650.0, "fallback: 6.65 TB/s, an earlier measurement on this pool"
    achieved = traffic / (ms * 1e-3) / 1e9
    return {"achieved": achieved, "peak": gbs, "unit": "GB/s", "frac": achieved / gbs,
            "peak_source": src}


def build_roofline(wfn, build_ms, peak64, npts):
    """The table build against the FP64 peak: E-coefficients, Hermite table and
    G contraction of every primitive pair over the build time.  The point
    screen is left out of the count: the reference's brute-force screen
    (8 FLOP per pair and point) is quoted beside it, but the build here prunes
    it over point-block bounding boxes and does a small fraction of that work."""
    if build_ms is None:
        return None
    fl = build_flops(wfn)
    npair = build_pairs_count(wfn)
    return {"ms": build_ms, "primitive_pairs": npair, "flops": fl,
            "achieved": fl / (build_ms * 1e-3) / 1e12, "peak": peak64 / 1e12, "unit": "TFLOP/s",
            "frac": fl / (build_ms * 1e-3) / peak64,
            "bruteforce_screen_flops": 8.0 * npair * npts}


def algorithmic_flops(counts, npts):
    from fastesp_b200 import hermite as H
    return float(sum(c * H.eval_flops(L) for L, c in enumerate(counts))) * npts


def run_ours(args):
    import torch
    import torch.distributed as dist
    from fastesp_b200 import _lib, build_table, synth
    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    wfn, basis, P, _ = synth.load_workload("frag54", 10, seed=0)
    pts = rank_points(wfn.symbols, wfn.coords, args.points, rank)    # weak scaling
    dev = torch.device("cuda", local)
    P_d = torch.as_tensor(P, device=dev)
    pts_d = torch.as_tensor(pts, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # table build (device-resident inputs)
    tab = build_table(wfn, basis, P_d, pts_d, tol=1e-12)
    counts = tab.counts
    prec = args.precision
    tb = []
    for i in range(0 if args.eval_only else args.warmup + max(3, args.steps // 2)):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        t2 = build_table(wfn, basis, P_d, pts_d, tol=1e-12)
        b.record()
        b.synchronize()
        if i >= args.warmup:
            tb.append(a.elapsed_time(b))
        del t2
    build_ms = statistics.median(tb) if tb else None

    # value: evaluation with the table resident, both precisions
    out = torch.empty(args.points, dtype=torch.float64, device=dev)
    L = _lib.lib()
    ws = torch.empty(max(256, tab.ws_bytes(args.points, "fp64"), tab.ws_bytes(args.points, "mixed")),
                     dtype=torch.uint8, device=dev)
    n64 = torch.zeros(1, dtype=torch.int64, device=dev)

    def step_fp64():
        _lib.check(L.fe_esp_fp64(_lib.ptr(tab._buf), _lib.ptr(pts_d), args.points, _lib.ptr(out),
                                 _lib.ptr(ws), ws.numel(), _lib.stream_ptr()))

    def step_mixed():
        _lib.check(L.fe_esp_mixed(_lib.ptr(tab._buf), _lib.ptr(pts_d), args.points, _lib.ptr(out),
                                  _lib.ptr(ws), ws.numel(), 0.0, None, _lib.stream_ptr()))

    def timed(step, clk=None):
        for _ in range(args.warmup):
            flush.zero_()
            step()
        barrier()
        times = []
        for _ in range(args.steps):
            flush.zero_()            # L2 flush between timed steps (not timed)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            step()
            b.record()
            b.synchronize()
            times.append(a.elapsed_time(b))
        barrier()
        t = sum(times)
        if world > 1:
            tt = torch.tensor([t], device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            t = float(tt[0])
        return t / args.steps

    main_step, other_step = (step_mixed, step_fp64) if prec == "mixed" else (step_fp64, step_mixed)
    with ClockSampler(local) as clk:
        ms_per_step = timed(main_step)
    ms_other = timed(other_step)
    ms_fp64, ms_mixed = (ms_other, ms_per_step) if prec == "mixed" else (ms_per_step, ms_other)
    if args.eval_only:
        if rank == 0:
            print(json.dumps({"eval_only": True, "mixed_ms": ms_mixed, "fp64_ms": ms_fp64,
                              "points": args.points, "pairs": int(sum(counts))}))
        if world > 1:
            dist.destroy_process_group()
        return
    if world > 1 and build_ms is not None:
        t = torch.tensor([build_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        build_ms = float(t[0])
    value = world * args.points / (ms_per_step * 1e-3)
    # accuracy of the mixed path against the FP64 path on this run's points
    step_fp64()
    v64 = out.clone()
    _lib.check(L.fe_esp_mixed(_lib.ptr(tab._buf), _lib.ptr(pts_d), args.points, _lib.ptr(out),
                              _lib.ptr(ws), ws.numel(), 0.0, _lib.ptr(n64), _lib.stream_ptr()))
    dv = (out - v64).abs()
    mixed_err = {"max_abs": float(dv.max()), "rms": float(dv.pow(2).mean().sqrt()),
                 "fp64_routed_pair_warp_evals": int(n64.item()),
                 # warps of 32 threads x 4 points each evaluate every pair
                 "pair_warp_evals": int(sum(counts)) * (((args.points + 511) // 512) * 4)}

    # e2e through the public API from pinned host buffers
    P_h = torch.as_tensor(P).pin_memory()
    pts_h = torch.as_tensor(pts).pin_memory()
    res_h = torch.empty(args.points, dtype=torch.float64).pin_memory()

    def e2e_step():
        t = build_table(wfn, basis, P_h, pts_h, tol=1e-12)
        v = t.esp(pts_h.to(dev, non_blocking=True), precision=prec)
        res_h.copy_(v, non_blocking=True)

    for _ in range(max(1, args.warmup)):
        e2e_step()
    barrier()
    e2e_t = []
    for _ in range(max(3, args.steps // 2)):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        e2e_step()
        b.record()
        b.synchronize()
        e2e_t.append(a.elapsed_time(b))
    e2e_ms = statistics.mean(e2e_t)
    if world > 1:
        t = torch.tensor([e2e_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t[0])
    e2e = {"value": world * args.points / (e2e_ms * 1e-3), "unit": "points/s",
           "h2d_bytes_per_step": int(P_h.numel() * 8 + 2 * pts_h.numel() * 8),
           "d2h_bytes_per_step": int(res_h.numel() * 8), "ms_per_step": e2e_ms,
           "includes": "H2D density+points, GPU table build, GPU evaluation, D2H result"}

    # parity check of this very run against the golden 300-point values
    from fastesp_b200 import build_table as bt
    g = np.load(ROOT / "tests" / "golden" / "frag54_300.npz")
    gt = bt(wfn, basis, P_d, g["points"], tol=1e-12)
    parity = float(np.abs(gt.esp() - g["esp_t12"]).max())
    status = _lib.status(clear=True)

    peak64 = peak_flops(torch, 1)
    peak32_scalar = peak_flops(torch, 0)
    peak32_packed = peak_flops(torch, 2)
    peak32 = max(peak32_scalar, peak32_packed)
    flops = algorithmic_flops(counts, args.points)
    achieved = flops / (ms_per_step * 1e-3)
    peak = peak32 if prec == "mixed" else peak64
    traffic = None
    prof = ROOT / "profiles" / f"eval_{'mixed' if prec == 'mixed' else 'f64'}_frag54_30000.json"
    if prof.exists():
        traffic = json.loads(prof.read_text()).get("dram_bytes_per_launch")
    # per step: the point order (bbox, count, scan, place, rank), the evaluator
    # kernel instances and the reduction
    launches = 5 + (6 if prec == "mixed" else 3)
    line = {
        "metric": METRIC, "value": value, "unit": "points/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if prec == "fp64" else "f32+f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "points_per_gpu": args.points,
                   "pairs": int(sum(counts)), "pairs_per_class": counts,
                   "precision": prec, "l2": "flushed (256 MiB write) between timed steps",
                   "parallelism": f"points sharded across {world} GPU(s), table per GPU"},
        "fp64_points_per_s": world * args.points / (ms_fp64 * 1e-3),
        "mixed_points_per_s": world * args.points / (ms_mixed * 1e-3),
        "mixed_over_fp64": ms_fp64 / ms_mixed,
        "mixed_error_vs_fp64": mixed_err,
        "table_build_ms": build_ms,
        "table_build_warp_screen_pairs": int(tab.info.n_warp_screen),
        "e2e": e2e,
        "roofline": {"bound": "fp32" if prec == "mixed" else "fp64",
                     "achieved": achieved / 1e12, "peak": peak / 1e12, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "peak_source": ("measured FMA throughput (fe_peak_run) on this GPU, this run: "
                                     "FP32 the larger of scalar FFMA and packed FFMA2 "
                                     f"({peak32_scalar / 1e12:.2f} / {peak32_packed / 1e12:.2f} "
                                     "TFLOP/s), FP64 DFMA"),
                     "flops_per_step": flops,
                     "fp64_path": {"achieved": flops / (ms_fp64 * 1e-3) / 1e12,
                                   "peak": peak64 / 1e12, "frac": flops / (ms_fp64 * 1e-3) / peak64},
                     "hbm_view": hbm_view(traffic, ms_per_step),
                     "build": build_roofline(wfn, build_ms, peak64, args.points),
                     "per_class": per_class_rates(torch, tab, pts_d, args.points, flush,
                                                  peak64, peak32)},
        "gpu_launches": args.steps * launches,
        "parity_frag54_300_max_abs": parity,
        "device_status": status,
        "published_reference": PUBLISHED,
    }
    line["clocks"] = clk.summary()
    if world == 1 and not args.no_extras:
        line["extras"] = run_extras(args, dev, flush)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(wfn, basis, P, pts, counts, budget_s=args.cpu_budget)
        # the reference's own GPU pipeline on the same points, as the GPU comparator
        line["reference_gpu"] = reference_cuda(wfn, basis, P, pts)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


# ---------------------------------------------------------------------------
# the other workloads: grid sweep, adjoint, batch (reported beside the headline)
# ---------------------------------------------------------------------------
def _median_ms(fn, reps, warm=2, flush=None):
    import torch
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        if flush is not None:
            flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        b.synchronize()
        ts.append(a.elapsed_time(b))
    return statistics.median(ts)


def run_extras(args, dev, flush, which=("grid", "adjoint", "batch")):
    """Grid sweep (mixed vs FP64 on a cubic grid), the adjoint on the 20-atom
    l<=2 system and at the headline size, and the 64-molecule batch against 64
    plain launches (``which`` selects)."""
    import torch
    from fastesp_b200 import build_table, synth
    from fastesp_b200.batch import BatchESP, separate_launches
    out = {}
    wfn, basis, P, _ = synth.load_workload("frag54", 10, seed=0)
    P_d = torch.as_tensor(P, device=dev)
    sweep = []
    for n in (args.grid_points if "grid" in which else []):
        pts = torch.as_tensor(synth.cubic_grid_points(wfn.coords, n, seed=2), device=dev)
        tb = _median_ms(lambda: build_table(wfn, basis, P_d, pts), 3, warm=1, flush=flush)
        tab = build_table(wfn, basis, P_d, pts)
        v64 = tab.esp(pts)
        vmx, n64 = tab.esp_stats(pts)
        d = (vmx - v64).abs()
        t64 = _median_ms(lambda: tab.esp(pts), 3, warm=1, flush=flush)
        tmx = _median_ms(lambda: tab.esp(pts, precision="mixed"), 3, warm=1, flush=flush)
        sweep.append({"points": int(pts.shape[0]), "pairs": tab.n_pairs, "build_ms": tb,
                      "fp64_ms": t64, "mixed_ms": tmx, "mixed_over_fp64": t64 / tmx,
                      "fp64_points_per_s": pts.shape[0] / (t64 * 1e-3),
                      "mixed_points_per_s": pts.shape[0] / (tmx * 1e-3),
                      "mixed_max_abs_err": float(d.max()), "mixed_rms_err": float(d.pow(2).mean().sqrt()),
                      "fp64_routed_pair_warp_evals": n64})
        del tab, pts, v64, vmx
    if "grid" in which:
        out["grid_sweep"] = {"workload": "frag54 on a cubic grid of 0.2 Bohr spacing, 4 Bohr margin, "
                                         "points within 0.3 Bohr of a nucleus dropped; errors of the "
                                         "mixed path against the FP64 path", "runs": sweep}
    if "adjoint" in which:
        # adjoint: 20 atoms l<=2, 500 surface points, L = 0.5 ||V - V_target||^2
        w3, b3, P3, p3 = synth.load_workload("adjoint20", 500, seed=0)
        P3d = torch.as_tensor(P3, device=dev)
        p3d = torch.as_tensor(p3, device=dev)
        rng = np.random.default_rng(7)
        E = rng.normal(0.0, 1e-3, P3.shape)
        vt = build_table(w3, b3, P3d + torch.as_tensor(0.5 * (E + E.T), device=dev), p3d).esp(p3d)
        t3 = build_table(w3, b3, P3d, p3d)
        wv = t3.esp(p3d) - vt
        t_fwd = _median_ms(lambda: build_table(w3, b3, P3d, p3d).esp(p3d), 5)
        t_adj = _median_ms(lambda: t3.adjoint(p3d, wv), 5)
        t_fld = _median_ms(lambda: t3.adjoint(p3d, wv, density=False), 5)
        out["adjoint"] = {"workload": f"adjoint20: 20 atoms, l<=2, {b3.n} Cartesian functions, 500 points",
                          "pairs": t3.n_pairs, "forward_ms": t_fwd, "adjoint_dP_dC_ms": t_adj,
                          "adjoint_dC_only_ms": t_fld}
        # the same adjoint at the headline size (54 atoms, l<=3, 30000 points)
        pts54 = torch.as_tensor(synth.vdw_surface_points(wfn.symbols, wfn.coords, 30000, seed=1),
                                device=dev)
        t54 = build_table(wfn, basis, P_d, pts54)
        w54 = torch.linspace(-1.0, 1.0, pts54.shape[0], dtype=torch.float64, device=dev)
        t_fwd54 = _median_ms(lambda: t54.esp(pts54), 3, warm=1)
        t_adj54 = _median_ms(lambda: t54.adjoint(pts54, w54), 3, warm=1)
        t_dc54 = _median_ms(lambda: t54.adjoint(pts54, w54, density=False), 3, warm=1)
        from fastesp_b200 import hermite as H
        n54 = int(pts54.shape[0])
        fl_field = float(sum(c * H.field_flops(L) for L, c in enumerate(t54.counts))) * n54
        fl_mom = float(sum(c * H.eval_flops(L) for L, c in enumerate(t54.counts))) * n54
        pk64 = peak_flops(torch, 1)
        out["adjoint"]["frag54_30000"] = {
            "pairs": t54.n_pairs, "forward_fp64_ms": t_fwd54, "adjoint_dP_dC_ms": t_adj54,
            "adjoint_dC_only_ms": t_dc54,
            "field_tflops": fl_field / (t_dc54 * 1e-3) / 1e12,
            "field_frac_of_fp64_peak": fl_field / (t_dc54 * 1e-3) / pk64,
            "density_part_tflops": fl_mom / max(1e-9, (t_adj54 - t_dc54) * 1e-3) / 1e12,
            "density_part_frac_of_fp64_peak": fl_mom / max(1e-9, (t_adj54 - t_dc54) * 1e-3) / pk64,
            "flops": "field: hermite.field_flops per (pair, point); density part (moments, "
                     "pair back-transform, gather): hermite.eval_flops per (pair, point)"}
        del t54, pts54
    if "batch" in which:
        # batch: 64 uneven molecules
        mols = synth.batch_workload(64, seed=0)
        tabs, pts = [], []
        for wfn_, basis_, P_, p_ in mols:
            pd = torch.as_tensor(p_, device=dev)
            tabs.append(build_table(wfn_, basis_, torch.as_tensor(P_, device=dev), pd))
            pts.append(pd)
        b = BatchESP(tabs, pts)
        _, run_sep = separate_launches(tabs, pts)
        tbat = _median_ms(b.run, 10, flush=flush)
        tsep = _median_ms(run_sep, 10, flush=flush)
        err = max(float((x - y).abs().max()) for x, y in zip(b.run(), run_sep()))
        npts = sum(int(p.shape[0]) for p in pts)
        out["batch"] = {"workload": "64 molecules, 5-60 atoms, l<=2, 200-5000 surface points each",
                        "points": npts, "pairs": sum(t.n_pairs for t in tabs),
                        "batched_graph_ms": tbat, "separate_launches_ms": tsep,
                        "speedup": tsep / tbat, "points_per_s": npts / (tbat * 1e-3),
                        "shape": list(b.shape), "items": b.n_items, "max_abs_diff": err,
                        "autotune_ms": {f"np{k[0]}_w{k[1]}_tile{k[2] // 1024}K": v
                                        for k, v in (b.tuning or {}).items()},
                        "shape_fields": "points per thread, work items per resident block, "
                                        "pair-tile bytes per stage"}
    return out


# ---------------------------------------------------------------------------
# reference CPU path (build_pairs + NumPy evaluator on a bounded sample)
# ---------------------------------------------------------------------------
def cpu_baseline(wfn, basis, P, pts, counts=None, budget_s=20.0, per_class=None):
    import oracle.esp_oracle as O
    from fastesp_b200 import basis_payload, hermite as H, write_basis_payload
    ncore = len(os.sched_getaffinity(0))
    exe = ROOT / "oracle" / "_ref" / "build_pairs"
    env = dict(os.environ, OMP_NUM_THREADS=str(ncore))
    with tempfile.TemporaryDirectory() as td:
        bb, pb = Path(td) / "basis.bin", Path(td) / "pairs.bin"
        write_basis_payload(bb, basis_payload(wfn, basis, P, pts))
        if exe.exists():
            t0 = time.perf_counter()
            subprocess.run([str(exe), str(bb), str(pb), "1e-12"], check=True, env=env,
                           capture_output=True)
            t_build = time.perf_counter() - t0
            tab = O.OracleTable.read(pb)
            kind = "reference"
        else:
            t0 = time.perf_counter()
            from fastesp_b200.molden import Z_OF
            Z = np.array([Z_OF[s] for s in wfn.symbols])
            tab = O.build_table(wfn.shells, wfn.coords, Z, P, pts, tol=1e-12, rule="native")
            t_build = time.perf_counter() - t0
            kind = "port"
    # NumPy evaluator (fastesp/table.py:73-93) on a per-class sample, scaled
    nt = tab.pp_nt
    by_nt = {H.n_terms(L): L for L in range(9)}
    cls = np.array([by_nt[int(t)] for t in nt])
    rng = np.random.default_rng(0)
    t_eval = 0.0
    sampled = 0
    per_class = per_class or max(2, int(budget_s * 4))
    for L in range(9):
        idx = np.nonzero(cls == L)[0]
        if not len(idx):
            continue
        take = rng.choice(idx, size=min(len(idx), per_class), replace=False)
        mask = np.zeros(tab.n_pairs, bool)
        mask[take] = True
        t0 = time.perf_counter()
        tab.electron(pts, pair_mask=mask)
        dt = time.perf_counter() - t0
        t_eval += dt * len(idx) / len(take)
        sampled += len(take)
    t_tot = t_build + t_eval
    return {"value": len(pts) / t_tot, "unit": "points/s", "cores": ncore, "kind": kind,
            "sample": (f"{'reference build_pairs (C++/OpenMP, ' + str(ncore) + ' threads)' if kind == 'reference' else 'oracle build (NumPy)'}"
                       f" on all {len(pts)} points: {t_build:.2f} s; NumPy evaluator (1 thread) "
                       f"timed on {sampled} sampled pairs (<= {per_class} per class) at all "
                       f"points and scaled by class pair counts: {t_eval:.1f} s estimated"),
            "build_s": t_build, "eval_s_estimated": t_eval, "n_pairs": int(tab.n_pairs),
            "sampled_pairs": int(sampled)}


def reference_cuda(wfn, basis, P, pts, repeats=5):
    """The reference's --backend cuda pipeline (fastesp/cli.py:143-168): its C++
    builder, then its CUDA evaluator (both compiled from the reference sources
    into oracle/_ref), timed as the reference times them: builder wall time,
    evaluator as the minimum of its own per-run timings."""
    import re
    from fastesp_b200 import basis_payload, write_basis_payload
    bp, eg = ROOT / "oracle" / "_ref" / "build_pairs", ROOT / "oracle" / "_ref" / "esp_gpu"
    if not (bp.exists() and eg.exists()):
        return {"unavailable": "oracle/_ref/build_pairs or esp_gpu not built"}
    env = dict(os.environ, OMP_NUM_THREADS=str(len(os.sched_getaffinity(0))))
    with tempfile.TemporaryDirectory() as td:
        bb, pb, out = Path(td) / "basis.bin", Path(td) / "pairs.bin", Path(td) / "esp.txt"
        write_basis_payload(bb, basis_payload(wfn, basis, P, pts))
        t0 = time.perf_counter()
        subprocess.run([str(bp), str(bb), str(pb), "1e-12"], check=True, env=env, capture_output=True)
        t_build = time.perf_counter() - t0
        r = subprocess.run([str(eg), str(pb), str(out), "--repeats", str(repeats)], check=True,
                           capture_output=True, text=True)
        ms = min(float(m) for m in re.findall(r"run \d+: ([0-9.]+) ms", r.stdout))
    return {"build_s": t_build, "solve_ms": ms, "points": int(len(pts)),
            "solve_points_per_s": len(pts) / (ms * 1e-3),
            "e2e_points_per_s": len(pts) / (t_build + ms * 1e-3),
            "what": "reference build_pairs (OpenMP, all cores) + reference esp_gpu (FP64 CUDA, "
                    "compiled for sm_100a), min of its own per-run host timings"}


def run_reference(args):
    rank, world, _ = rank_info()
    if rank != 0:
        return
    from fastesp_b200 import synth
    wfn, basis, P, _ = synth.load_workload("frag54", 10, seed=0)
    pts = synth.vdw_surface_points(wfn.symbols, wfn.coords, args.points, seed=1)
    est, wall = [], []
    base = None
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        cb = cpu_baseline(wfn, basis, P, pts, budget_s=2.0, per_class=6)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            est.append(len(pts) / cb["value"])
            wall.append(dt)
            base = cb
    ms_est = 1e3 * statistics.mean(est)
    value = len(pts) / (ms_est * 1e-3)
    base = dict(base, value=value)
    # A step runs the reference's full table build on all points plus its NumPy
    # evaluator on a bounded sample of pairs (at all points); ms_per_step is that
    # step's measured wall time.  ``value`` is the whole workload's throughput
    # estimated from it: the evaluation is exactly linear in the pairs of a
    # class, so the sampled pairs' time is scaled by the class pair counts.
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "points/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * statistics.mean(wall),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": WORKLOAD, "points_per_gpu": args.points,
                                             "precision": "fp64"},
            "value_is_estimate": True,
            "estimate": {"workload_ms_estimated": ms_est,
                         "how": ("reference build_pairs timed in full; reference NumPy evaluator "
                                 "timed on 6 sampled pairs per class at all points and scaled "
                                 "by the class pair counts (its cost per pair is the same "
                                 "within a class)"),
                         "scale_factor": base["n_pairs"] / max(1, base.get("sampled_pairs", 1))},
            "cpu_baseline": base,
            "e2e": {"value": value, "unit": "points/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    try:
        import torch
        if torch.cuda.is_available():
            line["reference_cuda"] = reference_cuda(wfn, basis, P, pts)
    except Exception as e:                      # reported, never fatal for the CPU arm
        line["reference_cuda"] = {"unavailable": f"{type(e).__name__}: {e}"[:200]}
    print(json.dumps(line))


def free_port() -> int:
    import socket
    with socket.socket() as s_:
        s_.bind(("127.0.0.1", 0))
        return s_.getsockname()[1]


def launcher_argv(n_gpus: int, argv, port: int) -> list:
    """This script as ``n_gpus`` ranks of one node under torch.distributed.run
    (one process per GPU; each reads RANK / LOCAL_RANK / WORLD_SIZE)."""
    return [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
            f"--nproc-per-node={n_gpus}", "--master-addr=127.0.0.1", f"--master-port={port}",
            str(Path(__file__).resolve()), *argv]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="mixed")
    ap.add_argument("--points", type=int, default=30000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the grid sweep, adjoint and batch measurements")
    ap.add_argument("--grid-points", type=int, nargs="*", default=[100000, 1000000])
    ap.add_argument("--only", choices=["grid", "adjoint", "batch"], default=None,
                    help="run one of the extra measurements alone and print its JSON")
    ap.add_argument("--eval-only", action="store_true",
                    help="time only the two evaluators (short run for profiling)")
    ap.add_argument("--print-ranks", action="store_true",
                    help="print this process's rank assignment as JSON and exit (no GPU work)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ and not args.only:
        # --gpus N without a launcher: become N ranks (one per GPU) of this node
        sys.stdout.flush()
        os.execv(sys.executable, launcher_argv(args.gpus, sys.argv[1:], free_port()))
    if args.print_ranks:
        rank, world, local = rank_info()
        print(json.dumps({"rank": rank, "local_rank": local, "world_size": world,
                          "gpus_asked": args.gpus}), flush=True)
        return
    if args.only:
        import torch
        dev = torch.device("cuda", 0)
        torch.cuda.set_device(dev)
        flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
        print(json.dumps({"only": args.only, **run_extras(args, dev, flush, which=(args.only,))}))
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
