"""Benchmark of the Z(w) sweep at 10,020 filaments x 32 frequencies.

Workload (the metric's configuration): the 167-leg meander — 1 mm legs at
40 um pitch, 20 um x 5 um copper, 10 x 3 filaments per segment — giving
10,020 filaments and 9,686 internal loops; 32 log-spaced frequencies from
1e5 to 1e10 Hz.  Synthetic geometry built in code (no dataset).

A step is one Z(w) sweep of the assembled system (MeshSystem.sweep: all 32
complex factorizations, solves, refinement and Schur complements) in the
mixed form (FP32 factors with split-BF16 x3 tensor-core trailing updates and
FP64-residual iterative refinement).  The FP64 form of the same sweep is
timed alongside it, and the error of every mixed Z entry against the FP64
form is reported.  Inputs (R_m, L_m: 1.5 GB) are resident in HBM and every
factorization streams 24 GB, far larger than the 126 MB L2, so no flush is
needed between steps.

``e2e`` is ``solve()`` through the C ABI from host geometry to host Z:
discretization, fill, congruence, sweep and the device-to-host copy.

``--impl reference`` times the CPU oracle (a C++ restatement of the
reference's Rust path; the Rust reference cannot be built here) on the full
metric system: its assembly once, then one full-size FP64 LU + Schur per step
at one of the 32 frequencies; the sweep time is the mean step x 32 plus the
assembly.  The default run's ``cpu_baseline`` leg does the same for the lowest
and highest frequency and reports the error of the GPU's FP64 and mixed Z
against those oracle values (``max_rel_err_*_vs_oracle``).

``--config c3`` sweeps 64 seeded spirals of uneven size (16 frequencies each,
mixed form) through one batched call: one persistent launch for all 1,024
(system, frequency) items, tile shapes from the autotuner.

``--config c5`` runs the matrix-free path instead (its own JSON line): the
square meander of 157 runs (99,224 filaments at 2 x 2) over a 4 mm x 4 mm
copper ground plane meshed 64 x 64 with one square hole (107,144 filaments in
all) with the precorrected-FFT operator (3 x 3 x 3 stencil, near-field radius
8 cells) and GMRES to 1e-8; a step is one Z(1 GHz) solve; the 49-run meander
over the same plane (17,720 filaments) is checked against the dense FP64
path.

Multi-GPU (torchrun, N ranks): replicas only — every rank sweeps its own
copy of the workload (frequencies and geometries are independent; nothing is
exchanged), timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Z(ω) sweep s at 10k filaments×32 freqs: mixed+IR vs FP64 LU at ≤1e-9 rel"
UNIT = "s"


def _workload(name):
    from fasterhenry_b200 import fixtures as F
    return {"metric": F.metric_meander, "metric_odd": F.metric_meander_odd, "c2": F.c2_meander,
            "c1": F.c1_spiral}[name]()


WORKLOADS = {
    "c3": ("batched uneven geometries: 64 seeded square spirals (turns 2-8, width 5-20 um, spacing 3-10 um, "
           "thickness 1-4 um, outer 150-600 um, nw 3-10 x nh 2-3), 16 freqs 1e7-1e10 Hz each", None),
    "c5": ("matrix-free: square meander of 157 runs (24,806 segments at 2 x 2: 99,224 filaments) over a 4 mm x 4 mm "
           "copper ground plane (top 50 um below the meander, 10 um thick, 64 x 64 cells, one 0.5 mm square hole: "
           "7,920 bars at 1 x 1), 107,144 filaments, Z at 1 GHz, pFFT p = 2 (3 x 3 x 3 stencil), near-field radius "
           "8 cells, GMRES(400) to 1e-8", None),
    "c4": ("impedance gradient: 6-turn square spiral (15 um wide, 5 um spacing, 3 um thick, 500 um outer), "
           "skin-depth graded at 1 GHz (cells <= 0.1 skin depth, ratio 1.4: 3,672 filaments), dZ/dp for the "
           "24 widths, 24 thicknesses and the x, y of its 25 nodes (98 parameters) at 1 GHz", None),
    "metric": ("meander 167 legs, 10,020 filaments, m = 9,686, 32 freqs 1e5-1e10 Hz", lambda: _workload("metric")),
    "metric_odd": ("meander 167 legs with one segment at 29 x 1, 10,019 filaments, m = 9,685 (odd), "
                   "32 freqs 1e5-1e10 Hz", lambda: _workload("metric_odd")),
    "c2": ("meander 40 legs, 2,400 filaments, m = 2,320, 32 freqs 1e5-1e10 Hz", lambda: _workload("c2")),
    "c1": ("4-turn spiral, 240 filaments, m = 224, 10 freqs 1e6-1e10 Hz", lambda: _workload("c1")),
}


def _peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return p, "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def max_over_ranks(value: float, world: int) -> float:
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def init_dist(world: int, local: int):
    if world <= 1:
        return
    import datetime
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))


def run_ours(args):
    import ctypes
    rank, world, local = dist_env()
    init_dist(world, local)
    import torch
    torch.cuda.set_device(local)
    import fasterhenry_b200 as fh
    from fasterhenry_b200 import fixtures as F
    from fasterhenry_b200 import _native as N

    deck, freqs = WORKLOADS[args.config][1]()
    geometry = fh.Geometry.from_deck(deck)
    system = fh.MeshSystem.assemble(geometry, deck.ports, deck.discretization)
    counts = system.counts()
    fill = fh.fill_stats(system)
    assembly = system.timing()
    # FP64 form (the plain form) once for the error reference and its time.
    torch.cuda.synchronize()
    r64 = system.sweep(freqs, fh.Precision.FP64)
    r64 = system.sweep(freqs, fh.Precision.FP64)
    lib = N.load()

    def sweep_device_s(precision):
        f = np.ascontiguousarray(freqs, dtype=np.float64)
        p = counts["ports"]
        z = np.zeros((len(f), p, p), dtype=np.complex128)
        it = np.zeros(len(f), dtype=np.int32)
        rs = np.zeros(len(f))
        rep = N.SweepReport(it.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), rs.ctypes.data_as(N.c_double_p))
        info = N.ErrorInfo()
        st = lib.fh_sweep(system._h, f.ctypes.data_as(N.c_double_p), len(f), int(precision),
                          z.ctypes.data_as(N.c_double_p), ctypes.byref(rep), ctypes.byref(info))
        if st:
            raise RuntimeError("sweep failed: %s" % N.last_error())
        return rep.solve_s, z, it, rs

    fp64_s = [sweep_device_s(fh.Precision.FP64)[0] for _ in range(2)]
    fp64_time = min(fp64_s)
    for _ in range(args.warmup):
        sweep_device_s(fh.Precision.MIXED_BF16X3)
    torch.cuda.synchronize()
    barrier(world)
    times = []
    zs = None
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize()
        for _ in range(args.steps):
            t, zs, iters, resid = sweep_device_s(fh.Precision.MIXED_BF16X3)
            times.append(t)
        torch.cuda.synchronize()
    barrier(world)
    # Per-kernel-class breakdown (and the roofline's launch times) from the
    # same number of sweeps run again with the event profiler on: its two
    # event records per launch stay out of the timed sweeps.
    with fh.Profiler() as prof:
        for _ in range(args.steps):
            sweep_device_s(fh.Precision.MIXED_BF16X3)
        torch.cuda.synchronize()
        profile = prof.read()
        # the look-ahead: diagonal-region launches (second stream) beside the deep update
        ov = prof.overlap(["panel", "trsm", "gemm_tc_inner"], ["gemm_tc", "gemm_tc_shared"])
    look_ahead = {"front_ms": round(ov["a_ms"] / args.steps, 3), "update_ms": round(ov["b_ms"] / args.steps, 3),
                  "overlap_ms": round(ov["both_ms"] / args.steps, 3),
                  "what": "per sweep, event-timed: time the diagonal-region launches ran, the deep update ran, "
                          "and both at once"}
    step_s = sum(times) / len(times)
    step_max = max_over_ranks(step_s, world)
    z64 = r64.impedance_ohm
    rel = [float(np.max(np.abs(zs[k] - z64[k])) / np.max(np.abs(z64[k]))) for k in range(len(freqs))]

    # e2e: solve() through the C ABI from host geometry to host Z, after two
    # untimed calls (the first systems of a process grow the device memory cache).
    for _ in range(2):
        fh.solve(geometry, deck.ports, deck.discretization, freqs, fh.Precision.MIXED_BF16X3)
    e2e_times, e2e_parts = [], []
    for _ in range(max(1, min(args.steps, 5))):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = fh.solve(geometry, deck.ports, deck.discretization, freqs, fh.Precision.MIXED_BF16X3)
        torch.cuda.synchronize()
        e2e_times.append(time.perf_counter() - t0)
        e2e_parts.append([round(res.timing.get(k, 0.0), 4) for k in ("inductance_s", "assembly_s", "solve_s")])
    e2e_s = max_over_ranks(statistics.median(e2e_times), world)
    h2d = counts["filaments"] * 256 + counts["filaments"] * 8 + len(freqs) * 8 + (2 * counts["filaments"]) * 12
    d2h = len(freqs) * counts["ports"] ** 2 * 16

    peaks, peak_kind = _peaks()
    # Roofline of the dominant kernel: the trailing-update GEMM.
    gemm_cls = "gemm_tc" if profile["gemm_tc"]["launches"] else "gemm_fp32"
    g = profile[gemm_cls]
    gemm_launches = max(1, g["launches"])
    per_launch_ms = g["ms"] / gemm_launches
    if gemm_cls == "gemm_tc":
        # bf16 tensor flops actually required: three split products per real product
        achieved = 3.0 * g["work"] / (g["ms"] * 1e-3) / 1e12
        peak = peaks.get("bf16_tflops", 1590.0)
        unit = "TFLOP/s"
        bound = "tensor"
    else:
        achieved = g["work"] / (g["ms"] * 1e-3) / 1e12 if g["ms"] else 0.0
        peak = 80.0  # FP32 SIMT nominal (no measured figure)
        unit = "TFLOP/s"
        bound = "fp32-simt"
    traffic = None
    if gemm_cls == "gemm_tc":
        # DRAM bytes per launch: the ncu capture of packed_update_kernel on the
        # 2,400-filament meander moved 0.985 x its algorithmic bytes (C read +
        # write, 16 B per entry, plus the packed operands once); scaled here to
        # the algorithmic C bytes of this run's average launch (work / 256 at
        # K = 512, i.e. 16 B per 8 * 512 flops).
        traffic = round(0.985 * (g["work"] / gemm_launches) / 256.0 * 1.03, 1)
    roofline = {"kernel": "packed_update_kernel (deep split-BF16x3 trailing update, K = 512)"
                if gemm_cls == "gemm_tc" else gemm_cls,
                "bound": bound, "achieved": round(achieved, 2), "peak": peak,
                "unit": unit, "frac": round(achieved / peak, 4) if peak else None,
                "peak_source": ("measured bf16 burst (MEASURED_PEAKS.json)" if peak_kind == "measured" else peak_kind)
                if gemm_cls == "gemm_tc" else "nominal",
                "traffic": traffic, "traffic_unit": "bytes per launch",
                "traffic_source": "ncu dram__bytes_read+write of packed_update_kernel (2,400-filament meander), "
                                  "scaled by algorithmic bytes",
                "per_launch_ms": round(per_launch_ms, 4), "launches": g["launches"]}
    if gemm_cls == "gemm_tc":
        roofline["launches_counted"] = ("the deep updates and the first parts of split updates, on every SM; "
                                        "the second parts below")
        sh = profile.get("gemm_tc_shared", {"launches": 0, "ms": 0.0, "work": 0.0})
        if sh["launches"]:
            sh_achieved = 3.0 * sh["work"] / (sh["ms"] * 1e-3) / 1e12
            roofline["shared_part"] = {
                "launches": sh["launches"], "per_launch_ms": round(sh["ms"] / sh["launches"], 4),
                "achieved": round(sh_achieved, 2), "frac": round(sh_achieved / peak, 4) if peak else None,
                "what": "second parts of split deep updates: 116 of 148 SMs while the next diagonal region runs "
                        "on the others, then all of them (a joining grid, not timed apart)"}
    launches = sum(v["launches"] for v in profile.values())

    out = {
        "metric": METRIC, "value": round(step_max, 6), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(step_max * 1e3, 3), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "c64+bf16x3 (FP64 residual)", "data": "synthetic",
        "config": {"workload": WORKLOADS[args.config][0],
                   "filaments": counts["filaments"], "internal_meshes": counts["internal_meshes"],
                   "frequencies": len(freqs), "precision": "mixed_bf16x3_ir", "l2": "inputs 24 GB >> L2 (no flush)",
                   "parallelism": "replicas" if world > 1 else "single"},
        "fp64_sweep_s": round(fp64_time, 6), "speedup_vs_fp64": round(fp64_time / step_max, 3),
        "max_rel_err_vs_fp64": max(rel), "rel_err_per_freq": rel,
        "refinement_iterations": [int(x) for x in iters], "fill": fill, "assembly": assembly,
        "e2e": {"value": round(e2e_s, 6), "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "samples": [round(t, 4) for t in e2e_times],
                "fill_assembly_sweep_s": e2e_parts,
                "what": "solve(): discretize + fill + congruence + mixed sweep + D2H of Z, via the C ABI"},
        "roofline": roofline, "profile": profile, "look_ahead": look_ahead, "gpu_launches": int(launches),
        "clocks": clocks.summary(),
    }
    if rank == 0 and world == 1:
        out["fp64_library_lu"] = library_fp64_lu(system, freqs, counts)
    if rank == 0 and world == 1 and not args.no_cpu and args.config == "metric":
        out["cpu_baseline"] = cpu_baseline(args, z64, zs)
        for key in ("max_rel_err_fp64_vs_oracle", "max_rel_err_mixed_vs_oracle"):
            if key in out["cpu_baseline"]:
                out[key] = out["cpu_baseline"][key]
    if rank == 0:
        print(json.dumps(out))
    system.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_c3(args):
    """64 independent spirals of uneven size, each swept over 16 frequencies
    in the mixed form, all through one batched call (fh_batch_sweep): the
    1,024 (system, frequency) items in ONE persistent launch, tile shapes per
    order bucket from the autotuner (measured on the first call, cached in a
    JSON file).  A step is the whole batch, host in/out.  Every Z is checked
    against the FP64 form of the same batch.  Rank 0 only (one GPU)."""
    import torch
    import fasterhenry_b200 as fh
    from fasterhenry_b200 import fixtures as F
    rank, world, local = dist_env()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    decks = F.random_spirals(64, seed=2026)
    t0 = time.perf_counter()
    systems = [fh.MeshSystem.assemble(fh.Geometry.from_deck(d), d.ports, d.discretization) for d in decks]
    assemble_s = time.perf_counter() - t0
    freqs = [F.logspace(7, 10, 16) for _ in systems]
    ref = fh.batch_sweep(systems, freqs, fh.Precision.FP64, concurrency=4)
    t1 = time.perf_counter()
    fh.batch_sweep(systems, freqs, fh.Precision.MIXED_BF16X3)  # first call: autotunes new buckets
    first_call_s = time.perf_counter() - t1
    for _ in range(args.warmup):
        fh.batch_sweep(systems, freqs, fh.Precision.MIXED_BF16X3)
    times = []
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            res = fh.batch_sweep(systems, freqs, fh.Precision.MIXED_BF16X3)
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t1)
    with fh.Profiler() as prof:
        fh.batch_sweep(systems, freqs, fh.Precision.MIXED_BF16X3)
        profile = prof.read()
    # the per-system path for comparison: each system's own mixed sweep in turn
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    for s, f in zip(systems, freqs):
        s.sweep(f, fh.Precision.MIXED_BF16X3)
    torch.cuda.synchronize()
    per_system_s = time.perf_counter() - t2
    step = statistics.median(times)
    rel = max(float(np.max(np.abs(m.impedance_ohm - r.impedance_ohm) / np.abs(r.impedance_ohm)))
              for m, r in zip(res, ref))
    counts = [s.counts() for s in systems]
    b = profile["batch"]
    peaks, _ = _peaks()
    cache = os.environ.get("FH_AUTOTUNE_CACHE") or os.path.join(
        os.environ.get("XDG_CACHE_HOME") or os.path.join(os.path.expanduser("~"), ".cache"),
        "fasterhenry_b200", "batch_tiles.json")
    try:
        with open(cache) as f:
            table = json.load(f)
    except Exception:
        table = None
    out = {
        "metric": "batched Z(w) sweeps of 64 uneven spirals x 16 freqs: mixed+IR, s", "value": round(step, 6),
        "unit": "s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(step * 1e3, 3),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "c64 (FP32 SIMT) + FP64 residual",
        "data": "synthetic",
        "config": {"workload": WORKLOADS["c3"][0], "systems": len(systems),
                   "filaments_min": min(c["filaments"] for c in counts),
                   "filaments_max": max(c["filaments"] for c in counts),
                   "internal_meshes_min": min(c["internal_meshes"] for c in counts),
                   "internal_meshes_max": max(c["internal_meshes"] for c in counts),
                   "internal_meshes_total": sum(c["internal_meshes"] for c in counts),
                   "items": sum(len(f) for f in freqs), "l2": "working sets of up to 4.3 MB per item; no flush"},
        "launches_per_step": b["launches"], "kernel_ms": round(b["ms"], 3),
        "kernel_tflops": round(b["work"] / (b["ms"] * 1e-3) / 1e12, 2) if b["ms"] else None,
        "autotune": {"first_call_s": round(first_call_s, 3), "table": table},
        "assemble_all_s": round(assemble_s, 3), "per_system_sweeps_s": round(per_system_s, 4),
        "max_rel_err_vs_fp64": rel, "clocks": clocks.summary(),
    }
    print(json.dumps(out))
    for s in systems:
        s.close()


def run_c4(args):
    """dZ/dp of the 6-turn skin-graded spiral at 1 GHz for its 98 parameters
    (24 widths, 24 thicknesses, x and y of 25 nodes) by the stationary form
    (fh_gradient: one FP64 solve, the width / thickness and the coordinate
    derivative fills, one product per derivative matrix); a step is one
    gradient through the public API.  For comparison, the cost of the same
    gradient by central differences through the public API is estimated as
    196 x (assembly + one FP64 solve) of the same spiral.  Rank 0 only."""
    import torch
    import fasterhenry_b200 as fh
    from fasterhenry_b200 import fixtures as F
    rank, world, local = dist_env()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    deck = F.c4_spiral()
    geometry = fh.Geometry.from_deck(deck)
    system = fh.MeshSystem.assemble(geometry, deck.ports, deck.discretization)
    nseg, nnodes = len(deck.segments), len(deck.nodes)
    params = ([fh.Param(k, s) for k in ("width", "thickness") for s in range(nseg)] +
              [fh.Param(k, v) for v in range(nnodes) for k in ("x", "y")])
    for _ in range(args.warmup):
        system.gradient(1e9, params)
    times, reports = [], []
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            g = system.gradient(1e9, params)
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t1)
            reports.append(g.report)
    step = statistics.median(times)
    fd_samples = []
    for _ in range(2):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        with fh.MeshSystem.assemble(geometry, deck.ports, deck.discretization) as s2:
            s2.impedance(1e9)
        torch.cuda.synchronize()
        fd_samples.append(time.perf_counter() - t0)
    counts = system.counts()
    fs = fh.fill_stats(system)
    med = lambda k: statistics.median(r[k] for r in reports)
    out = {
        "metric": "dZ/dp (98 params: widths, thicknesses, node x/y) of a 3,672-filament spiral at 1 GHz, s",
        "value": round(step, 6),
        "unit": "s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(step * 1e3, 3),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOADS["c4"][0], "filaments": counts["filaments"],
                   "internal_meshes": counts["internal_meshes"], "params": len(g.params),
                   "l2": "derivative matrices 647 MB (> L2); no flush"},
        "solve_s": round(med("solve_s"), 6), "derivative_fill_s": round(med("derivative_fill_s"), 6),
        "contract_s": round(med("contract_s"), 6), "pairs": int(reports[-1]["pairs"]),
        "fill_methods": {k: fs[k] for k in ("point_quadrature", "closed_form", "aligned_quadrature", "orthogonal")},
        "fd_equivalent_s": round(2 * len(params) * min(fd_samples), 3),
        "dz_dx_node0": [g.gradient[2 * nseg, 0, 0].real, g.gradient[2 * nseg, 0, 0].imag],
        "translation_residual": float(np.max(np.abs(g.gradient[2 * nseg::2].sum(axis=0))) /
                                      np.max(np.abs(g.gradient[2 * nseg:]))),
        "z_ohm": [g.impedance_ohm[0, 0].real, g.impedance_ohm[0, 0].imag],
        "clocks": clocks.summary(),
    }
    print(json.dumps(out))
    system.close()


def run_c5(args):
    """The matrix-free path at the 99,224-filament meander over its ground
    plane (107,144 filaments): IterativeSystem assembly (pFFT set-up) and
    Z(1 GHz) by GMRES, each step one solve; the 9,800-filament meander over the
    same plane is checked against the dense FP64 path (bound 1e-4 on Z).
    Rank 0 only (one GPU)."""
    import torch
    import fasterhenry_b200 as fh
    from fasterhenry_b200 import fixtures as F
    rank, world, local = dist_env()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    # GMRES restarted every 400 iterations: the plane's cell loops make
    # GMRES(100) (the library default) lose most of its progress at each
    # restart (1,129 iterations against 491).
    params = fh.IterativeParams(pfft=fh.PfftParams(near_field_radius=8.0, interpolation_order=2, fft_fp32=True),
                                gmres=fh.GmresParams(tolerance=1e-8, restart=400))
    deck = F.meander_over_plane(157)
    geometry = fh.Geometry.from_deck(deck)
    t0 = time.perf_counter()
    system = fh.IterativeSystem.assemble(geometry, deck.ports, deck.discretization, params)
    assemble_s = time.perf_counter() - t0
    for _ in range(args.warmup):
        system.impedance(1e9)
    times = []
    with ClockSampler(local) as clocks, fh.Profiler() as prof:
        for _ in range(args.steps):
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            z = system.impedance(1e9)
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t1)
        profile = prof.read()
    step = statistics.median(times)
    stats = system.operator_stats()
    outcome = system.last_outcomes[0][0]
    pa = profile["pfft_apply"]
    # The parity check after the timed solves (so that a launch list of this
    # command starts with the full-size system's kernels).
    sub = F.meander_over_plane(49)
    g = fh.Geometry.from_deck(sub)
    with fh.IterativeSystem.assemble(g, sub.ports, sub.discretization, params) as s:
        z_it = s.impedance(1e9)
    with fh.MeshSystem.assemble(g, sub.ports, sub.discretization) as d:
        z_d = d.impedance(1e9)
    subset_rel = float(np.max(np.abs(z_it - z_d) / np.abs(z_d)))
    peaks, peak_kind = _peaks()
    hbm = peaks.get("hbm_gbs", 6650.0)
    achieved = pa["work"] / (pa["ms"] * 1e-3) / 1e9 if pa["ms"] else 0.0
    out = {
        "metric": "matrix-free Z(1 GHz) at 107,144 filaments (99,224-filament meander over a ground plane): "
                  "GMRES solve s (pFFT operator)",
        "value": round(step, 6), "unit": "s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(step * 1e3, 3), "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOADS["c5"][0], "filaments": stats["filaments"],
                   "internal_meshes": system.counts()["internal_meshes"], "grid_dims": stats["grid_dims"],
                   "fft_dims": stats["fft_dims"], "projection_entries": stats["projection_entries"],
                   "near_entries": stats["near_entries"], "l2": "FFT grids of %.0f MB each >> L2 (no flush)"
                   % (16 * np.prod(stats["fft_dims"]) / 1e6)},
        "assemble_s": round(assemble_s, 3), "setup_host_s": round(stats["setup_host_s"], 3),
        "setup_device_s": round(stats["setup_device_s"], 3), "setup_near_s": round(stats["setup_near_s"], 3),
        "gmres": {"iterations": outcome.iterations, "relative_residual": outcome.relative_residual},
        "z_ohm": [float(z[0, 0].real), float(z[0, 0].imag)],
        "subset_rel_err_vs_dense": subset_rel,
        "subset": "meander of 49 runs (9,800 filaments) over the same plane: 17,720 filaments, dense FP64 vs matrix-free",
        "roofline": {"kernel": "pfft apply (near SpMV, spread, FFTs, interpolation)", "bound": "hbm",
                     "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                     "frac": round(achieved / hbm, 4) if hbm else None, "peak_source": peak_kind, "traffic": None,
                     "launches": pa["launches"], "per_launch_ms": round(pa["ms"] / max(1, pa["launches"]), 4)},
        "profile": profile, "clocks": clocks.summary(),
    }
    print(json.dumps(out))
    system.close()


def library_fp64_lu(system, freqs, counts):
    """A library FP64 GPU LU for context: cuSOLVER's complex128 getrf (through
    torch.linalg.lu_factor) on one frequency's m x m matrix R_ee + j w L_ee,
    timed with CUDA events and multiplied by the number of frequencies (each
    frequency is an independent factorization).  Not on the product path."""
    import torch
    m = counts["internal_meshes"]
    R, L = system.mesh_matrices()
    w = 2.0 * np.pi * freqs[len(freqs) // 2]
    a = torch.from_numpy(np.ascontiguousarray(R[:m, :m] + 1j * w * L[:m, :m])).to("cuda")
    torch.linalg.lu_factor(a)  # warm-up (workspace, handles)
    torch.cuda.synchronize()
    ms = []
    for _ in range(2):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.linalg.lu_factor(a)
        e1.record()
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    one = min(ms) * 1e-3
    del a
    torch.cuda.empty_cache()
    return {"one_matrix_s": round(one, 6), "sweep_s": round(one * len(freqs), 6),
            "what": "torch.linalg.lu_factor complex128 (cuSOLVER getrf) of one m x m matrix x %d frequencies"
                    % len(freqs)}


def _oracle_metric_system(threads):
    """The oracle's assembly of the full metric system (10,020 filaments: fill,
    loop basis, congruence), timed."""
    from oracle import oracle as O
    deck, freqs = _workload("metric")
    t0 = time.perf_counter()
    s = O.System(deck, threads=threads)
    return s, freqs, time.perf_counter() - t0


def cpu_baseline(args, z64=None, zmx=None):
    """The oracle (C++ restatement of the reference's dense path) on the full
    metric system: its assembly, then the FP64 LU + Schur at the lowest and the
    highest of the 32 frequencies, each an m = 9,686 factorization.  Every
    frequency of the sweep is a factorization of the same order, so the sweep
    time is the mean per-frequency time x 32, plus the assembly.  The two
    oracle Z values also check the GPU's FP64 and mixed Z at full size."""
    threads = os.cpu_count() or 1
    s, freqs, assemble_s = _oracle_metric_system(threads)
    picks = [0, len(freqs) - 1]
    per, err64, errmx = [], [], []
    for k in picks:
        t1 = time.perf_counter()
        z = s.impedance(freqs[k])
        per.append(time.perf_counter() - t1)
        if z64 is not None:
            err64.append(float(np.max(np.abs(z64[k] - z)) / np.max(np.abs(z))))
        if zmx is not None:
            errmx.append(float(np.max(np.abs(zmx[k] - z)) / np.max(np.abs(z))))
    one = statistics.mean(per)
    value = one * len(freqs) + assemble_s
    out = {"value": round(value, 3), "unit": UNIT, "cores": threads, "kind": "port",
           "sample": "oracle on the full 10,020-filament system: assembly %.2f s, FP64 LU + Schur (m = %d) at "
                     "%s Hz, %s s; value = mean per-frequency time x %d + assembly"
                     % (assemble_s, s.counts["internal_meshes"], ", ".join("%.0e" % freqs[k] for k in picks),
                        ", ".join("%.2f" % t for t in per), len(freqs)),
           "sample_assemble_s": round(assemble_s, 3), "per_frequency_s": [round(t, 3) for t in per],
           "oracle_frequency_indices": picks}
    if err64:
        out["max_rel_err_fp64_vs_oracle"] = max(err64)
    if errmx:
        out["max_rel_err_mixed_vs_oracle"] = max(errmx)
    return out


def run_reference(args):
    """The reference arm: the oracle (C++ OpenMP restatement of the
    reference's Rust dense path, which cannot be built here) on the metric
    system itself.  The full 10,020-filament assembly is timed once; each step
    is one full-size (m = 9,686) FP64 LU + Schur at one of the 32 metric
    frequencies, cycling through them.  value = mean step x 32 + assembly:
    every frequency is a factorization of the same order, so only the number
    of frequencies is scaled."""
    rank, world, local = dist_env()
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    s, freqs, assemble_s = _oracle_metric_system(threads)
    k = 0
    for _ in range(args.warmup):
        s.impedance(freqs[k % len(freqs)])
        k += 1
    times, zs = [], {}
    for _ in range(args.steps):
        f = freqs[k % len(freqs)]
        t0 = time.perf_counter()
        z = s.impedance(f)
        times.append(time.perf_counter() - t0)
        zs["%.6e" % f] = [float(z[0, 0].real), float(z[0, 0].imag)]
        k += 1
    one = statistics.mean(times)
    value = one * len(freqs) + assemble_s
    sample = ("oracle (C++ restatement of the reference's Rust dense path) on the full 10,020-filament metric "
              "system: assembly %.2f s once, then per step one m = %d FP64 LU + Schur at one of the 32 "
              "frequencies (cycling), mean %.2f s; value = mean x 32 + assembly"
              % (assemble_s, s.counts["internal_meshes"], one))
    out = {"impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(one * 1e3, 3),
           "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
           "config": {"workload": WORKLOADS["metric"][0], "filaments": s.counts["filaments"],
                      "internal_meshes": s.counts["internal_meshes"], "frequencies": len(freqs),
                      "precision": "fp64"},
           "assemble_s": round(assemble_s, 3), "step_s": [round(t, 3) for t in times], "z_ohm": zs,
           "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": threads, "kind": "port",
                            "sample": sample},
           "e2e": {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline leg")
    ap.add_argument("--config", default="metric", choices=sorted(WORKLOADS),
                    help="workload: the metric's 10k-filament meander (default) or a smaller parity config "
                         "(used for profiling captures)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.config == "c5":
        run_c5(args)
    elif args.config == "c3":
        run_c3(args)
    elif args.config == "c4":
        run_c4(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
