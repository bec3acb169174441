#!/usr/bin/env python
"""Benchmark: elastic FWI gradient shots/s on B200.

Workload (the FWI-gradient configuration): 300^3 interior + 40-cell sponge
(392 x 392 x 388 cells with the FAT ring), dx = 10 m, 2500 coarse samples at
2 ms (9996 fine steps), explosive Ricker 10 Hz source, 150 x 150 receivers
(all nine components), L2 misfit.  True model = smooth background + two
Gaussian anomalies; the gradient is taken at the background model.  Inputs are
seeded synthetic data (no dataset is involved).

One step = one shot's FWI gradient per GPU through ``ElasticFwiMisfit``
(autograd forward + backward): the model and the observed traces are copied in
from pinned host memory, the nonlinear forward runs with on-device
checkpoints, the residual is formed at the receivers, the Born adjoint of the
residual runs with the source wavefield recomputed from the checkpoints, and
the gradient (and the misfit) are copied back to pinned host memory.  One
timed loop gives both figures: ``value`` from the device time between the
input copies and the gradient copy of each step (inputs resident in HBM),
``e2e`` from the whole loop including the copies.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU (torchrun): every rank takes its own shot each step (weak scaling) and
the misfit and gradient are summed with one all-reduce; the time is the max over
ranks.  --impl reference times the oracle port of the path on the host cores
(rank 0 only), without loading this package's native library.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FWI gradient shots/s (Born-adjoint gradient, 300^3+40 sponge, 2500 samples)"
UNIT = "shots/s"
# Timed kernel kinds of the gradient (e3d_kernel_timing_read) and their algorithmic bytes per
# updated cell (fp32 fields):
#   0 forward stepper: read old 9 + current 9 + medium 8, write new 9 = 140 B (the forward pass
#     and the source recompute, whose fine levels go to a ring of sub+1 levels)
#   1 exact-adjoint stepper on the premultiplied-only state (the time-reversed stepper on
#     premultiplied levels): read old 9 + current 9 (both premultiplied) + medium 8, write new 9
#     = 140 B (where the medium's premultiplication is well conditioned)
#   2 the same on the dual state (raw + premultiplied levels): read old raw 9, current
#     premultiplied 9, medium 8, write new raw 9 and new premultiplied 9 = 176 B
#   6 block imaging, once per coarse block: read the sub adjoint levels (sub*36 B), V(t-1..t+2)
#     (48 B), the eight image planes (32 B) and write them (32 B) = 256 B at sub = 4, and with a
#     premultiplied-only adjoint the eight medium planes (32 B) to convert its sums back
#   7 source-velocity decimation, once per recomputed block: read sub levels x 3 fields (48 B),
#     V[b] (12 B), write V[b] and V[b+1] (24 B) = 84 B at sub = 4
#   with --decimation acc: 3 = forward + 3-field accumulators (188 B), 5 = dual adjoint + 9-field
#     accumulators (320 B)
KIND_NAMES = {0: "forward stepper", 1: "exact-adjoint stepper on premultiplied levels",
              2: "dual-state exact-adjoint stepper", 6: "block imaging from the adjoint ring",
              7: "source-velocity decimation", 3: "forward stepper + 3-field decimation accumulators",
              5: "dual adjoint stepper + 9-field accumulators"}
# ncu summaries (DRAM bytes per updated cell) of the kernels each stepper choice runs
PROFILES = {
    "split": {0: "profiles/kStepSplit_forward_392x392x104.txt",
              1: "profiles/kStepSplit_adjoint_premultiplied_392x392x104.txt"},
    "split-pair": {0: "profiles/kStepSplitPair_forward_392x392x104.txt",
                   1: "profiles/kStepSplitPair_time_reversed_392x392x104.txt"},
}
PROFILE_COMMON = {2: "profiles/kStepTma_adjoint_dual_392x392x104.txt", 6: "profiles/kImagingTma_280x280x280.txt"}


def kind_names(args):
    """The kernel each timed kind runs with this command's stepper and imaging choices."""
    fwd = {"split": "kStepSplit<0,3,3>: velocity and stress CTA roles",
           "split-pair": "kStepSplitPair<0,3,3>: velocity and stress CTA roles, two z cells per thread",
           "tma": "kStepTma<0,8,2>", "plain": "kStep<0,8>: plain loads", "auto": "autotuned stepper"}[args.variant]
    rev = {"split": "kStepSplit<1,3,3>", "split-pair": "kStepSplitPair<1,3,3>", "tma": "kStepTma<1,8,2>",
           "plain": "kStep<1,8>: plain loads", "auto": "autotuned stepper"}[args.variant]
    img = {"auto": "kImagingBlock" if args.variant == "plain" else "kImagingTma", "tma": "kImagingTma",
           "tma-levels": "kImagingLev: levels staged by TMA",
           "tma-levels-4": "kImagingLev, 4-wide tiles: levels staged by TMA",
           "cells": "kImagingBlock"}[args.imaging]
    plain = args.variant == "plain"
    acc = "kStep<0,8>: plain loads" if plain else "kStepTma<0,8>"
    # without a TMA loader the exact adjoint keeps one raw state and premultiplies its neighbours
    adj = "kStep<2,8>: plain loads, neighbours premultiplied on the fly" if plain else "kStepTma<2,8,2>"
    return {0: f"forward stepper ({fwd})",
            1: f"exact-adjoint stepper on premultiplied levels ({rev}, the time-reversed update on P)",
            2: f"exact-adjoint stepper ({adj})" if plain else "dual-state exact-adjoint stepper (kStepTma<2,8,2>)",
            6: f"block imaging from the adjoint ring ({img})",
            7: "source-velocity decimation (kDecimateVelocity)",
            3: f"forward stepper + 3-field decimation accumulators ({acc})",
            5: f"exact-adjoint stepper + 9-field accumulators ({adj})"}


def profiled(kind, args):
    """The ncu summary whose DRAM bytes per cell stand for this kind's launches, where it profiled
    the same kernel."""
    table = {**PROFILE_COMMON, **PROFILES[args.variant]} if args.variant in PROFILES else {}
    if kind not in table:
        return None
    if kind == 6 and args.imaging not in ("auto", "tma"):
        return None
    return os.path.join(ROOT, table[kind])


def kind_bytes(kind, sub, prem=False, dual=True):
    """Algorithmic bytes per updated cell of a timed kind; dual=False: the exact adjoint keeps one
    raw state (the plain-load stepper premultiplies its neighbours on the fly), 140 B and 284 B
    with the 9-field accumulators."""
    adj, adj_acc = (176.0, 320.0) if dual else (140.0, 284.0)
    return {0: 140.0, 1: 140.0, 2: adj, 6: sub * 36.0 + 48.0 + 64.0 + (32.0 if prem else 0.0), 7: sub * 12.0 + 36.0,
            3: 188.0, 5: adj_acc}[kind]


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nts", type=int, default=2500)
    ap.add_argument("--interior", type=int, default=300)
    ap.add_argument("--variant", default="split-pair", choices=["split", "split-pair", "tma", "plain", "auto"],
                    help="stepper: split-pair (default: velocity and stress updates as two CTA roles with 3-stage "
                         "TMA pipelines and two z cells per thread for the forward-type steps, the 2-stage TMA "
                         "stepper for the dual-state adjoint), split (the same with one cell per thread), tma "
                         "(2-stage TMA stepper for every step), plain (plain loads, no dual-state adjoint), auto "
                         "(autotuned)")
    ap.add_argument("--ckpt", default="auto", choices=["auto", "fp32", "fp16", "bf16"])
    ap.add_argument("--velocity", default="auto", choices=["auto", "fp32", "fp16"],
                    help="storage of the decimated source velocity slots (fp32 with --ckpt fp32: the "
                         "all-FP32 plan)")
    ap.add_argument("--decimation", default="ring", choices=["ring", "acc"],
                    help="gradient passes: decimate from a ring of fine levels once per coarse block (ring) "
                         "or through accumulators fused into every fine step (acc)")
    ap.add_argument("--imaging", default="auto", choices=["auto", "cells", "tma", "tma-levels", "tma-levels-4"],
                    help="block imaging kernel of the decimation ring (Propagator.set_imaging_variant)")
    ap.add_argument("--adjoint-state", default="auto", choices=["auto", "dual"],
                    help="gradient adjoint pass: premultiplied levels only where the medium allows (auto) or "
                         "the dual raw + premultiplied state everywhere")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--breakdown", action="store_true",
                    help="after the measurement, print the device time per kernel of one more gradient")
    return ap.parse_args(argv)


class ClockSampler:
    """nvidia-smi clock and throttle-reason samples during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}




def build_problem(args, device):
    """Background survey, the FWI problem on it and one shot whose observed traces are the
    nonlinear forward of the true model (computed on the device)."""
    import torch
    from elasticisolib_3d_b200 import fwi as F
    from elasticisolib_3d_b200 import hostprep as H
    from elasticisolib_3d_b200 import synthetic as S
    n = args.interior
    sv, true_el = S.fwi_gradient_survey(nzi=n, nxi=n, nyi=n, nts=args.nts, with_true=True)
    fd = H.FdParam(sv.elastic, sv.axes, sv.par)
    ax7 = H.grid_axes(*(a.n for a in sv.axes), *(a.o for a in sv.axes), *(a.d for a in sv.axes))
    variant = {"split": (8, 3, "split-fwd"), "split-pair": (8, 3, "split-pair"), "tma": (8, 2, "tma"),
               "plain": (8, 2, "plain"),
               "auto": "auto"}[args.variant]
    prob = F.FwiProblem(fd, device=device, ckpt=args.ckpt, variant=variant, velocity=args.velocity,
                        decimation_ring=args.decimation == "ring", premultiplied=args.adjoint_state == "auto")
    prob.prop.set_imaging_variant(args.imaging)
    rank = int(os.environ.get("RANK", "0"))
    shot_id = rank % len(sv.src_xyz)
    src = H.build_devices(*sv.src_xyz[shot_id], ax7, fd.nts, sv.par)
    rec = H.build_devices(*sv.rec_xyz, ax7, fd.nts, sv.par)
    irr = [np.zeros((1, fd.nts), dtype=np.float32) for _ in range(9)]
    for k in (3, 4, 5):
        irr[k][0] = sv.wavelet
    shot = F.make_shot(src, rec, irr, None, device)
    mt = [torch.tensor(true_el[k], device=device) for k in range(3)]
    planes = prob.set_model(*mt)
    shot.d_obs, _ = prob.forward_data(shot, planes)
    del planes, mt
    prob.shots.append(shot)
    torch.cuda.synchronize()
    return sv, fd, prob


def oracle_grid(args):
    """Grid, medium planes and propagation constants of the workload for the host-core runs,
    from the oracle's own host preparation (this package's native library is not loaded)."""
    from elasticisolib_3d_b200 import synthetic as S
    from oracle import oracle as O
    n = args.interior
    sv = S.fwi_gradient_survey(nzi=n, nxi=n, nyi=n, nts=args.nts)
    par = sv.par
    nts, dts = par.getInt("nts"), par.getFloat("dts")
    sub, _, dtw = O.time_axes(nts, dts, par.getInt("sub"))
    za, xa, ya = sv.axes
    # one sponge width for all faces: the smaller z and x pads (fdParamElastic_3D.cpp minPad rule)
    min_pad = min(par.getInt("zPadMinus"), par.getInt("zPadPlus"), par.getInt("xPadMinus"), par.getInt("xPadPlus"))
    p = O.PropParams(za.n, xa.n, ya.n, nts, sub, min_pad, float(za.d), float(xa.d), float(ya.d), float(dts))
    med = O.medium_planes(sv.elastic, dtw)
    return p, med


class OracleSteps:
    """The oracle's FP32 stepper (C++/OpenMP restatement of the reference's kernels, sponge fused)
    on the full grid, on all host cores; one sample = 2 forward + 1 exact-adjoint fine steps, the
    mix of a gradient (forward pass, source wavefield, adjoint pass)."""

    def __init__(self, p, med, threads=0):
        import ctypes
        from oracle import oracle as O
        self.ctypes = ctypes
        self.L = O.lib()
        self.threads = int(self.L.oracle_num_threads(threads or os.cpu_count() or 1))
        shape = (p.ny, p.nx, p.nz)
        rng = np.random.default_rng(0)
        self.keep = [np.ascontiguousarray(m, dtype=np.float32) for m in med]
        self.p0 = [np.zeros(shape, np.float32) for _ in range(9)]
        self.p1 = [rng.standard_normal(shape, dtype=np.float32) * 1e-3 for _ in range(9)]
        self.a, _ = O._ptrs(self.p0)
        self.b, _ = O._ptrs(self.p1)
        self.m, _ = O._ptrs(self.keep)
        self.prm = p.c()
        self.steps_per_gradient = (p.nts - 1) * p.sub  # fine steps of each of the three passes

    def sample(self):
        """Seconds of one 2-forward + 1-adjoint sample."""
        L, by = self.L, self.ctypes.byref
        t0 = time.perf_counter()
        L.oracle_step_f32(by(self.prm), self.a, self.b, self.m, 0, 1)
        L.oracle_step_f32(by(self.prm), self.a, self.b, self.m, 0, 1)
        L.oracle_step_f32(by(self.prm), self.a, self.b, self.m, 2, 1)
        return time.perf_counter() - t0


def cpu_baseline(fd, n_samples=3, threads=0):
    """The oracle port timed on the host cores over a bounded sample of the same workload
    (n_samples samples of 2 forward + 1 adjoint fine steps on the full grid after one warm-up
    sample), extrapolated to one gradient.  fd: the workload's fdParamElastic_3D (grid, time axes
    and medium planes); threads: host threads (0: all cores)."""
    from oracle import oracle as O
    p = O.PropParams(fd.nz, fd.nx, fd.ny, fd.nts, fd.sub, fd.minPad, float(fd.dz), float(fd.dx), float(fd.dy),
                     float(fd.dts))
    o = OracleSteps(p, fd.planes, threads)
    o.sample()
    t = statistics.mean(o.sample() for _ in range(n_samples))
    return {"value": 1.0 / (t * o.steps_per_gradient), "unit": UNIT, "cores": o.threads, "kind": "port",
            "sample": f"{n_samples} samples of 2 forward + 1 exact-adjoint fine steps of the oracle's FP32 stepper "
                      f"on the full {p.nz}x{p.nx}x{p.ny} grid ({3 * n_samples} fine steps after 3 warm-up steps), "
                      f"extrapolated to the gradient's 3 x {o.steps_per_gradient} fine steps"}


def run_reference(args):
    """Reference arm: the reference's path has no CPU implementation, so the oracle port (its
    kernels restated in C++/OpenMP) runs on the host cores, rank 0 only.  One step = one bounded
    sample of the workload: 2 forward + 1 exact-adjoint fine steps on the full grid (1/9996 of a
    gradient); shots/s is extrapolated from the timed window of K samples."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    p, med = oracle_grid(args)
    o = OracleSteps(p, med)
    for _ in range(args.warmup):
        o.sample()
    times = [o.sample() for _ in range(args.steps)]
    t = statistics.mean(times)
    v = 1.0 / (t * o.steps_per_gradient)
    cb = {"value": v, "unit": UNIT, "cores": o.threads, "kind": "port",
          "sample": f"{args.steps} timed samples (after {args.warmup} warm-up samples) of 2 forward + 1 exact-adjoint "
                    f"fine steps of the oracle's FP32 stepper on the full {p.nz}x{p.nx}x{p.ny} grid, i.e. a window of "
                    f"{3 * args.steps} fine steps after {3 * args.warmup}; shots/s extrapolated to the gradient's "
                    f"3 x {o.steps_per_gradient} fine steps"}
    out = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": 1e3 * t, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)", "impl": "reference",
           "config": {"workload": f"fwi-gradient {args.interior}^3+40 sponge ({p.nz}x{p.nx}x{p.ny}), {p.nts} samples "
                                  f"({(p.nts - 1) * p.sub} fine steps), 150x150 receivers x 9 components, Ricker 10 Hz, "
                                  f"one shot per gradient",
                      "step": "one bounded sample: 2 forward + 1 exact-adjoint fine steps on the full grid; "
                              "ms_per_step is the sample's time, value the extrapolated gradient throughput",
                      "l2_flush": "inputs larger than L2"},
           "cpu_baseline": cb, "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def run_ours(args):
    import torch
    import torch.distributed as dist
    from elasticisolib_3d_b200 import fwi as F
    from elasticisolib_3d_b200.engine import checkpoint_schedule

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        import datetime
        # bounded so that ranks left waiting on a failed peer end with an error: the longest gap
        # between collectives is one gradient plus set-up skew
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=device)

    sv, fd, prob = build_problem(args, device)
    # every rank holds its own shot; under torchrun the misfit and gradient of the step are
    # summed over ranks with one all-reduce, as an FWI iteration needs
    prob.distributed = world > 1
    # the CPU baseline runs on all host cores but two (kept for the GPU's launch thread) while the
    # untimed warm-up steps run, and is finished before the timed region starts
    cb_box = {}
    cb_thread = None
    if world == 1 and rank == 0 and not args.no_cpu:
        cb_thread = threading.Thread(
            target=lambda: cb_box.update(cb=cpu_baseline(fd, threads=max(1, (os.cpu_count() or 1) - 2))))
        cb_thread.start()

    # inputs and output in pinned host memory: the model, the shot's observed traces, the gradient
    shot = prob.shots[0]
    host_model = [torch.from_numpy(np.ascontiguousarray(sv.elastic[k])).pin_memory() for k in range(3)]
    host_obs = shot.d_obs.cpu().pin_memory()
    host_grad = [torch.empty_like(h).pin_memory() for h in host_model]
    h2d = sum(h.numel() * 4 for h in host_model) + host_obs.numel() * 4
    d2h = sum(h.numel() * 4 for h in host_grad) + 8
    stream = torch.cuda.current_stream(device)

    def step(ev=None):
        if ev:
            ev[0].record(stream)
        md = [h.to(device, non_blocking=True).requires_grad_(True) for h in host_model]
        shot.d_obs.copy_(host_obs, non_blocking=True)
        if ev:
            ev[1].record(stream)
        loss = F.ElasticFwiMisfit.apply(md[0], md[1], md[2], prob, [0])
        loss.backward()
        if ev:
            ev[2].record(stream)
        for hg, x in zip(host_grad, md):
            hg.copy_(x.grad, non_blocking=True)
        lv = loss.item()
        if ev:
            ev[3].record(stream)
        return lv

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if cb_thread is not None:
        cb_thread.join()
    cb = cb_box.get("cb")

    prob.prop.kernel_timing(16)
    for kind in KIND_NAMES:
        prob.prop.kernel_timing_read(kind)
    launches0 = prob.prop.launch_count
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(args.steps)]
    clocks = ClockSampler(local)
    clocks.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    loss_value = None
    for i in range(args.steps):
        loss_value = step(evs[i])
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    launches = prob.prop.launch_count - launches0
    device_ms = sum(e[1].elapsed_time(e[2]) for e in evs)   # inputs resident, gradient on the device
    e2e_ms = evs[0][0].elapsed_time(evs[-1][3])              # the whole loop, copies included
    sampled = {kind: prob.prop.kernel_timing_read(kind) for kind in KIND_NAMES}
    prob.prop.kernel_timing(0)
    t = torch.tensor([device_ms, e2e_ms], device=device, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    device_ms, e2e_ms = float(t[0].item()), float(t[1].item())
    value = world * args.steps / (device_ms / 1e3)

    if rank == 0:
        cells = prob.prop.cells_per_step
        peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
        if os.path.exists(peaks_path):
            with open(peaks_path) as f:
                peak = float(json.load(f)["hbm_gbs"])
            peak_src = "measured (MEASURED_PEAKS.json hbm_gbs)"
        else:
            peak, peak_src = 6650.0, "fallback"
        steps_per_pass = (fd.nts - 1) * fd.sub
        blocks = fd.nts - 1
        seg = prob.prop.checkpoint_segment or blocks
        _, recompute_blocks = checkpoint_schedule(blocks, seg)
        cell_updates = cells * (steps_per_pass + recompute_blocks * fd.sub + steps_per_pass)
        ring = args.decimation == "ring"
        # launches of each kind in one gradient
        prem = sampled.get(1, (0, 0))[1] > 0
        per_step = ({0: steps_per_pass + recompute_blocks * fd.sub, (1 if prem else 2): steps_per_pass, 6: blocks,
                     7: recompute_blocks + seg + 1} if ring else
                    {0: max(blocks - seg - 1, 0) * fd.sub, 3: (min(seg + 1, blocks) + recompute_blocks) * fd.sub,
                     5: steps_per_pass})
        kernels = {}
        for kind, (avg, cnt) in sampled.items():
            if cnt == 0 or kind not in per_step:
                continue
            traffic_per_cell = None
            prof = profiled(kind, args)
            if prof and os.path.exists(prof):
                for line in open(prof):
                    if line.startswith("dram_bytes_per_cell:"):
                        traffic_per_cell = float(line.split(":")[1])
            nbytes = kind_bytes(kind, fd.sub, prem, dual=args.variant != "plain")
            ach = nbytes * cells / (avg / 1e3) / 1e9 if avg > 0 else None
            kernels[kind] = {"kernel": kind_names(args)[kind], "bound": "hbm", "achieved": ach, "peak": peak,
                             "peak_source": peak_src, "unit": "GB/s", "frac": (ach / peak) if ach else None,
                             "traffic": traffic_per_cell * cells if traffic_per_cell else None,
                             "algorithmic_bytes_per_cell": nbytes, "cells_per_launch": cells,
                             "avg_launch_ms": avg, "sampled_launches": cnt, "launches_per_step": per_step[kind],
                             "share_of_step_est": avg * per_step[kind] / (device_ms / args.steps)}
        dom = max(kernels, key=lambda k: kernels[k]["share_of_step_est"] or 0.0)
        roofline = dict(kernels[dom])
        roofline["other_kernels"] = [kernels[k] for k in kernels if k != dom]
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": device_ms / args.steps, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
               "config": {"workload": f"fwi-gradient {args.interior}^3+40 sponge ({fd.nz}x{fd.nx}x{fd.ny}), "
                                      f"{fd.nts} samples ({steps_per_pass} fine steps), 150x150 receivers x 9 "
                                      f"components, Ricker 10 Hz, one shot per step per GPU",
                          "parallelism": f"shots sharded over {world} GPU(s)",
                          "l2_flush": "inputs larger than L2 (each field 238 MB, working set > 14 GB)",
                          "checkpoint_segment_blocks": seg, "recomputed_blocks": recompute_blocks,
                          "stepper": args.variant, "decimation": args.decimation,
                          "checkpoints": prob.prop.checkpoint_type, "velocity_slots": prob.prop.velocity_storage},
               "gcell_updates_per_s": world * args.steps * cell_updates / (device_ms / 1e3) / 1e9,
               "roofline": roofline,
               "gpu_launches": int(launches), "clocks": clk,
               "e2e": {"value": world * args.steps / (e2e_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                       "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_ms / args.steps, "loss": loss_value}}
        if cb is not None:
            out["cpu_baseline"] = cb
        print(json.dumps(out), flush=True)
    if args.breakdown and world == 1:
        kernel_breakdown(step)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def kernel_breakdown(step, top=16):
    """Device time per kernel of one more gradient after the measurement, from the CUDA activity
    trace (torch.profiler), printed to stderr; the JSON line is not affected."""
    import collections
    import torch
    from torch.profiler import ProfilerActivity, profile
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        step()
        torch.cuda.synchronize()
    agg = collections.defaultdict(lambda: [0, 0.0])
    for ev in prof.events():
        if ev.device_type == torch.autograd.DeviceType.CUDA:
            a = agg[ev.name.split("(")[0][:80]]
            a[0] += 1
            a[1] += ev.device_time_total
    tot = sum(v[1] for v in agg.values())
    print(f"kernel breakdown of one gradient: {tot / 1e3:.1f} ms device time", file=sys.stderr)
    for name, (cnt, us) in sorted(agg.items(), key=lambda kv: -kv[1][1])[:top]:
        print(f"  {us / 1e3:9.1f} ms {100 * us / tot:6.2f} % {cnt:7d}  {name}", file=sys.stderr)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
