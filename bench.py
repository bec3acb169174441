#!/usr/bin/env python
"""Benchmark: elastic FWI gradient shots/s on B200.

Workload (the FWI-gradient configuration): 300^3 interior + 40-cell sponge
(392 x 392 x 388 cells with the FAT ring), dx = 10 m, 2500 coarse samples at
2 ms (9996 fine steps), explosive Ricker 10 Hz source, 150 x 150 receivers
(all nine components), L2 misfit.  True model = smooth background + two
Gaussian anomalies; the gradient is taken at the background model.  Inputs are
seeded synthetic data (no dataset is involved).

One step = one shot's FWI gradient per GPU: nonlinear forward with on-device
checkpoints, residual at the receivers, Born adjoint of the residual with the
source wavefield recomputed from the checkpoints, and the Born model
post-processing, through ``ElasticFwiMisfit`` (autograd forward+backward);
with several GPUs the misfit and gradient are then summed over ranks (one
NCCL all-reduce of the flat gradient).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU (torchrun): every rank takes its own shot each step (weak scaling) and
the gradients are summed with one all-reduce; the time is the max over ranks.
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
# Algorithmic bytes per updated cell of the three stepper launches of a gradient (fp32 fields):
#   0 forward (checkpointed forward pass): read old 9 + current 9 + medium 8, write new 9 = 140 B
#   3 forward with the 3 velocity fields decimated into two accumulators (source recompute): +48 B
#   5 dual-state exact adjoint (raw + premultiplied levels: +36 B) with all 9 fields decimated
#     into two accumulators (+144 B) = 320 B
STEPPER_BYTES = {0: 140.0, 3: 188.0, 5: 320.0}
STEPPER_NAMES = {0: "forward stepper (kStepTma<0>)", 3: "forward stepper + 3-field decimation (kStepTma<0>)",
                 5: "exact-adjoint stepper, dual state + 9-field decimation (kStepTma<2>)"}
PROFILE = {5: "profiles/kStepTma_adjoint_decimated_392x392x104.txt",
           0: "profiles/kStepTma_forward_392x392x104.txt"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nts", type=int, default=2500)
    ap.add_argument("--interior", type=int, default=300)
    ap.add_argument("--variant", default="tma", choices=["tma", "plain", "auto"],
                    help="stepper: tma (8-wide, 2 stages, TMA; default), plain (plain loads, no dual-state "
                         "adjoint), auto (autotuned)")
    ap.add_argument("--ckpt", default="auto", choices=["auto", "fp32", "fp16", "bf16"])
    ap.add_argument("--velocity", default="auto", choices=["auto", "fp32", "fp16"],
                    help="storage of the decimated source velocity slots (fp32 with --ckpt fp32: the "
                         "all-FP32 plan)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--breakdown", action="store_true",
                    help="after the measurement, print the device time per kernel of one more gradient")
    return ap.parse_args()


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
    import torch
    from elasticisolib_3d_b200 import fwi as F
    from elasticisolib_3d_b200 import hostprep as H
    from elasticisolib_3d_b200 import synthetic as S
    n = args.interior
    sv = S.fwi_gradient_survey(nzi=n, nxi=n, nyi=n, nts=args.nts, true_model=False)
    svt = S.fwi_gradient_survey(nzi=n, nxi=n, nyi=n, nts=args.nts, true_model=True)
    fd = H.FdParam(sv.elastic, sv.axes, sv.par)
    ax7 = H.grid_axes(*(a.n for a in sv.axes), *(a.o for a in sv.axes), *(a.d for a in sv.axes))
    variant = {"tma": (8, 2, "tma"), "plain": (8, 2, "plain"), "auto": "auto"}[args.variant]
    prob = F.FwiProblem(fd, device=device, ckpt=args.ckpt, variant=variant, velocity=args.velocity)
    rank = int(os.environ.get("RANK", "0"))
    shot_id = rank % len(sv.src_xyz)
    src = H.build_devices(*sv.src_xyz[shot_id], ax7, fd.nts, sv.par)
    rec = H.build_devices(*sv.rec_xyz, ax7, fd.nts, sv.par)
    irr = [np.zeros((1, fd.nts), dtype=np.float32) for _ in range(9)]
    for k in (3, 4, 5):
        irr[k][0] = sv.wavelet
    shot = F.make_shot(src, rec, irr, None, device)
    # observed data: nonlinear forward on the true model
    mt = [torch.tensor(svt.elastic[k], device=device) for k in range(3)]
    planes = prob.set_model(*mt)
    shot.d_obs, _ = prob.forward_data(shot, planes)
    del planes, mt
    prob.shots.append(shot)
    torch.cuda.synchronize()
    return sv, fd, prob


def cpu_baseline(fd, n_sample_fwd=2, n_sample_adj=1):
    """Oracle (C++/OpenMP restatement) stepper timed on the host cores over a bounded sample of the
    same grid, extrapolated to one gradient (2 forward-type passes + 1 adjoint pass)."""
    import ctypes
    from oracle import oracle as O
    L = O.lib()
    threads = L.oracle_num_threads(os.cpu_count() or 1)
    p = O.PropParams(fd.nz, fd.nx, fd.ny, fd.nts, fd.sub, fd.minPad, float(fd.dz), float(fd.dx), float(fd.dy),
                     float(fd.dts))
    shape = (fd.ny, fd.nx, fd.nz)
    rng = np.random.default_rng(0)
    med = [np.asarray(fd.planes[k]) for k in range(8)]
    p0 = [np.zeros(shape, np.float32) for _ in range(9)]
    p1 = [rng.standard_normal(shape, dtype=np.float32) * 1e-3 for _ in range(9)]
    a, k1 = O._ptrs(p0)
    b, k2 = O._ptrs(p1)
    m, k3 = O._ptrs(med)
    prm = p.c()
    t0 = time.perf_counter()
    for _ in range(n_sample_fwd):
        L.oracle_step_f32(ctypes.byref(prm), a, b, m, 0, 1)
    t_fwd = (time.perf_counter() - t0) / n_sample_fwd
    t0 = time.perf_counter()
    for _ in range(n_sample_adj):
        L.oracle_step_f32(ctypes.byref(prm), a, b, m, 2, 1)
    t_adj = (time.perf_counter() - t0) / n_sample_adj
    steps = (fd.nts - 1) * fd.sub
    t_shot = 2 * steps * t_fwd + steps * t_adj
    return {"value": 1.0 / t_shot, "unit": UNIT, "cores": int(threads), "kind": "port",
            "sample": f"{n_sample_fwd} forward + {n_sample_adj} exact-adjoint fine steps of the oracle stepper "
                      f"(FP32, fused sponge) on the full {fd.nz}x{fd.nx}x{fd.ny} grid, extrapolated to "
                      f"2x{steps} forward + {steps} adjoint steps per gradient"}


def run_reference(args):
    """Reference arm: the reference's path has no CPU implementation, so the oracle port runs on the
    host cores (rank 0 only)."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    from elasticisolib_3d_b200 import hostprep as H
    from elasticisolib_3d_b200 import synthetic as S
    n = args.interior
    sv = S.fwi_gradient_survey(nzi=n, nxi=n, nyi=n, nts=args.nts)
    fd = H.FdParam(sv.elastic, sv.axes, sv.par)
    vals = []
    for i in range(args.warmup + args.steps):
        cb = cpu_baseline(fd, 1, 1)
        if i >= args.warmup:
            vals.append(cb["value"])
    v = float(np.mean(vals))
    cb["value"] = v
    out = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": 1e3 / v, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)", "impl": "reference",
           "config": {"workload": f"fwi-gradient {args.interior}^3+40 sponge ({fd.nz}x{fd.nx}x{fd.ny}), "
                                  f"{fd.nts} samples ({(fd.nts - 1) * fd.sub} fine steps), 150x150 receivers x 9 "
                                  f"components, Ricker 10 Hz, one shot per step",
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
        # between collectives is one gradient (about 90 s at the default size) plus set-up skew
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=device)

    sv, fd, prob = build_problem(args, device)
    # every rank holds its own shot; under torchrun the misfit and gradient of the step are
    # summed over ranks with one all-reduce, as an FWI iteration needs
    prob.distributed = world > 1
    m = [torch.tensor(sv.elastic[k], device=device, requires_grad=True) for k in range(3)]

    def step():
        loss = F.ElasticFwiMisfit.apply(m[0], m[1], m[2], prob, [0])
        loss.backward()
        for x in m:
            x.grad = None
        return loss

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    stream = torch.cuda.current_stream(device)
    prob.prop.kernel_timing(16)
    for mode in STEPPER_BYTES:
        prob.prop.kernel_timing_read(mode)
    launches0 = prob.prop.launch_count
    clocks = ClockSampler(local)
    clocks.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    launches = prob.prop.launch_count - launches0
    ms = e0.elapsed_time(e1)
    sampled = {mode: prob.prop.kernel_timing_read(mode) for mode in STEPPER_BYTES}
    prob.prop.kernel_timing(0)
    stepper_bytes, stepper_names = dict(STEPPER_BYTES), dict(STEPPER_NAMES)
    if args.variant == "plain":
        # plain loads: the adjoint runs on the raw state only (medium applied at the halo), no dual level
        stepper_bytes[5] = 284.0
        stepper_names = {0: "forward stepper (kStep<0>, plain loads)",
                         3: "forward stepper + 3-field decimation (kStep<0>, plain loads)",
                         5: "exact-adjoint stepper + 9-field decimation (kStep<2>, plain loads)"}
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = world * args.steps / (ms_max / 1e3)

    # end to end through the public API: model and observed data from pinned host memory,
    # gradient back to pinned host memory, every step
    e2e = None
    if not args.no_e2e:
        host_model = [torch.from_numpy(np.ascontiguousarray(sv.elastic[k])).pin_memory() for k in range(3)]
        shot = prob.shots[0]
        host_obs = shot.d_obs.cpu().pin_memory()
        host_grad = [torch.empty_like(h).pin_memory() for h in host_model]
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        for _ in range(args.steps):
            md = [h.to(device, non_blocking=True).requires_grad_(True) for h in host_model]
            shot.d_obs = host_obs.to(device, non_blocking=True)
            loss = F.ElasticFwiMisfit.apply(md[0], md[1], md[2], prob, [0])
            loss.backward()
            for hg, x in zip(host_grad, md):
                hg.copy_(x.grad, non_blocking=True)
            lv = loss.item()
        a1.record(stream)
        torch.cuda.synchronize()
        t2 = torch.tensor([a0.elapsed_time(a1)], device=device, dtype=torch.float64)
        if world > 1:
            dist.all_reduce(t2, op=dist.ReduceOp.MAX)
        h2d = sum(h.numel() * 4 for h in host_model) + host_obs.numel() * 4
        d2h = sum(h.numel() * 4 for h in host_grad) + 8
        e2e = {"value": world * args.steps / (float(t2.item()) / 1e3), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "loss": lv}

    if rank == 0:
        cells = prob.prop.cells_per_step
        peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
        if os.path.exists(peaks_path):
            with open(peaks_path) as f:
                peak = float(json.load(f)["hbm_gbs"])
            peak_src = "measured"
        else:
            peak, peak_src = 6650.0, "fallback"
        steps_per_pass = (fd.nts - 1) * fd.sub
        blocks = fd.nts - 1
        seg = prob.prop.checkpoint_segment or blocks
        _, recompute_blocks = checkpoint_schedule(blocks, seg)
        # the forward pass decimates from the block before the last segment on
        plain_fwd = max(blocks - seg - 1, 0) if seg < blocks else 0
        cell_updates = cells * (steps_per_pass + recompute_blocks * fd.sub + steps_per_pass)
        launches_per_step = {0: plain_fwd * fd.sub, 3: (blocks - plain_fwd + recompute_blocks) * fd.sub,
                             5: steps_per_pass}
        kernels = {}
        for mode, (avg, cnt) in sampled.items():
            if cnt == 0:
                continue  # e.g. the plain forward stepper when the whole record is decimated in the forward pass
            traffic_per_cell = None
            prof = os.path.join(ROOT, PROFILE[mode]) if mode in PROFILE and args.variant != "plain" else None
            if prof and os.path.exists(prof):
                for line in open(prof):
                    if line.startswith("dram_bytes_per_cell:"):
                        traffic_per_cell = float(line.split(":")[1])
            ach = stepper_bytes[mode] * cells / (avg / 1e3) / 1e9 if avg > 0 else None
            kernels[mode] = {"kernel": stepper_names[mode], "bound": "hbm", "achieved": ach, "peak": peak,
                             "peak_source": peak_src, "unit": "GB/s", "frac": (ach / peak) if ach else None,
                             "traffic": traffic_per_cell * cells if traffic_per_cell else None,
                             "algorithmic_bytes_per_cell": stepper_bytes[mode], "avg_launch_ms": avg,
                             "sampled_launches": cnt,
                             "share_of_step_est": avg * launches_per_step[mode] / (ms_max / args.steps)}
        # the dominant kernel: largest estimated share of the step
        dom = max(kernels, key=lambda m: kernels[m]["share_of_step_est"] or 0.0)
        roofline = dict(kernels[dom])
        roofline["other_kernels"] = [kernels[m] for m in kernels if m != dom]
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
               "config": {"workload": f"fwi-gradient {args.interior}^3+40 sponge ({fd.nz}x{fd.nx}x{fd.ny}), "
                                      f"{fd.nts} samples ({steps_per_pass} fine steps), 150x150 receivers x 9 "
                                      f"components, Ricker 10 Hz, one shot per step per GPU",
                          "parallelism": f"shots sharded over {world} GPU(s)",
                          "l2_flush": "inputs larger than L2 (each field 238 MB, working set > 14 GB)",
                          "checkpoint_segment_blocks": seg, "stepper": args.variant, "checkpoints": prob.prop.checkpoint_type,
                          "velocity_slots": prob.prop.velocity_storage},
               "gcell_updates_per_s": world * args.steps * cell_updates / (ms_max / 1e3) / 1e9,
               "roofline": roofline,
               "gpu_launches": int(launches), "clocks": clk, "e2e": e2e}
        if world == 1 and not args.no_cpu:
            out["cpu_baseline"] = cpu_baseline(fd)
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
