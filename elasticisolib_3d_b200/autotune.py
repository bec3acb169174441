"""Stepper autotuner: time the stepper variants on a context's own grid and keep the fastest.

Candidates are the (x tile width, pipeline stages, loader) forms the engine builds, timed with
CUDA events on the context's stream over a few bare steps of the mode that will dominate
(0 forward / 1 time-reversed / 2 the FWI adjoint: exact transpose on the dual state).  Variants
the grid cannot run (cp.async and TMA need nz % 4 == 0) are skipped.  The working wavefields of the context are overwritten; call it before propagating.
The y-chunking of the stepper grid stays automatic (a measured per-mode rule in the engine).
"""
from __future__ import annotations

import torch

from .engine import Propagator

CANDIDATES = [(8, 3, "split-fwd"), (8, 3, "split-pair"), (8, 2, "split-pair"), (8, 3, "split"), (8, 2, "split"),
              (8, 2, "tma"), (16, 2, "tma"), (8, 3, "tma"),
              (8, 2, "cpasync"), (16, 2, "cpasync"), (8, 2, "plain"), (8, 2, "tma-ring"), (8, 2, "tma-ring-ldg")]
TMA_LOADERS = ("tma", "split", "split-fwd", "split-pair")


def autotune(prop: Propagator, mode: int = 0, steps: int = 6, warmup: int = 2, candidates=None):
    """Time each candidate on `prop`'s grid, select the fastest and return
    (best, {variant: ms_per_step}).  The medium must be set."""
    cands = list(candidates or CANDIDATES)
    if prop.nz % 4 != 0:
        cands = [c for c in cands if c[2] == "plain"]
    if mode in (2, 5):
        # the dual-state adjoint runs on the TMA steppers only
        cands = [c for c in cands if c[2] in TMA_LOADERS]
    if not cands:
        return (8, 2, "plain"), {}
    stream = torch.cuda.current_stream()
    prop.set_stream(stream)
    times = {}
    for v in cands:
        prop.set_stepper_variant(*v)
        prop.step_only(mode, warmup)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        prop.step_only(mode, steps)
        e1.record(stream)
        e1.synchronize()
        times[v] = e0.elapsed_time(e1) / steps
    best = min(times, key=times.get)
    prop.set_stepper_variant(*best)
    return best, times


def autotune_gradient(prop: Propagator, steps: int = 4, warmup: int = 2):
    """Variant for the FWI gradient, whose passes are a forward and a source recompute (mode 0 each,
    their fine levels decimated from a ring once per block) and the dual-state exact adjoint
    (mode 2): minimises 2*t0 + t2 over the TMA candidates (the dual adjoint runs on TMA only).
    Returns (best, {variant: (t0, t2)})."""
    cands = [c for c in CANDIDATES if c[2] in TMA_LOADERS]
    if prop.nz % 4 != 0:
        # no TMA form fits the grid; the plain stepper runs every pass
        prop.set_stepper_variant(8, 2, "plain")
        return (8, 2, "plain"), {}
    per = {}
    for mode in (0, 2):
        _, t = autotune(prop, mode, steps, warmup, cands)
        for v, ms in t.items():
            per.setdefault(v, []).append(ms)
    best = min(per, key=lambda v: 2 * per[v][0] + per[v][1])
    prop.set_stepper_variant(*best)
    return best, {v: tuple(t) for v, t in per.items()}

