"""Stepper benchmark: bare fine steps of one stepper variant on a synthetic grid.

  python -m elasticisolib_3d_b200.stepbench --nz 392 --nx 392 --ny 104 --mode 0 --steps 20 --warmup 3 \
      [--tx 8 --stages 2 --loader tma]

Modes: 0 forward, 1 time-reversed, 2 exact transpose (run on the dual raw +
premultiplied state with the TMA loader, as the FWI adjoint pass does);
3..5 the same with the new level decimated into two coarse accumulators
(3 velocity fields for 3 and 4; 9 fields for 5), as the fused-accumulator
passes do.  The ring adjoint pass's exact transpose on the premultiplied-only
state is mode 1 on premultiplied levels (140 B per cell).  The
medium is homogeneous (vp 2500 m/s, vs 1443 m/s, rho 2000 kg/m^3, dtw 0.5 ms);
the wavefields start at zero.  Prints one JSON line with the mean step time
(CUDA events on the launching stream), the updated cells per step, the
algorithmic bytes per cell (forward/time-reversed: read old 9 + current 9 +
medium 8, write new 9 fields = 140 B; dual exact adjoint: 9 more reads of the
premultiplied level and 9 more writes = 176 B; each decimated field adds a
read and a write of two accumulators = 16 B) and the resulting GB/s.  It is
the command the stepper's ncu captures run.
"""
from __future__ import annotations

import argparse
import json

import torch

from .engine import Propagator
from .fwi import medium_planes

BYTES_PER_CELL = {0: 140.0, 1: 140.0, 2: 176.0, 3: 188.0, 4: 188.0, 5: 320.0}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--nz", type=int, default=392)
    ap.add_argument("--nx", type=int, default=392)
    ap.add_argument("--ny", type=int, default=104)
    ap.add_argument("--mode", type=int, default=0, choices=[0, 1, 2, 3, 4, 5])
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--tx", type=int, default=8)
    ap.add_argument("--stages", type=int, default=2)
    ap.add_argument("--loader", default="tma", choices=sorted(Propagator.LOADERS))
    ap.add_argument("--chunks", type=int, default=0, help="y chunks of the stepper grid (0 = automatic)")
    a = ap.parse_args(argv)
    dev = torch.device("cuda", torch.cuda.current_device())
    shape = (a.ny, a.nx, a.nz)
    rho = torch.full(shape, 2000.0, device=dev)
    vp, vs = 2500.0, 2500.0 / 1.732
    mu = torch.full(shape, 2000.0 * vs * vs, device=dev)
    lam = torch.full(shape, 2000.0 * vp * vp, device=dev) - 2 * mu
    planes = medium_planes(rho, lam, mu, 0.0005)
    pr = Propagator(a.nz, a.nx, a.ny, 10, 4, 30, 10.0, 10.0, 10.0, 0.002, device=dev.index or 0)
    pr.set_stepper_variant(a.tx, a.stages, a.loader)
    pr.set_stepper_chunks(a.chunks)
    pr.set_stream(torch.cuda.current_stream(dev))
    pr.set_medium(planes)
    pr.step_only(a.mode, a.warmup)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    pr.step_only(a.mode, a.steps)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / a.steps
    cells = pr.cells_per_step
    b = BYTES_PER_CELL[a.mode]
    print(json.dumps({"grid": [a.nz, a.nx, a.ny], "mode": a.mode, "variant": [a.tx, a.stages, a.loader], "chunks": a.chunks,
                      "ms_per_step": ms, "cells_per_step": cells, "gcells_per_s": cells / ms / 1e6,
                      "algorithmic_bytes_per_cell": b, "achieved_gbs": b * cells / ms / 1e6}), flush=True)
    pr.close()


if __name__ == "__main__":
    main()
