"""Forward-modelling benchmark: shots/s of the nonlinear forward on the batched-forward workload
(400 x 400 x 300 interior + 40 sponge: 392 x 488 x 488 cells with the FAT ring; Gardner model
family; explosive Ricker 15 Hz sources on the 4 x 4 surface grid; 200 x 200 receivers).  The same
shots run one launch sequence per shot (batch of one) and advanced together by one stepper launch
per fine step (e3d_nl_forward_batch_device).

  python -m elasticisolib_3d_b200.forwardbench --shots 4 --nts 200

Inputs and outputs stay on the device (regular-grid, time-major); CUDA events on the context's
stream time each mode after one warm-up run of it.  Prints one JSON line.
"""
from __future__ import annotations

import argparse
import json

import numpy as np
import torch

from . import hostprep as H
from . import operators as OP
from . import synthetic as S
from .engine import COMP_GRID, Propagator


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--shots", type=int, default=4)
    ap.add_argument("--nts", type=int, default=200)
    a = ap.parse_args(argv)
    sv = S.batched_forward_survey(nts=a.nts, nshots=a.shots)
    fd = H.FdParam(sv.elastic, sv.axes, sv.par)
    za, xa, ya = sv.axes
    ax7 = H.grid_axes(za.n, xa.n, ya.n, za.o, xa.o, ya.o, za.d, xa.d, ya.d)
    rpos = [d.getRegPosUnique() for d in H.build_devices(*sv.rec_xyz, ax7, fd.nts, sv.par)]
    pr = Propagator(fd.nz, fd.nx, fd.ny, fd.nts, fd.sub, fd.minPad, float(fd.dz), float(fd.dx), float(fd.dy),
                    float(fd.dts), float(fd.alphaCos), q2compat=0)
    pr.set_stepper_variant(8, 3, "split-fwd")
    pr.set_medium(fd.planes)
    st = torch.cuda.Stream(torch.device("cuda", 0))
    pr.set_stream(st)
    spos, models = [], []
    for s in range(a.shots):
        src = H.build_devices(*sv.src_xyz[s], ax7, fd.nts, sv.par)
        irr = [np.zeros((1, fd.nts), np.float32) for _ in range(9)]
        for k in (3, 4, 5):
            irr[k][0] = sv.wavelet
        sig = [src[COMP_GRID[k]].adjoint(False, None, irr[k]) for k in range(9)]
        OP.scale_signals(sig, src, fd.planes, fd.dx, fd.dy, fd.dz)
        spos.append([d.getRegPosUnique() for d in src])
        models.append(sig)
    single = [pr.batch_tables([models[s]], [spos[s]], rpos) for s in range(a.shots)]
    batched = [pr.batch_tables(models, spos, rpos)]
    res = {}
    for name, groups in (("sequential", single), ("batched", batched)):
        for bt in groups:
            pr.nl_forward_batch_device(bt)
        st.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for bt in groups:
            pr.nl_forward_batch_device(bt)
        e1.record(st)
        e1.synchronize()
        res[name] = e0.elapsed_time(e1) / 1e3
    one = single[-1].rec_sig
    nb = batched[0].split(batched[0].rec_sig.cpu().numpy().T)[a.shots - 1]
    ns = single[-1].split(one.cpu().numpy().T)[0]
    diff = max(float(np.abs(x - y).max()) for x, y in zip(nb, ns))
    scale = max(float(np.abs(y).max()) for y in ns)
    cells = (fd.nz - 8) * (fd.nx - 8) * (fd.ny - 8) * (fd.nts - 1) * fd.sub * a.shots
    print(json.dumps({"workload": f"batched forward {fd.nz}x{fd.nx}x{fd.ny} cells, {fd.nts} samples, sub {fd.sub}, "
                                  f"{a.shots} shots",
                      "sequential_s": round(res["sequential"], 4), "batched_s": round(res["batched"], 4),
                      "sequential_shots_per_s": a.shots / res["sequential"],
                      "batched_shots_per_s": a.shots / res["batched"],
                      "speedup": res["sequential"] / res["batched"],
                      "batched_gcells_per_s": cells / res["batched"] / 1e9,
                      "last_shot_max_abs_diff": diff, "last_shot_max_abs": scale}), flush=True)
    pr.close()


if __name__ == "__main__":
    main()
