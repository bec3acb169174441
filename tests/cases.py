"""Shared test cases: one small survey prepared by the oracle and by the product."""
from __future__ import annotations

import numpy as np

from elasticisolib_3d_b200 import hostprep as H
from elasticisolib_3d_b200 import synthetic as S
from oracle import oracle as O


def prepared(seed=0, **kw):
    """Survey + oracle-side preparation (medium planes, devices, regular signals)."""
    sv = S.small_survey(seed=seed, **kw)
    par = sv.par
    sub, ntw, dtw = O.time_axes(par.getInt("nts"), par.getFloat("dts"), par.getInt("sub"))
    za, xa, ya = sv.axes
    med = O.medium_planes(sv.elastic, dtw, np.float32)
    ax7 = O.staggered_axes(za.n, xa.n, ya.n, za.o, xa.o, ya.o, za.d, xa.d, ya.d)
    pads = dict(fat=4, zPadMinus=par.getInt("zPadMinus"), zPadPlus=par.getInt("zPadPlus"),
                xPadMinus=par.getInt("xPadMinus"), xPadPlus=par.getInt("xPadPlus"), yPad=par.getInt("yPad"))
    z, x, y = sv.src_xyz[0]
    src = O.build_devices(z, x, y, ax7, pads, par.getInt("nts"))
    rz, rx, ry = sv.rec_xyz
    rec = O.build_devices(rz, rx, ry, ax7, pads, par.getInt("nts"))
    p = O.PropParams(za.n, xa.n, ya.n, par.getInt("nts"), sub, min(pads["zPadMinus"], pads["zPadPlus"],
                                                                   pads["xPadMinus"], pads["xPadPlus"]),
                     float(za.d), float(xa.d), float(ya.d), float(par.getFloat("dts")))
    return sv, p, med, src, rec, dtw


def random_signals(pos7, nts, rng, dtype=np.float32):
    return [rng.standard_normal((len(pos7[O.COMP_GRID[k]]), nts)).astype(dtype) for k in range(9)]


def rel_l2(a, b):
    a = np.concatenate([np.asarray(x, dtype=np.float64).ravel() for x in a])
    b = np.concatenate([np.asarray(x, dtype=np.float64).ravel() for x in b])
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
