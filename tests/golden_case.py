"""The seeded inputs behind tests/golden/ref_small.npz (shared by the fixture
generator and the tests that read the fixture)."""
from __future__ import annotations

import hashlib

import numpy as np

from elasticisolib_3d_b200 import synthetic as S
from oracle import oracle as O

SEED = 11
SUBSAMPLE = 2  # the Born-adjoint image is stored on every 2nd cell along each axis


def golden_inputs():
    sv = S.small_survey(seed=SEED, nzi=16, nxi=16, nyi=16, pad=4, nts=16, nrec=5)
    par = sv.par
    sub, ntw, dtw = O.time_axes(par.getInt("nts"), par.getFloat("dts"), par.getInt("sub"))
    za, xa, ya = sv.axes
    med32 = O.medium_planes(sv.elastic, dtw, np.float32)
    # the FP64 tree reads dts as float and divides in double (fdParamElastic_3D.cpp:21-33)
    dtw64 = float(np.float32(par.getFloat("dts"))) / sub
    med64 = O.medium_planes(sv.elastic.astype(np.float64), dtw64, np.float64)
    ax7 = O.staggered_axes(za.n, xa.n, ya.n, za.o, xa.o, ya.o, za.d, xa.d, ya.d)
    pads = dict(fat=4, zPadMinus=par.getInt("zPadMinus"), zPadPlus=par.getInt("zPadPlus"),
                xPadMinus=par.getInt("xPadMinus"), xPadPlus=par.getInt("xPadPlus"), yPad=par.getInt("yPad"))
    z, x, y = sv.src_xyz[0]
    src = O.build_devices(z, x, y, ax7, pads, par.getInt("nts"))
    rz, rx, ry = sv.rec_xyz
    rec = O.build_devices(rz, rx, ry, ax7, pads, par.getInt("nts"))
    minPad = min(pads["zPadMinus"], pads["zPadPlus"], pads["xPadMinus"], pads["xPadPlus"])
    # dts and alphaCos come from the parameter file as float in both trees
    p = O.PropParams(za.n, xa.n, ya.n, par.getInt("nts"), sub, minPad, float(za.d), float(xa.d), float(ya.d),
                     float(np.float32(par.getFloat("dts"))), alphaCos=float(np.float32(0.99)))
    spos = [d.unique for d in src]
    rpos = [d.unique for d in rec]
    rng = np.random.default_rng(SEED + 1)
    nts = p.nts
    sig = [rng.standard_normal((len(spos[O.COMP_GRID[k]]), nts)) for k in range(9)]
    dat = [rng.standard_normal((len(rpos[O.COMP_GRID[k]]), nts)) for k in range(9)]
    pert64 = rng.standard_normal((8,) + med32.shape[1:]) * 1e-2
    h = hashlib.sha256()
    for a in [med32] + spos + rpos:
        h.update(np.ascontiguousarray(a).tobytes())
    return dict(params=p, med32=med32, med64=med64, spos=spos, rpos=rpos, sig=sig, dat=dat,
                pert32=pert64.astype(np.float32), pert64=pert64, digest=h.digest(), src=src, rec=rec,
                survey=sv, dtw=dtw)
