"""A small FWI problem prepared for both the product (torch / CUDA) and the oracle (FP64)."""
from __future__ import annotations

import numpy as np

from elasticisolib_3d_b200 import hostprep as H
from elasticisolib_3d_b200 import synthetic as S
from oracle import oracle as O


def survey(seed=3, nts=32):
    sv = S.small_survey(seed=seed, nzi=16, nxi=16, nyi=16, pad=4, nts=nts, nrec=10)
    rng = np.random.default_rng(seed + 50)
    true = sv.elastic.astype(np.float64).copy()
    true[0, 4:-4, 4:-4, 4:-4] *= 1 + 0.01 * rng.standard_normal(true[0, 4:-4, 4:-4, 4:-4].shape)
    true[1:, 4:-4, 4:-4, 4:-4] *= 1 + 0.02 * rng.standard_normal(true[1:, 4:-4, 4:-4, 4:-4].shape)
    return sv, true.astype(np.float32)


def explosive(nts, wavelet):
    """Irregular source blocks for one explosive point source (sxx = syy = szz = wavelet)."""
    irr = [np.zeros((1, nts), dtype=np.float32) for _ in range(9)]
    for k in (3, 4, 5):
        irr[k][0] = wavelet
    return irr


class OracleFwi:
    """FP64 oracle of the misfit and its Born-adjoint gradient for one shot."""

    def __init__(self, sv):
        par = sv.par
        self.sub = 2 * par.getInt("sub")
        self.dtw = float(np.float32(par.getFloat("dts"))) / self.sub
        za, xa, ya = sv.axes
        ax7 = O.staggered_axes(za.n, xa.n, ya.n, za.o, xa.o, ya.o, za.d, xa.d, ya.d)
        pads = dict(fat=4, zPadMinus=par.getInt("zPadMinus"), zPadPlus=par.getInt("zPadPlus"),
                    xPadMinus=par.getInt("xPadMinus"), xPadPlus=par.getInt("xPadPlus"), yPad=par.getInt("yPad"))
        self.src = O.build_devices(*sv.src_xyz[0], ax7, pads, par.getInt("nts"))
        self.rec = O.build_devices(*sv.rec_xyz, ax7, pads, par.getInt("nts"))
        minPad = min(pads["zPadMinus"], pads["zPadPlus"], pads["xPadMinus"], pads["xPadPlus"])
        self.p = O.PropParams(za.n, xa.n, ya.n, par.getInt("nts"), self.sub, minPad, float(za.d), float(xa.d),
                              float(ya.d), float(np.float32(par.getFloat("dts"))), alphaCos=float(np.float32(0.99)))
        self.spos = [d.unique for d in self.src]
        self.rpos = [d.unique for d in self.rec]
        self.irr = [x.astype(np.float64) for x in explosive(self.p.nts, sv.wavelet)]
        self.d = (float(za.d), float(xa.d), float(ya.d))

    def src_reg(self, med):
        reg = [self.src[O.COMP_GRID[k]].adjoint(self.irr[k]) for k in range(9)]
        O.scale_signals(reg, self.src, med, self.d[1], self.d[2], self.d[0])
        return reg

    def data(self, ep):
        med = O.medium_planes(np.asarray(ep, dtype=np.float64), self.dtw, np.float64)
        d = O.nl_forward_reg(self.p, med, self.src_reg(med), self.spos, self.rpos, np.float64)
        return np.stack([self.rec[O.COMP_GRID[k]].forward(d[k]) for k in range(9)]), med

    def misfit(self, ep, d_obs):
        d, _ = self.data(ep)
        res = d - np.asarray(d_obs, dtype=np.float64)
        return 0.5 * float(np.sum(res * res))

    def misfit_and_gradient(self, ep, d_obs):
        d, med = self.data(ep)
        res = d - np.asarray(d_obs, dtype=np.float64)
        loss = 0.5 * float(np.sum(res * res))
        rreg = [self.rec[O.COMP_GRID[k]].adjoint(res[k]) for k in range(9)]
        g8 = O.born_adjoint_reg(self.p, med, self.src_reg(med), rreg, self.spos, self.rpos, None, np.float64)
        g = O.born_planes_to_model(g8, med[0:3], self.dtw, None, np.float64)
        return loss, g
