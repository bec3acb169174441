"""A two-shot survey prepared for the drop-in operator classes and for the oracle pipeline
(spatial interpolation, medium scaling and propagation restated on the CPU)."""
from __future__ import annotations

import numpy as np

from elasticisolib_3d_b200 import hostprep as H
from elasticisolib_3d_b200 import synthetic as S
from oracle import oracle as O


class OperatorCase:
    def __init__(self, seed=4, nts=20):
        sv = S.small_survey(seed=seed, nzi=16, nxi=16, nyi=16, pad=4, nts=nts, nrec=7, nshots=2)
        self.sv = sv
        par = sv.par
        self.par = par
        self.nts = par.getInt("nts")
        za, xa, ya = sv.axes
        self.axes = sv.axes
        ax7 = H.grid_axes(za.n, xa.n, ya.n, za.o, xa.o, ya.o, za.d, xa.d, ya.d)
        self.src_dev = [H.build_devices(*s, ax7, self.nts, par) for s in sv.src_xyz]
        self.rec_dev = H.build_devices(*sv.rec_xyz, ax7, self.nts, par)
        # reference-style argument lists: per grid, one entry per shot (receivers: one for all)
        self.devices14 = [[self.src_dev[i][g] for i in range(2)] for g in range(7)] + \
                         [[self.rec_dev[g]] for g in range(7)]
        self.n_sim = self.src_dev[0][0].getNDeviceIrreg()
        self.n_rec = self.rec_dev[0].getNDeviceIrreg()
        # oracle side
        sub, ntw, dtw = O.time_axes(self.nts, par.getFloat("dts"), par.getInt("sub"))
        self.dtw = dtw
        oax7 = O.staggered_axes(za.n, xa.n, ya.n, za.o, xa.o, ya.o, za.d, xa.d, ya.d)
        pads = dict(fat=4, zPadMinus=par.getInt("zPadMinus"), zPadPlus=par.getInt("zPadPlus"),
                    xPadMinus=par.getInt("xPadMinus"), xPadPlus=par.getInt("xPadPlus"), yPad=par.getInt("yPad"))
        self.o_src = [O.build_devices(*s, oax7, pads, self.nts) for s in sv.src_xyz]
        self.o_rec = O.build_devices(*sv.rec_xyz, oax7, pads, self.nts)
        minPad = min(pads["zPadMinus"], pads["zPadPlus"], pads["xPadMinus"], pads["xPadPlus"])
        self.p = O.PropParams(za.n, xa.n, ya.n, self.nts, sub, minPad, float(za.d), float(xa.d), float(ya.d),
                              float(np.float32(par.getFloat("dts"))), alphaCos=float(np.float32(0.99)))
        self.d = (float(za.d), float(xa.d), float(ya.d))

    def med(self, ep, dtype=np.float32):
        return O.medium_planes(np.asarray(ep, dtype=dtype), self.dtw if dtype == np.float32 else
                               float(np.float32(self.par.getFloat("dts"))) / self.p.sub, dtype)

    def src_reg(self, i, model9, med, dtype):
        reg = [self.o_src[i][O.COMP_GRID[k]].adjoint(np.asarray(model9[k], dtype=dtype)) for k in range(9)]
        O.scale_signals(reg, self.o_src[i], med, self.d[1], self.d[2], self.d[0])
        return reg

    def nl_forward(self, ep, model, dtype=np.float64):
        med = self.med(ep, dtype)
        out = []
        for i in range(2):
            reg = self.src_reg(i, model[0 if model.shape[0] == 1 else i], med, dtype)
            d = O.nl_forward_reg(self.p, med, reg, [x.unique for x in self.o_src[i]],
                                 [x.unique for x in self.o_rec], dtype)
            out.append(np.stack([self.o_rec[O.COMP_GRID[k]].forward(d[k]) for k in range(9)]))
        return np.stack(out)

    def born_forward(self, ep, sources, model3, dtype=np.float64):
        med = self.med(ep, dtype)
        pert = O.born_model_to_planes(model3, med[0:3], self.dtw if dtype == np.float32 else
                                      float(np.float32(self.par.getFloat("dts"))) / self.p.sub, dtype)
        out = []
        for i in range(2):
            reg = self.src_reg(i, sources[0], med, dtype)
            d = O.born_forward_reg(self.p, med, reg, pert, [x.unique for x in self.o_src[i]],
                                   [x.unique for x in self.o_rec], dtype)
            out.append(np.stack([self.o_rec[O.COMP_GRID[k]].forward(d[k]) for k in range(9)]))
        return np.stack(out)
