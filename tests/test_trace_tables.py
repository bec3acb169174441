"""CPU: the FWI trace map (the tables kTraceGather / kTraceSpread read on the device) reproduces
spaceInterpGpu_3D forward and adjoint for any tap count: trilinear (8), dipole (16) and sinc
((2h)^3) receivers.  The sums run in another order than the host loops, hence a tolerance."""
import numpy as np
import pytest
import torch

from elasticisolib_3d_b200 import fwi as F
from elasticisolib_3d_b200 import hostprep as H
from elasticisolib_3d_b200 import synthetic as S
from elasticisolib_3d_b200.engine import COMP_GRID


@pytest.mark.parametrize("method,h,dipole", [("linear", 1, 0), ("linear", 1, 1), ("sinc", 2, 0), ("sinc", 2, 1)])
def test_trace_map_matches_space_interp(method, h, dipole):
    sv = S.small_survey(seed=5, nzi=16, nxi=16, nyi=16, pad=4, nts=7, nrec=5)
    za, xa, ya = sv.axes
    ax7 = H.grid_axes(za.n, xa.n, ya.n, za.o, xa.o, ya.o, za.d, xa.d, ya.d)
    rz, rx, ry = sv.rec_xyz
    # dipole poles one cell deeper, which stays inside the model for these receivers
    rec7 = H.build_devices(rz, rx, ry, ax7, 7, sv.par, dipole=dipole, shifts=(float(za.d), 0.0, 0.0),
                           method=method, hFilter1d=h, compat=False)
    rec = F.DeviceSet.from_devices(rec7, "cpu")
    tt = F.TraceTables.from_set(rec, "cpu")
    assert tt.n_taps == (2 * h) ** 3 * (2 if dipole else 1)
    rng = np.random.default_rng(9)
    nts = 7
    reg = rng.standard_normal((rec.off[9], nts)).astype(np.float32)
    # gather: irregular row r = sum over its taps of weight * regular trace
    slot = tt.slot.numpy().reshape(-1, tt.n_taps)
    wt = tt.weight.numpy().reshape(-1, tt.n_taps).astype(np.float64)
    irr = np.einsum("rt,rts->rs", wt, reg.astype(np.float64)[slot])
    # spread: regular row q = sum over its CSR entries of w * irregular trace
    row_ptr, idx, w = tt.row_ptr.numpy(), tt.idx.numpy(), tt.w.numpy().astype(np.float64)
    back = np.zeros_like(reg, dtype=np.float64)
    for q in range(rec.off[9]):
        for e in range(row_ptr[q], row_ptr[q + 1]):
            back[q] += w[e] * irr[idx[e]]
    n = rec.n_irreg
    for k in range(9):
        dev = rec7[COMP_GRID[k]]
        fwd = dev.forward(False, reg[rec.comp(k)])
        np.testing.assert_allclose(irr[k * n:(k + 1) * n], fwd, rtol=1e-5, atol=1e-5)
        adj = dev.adjoint(False, None, irr[k * n:(k + 1) * n].astype(np.float32))
        np.testing.assert_allclose(back[rec.comp(k)], adj, rtol=1e-4, atol=1e-4)


def test_empty_device_sets():
    """No receivers: empty tables, empty traces, and a trace map with no rows (the engine's
    gather and spread launch nothing for it)."""
    sv = S.small_survey(seed=5, nzi=16, nxi=16, nyi=16, pad=4, nts=7, nrec=5)
    za, xa, ya = sv.axes
    ax7 = H.grid_axes(za.n, xa.n, ya.n, za.o, xa.o, ya.o, za.d, xa.d, ya.d)
    e = np.zeros(0, np.float32)
    d7 = H.build_devices(e, e, e, ax7, 7, sv.par)
    assert all(d.getNDeviceReg() == 0 and d.getNDeviceIrreg() == 0 for d in d7)
    assert d7[0].forward(False, np.zeros((0, 7), np.float32)).shape == (0, 7)
    assert d7[0].adjoint(False, None, np.zeros((0, 7), np.float32)).shape == (0, 7)
    rec = F.DeviceSet.from_devices(d7, "cpu")
    tt = F.TraceTables.from_set(rec, "cpu")
    assert tt.n_irreg == 0 and tt.slot.numel() == 0 and tt.row_ptr.tolist() == [0]
