"""CPU: the oracle's free surface (new physics: the reference parses freeSurface but implements
none, so this path has no reference output and is pinned by physics instead):

  * zero traction on the surface: szz recorded on the surface is exactly zero, and sxz, syz
    interpolated onto the surface vanish (odd images);
  * in a homogeneous half-space a vertical surface force sends a Rayleigh wave whose moveout
    between two surface receivers travels at c_R = 0.9194 vs (Poisson ratio 0.25), within 3 %;
    without the free surface the same receivers see a clearly faster arrival.

The GPU tests compare the CUDA path with this oracle and repeat the checks on its output.
"""
import numpy as np

from elasticisolib_3d_b200 import hostprep as H
from elasticisolib_3d_b200 import synthetic as S
from elasticisolib_3d_b200.engine import COMP_GRID
from free_surface_case import half_space, moveout_velocity, oracle_params, prep
from oracle import oracle as O


def test_oracle_zero_traction_on_the_surface():
    el, axes, par = half_space(24, 32, 24, 6, nts=60)
    fd, ax7 = prep(el, axes, par)
    src = H.build_devices(np.array([30.0]), np.array([150.0]), np.array([110.0]), ax7, fd.nts, par)
    xs = np.linspace(60.0, 250.0, 8)
    rec = H.build_devices(np.zeros(8), xs, np.full(8, 115.0), ax7, fd.nts, par)
    irr = [np.zeros((1, fd.nts), np.float32) for _ in range(9)]
    w = S.ricker(fd.nts, 0.002, 20.0, 0.05)
    for k in (2, 3, 4, 5):
        irr[k][0] = w
    sig = [src[COMP_GRID[k]].adjoint(False, None, irr[k]) for k in range(9)]
    p = oracle_params(fd, 1)
    p.q2compat = 0   # sxz receivers on their own grid
    data = O.nl_forward_reg(p, fd.planes, sig, [d.getRegPosUnique() for d in src],
                            [d.getRegPosUnique() for d in rec], np.float32)
    tr = [rec[COMP_GRID[k]].forward(False, data[k]) for k in range(9)]
    scale = max(float(np.abs(tr[k]).max()) for k in (3, 4))
    assert scale > 0
    assert float(np.abs(tr[5]).max()) == 0.0
    assert float(np.abs(tr[6]).max()) <= 1e-6 * scale
    assert float(np.abs(tr[8]).max()) <= 1e-6 * scale


def _surface_vz(free_surface):
    el, axes, par = half_space(24, 80, 24, 14, d=10.0, nts=360)
    fd, ax7 = prep(el, axes, par)
    src = H.build_devices(np.array([0.0]), np.array([100.0]), np.array([120.0]), ax7, fd.nts, par)
    xr = np.array([250.0, 650.0])
    rec = H.build_devices(np.full(2, 10.0), xr, np.full(2, 120.0), ax7, fd.nts, par)
    irr = [np.zeros((1, fd.nts), np.float32) for _ in range(9)]
    irr[2][0] = S.ricker(fd.nts, 0.002, 10.0, 0.12)   # vertical force
    sig = [src[COMP_GRID[k]].adjoint(False, None, irr[k]) for k in range(9)]
    data = O.nl_forward_reg(oracle_params(fd, free_surface), fd.planes, sig, [x.getRegPosUnique() for x in src],
                            [x.getRegPosUnique() for x in rec], np.float32)
    return rec[COMP_GRID[2]].forward(False, data[2]).astype(np.float64), xr[1] - xr[0]


def test_oracle_rayleigh_wave_moveout():
    vs = 2500.0 / np.sqrt(3.0)
    c_r = 0.9194 * vs
    c = moveout_velocity(*_surface_vz(1))
    assert abs(c - c_r) / c_r < 0.03, (c, c_r)
    c0 = moveout_velocity(*_surface_vz(0))
    assert c0 > 1.2 * vs, c0
