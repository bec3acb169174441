"""GPU: the free surface (new physics; the reference parses freeSurface but implements none).

The surface is the first updated row z = FAT, where the normal stresses live.  Checks:
  * parity with the oracle's restatement of the same conditions (FP64, relative L2 1e-5),
    forward and time-reversed adjoint, plain and TMA steppers;
  * zero traction on the surface: szz recorded on the surface is exactly zero, and sxz, syz
    interpolated onto the surface vanish (odd images);
  * a physical check: in a homogeneous half-space a vertical surface force sends a Rayleigh
    wave whose moveout between two surface receivers travels at c_R = 0.9194 vs (Poisson
    ratio 0.25), within 3 %, clearly below vs;
  * the Born / FWI paths, which have no exact adjoint of it, refuse it.
"""
import numpy as np
import pytest

from elasticisolib_3d_b200 import hostprep as H
from elasticisolib_3d_b200 import synthetic as S
from elasticisolib_3d_b200._native import E3DError
from elasticisolib_3d_b200.engine import COMP_GRID, Propagator
from free_surface_case import half_space, moveout_velocity, oracle_params, prep
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _prop(fd, free_surface, q2compat=1):
    return Propagator(fd.nz, fd.nx, fd.ny, fd.nts, fd.sub, fd.minPad, float(fd.dz), float(fd.dx), float(fd.dy),
                      float(fd.dts), float(fd.alphaCos), q2compat=q2compat, free_surface=free_surface)


def _rel(a, b):
    a = np.concatenate([np.asarray(x, np.float64).ravel() for x in a])
    b = np.concatenate([np.asarray(x, np.float64).ravel() for x in b])
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("loader", ["plain", "tma"])
def test_free_surface_matches_oracle(loader):
    el, axes, par = half_space(24, 24, 16, 6, nts=40, smooth=0.08, seed=2)
    fd, ax7 = prep(el, axes, par)
    rng = np.random.default_rng(3)
    src = H.build_devices(np.array([20.0]), np.array([110.0]), np.array([70.0]), ax7, fd.nts, par)
    rz, rx, ry = rng.uniform(0.0, 150.0, 12), rng.uniform(10.0, 220.0, 12), rng.uniform(10.0, 140.0, 12)
    rz[:4] = 0.0  # some receivers on the surface
    rec = H.build_devices(rz, rx, ry, ax7, fd.nts, par)
    spos = [d.getRegPosUnique() for d in src]
    rpos = [d.getRegPosUnique() for d in rec]
    sig = [rng.standard_normal((len(spos[COMP_GRID[k]]), fd.nts)).astype(np.float32) for k in range(9)]
    pr = _prop(fd, 1)
    pr.set_stepper_variant(8, 2, loader)
    pr.set_medium(fd.planes)
    got = pr.nl_forward(sig, spos, rpos)
    p = oracle_params(fd, 1)
    ref64 = O.nl_forward_reg(p, fd.planes.astype(np.float64), [s.astype(np.float64) for s in sig], spos, rpos,
                             np.float64)
    assert _rel(got, ref64) < 1e-5
    # without the free surface the traces differ clearly (the check above is not vacuous)
    ref_nofs = O.nl_forward_reg(oracle_params(fd, 0), fd.planes, sig, spos, rpos, np.float32)
    assert _rel(got, ref_nofs) > 1e-2
    dat = [rng.standard_normal((len(rpos[COMP_GRID[k]]), fd.nts)).astype(np.float32) for k in range(9)]
    got_a = pr.nl_adjoint(dat, spos, rpos)
    ref_a = O.nl_adjoint_reg(p, fd.planes.astype(np.float64), [x.astype(np.float64) for x in dat], spos, rpos,
                             np.float64)
    assert _rel(got_a, ref_a) < 1e-5


def test_zero_traction_on_the_surface():
    el, axes, par = half_space(24, 32, 24, 6, nts=60)
    fd, ax7 = prep(el, axes, par)
    src = H.build_devices(np.array([30.0]), np.array([150.0]), np.array([110.0]), ax7, fd.nts, par)
    xs = np.linspace(60.0, 250.0, 8)
    rec = H.build_devices(np.zeros(8), xs, np.full(8, 115.0), ax7, fd.nts, par)
    spos = [d.getRegPosUnique() for d in src]
    irr = [np.zeros((1, fd.nts), np.float32) for _ in range(9)]
    w = S.ricker(fd.nts, 0.002, 20.0, 0.05)
    for k in (2, 3, 4, 5):
        irr[k][0] = w
    sig = [src[COMP_GRID[k]].adjoint(False, None, irr[k]) for k in range(9)]
    pr = _prop(fd, 1, q2compat=0)
    pr.set_medium(fd.planes)
    data = pr.nl_forward(sig, spos, [d.getRegPosUnique() for d in rec])
    tr = [rec[COMP_GRID[k]].forward(False, data[k]) for k in range(9)]
    scale = max(float(np.abs(tr[k]).max()) for k in (3, 4))
    assert scale > 0
    assert float(np.abs(tr[5]).max()) == 0.0        # szz on the surface
    assert float(np.abs(tr[6]).max()) <= 1e-6 * scale  # sxz
    assert float(np.abs(tr[8]).max()) <= 1e-6 * scale  # syz


def _surface_vz(free_surface):
    d = 10.0
    el, axes, par = half_space(40, 140, 40, 20, d=d, nts=520)
    fd, ax7 = prep(el, axes, par)
    src = H.build_devices(np.array([0.0]), np.array([100.0]), np.array([200.0]), ax7, fd.nts, par)
    xr = np.array([500.0, 1100.0])
    rec = H.build_devices(np.full(2, 10.0), xr, np.full(2, 200.0), ax7, fd.nts, par)
    irr = [np.zeros((1, fd.nts), np.float32) for _ in range(9)]
    irr[2][0] = S.ricker(fd.nts, 0.002, 10.0, 0.12)   # vertical force
    sig = [src[COMP_GRID[k]].adjoint(False, None, irr[k]) for k in range(9)]
    pr = _prop(fd, free_surface)
    pr.set_medium(fd.planes)
    data = pr.nl_forward(sig, [x.getRegPosUnique() for x in src], [x.getRegPosUnique() for x in rec])
    vz = rec[COMP_GRID[2]].forward(False, data[2])
    return vz.astype(np.float64), xr[1] - xr[0]


def test_rayleigh_wave_moveout():
    vs = 2500.0 / np.sqrt(3.0)
    c_r = 0.9194 * vs
    vz, dx = _surface_vz(1)
    c = moveout_velocity(vz, dx)
    assert abs(c - c_r) / c_r < 0.03, (c, c_r)
    assert c < 0.97 * vs


def test_born_and_fwi_refuse_the_free_surface():
    el, axes, par = half_space(24, 24, 16, 6, nts=20)
    fd, ax7 = prep(el, axes, par)
    src = H.build_devices(np.array([20.0]), np.array([110.0]), np.array([70.0]), ax7, fd.nts, par)
    rec = H.build_devices(np.array([0.0]), np.array([50.0]), np.array([50.0]), ax7, fd.nts, par)
    spos = [d.getRegPosUnique() for d in src]
    rpos = [d.getRegPosUnique() for d in rec]
    sig = [np.zeros((len(spos[COMP_GRID[k]]), fd.nts), np.float32) for k in range(9)]
    pr = _prop(fd, 1)
    pr.set_medium(fd.planes)
    with pytest.raises(E3DError):
        pr.born_forward(sig, np.zeros_like(fd.planes), spos, rpos)
