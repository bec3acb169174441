"""GPU: the parametrisation operators on device tensors, and sinc and corrected-dipole acquisition
through a GPU propagation.

* ElasticConv_3D / ElasticConvJab_3D (elasticParamConvertModule_3D.py:30-108) on CUDA tensors
  against the same operators on FP64 numpy arrays (relative 1e-6, FP32 rounding), and FWI in
  (vp, vs, rho): autograd through vpvsrho_to_rholammu into ElasticFwiMisfit equals the Jacobian's
  adjoint applied to the (rho, lambda, mu) gradient (relative 1e-5).
* The nonlinear forward with sinc receivers and sources (8 taps per axis) and with the corrected
  dipole (compat = False), host tables from this library's spaceInterpGpu_3D, against the FP64
  oracle on the oracle's own tables (oracle.space_interp_sinc / space_interp_linear): irregular
  traces within 1e-5 relative L2.
"""
import numpy as np
import pytest
import torch

from fwi_case import explosive, survey
from elasticisolib_3d_b200 import fwi as F
from elasticisolib_3d_b200 import hostprep as H
from elasticisolib_3d_b200 import operators as OP
from elasticisolib_3d_b200 import params as P
from elasticisolib_3d_b200 import synthetic as S
from elasticisolib_3d_b200.engine import COMP_GRID, Propagator
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _model(seed=0, shape=(24, 20, 28)):
    rng = np.random.default_rng(seed)
    vp = 2500.0 + 500.0 * rng.random(shape)
    vs = vp / 1.8
    rho = 2000.0 + 300.0 * rng.random(shape)
    return np.stack([vp, vs, rho])


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_conversions_and_jacobian_on_cuda_tensors():
    m = _model()
    dm = np.random.default_rng(1).standard_normal(m.shape) * np.array([10.0, 5.0, 3.0])[:, None, None, None]
    mg = torch.tensor(m, dtype=torch.float32, device="cuda")
    dmg = torch.tensor(dm, dtype=torch.float32, device="cuda")
    for ct in (1, -1):
        ref = np.zeros_like(m)
        got = torch.zeros_like(mg)
        src = m if ct == 1 else P.vpvsrho_to_rholammu(m[0], m[1], m[2])
        src = np.stack(src) if ct == -1 else src
        P.ElasticConv_3D(src, ct).forward(False, src, ref)
        srcg = torch.tensor(src, dtype=torch.float32, device="cuda")
        P.ElasticConv_3D(srcg, ct).forward(False, srcg, got)
        assert _rel(got.double().cpu().numpy(), ref) < 1e-6
    J, Jg = P.ElasticConvJab_3D(m, m, 1), P.ElasticConvJab_3D(mg, mg, 1)
    ref, got = np.zeros_like(m), torch.zeros_like(mg)
    J.forward(False, dm, ref)
    Jg.forward(False, dmg, got)
    assert _rel(got.double().cpu().numpy(), ref) < 1e-6
    ref, got = np.zeros_like(m), torch.zeros_like(mg)
    J.adjoint(False, ref, dm)
    Jg.adjoint(False, got, dmg)
    assert _rel(got.double().cpu().numpy(), ref) < 1e-6


def test_fwi_in_vp_vs_rho_chains_the_jacobian_adjoint():
    sv, true = survey()
    fd = H.FdParam(sv.elastic, sv.axes, sv.par)
    ax7 = H.grid_axes(*(a.n for a in sv.axes), *(a.o for a in sv.axes), *(a.d for a in sv.axes))
    src = H.build_devices(*sv.src_xyz[0], ax7, fd.nts, sv.par)
    rec = H.build_devices(*sv.rec_xyz, ax7, fd.nts, sv.par)
    prob = F.FwiProblem(fd, ckpt="fp32")
    shot = F.make_shot(src, rec, explosive(fd.nts, sv.wavelet), None, "cuda")
    planes = prob.set_model(*[torch.tensor(true[k], device="cuda") for k in range(3)])
    shot.d_obs, _ = prob.forward_data(shot, planes)
    prob.shots.append(shot)
    rho, lam, mu = (torch.tensor(sv.elastic[k], device="cuda", dtype=torch.float64) for k in range(3))
    vpvsrho = [x.float() for x in P.rholammu_to_vpvsrho(rho, lam, mu)]
    # (vp, vs, rho) gradient by autograd through the conversion
    v = [x.clone().requires_grad_(True) for x in vpvsrho]
    r, l, u = P.vpvsrho_to_rholammu(v[0], v[1], v[2])
    F.ElasticFwiMisfit.apply(r, l, u, prob).backward()
    got = torch.stack([x.grad for x in v]).double().cpu().numpy()
    # (rho, lambda, mu) gradient at the same medium (the conversion's FP32 output)
    m = [x.detach().clone().requires_grad_(True) for x in (r, l, u)]
    F.ElasticFwiMisfit.apply(m[0], m[1], m[2], prob).backward()
    g_rlm = torch.stack([x.grad for x in m]).double().cpu().numpy()
    bg = torch.stack(vpvsrho).double().cpu().numpy()
    ref = np.zeros_like(bg)
    P.ElasticConvJab_3D(bg, bg, 1).adjoint(False, ref, g_rlm)
    for k in range(3):
        assert _rel(got[k], ref[k]) < 1e-5, k


def _oracle_devices(sv, method, h, dipole, shifts, compat):
    par = sv.par
    za, xa, ya = sv.axes
    ax7 = O.staggered_axes(za.n, xa.n, ya.n, za.o, xa.o, ya.o, za.d, xa.d, ya.d)
    pads = dict(fat=4, zPadMinus=par.getInt("zPadMinus"), zPadPlus=par.getInt("zPadPlus"),
                xPadMinus=par.getInt("xPadMinus"), xPadPlus=par.getInt("xPadPlus"), yPad=par.getInt("yPad"))
    nt = par.getInt("nts")

    def make(z, x, y):
        if method == "sinc":
            return [O.space_interp_sinc(z, x, y, ax7[g], pads, nt, h, dipole, shifts, compat) for g in O.GRIDS]
        return [O.space_interp_linear(z, x, y, ax7[g], pads, nt, dipole, shifts, compat) for g in O.GRIDS]
    return make(*sv.src_xyz[0]), make(*sv.rec_xyz)


def acquisition_survey():
    """32^3 interior + 6 sponge; sources and receivers at least 6 cells inside the interior, so that
    8-point sinc stencils and dipole poles stay in the updated cells."""
    sv = S.small_survey(seed=2, nzi=32, nxi=32, nyi=32, pad=6, nts=30, nrec=12)
    rng = np.random.default_rng(40)
    r = 60.0 + 180.0 * rng.random((12, 3))
    sv.rec_xyz = (r[:, 0], r[:, 1], r[:, 2])
    sv.src_xyz = [(np.array([150.0]), np.array([155.0]), np.array([145.0]))]
    return sv


@pytest.mark.parametrize("method,h,dipole", [("sinc", 4, 0), ("linear", 1, 1), ("sinc", 3, 1)])
def test_forward_with_sinc_and_corrected_dipole_acquisition_matches_fp64_oracle(method, h, dipole):
    """Both sides with the sxz receivers on their own grid (q2compat = 0): with a dipole the xz grid
    has more points than the z grid, whose table the reference's quirk Q2 would read."""
    sv = acquisition_survey()
    shifts = (10.0, 10.0, 10.0) if dipole else (0.0, 0.0, 0.0)
    fd = H.FdParam(sv.elastic, sv.axes, sv.par)
    ax7 = H.grid_axes(*(a.n for a in sv.axes), *(a.o for a in sv.axes), *(a.d for a in sv.axes))
    kw = dict(dipole=dipole, shifts=shifts, method=method, hFilter1d=h, compat=False)
    src = H.build_devices(*sv.src_xyz[0], ax7, fd.nts, sv.par, **kw)
    rec = H.build_devices(*sv.rec_xyz, ax7, fd.nts, sv.par, **kw)
    irr = explosive(fd.nts, sv.wavelet)
    for k in (0, 1, 2):   # a force source as well, so that every component carries signal
        irr[k][0] = sv.wavelet * 1e-3
    sig = [src[COMP_GRID[k]].adjoint(False, None, irr[k]) for k in range(9)]
    OP.scale_signals(sig, src, fd.planes, fd.dx, fd.dy, fd.dz)
    pr = Propagator(fd.nz, fd.nx, fd.ny, fd.nts, fd.sub, fd.minPad, float(fd.dz), float(fd.dx), float(fd.dy),
                    float(fd.dts), float(fd.alphaCos), q2compat=0)
    pr.set_medium(fd.planes)
    reg = pr.nl_forward(sig, [d.getRegPosUnique() for d in src], [d.getRegPosUnique() for d in rec])
    pr.close()
    got = np.concatenate([rec[COMP_GRID[k]].forward(False, reg[k]) for k in range(9)])
    # the oracle on its own tables, in FP64
    osrc, orec = _oracle_devices(sv, method, h, dipole, shifts, False)
    for g in range(7):
        np.testing.assert_array_equal(osrc[g].unique, src[g].getRegPosUnique())
        np.testing.assert_array_equal(orec[g].unique, rec[g].getRegPosUnique())
    dtw = float(fd.dtw)
    med = O.medium_planes(sv.elastic.astype(np.float64), dtw, np.float64)
    sreg = [osrc[O.COMP_GRID[k]].adjoint(np.asarray(irr[k], np.float64)) for k in range(9)]
    O.scale_signals(sreg, osrc, med, float(fd.dx), float(fd.dy), float(fd.dz))
    p = O.PropParams(fd.nz, fd.nx, fd.ny, fd.nts, fd.sub, fd.minPad, float(fd.dz), float(fd.dx), float(fd.dy),
                     float(fd.dts), alphaCos=float(fd.alphaCos), q2compat=0)
    dreg = O.nl_forward_reg(p, med, sreg, [d.unique for d in osrc], [d.unique for d in orec], np.float64)
    ref = np.concatenate([orec[O.COMP_GRID[k]].forward(dreg[k]) for k in range(9)])
    assert np.abs(ref).max() > 0
    e = _rel(got, ref)
    print(f"{method} h={h} dipole={dipole} (corrected): traces vs FP64 oracle {e:.2e}")
    assert e < 1e-5
