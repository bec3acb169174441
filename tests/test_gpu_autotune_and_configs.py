"""GPU: the stepper autotuner, and the Born configuration's grid (256^3 interior + 32-cell sponge,
328^3 cells with FAT) through the Born pair's dot-product test."""
import numpy as np
import pytest
import torch

from cases import prepared, random_signals, rel_l2
from elasticisolib_3d_b200 import autotune as AT
from elasticisolib_3d_b200 import hostprep as H
from elasticisolib_3d_b200 import synthetic as S
from elasticisolib_3d_b200.engine import COMP_GRID, Propagator
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_autotuner_picks_a_variant_that_keeps_parity():
    sv, p, med, src, rec, dtw = prepared(seed=1)
    rng = np.random.default_rng(5)
    spos = [d.unique for d in src]
    rpos = [d.unique for d in rec]
    sig = random_signals(spos, p.nts, rng)
    pr = Propagator(p.nz, p.nx, p.ny, p.nts, p.sub, p.minPad, p.dz, p.dx, p.dy, p.dts, p.alphaCos)
    pr.set_medium(med)
    best, times = AT.autotune(pr, mode=0, steps=3, warmup=1)
    assert best in times and all(t > 0 for t in times.values())
    assert times[best] == min(times.values())
    got = pr.nl_forward(sig, spos, rpos)
    assert rel_l2(got, O.nl_forward_reg(p, med, sig, spos, rpos, np.float32)) < 1e-5
    best_g, per = AT.autotune_gradient(pr, steps=2, warmup=1)
    assert best_g[2] in AT.TMA_LOADERS and len(per[best_g]) == 2


def test_born_dot_test_on_the_born_configuration_grid():
    """256^3 interior + 32 sponge, smooth background (vp 2500, vs vp/1.732, rho 2000, +-10 %),
    sparse +-5 % (drho, dlambda, dmu) at 1 % of the cells, 128 x 128 receivers; 200 samples
    (instead of 1500) keep the test short.  Reference tolerance 1e-5 (operator.h:50)."""
    d = 10.0
    axes, pads = S.make_grid(256, 256, 256, 32, d)
    shape = (axes[2].n, axes[1].n, axes[0].n)
    vp, vs, rho = S.gaussian_perturbed_model(shape, 2500.0, 2500.0 / 1.732, 2000.0, 0.10, 5.0, 2)
    el = S.elastic_from_velocity(vp, vs, rho)
    par = S.base_params(axes, pads, 200, 0.002, 2, 25.0)
    fd = H.FdParam(el, axes, par)
    za, xa, ya = axes
    ax7 = H.grid_axes(za.n, xa.n, ya.n, za.o, xa.o, ya.o, za.d, xa.d, ya.d)
    src = H.build_devices(np.array([20.0]), np.array([1280.0]), np.array([1280.0]), ax7, fd.nts, par)
    g = np.linspace(0.0, 2540.0, 128)
    X, Y = np.meshgrid(g, g, indexing="ij")
    rec = H.build_devices(np.full(X.size, 10.0), X.ravel(), Y.ravel(), ax7, fd.nts, par)
    spos = [x.getRegPosUnique() for x in src]
    rpos = [x.getRegPosUnique() for x in rec]
    rng = np.random.default_rng(2)
    wav = S.ricker(fd.nts, 0.002, 15.0, 1.0 / 15.0)
    sig = [np.zeros((len(spos[COMP_GRID[k]]), fd.nts), np.float32) for k in range(9)]
    for k in (3, 4, 5):
        sig[k][:] = wav[None, :] * 1e6
    pert = np.zeros((8,) + shape, np.float32)
    mask = rng.random(shape) < 0.01
    for k in range(8):
        pert[k][mask] = (0.05 * rng.uniform(-1, 1, mask.sum()) * np.abs(fd.planes[k][mask])).astype(np.float32)
    dat = [rng.standard_normal((len(rpos[COMP_GRID[k]]), fd.nts)).astype(np.float32) for k in range(9)]
    pr = Propagator(fd.nz, fd.nx, fd.ny, fd.nts, fd.sub, fd.minPad, float(fd.dz), float(fd.dx), float(fd.dy),
                    float(fd.dts), float(fd.alphaCos))
    pr.set_medium(fd.planes)
    Bm = pr.born_forward(sig, pert, spos, rpos)
    Btd = pr.born_adjoint(sig, dat, spos, rpos)
    lhs = sum(float(np.dot(a.ravel().astype(np.float64), b.ravel())) for a, b in zip(Bm, dat))
    rhs = sum(float(np.dot(a.ravel().astype(np.float64), b.ravel())) for a, b in zip(pert, Btd))
    err = abs(lhs - rhs) / abs(rhs)
    print(f"born dot test 328^3 x 200 samples: <Bm,d> {lhs:.10e} <m,B'd> {rhs:.10e} rel {err:.3e}", flush=True)
    assert np.isfinite(lhs) and lhs != 0.0
    assert err < 1e-5


def test_batched_forward_configuration_two_shots_linear_in_the_source():
    """The batched-forward workload's full grid (400 x 400 x 300 interior + 40 sponge, 392 x 488 x 488
    cells, 93 M), 200 x 200 receivers, two of the 4 x 4 surface shots through the drop-in operator,
    40 samples.  Size-independent checks: the traces are linear in the source signals (scaling by
    -2.5 scales them to 1e-6), finite, non-zero, and differ between the shots."""
    from elasticisolib_3d_b200 import operators as OP
    sv = S.batched_forward_survey(nts=40, nshots=2)
    par = sv.par
    za, xa, ya = sv.axes
    ax7 = H.grid_axes(za.n, xa.n, ya.n, za.o, xa.o, ya.o, za.d, xa.d, ya.d)
    nts = par.getInt("nts")
    src = [H.build_devices(*s, ax7, nts, par) for s in sv.src_xyz]
    rec = H.build_devices(*sv.rec_xyz, ax7, nts, par)
    devices14 = [[s[g] for s in src] for g in range(7)] + [[rec[g]] for g in range(7)]
    model = np.zeros((1, 9, 1, nts), np.float32)
    for k in (3, 4, 5):
        model[0, k, 0] = sv.wavelet
    data = np.zeros((2, 9, len(sv.rec_xyz[0]), nts), np.float32)
    op = OP.nonlinearPropElasticShotsGpu_3D(model, data, sv.elastic, par, *devices14)
    op.forward(False, model, data)
    d1 = data.copy()
    op.forward(False, -2.5 * model, data)
    assert np.isfinite(d1).all() and np.abs(d1).max() > 0
    assert np.linalg.norm(data + 2.5 * d1) / np.linalg.norm(2.5 * d1) < 1e-6
    assert np.linalg.norm(d1[0] - d1[1]) > 1e-3 * np.linalg.norm(d1[0])


def test_plain_forward_configuration_with_free_surface_matches_oracle():
    """The plain-forward workload (120^3 + 30 sponge, free surface on top as the configuration asks)
    through the drop-in operator and ElasticDatComp_3D (vx, vy, vz, p), against the oracle's FP32
    pipeline with the same free surface; 60 samples keep the CPU side short."""
    from elasticisolib_3d_b200 import operators as OP
    sv = S.plain_forward_survey(nts=60)
    par = sv.par
    assert par.getInt("freeSurface") == 1
    fd = H.FdParam(sv.elastic, sv.axes, par)
    za, xa, ya = sv.axes
    ax7 = H.grid_axes(za.n, xa.n, ya.n, za.o, xa.o, ya.o, za.d, xa.d, ya.d)
    src = H.build_devices(*sv.src_xyz[0], ax7, fd.nts, par)
    rec = H.build_devices(*sv.rec_xyz, ax7, fd.nts, par)
    devices14 = [[src[g]] for g in range(7)] + [[rec[g]] for g in range(7)]
    model = np.zeros((1, 9, 1, fd.nts), np.float32)
    for k in (3, 4, 5):
        model[0, k, 0] = sv.wavelet
    data = np.zeros((1, 9, len(sv.rec_xyz[0]), fd.nts), np.float32)
    op = OP.nonlinearPropElasticShotsGpu_3D(model, data, sv.elastic, par, *devices14)
    op.forward(False, model, data)
    comp = OP.ElasticDatComp_3D("vx,vy,vz,p", data)
    got = np.zeros(comp.range_shape, np.float32)
    comp.forward(False, data, got)
    # oracle pipeline, FP32, same free surface
    reg = [src[COMP_GRID[k]].adjoint(False, None, model[0, k]) for k in range(9)]
    OP.scale_signals(reg, src, fd.planes, fd.dx, fd.dy, fd.dz)
    p = O.PropParams(fd.nz, fd.nx, fd.ny, fd.nts, fd.sub, fd.minPad, float(fd.dz), float(fd.dx), float(fd.dy),
                     float(fd.dts), alphaCos=float(fd.alphaCos), free_surface=1)
    dreg = O.nl_forward_reg(p, fd.planes, reg, [x.getRegPosUnique() for x in src],
                            [x.getRegPosUnique() for x in rec], np.float32)
    ref9 = np.stack([rec[COMP_GRID[k]].forward(False, dreg[k]) for k in range(9)])[None]
    ref = np.zeros_like(got)
    comp.forward(False, ref9, ref)
    assert np.abs(ref).max() > 0
    assert rel_l2([got], [ref]) < 1e-5
