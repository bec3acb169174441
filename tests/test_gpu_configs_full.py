"""GPU: the benchmark configurations at their full grid sizes, against pinned references, with
short records (stated per test) so that the references finish in minutes.

* batched forward modelling, 400 x 400 x 300 interior + 40 sponge (392 x 488 x 488 cells): one
  shot through this library's nonlinear forward against the reference's own elastic_iso_double
  CUDA drivers (oracle/_ref, built from the reference sources), 1e-5 relative L2;
* Born forward and adjoint, 256^3 interior + 32 sponge (328^3 cells), sparse +-5 % reflectivity:
  against the reference's FP32 and FP64 Born CUDA drivers (data 5e-5 / image 1e-4 against FP32,
  the bounds of the 120^3 comparison; 1e-4 / 2e-4 against FP64, whose FP32-vs-FP64 gap this adds);
  the record is short because the reference keeps 3*N*nts source-wavefield values in pinned host
  memory;
* the FWI gradient, 300^3 interior + 40 sponge (392^3 cells), 150 x 150 receivers: the misfit and
  the gradient with 16-bit checkpoints and 16-bit velocity slots cut into four segments, against
  the FP64 oracle (misfit 1e-4, gradient 1e-3).
With -s each test prints its measured errors.
"""
import ctypes
import json
import os

import numpy as np
import pytest
import torch

from elasticisolib_3d_b200 import fwi as F
from elasticisolib_3d_b200 import hostprep as H
from elasticisolib_3d_b200 import operators as OP
from elasticisolib_3d_b200 import synthetic as S
from elasticisolib_3d_b200.engine import COMP_GRID, Propagator
from oracle import oracle as O

pytestmark = pytest.mark.gpu

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref")


def _pp(arrs):
    return (ctypes.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])


def _rel(a, b):
    a = np.concatenate([np.asarray(x, np.float64).ravel() for x in a])
    b = np.concatenate([np.asarray(x, np.float64).ravel() for x in b])
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


class _Points:
    def __init__(self, unique):
        self.unique = unique


def _prepare(sv, shot=0):
    par = sv.par
    fd = H.FdParam(sv.elastic, sv.axes, par)
    za, xa, ya = sv.axes
    ax7 = H.grid_axes(za.n, xa.n, ya.n, za.o, xa.o, ya.o, za.d, xa.d, ya.d)
    src = H.build_devices(*sv.src_xyz[shot], ax7, fd.nts, par)
    rec = H.build_devices(*sv.rec_xyz, ax7, fd.nts, par)
    irr = [np.zeros((1, fd.nts), np.float32) for _ in range(9)]
    for k in (3, 4, 5):
        irr[k][0] = sv.wavelet
    sig = [src[COMP_GRID[k]].adjoint(False, None, irr[k]) for k in range(9)]
    OP.scale_signals(sig, src, fd.planes, fd.dx, fd.dy, fd.dz)
    return fd, src, rec, irr, sig


def _ref_args(fd):
    dims = (ctypes.c_int * 6)(fd.nz, fd.nx, fd.ny, fd.nts, fd.sub, fd.minPad)
    reals = (ctypes.c_double * 5)(float(fd.dz), float(fd.dx), float(fd.dy), float(fd.dts), float(fd.alphaCos))
    return dims, reals


def _sig64(sv, fd, src, irr):
    """The source signals and medium planes of the FP64 drivers, prepared in double."""
    med64 = O.medium_planes(sv.elastic.astype(np.float64), float(fd.dts) / fd.sub, np.float64)
    sig64 = [src[COMP_GRID[k]].adjoint(False, None, irr[k]).astype(np.float64) for k in range(9)]
    O.scale_signals(sig64, [_Points(d.getRegPosUnique()) for d in src], med64, float(fd.dx), float(fd.dy),
                    float(fd.dz))
    return med64, sig64


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "libref_nl_f64.so")),
                    reason="the reference's CUDA drivers were not built (make -C oracle ref)")
def test_batched_forward_grid_matches_reference_fp64_cuda():
    """392 x 488 x 488 cells (93 M), 200 x 200 receivers, shot 0 of the 4 x 4 surface grid; 120
    samples (476 fine steps) instead of 2000."""
    sv = S.batched_forward_survey(nts=120)
    fd, src, rec, irr, sig = _prepare(sv)
    spos = [d.getRegPosUnique() for d in src]
    rpos = [d.getRegPosUnique() for d in rec]
    pr = Propagator(fd.nz, fd.nx, fd.ny, fd.nts, fd.sub, fd.minPad, float(fd.dz), float(fd.dx), float(fd.dy),
                    float(fd.dts), float(fd.alphaCos))
    pr.set_medium(fd.planes)
    got = pr.nl_forward(sig, spos, rpos)
    pr.close()
    med64, sig64 = _sig64(sv, fd, src, irr)
    dims, reals = _ref_args(fd)
    dat = [np.zeros((len(rpos[COMP_GRID[k]]), fd.nts), np.float64) for k in range(9)]
    sp = [np.ascontiguousarray(x, dtype=np.int64) for x in spos]
    rp = [np.ascontiguousarray(x, dtype=np.int64) for x in rpos]
    lib = ctypes.CDLL(os.path.join(REF, "libref_nl_f64.so"))
    st = lib.ref_nl_run(0, dims, reals, _pp([np.ascontiguousarray(m) for m in med64]),
                        _pp([np.ascontiguousarray(s) for s in sig64]), _pp(dat), _pp(sp),
                        (ctypes.c_longlong * 7)(*[len(x) for x in sp]), _pp(rp),
                        (ctypes.c_longlong * 7)(*[len(x) for x in rp]))
    assert st == 0
    e = _rel(got, dat)
    print(json.dumps({"workload": f"batched-forward grid {fd.nz}x{fd.nx}x{fd.ny}, {fd.nts} samples",
                      "rel_l2_vs_ref_fp64_cuda": e}), flush=True)
    assert max(float(np.abs(x).max()) for x in dat) > 0
    assert e < 1e-5


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "libref_born_f64.so")),
                    reason="the reference's CUDA drivers were not built (make -C oracle ref)")
def test_born_grid_matches_reference_cuda():
    """328^3 cells, sparse +-5 % (drho, dlambda, dmu) at 1 % of the cells, a 32 x 32 receiver patch
    (10 m spacing) 20 m above the source, so that the scattered field reaches it within the short
    record; 20 samples (76 fine steps) against the FP32 drivers and 10 against the FP64 ones (8.5 GB
    of pinned host memory each) instead of 1500."""
    d = 10.0
    axes, pads = S.make_grid(256, 256, 256, 32, d)
    shape = (axes[2].n, axes[1].n, axes[0].n)
    vp, vs, rho = S.gaussian_perturbed_model(shape, 2500.0, 2500.0 / 1.732, 2000.0, 0.10, 5.0, 4)
    el = S.elastic_from_velocity(vp, vs, rho)
    rng = np.random.default_rng(17)
    mask = rng.random(shape) < 0.01
    out = {}
    for nts, tree in ((20, "f32"), (10, "f64")):
        par = S.base_params(axes, pads, nts, 0.002, 2, 40.0)
        fd = H.FdParam(el, axes, par)
        za, xa, ya = axes
        ax7 = H.grid_axes(za.n, xa.n, ya.n, za.o, xa.o, ya.o, za.d, xa.d, ya.d)
        c = 1280.0
        src = H.build_devices(np.array([c]), np.array([c]), np.array([c]), ax7, fd.nts, par)
        g = c + (np.arange(32) - 15.5) * 10.0
        X, Y = np.meshgrid(g, g, indexing="ij")
        rec = H.build_devices(np.full(X.size, c - 20.0), X.ravel(), Y.ravel(), ax7, fd.nts, par)
        spos = [x.getRegPosUnique() for x in src]
        rpos = [x.getRegPosUnique() for x in rec]
        irr = [np.zeros((1, fd.nts), np.float32) for _ in range(9)]
        for k in (3, 4, 5):
            irr[k][0] = S.ricker(fd.nts, 0.002, 25.0, 0.0)
        sig = [src[COMP_GRID[k]].adjoint(False, None, irr[k]) for k in range(9)]
        OP.scale_signals(sig, src, fd.planes, fd.dx, fd.dy, fd.dz)
        prng = np.random.default_rng(9)
        pert = np.zeros((8,) + shape, np.float32)
        for k in range(8):
            pert[k][mask] = (0.05 * prng.uniform(-1, 1, mask.sum()) * np.abs(fd.planes[k][mask])).astype(np.float32)
        dat = [prng.standard_normal((len(rpos[COMP_GRID[k]]), fd.nts)).astype(np.float32) for k in range(9)]
        pr = Propagator(fd.nz, fd.nx, fd.ny, fd.nts, fd.sub, fd.minPad, float(fd.dz), float(fd.dx), float(fd.dy),
                        float(fd.dts), float(fd.alphaCos))
        pr.set_medium(fd.planes)
        ours_d = pr.born_forward(sig, pert, spos, rpos)
        ours_g = pr.born_adjoint(sig, dat, spos, rpos)
        pr.close()
        real = np.float32 if tree == "f32" else np.float64
        if tree == "f32":
            med, sg = fd.planes, sig
        else:
            med, sg = _sig64(S.Survey(el, axes, par), fd, src, irr)
        lib = ctypes.CDLL(os.path.join(REF, f"libref_born_{tree}.so"))
        dims, reals = _ref_args(fd)
        medc = [np.ascontiguousarray(m, dtype=real) for m in med]
        sgc = [np.ascontiguousarray(x, dtype=real) for x in sg]
        sp = [np.ascontiguousarray(x, dtype=np.int64) for x in spos]
        rp = [np.ascontiguousarray(x, dtype=np.int64) for x in rpos]
        sn = (ctypes.c_longlong * 7)(*[len(x) for x in sp])
        rn = (ctypes.c_longlong * 7)(*[len(x) for x in rp])
        ref_d = [np.zeros((len(rpos[COMP_GRID[k]]), fd.nts), real) for k in range(9)]
        assert lib.ref_born_run(0, dims, reals, _pp(medc), _pp(sgc), _pp(ref_d), _pp(sp), sn, _pp(rp), rn,
                                _pp([np.ascontiguousarray(pert[k], dtype=real) for k in range(8)])) == 0
        ref_g = [np.zeros(shape, real) for _ in range(8)]
        assert lib.ref_born_run(1, dims, reals, _pp(medc), _pp(sgc), _pp([np.ascontiguousarray(x, dtype=real)
                                                                          for x in dat]),
                                _pp(sp), sn, _pp(rp), rn, _pp(ref_g)) == 0
        out[tree] = (_rel(ours_d, ref_d), _rel(ours_g, ref_g))
        del ref_g, ref_d, pert
    print(json.dumps({"workload": "Born grid 328^3", "fp32_drivers_20_samples": {"data": out["f32"][0],
                                                                                 "image": out["f32"][1]},
                      "fp64_drivers_10_samples": {"data": out["f64"][0], "image": out["f64"][1]}}), flush=True)
    assert out["f32"][0] < 5e-5 and out["f32"][1] < 1e-4
    assert out["f64"][0] < 1e-4 and out["f64"][1] < 2e-4


def test_fwi_gradient_grid_with_16_bit_plan_matches_fp64_oracle():
    """392^3 cells, 150 x 150 receivers (nine components), Ricker 10 Hz, gradient at the background;
    8 samples (28 fine steps) instead of 2500, cut into four segments (segment length 2) with FP16
    states and FP16 velocity slots.  In 14 ms the wavefield travels about 35 m, far short of the
    configuration's two deep anomalies, so the true model here is the background with its top 40
    interior cells (the slab holding the source and the receivers) 3 % faster and denser, which
    the short record does see."""
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from fwi_case import OracleFwi, explosive
    sv = S.fwi_gradient_survey(nts=8)
    true_el = sv.elastic.copy()
    z0 = 4 + sv.par.getInt("zPadMinus")   # first interior cell
    true_el[:, :, :, z0:z0 + 40] *= np.float32(1.03)
    orc = OracleFwi(sv)
    d_obs, _ = orc.data(true_el)
    loss_ref, g_ref = orc.misfit_and_gradient(sv.elastic, d_obs)
    fd = H.FdParam(sv.elastic, sv.axes, sv.par)
    prob = F.FwiProblem(fd, ckpt="fp16", segment=2, velocity="fp16")
    ax7 = H.grid_axes(*(a.n for a in sv.axes), *(a.o for a in sv.axes), *(a.d for a in sv.axes))
    src = H.build_devices(*sv.src_xyz[0], ax7, fd.nts, sv.par)
    rec = H.build_devices(*sv.rec_xyz, ax7, fd.nts, sv.par)
    prob.shots.append(F.make_shot(src, rec, explosive(fd.nts, sv.wavelet), d_obs.astype(np.float32), "cuda"))
    m = [torch.tensor(sv.elastic[k], device="cuda", requires_grad=True) for k in range(3)]
    loss = F.ElasticFwiMisfit.apply(m[0], m[1], m[2], prob)
    loss.backward()
    assert prob.prop.checkpoint_segment == 2 and prob.prop.velocity_storage == "fp16"
    e_loss = abs(loss.item() - loss_ref) / loss_ref
    errs = [float(np.linalg.norm(m[k].grad.double().cpu().numpy() - g_ref[k]) / np.linalg.norm(g_ref[k]))
            for k in range(3)]
    print(json.dumps({"workload": f"FWI gradient grid {fd.nz}x{fd.nx}x{fd.ny}, {fd.nts} samples, 4 segments FP16",
                      "misfit_rel_err": e_loss, "gradient_rel_err": errs}), flush=True)
    prob.prop.close()
    assert e_loss < 1e-4
    for k in range(3):
        assert errs[k] < 1e-3, (k, errs[k])
