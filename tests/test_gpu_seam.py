"""GPU: the drop-in seam -- the reference-named driver functions exported by libelastic3d_b200.so
(initNonlinearElasticGpu_3D, allocateNonlinearElasticGpu_3D, propElasticFwdGpu_3D,
propElasticAdjGpu_3D, deallocateNonlinearElasticGpu_3D and their Born counterparts, declared in
include/elastic3d_b200.h after nonlinearPropElasticGpuFunctions_3D.h:10-19 and
BornElasticGpuFunctions_3D.h:9-22) -- called with data, exactly as a reference caller would (one
init for the slots of a shot loop, one allocate per slot, then propagations), against the
reference's own CUDA drivers driven with the same inputs (oracle/ref_shim.cpp).

Two slots (iGpu 0 and 1, both on device 0) hold two different media; each slot's traces match the
reference's traces of its own medium, which shows the slots are kept apart.  Bounds: 1e-5 relative
L2 for the nonlinear traces (FP32 and FP64 drivers), the Born bounds of the 120^3 comparison (data
5e-5, image 1e-4) against the FP32 Born drivers.
"""
import ctypes
import os

import numpy as np
import pytest

from elasticisolib_3d_b200 import _native as N
from elasticisolib_3d_b200 import hostprep as H
from elasticisolib_3d_b200 import operators as OP
from elasticisolib_3d_b200 import synthetic as S
from elasticisolib_3d_b200.engine import COMP_GRID
from oracle import oracle as O

pytestmark = pytest.mark.gpu

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref")
need_ref = pytest.mark.skipif(not all(os.path.exists(os.path.join(REF, f"libref_{n}.so"))
                                      for n in ("nl_f32", "nl_f64", "born_f32")),
                              reason="the reference's CUDA drivers were not built (make -C oracle ref)")

F = ctypes.POINTER(ctypes.c_float)
LL = ctypes.POINTER(ctypes.c_longlong)
c_ll = ctypes.c_longlong


def _seam_lib():
    lib = ctypes.CDLL(N.LIB_PATH)
    init = [ctypes.c_float] * 3 + [ctypes.c_int] * 4 + [ctypes.c_float] + [ctypes.c_int] * 3 + [ctypes.c_float] + \
        [ctypes.c_int] * 3
    for nm in ("initNonlinearElasticGpu_3D", "initBornElasticGpu_3D"):
        getattr(lib, nm).argtypes = init
    for nm in ("allocateNonlinearElasticGpu_3D", "allocateBornElasticGpu_3D"):
        getattr(lib, nm).argtypes = [F] * 8 + [ctypes.c_int] * 5
    for nm in ("deallocateNonlinearElasticGpu_3D", "deallocateBornElasticGpu_3D", "deallocatePinBornElasticGpu_3D"):
        getattr(lib, nm).argtypes = [ctypes.c_int] * 2
    lib.allocatePinBornElasticGpu_3D.argtypes = [ctypes.c_int] * 8
    prop = [F] * 18 + [LL, c_ll] * 14 + [ctypes.c_int] * 5
    for nm in ("propElasticFwdGpu_3D", "propElasticAdjGpu_3D"):
        getattr(lib, nm).argtypes = prop
    for nm in ("BornElasticFwdGpu_3D", "BornElasticAdjGpu_3D"):
        getattr(lib, nm).argtypes = [F] * 18 + [LL, c_ll] * 14 + [F] * 8 + [ctypes.c_int] * 5
    for nm in list(("initNonlinearElasticGpu_3D", "initBornElasticGpu_3D", "allocateNonlinearElasticGpu_3D",
                    "allocateBornElasticGpu_3D", "deallocateNonlinearElasticGpu_3D", "deallocateBornElasticGpu_3D",
                    "allocatePinBornElasticGpu_3D", "deallocatePinBornElasticGpu_3D", "propElasticFwdGpu_3D",
                    "propElasticAdjGpu_3D", "BornElasticFwdGpu_3D", "BornElasticAdjGpu_3D")):
        getattr(lib, nm).restype = ctypes.c_int
    return lib


def _fp(a):
    return a.ctypes.data_as(F)


def _geom_args(spos, rpos):
    out = []
    for tab in (spos, rpos):
        for g in range(7):
            out += [tab[g].ctypes.data_as(LL), c_ll(len(tab[g]))]
    return out


def _case(nts=300, scale_rho=1.0):
    d = 10.0
    axes, pads = S.make_grid(80, 80, 80, 16, d)
    shape = (axes[2].n, axes[1].n, axes[0].n)
    vp, vs, rho = S.gaussian_perturbed_model(shape, 2500.0, 2500.0 / 1.732, 2000.0 * scale_rho, 0.10, 4.0, 5)
    el = S.elastic_from_velocity(vp, vs, rho)
    par = S.base_params(axes, pads, nts, 0.002, 2, 40.0)
    fd = H.FdParam(el, axes, par)
    za, xa, ya = axes
    ax7 = H.grid_axes(za.n, xa.n, ya.n, za.o, xa.o, ya.o, za.d, xa.d, ya.d)
    src = H.build_devices(np.array([300.0]), np.array([400.0]), np.array([400.0]), ax7, fd.nts, par)
    g = np.linspace(100.0, 700.0, 20)
    X, Y = np.meshgrid(g, g, indexing="ij")
    rec = H.build_devices(np.full(X.size, 20.0), X.ravel(), Y.ravel(), ax7, fd.nts, par)
    spos = [np.ascontiguousarray(x.getRegPosUnique(), dtype=np.int64) for x in src]
    rpos = [np.ascontiguousarray(x.getRegPosUnique(), dtype=np.int64) for x in rec]
    irr = [np.zeros((1, fd.nts), np.float32) for _ in range(9)]
    for k in (3, 4, 5):
        irr[k][0] = S.ricker(fd.nts, 0.002, 15.0, 1.0 / 15.0)
    sig = [np.ascontiguousarray(src[COMP_GRID[k]].adjoint(False, None, irr[k])) for k in range(9)]
    OP.scale_signals(sig, src, fd.planes, fd.dx, fd.dy, fd.dz)
    med = [np.ascontiguousarray(m) for m in fd.planes]
    return fd, el, med, sig, spos, rpos, src, irr


def _pp(arrs):
    return (ctypes.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])


def _ref_nl(tree, adjoint, fd, med, sig, dat, spos, rpos):
    lib = ctypes.CDLL(os.path.join(REF, f"libref_nl_{tree}.so"))
    dims = (ctypes.c_int * 6)(fd.nz, fd.nx, fd.ny, fd.nts, fd.sub, fd.minPad)
    reals = (ctypes.c_double * 5)(float(fd.dz), float(fd.dx), float(fd.dy), float(fd.dts), float(fd.alphaCos))
    st = lib.ref_nl_run(int(adjoint), dims, reals, _pp(med), _pp(sig), _pp(dat), _pp(spos),
                        (c_ll * 7)(*[len(x) for x in spos]), _pp(rpos), (c_ll * 7)(*[len(x) for x in rpos]))
    assert st == 0


def _rel(a, b):
    a = np.concatenate([np.asarray(x, np.float64).ravel() for x in a])
    b = np.concatenate([np.asarray(x, np.float64).ravel() for x in b])
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@need_ref
def test_nonlinear_seam_two_slots_match_reference_cuda():
    lib = _seam_lib()
    cases = [_case(scale_rho=1.0), _case(scale_rho=1.15)]   # slot 0 and slot 1: two media
    fd = cases[0][0]
    assert lib.initNonlinearElasticGpu_3D(float(fd.dz), float(fd.dx), float(fd.dy), fd.nz, fd.nx, fd.ny, fd.nts,
                                          float(fd.dts), fd.sub, fd.minPad, 16, float(fd.alphaCos), 2, 0, 0) == 0
    for slot, (fdk, el, med, sig, spos, rpos, src, irr) in enumerate(cases):
        assert lib.allocateNonlinearElasticGpu_3D(*[_fp(m) for m in med], fd.nx, fd.ny, fd.nz, slot, 0) == 0
    try:
        for slot, (fdk, el, med, sig, spos, rpos, src, irr) in enumerate(cases):
            dat = [np.zeros((len(rpos[COMP_GRID[k]]), fd.nts), np.float32) for k in range(9)]
            assert lib.propElasticFwdGpu_3D(*[_fp(x) for x in sig], *[_fp(x) for x in dat], *_geom_args(spos, rpos),
                                            fd.nx, fd.ny, fd.nz, slot, 0) == 0
            ref32 = [np.zeros_like(x) for x in dat]
            _ref_nl("f32", False, fdk, med, sig, ref32, spos, rpos)
            med64 = [np.ascontiguousarray(m) for m in O.medium_planes(el.astype(np.float64),
                                                                      float(fdk.dts) / fdk.sub, np.float64)]
            sig64 = [np.ascontiguousarray(src[COMP_GRID[k]].adjoint(False, None, irr[k]), dtype=np.float64)
                     for k in range(9)]

            class _P:
                def __init__(self, u):
                    self.unique = u
            O.scale_signals(sig64, [_P(x.getRegPosUnique()) for x in src], med64, float(fdk.dx), float(fdk.dy),
                            float(fdk.dz))
            ref64 = [np.zeros(x.shape, np.float64) for x in dat]
            _ref_nl("f64", False, fdk, med64, sig64, ref64, spos, rpos)
            e32, e64 = _rel(dat, ref32), _rel(dat, ref64)
            print(f"seam slot {slot}: forward vs reference FP32 {e32:.2e}, FP64 {e64:.2e}")
            assert e32 < 1e-5 and e64 < 1e-5
            # adjoint through the seam (the reference's time-reversed stepper)
            rng = np.random.default_rng(3 + slot)
            din = [rng.standard_normal(x.shape).astype(np.float32) for x in dat]
            mout = [np.full(x.shape, 9.0, np.float32) for x in sig]
            assert lib.propElasticAdjGpu_3D(*[_fp(x) for x in mout], *[_fp(x) for x in din], *_geom_args(spos, rpos),
                                            fd.nx, fd.ny, fd.nz, slot, 0) == 0
            refm = [np.zeros_like(x) for x in mout]
            _ref_nl("f32", True, fdk, med, refm, din, spos, rpos)
            ea = _rel(mout, refm)
            print(f"seam slot {slot}: adjoint vs reference FP32 {ea:.2e}")
            assert ea < 1e-5
    finally:
        for slot in range(2):
            lib.deallocateNonlinearElasticGpu_3D(slot, 0)


@need_ref
def test_born_seam_matches_reference_cuda():
    lib = _seam_lib()
    fd, el, med, sig, spos, rpos, src, irr = _case(nts=200)
    shape = med[0].shape
    rng = np.random.default_rng(9)
    mask = rng.random(shape) < 0.01
    pert = [np.zeros(shape, np.float32) for _ in range(8)]
    for k in range(8):
        pert[k][mask] = (0.05 * rng.uniform(-1, 1, mask.sum()) * np.abs(med[k][mask])).astype(np.float32)
    assert lib.initBornElasticGpu_3D(float(fd.dz), float(fd.dx), float(fd.dy), fd.nz, fd.nx, fd.ny, fd.nts,
                                     float(fd.dts), fd.sub, fd.minPad, 16, float(fd.alphaCos), 1, 0, 0) == 0
    assert lib.allocateBornElasticGpu_3D(*[_fp(m) for m in med], fd.nx, fd.ny, fd.nz, 0, 0) == 0
    assert lib.allocatePinBornElasticGpu_3D(fd.nx, fd.ny, fd.nz, fd.nts, 1, 0, 0, 0) == 0
    try:
        dat = [np.zeros((len(rpos[COMP_GRID[k]]), fd.nts), np.float32) for k in range(9)]
        assert lib.BornElasticFwdGpu_3D(*[_fp(x) for x in sig], *[_fp(x) for x in dat], *_geom_args(spos, rpos),
                                        *[_fp(x) for x in pert], fd.nx, fd.ny, fd.nz, 0, 0) == 0
        din = [rng.standard_normal(x.shape).astype(np.float32) for x in dat]
        img = [np.zeros(shape, np.float32) for _ in range(8)]
        assert lib.BornElasticAdjGpu_3D(*[_fp(x) for x in sig], *[_fp(x) for x in din], *_geom_args(spos, rpos),
                                        *[_fp(x) for x in img], fd.nx, fd.ny, fd.nz, 0, 0) == 0
    finally:
        lib.deallocatePinBornElasticGpu_3D(0, 0)
        lib.deallocateBornElasticGpu_3D(0, 0)
    ref = ctypes.CDLL(os.path.join(REF, "libref_born_f32.so"))
    dims = (ctypes.c_int * 6)(fd.nz, fd.nx, fd.ny, fd.nts, fd.sub, fd.minPad)
    reals = (ctypes.c_double * 5)(float(fd.dz), float(fd.dx), float(fd.dy), float(fd.dts), float(fd.alphaCos))
    sn = (c_ll * 7)(*[len(x) for x in spos])
    rn = (c_ll * 7)(*[len(x) for x in rpos])
    ref_d = [np.zeros_like(x) for x in dat]
    assert ref.ref_born_run(0, dims, reals, _pp(med), _pp(sig), _pp(ref_d), _pp(spos), sn, _pp(rpos), rn,
                            _pp(pert)) == 0
    ref_g = [np.zeros(shape, np.float32) for _ in range(8)]
    assert ref.ref_born_run(1, dims, reals, _pp(med), _pp(sig), _pp(din), _pp(spos), sn, _pp(rpos), rn,
                            _pp(ref_g)) == 0
    e_d, e_g = _rel(dat, ref_d), _rel(img, ref_g)
    print(f"Born seam: data {e_d:.2e}, image {e_g:.2e}")
    assert e_d < 5e-5 and e_g < 1e-4
