"""GPU: y-slab domain decomposition through the reference-named seam
(propElasticFwdGpudomDec_3D / propElasticAdjGpudomDec_3D, declared in include/elastic3d_b200.h
after nonlinearPropElasticGpuFunctions_3D.h:15-19), called as the reference's
nonlinearPropElasticGpu_3D does: one init with the whole grid's ny, one allocate per slab with
ny_domDec[iGpu] planes of the shifted medium, then the decomposed propagation.

The slabs here share device 0 (runs get one GPU; the cross-GPU path is the same copies between
devices).  Every cell is updated with the undivided grid's arithmetic and the boundary planes are
exchanged after every fine step, so the traces equal propElasticFwdGpu_3D / propElasticAdjGpu_3D on
the whole grid bit for bit (checked at 1e-7 relative L2)."""
import ctypes

import numpy as np
import pytest

from elasticisolib_3d_b200 import _native as N
from elasticisolib_3d_b200.engine import domain_decomposition
from test_gpu_seam import _case, _fp, _geom_args, _rel, _seam_lib

pytestmark = pytest.mark.gpu

FAT = 4


def _domdec_lib():
    lib = _seam_lib()
    F = ctypes.POINTER(ctypes.c_float)
    LL = ctypes.POINTER(ctypes.c_longlong)
    for nm in ("propElasticFwdGpudomDec_3D", "propElasticAdjGpudomDec_3D"):
        fn = getattr(lib, nm)
        fn.argtypes = [F] * 18 + [LL, ctypes.c_longlong] * 14 + [ctypes.c_int] * 3 + \
            [ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_int]
        fn.restype = ctypes.c_int
    return lib


def _init(lib, fd, n_slots):
    st = lib.initNonlinearElasticGpu_3D(float(fd.dz), float(fd.dx), float(fd.dy), fd.nz, fd.nx, fd.ny, fd.nts,
                                        float(fd.dts), fd.sub, fd.minPad, 16, float(fd.alphaCos), n_slots, 0, 0)
    assert st == 0


def _alloc(lib, med, y0, ny, slot):
    planes = [np.ascontiguousarray(m[y0:y0 + ny]) for m in med]
    st = lib.allocateNonlinearElasticGpu_3D(*[_fp(p) for p in planes], med[0].shape[1], ny, med[0].shape[2], slot, 0)
    assert st == 0, N.lib().e3d_last_error().decode()
    return planes


def _run(lib, name, fd, sig, dat, spos, rpos, tail):
    args = [_fp(a) for a in sig] + [_fp(a) for a in dat] + _geom_args(spos, rpos) + [fd.nx, fd.ny, fd.nz] + tail
    return getattr(lib, name)(*args)


@pytest.mark.parametrize("n_slabs", [2, 3])
@pytest.mark.parametrize("adjoint", [False, True])
def test_decomposed_propagation_equals_the_whole_grid(n_slabs, adjoint):
    fd, el, med, sig, spos, rpos, src, irr = _case(nts=120)
    lib = _domdec_lib()
    sizes = domain_decomposition(fd.ny, n_slabs, FAT, fd.minPad)
    _init(lib, fd, n_slabs + 1)
    keep = []
    y0 = 0
    for s, ny in enumerate(sizes):
        keep.append(_alloc(lib, med, y0, ny, s))
        y0 += ny - 2 * FAT
    keep.append(_alloc(lib, med, 0, fd.ny, n_slabs))   # the whole grid in the next slot
    rng = np.random.default_rng(3)
    if adjoint:
        dat = [np.ascontiguousarray(rng.standard_normal((len(rpos[g]), fd.nts)).astype(np.float32))
               for g in (1, 2, 3, 0, 0, 0, 4, 5, 6)]
        whole = [np.zeros_like(a) for a in sig]
        part = [np.zeros_like(a) for a in sig]
        name = "propElasticAdjGpu_3D"
        assert _run(lib, name, fd, whole, dat, spos, rpos, [n_slabs, 0]) == 0
        nd = (ctypes.c_int * n_slabs)(*sizes)
        gl = (ctypes.c_int * n_slabs)(*([0] * n_slabs))
        assert _run(lib, "propElasticAdjGpudomDec_3D", fd, part, dat, spos, rpos, [nd, n_slabs, gl, n_slabs]) == 0
        out, ref = part, whole
    else:
        n_rec = [len(rpos[g]) for g in (1, 2, 3, 0, 0, 0, 4, 5, 6)]
        whole = [np.zeros((n, fd.nts), np.float32) for n in n_rec]
        part = [np.zeros((n, fd.nts), np.float32) for n in n_rec]
        assert _run(lib, "propElasticFwdGpu_3D", fd, sig, whole, spos, rpos, [n_slabs, 0]) == 0
        nd = (ctypes.c_int * n_slabs)(*sizes)
        gl = (ctypes.c_int * n_slabs)(*([0] * n_slabs))
        assert _run(lib, "propElasticFwdGpudomDec_3D", fd, sig, part, spos, rpos, [nd, n_slabs, gl, n_slabs]) == 0
        out, ref = part, whole
    scale = max(float(np.abs(x).max()) for x in ref)
    e = _rel(out, ref)
    print(f"{n_slabs} slabs {sizes}, {'adjoint' if adjoint else 'forward'}: relative L2 {e:.2e}, "
          f"max |diff| {max(float(np.abs(a - b).max()) for a, b in zip(out, ref)):.2e} of {scale:.2e}")
    assert scale > 0 and e < 1e-7
    for s in range(n_slabs + 1):
        assert lib.deallocateNonlinearElasticGpu_3D(s, 0) == 0


def test_decomposition_refuses_sizes_that_do_not_cover_the_grid():
    fd, el, med, sig, spos, rpos, src, irr = _case(nts=20)
    lib = _domdec_lib()
    sizes = domain_decomposition(fd.ny, 2, FAT, fd.minPad)
    _init(lib, fd, 2)
    keep = [_alloc(lib, med, 0, sizes[0], 0), _alloc(lib, med, sizes[0] - 2 * FAT, sizes[1] - 1, 1)]
    n_rec = [len(rpos[g]) for g in (1, 2, 3, 0, 0, 0, 4, 5, 6)]
    data = [np.zeros((n, fd.nts), np.float32) for n in n_rec]
    nd = (ctypes.c_int * 2)(sizes[0], sizes[1] - 1)
    gl = (ctypes.c_int * 2)(0, 0)
    assert _run(lib, "propElasticFwdGpudomDec_3D", fd, sig, data, spos, rpos, [nd, 2, gl, 2]) == 1
    del keep
    for s in range(2):
        assert lib.deallocateNonlinearElasticGpu_3D(s, 0) == 0


def test_operator_with_domdec_equals_the_undivided_operator():
    """The drop-in operator with domDec=1 (every shot over y-slabs, here two slabs sharing device 0
    through iGpu=0,0) models and back-propagates as the undivided operator does."""
    from operator_case import OperatorCase
    from elasticisolib_3d_b200 import hostprep as H
    from elasticisolib_3d_b200 import operators as OP
    c = OperatorCase()
    rng = np.random.default_rng(11)
    model = rng.standard_normal((2, 9, c.n_sim, c.nts)).astype(np.float32)
    data = np.zeros((2, 9, c.n_rec, c.nts), np.float32)
    par_dd = H.ParamObj(c.par)
    par_dd["domDec"] = 1
    par_dd["iGpu"] = "0,0"
    whole = OP.nonlinearPropElasticShotsGpu_3D(model, data, c.sv.elastic, c.par, *c.devices14)
    split = OP.nonlinearPropElasticShotsGpu_3D(model, data, c.sv.elastic, par_dd, *c.devices14)
    assert split.domDec and len(split.props[0].slabs) == 2
    d_whole, d_split = np.zeros_like(data), np.zeros_like(data)
    whole.forward(False, model, d_whole)
    split.forward(False, model, d_split)
    e = _rel([d_split], [d_whole])
    print(f"operator forward, domDec=1 vs undivided: {e:.2e}")
    assert np.abs(d_whole).max() > 0 and e < 1e-7
    m_whole, m_split = np.zeros_like(model), np.zeros_like(model)
    whole.adjoint(False, m_whole, d_whole)
    split.adjoint(False, m_split, d_whole)
    e = _rel([m_split], [m_whole])
    print(f"operator adjoint, domDec=1 vs undivided: {e:.2e}")
    assert e < 1e-7
