"""GPU: the product against the reference's own CUDA drivers on the plain nonlinear-forward
workload at full size (120^3 interior + 30-cell sponge, 168 x 200 x 188 cells, explosive 15 Hz
Ricker, 40 x 40 receivers, 1000 samples at 2 ms, 3996 fine steps).

The reference drivers (elastic_iso_float and elastic_iso_double trees) are compiled from the
reference sources into oracle/_ref by oracle/Makefile (target ref); the test is skipped where
they were not built.  Both sides get the same regular-grid inputs from this library's host
preparation.  Bound: FP32 traces within 1e-5 relative L2 of the reference's FP64 traces and of
its FP32 traces.  With -s the test prints the end-to-end time of each call (host buffers in,
traces out, device allocation and copies included on both sides).
"""
import ctypes
import json
import os
import time

import numpy as np
import pytest

from elasticisolib_3d_b200 import hostprep as H
from elasticisolib_3d_b200 import operators as OP
from elasticisolib_3d_b200 import synthetic as S
from elasticisolib_3d_b200.engine import COMP_GRID, Propagator
from oracle import oracle as O

pytestmark = pytest.mark.gpu

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref")


class _Points:
    """The oracle's view of a device set: its unique regular-grid points."""

    def __init__(self, unique):
        self.unique = unique


def _pp(arrs):
    return (ctypes.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])


def _ref_nl_forward(lib, dims, reals, med, sig, spos, rpos, nts, dtype):
    med = [np.ascontiguousarray(m, dtype=dtype) for m in med]
    sig = [np.ascontiguousarray(x, dtype=dtype) for x in sig]
    dat = [np.zeros((len(rpos[COMP_GRID[k]]), nts), dtype=dtype) for k in range(9)]
    sp = [np.ascontiguousarray(x, dtype=np.int64) for x in spos]
    rp = [np.ascontiguousarray(x, dtype=np.int64) for x in rpos]
    sn = (ctypes.c_longlong * 7)(*[len(x) for x in sp])
    rn = (ctypes.c_longlong * 7)(*[len(x) for x in rp])
    t0 = time.perf_counter()
    st = lib.ref_nl_run(0, dims, reals, _pp(med), _pp(sig), _pp(dat), _pp(sp), sn, _pp(rp), rn)
    t = time.perf_counter() - t0
    assert st == 0
    return dat, t


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "libref_nl_f64.so")),
                    reason="the reference's CUDA drivers were not built (make -C oracle ref)")
def test_plain_forward_matches_reference_cuda_fp64_and_fp32():
    sv = S.plain_forward_survey(nts=1000)
    par = sv.par
    fd = H.FdParam(sv.elastic, sv.axes, par)
    za, xa, ya = sv.axes
    ax7 = H.grid_axes(za.n, xa.n, ya.n, za.o, xa.o, ya.o, za.d, xa.d, ya.d)
    src = H.build_devices(*sv.src_xyz[0], ax7, fd.nts, par)
    rec = H.build_devices(*sv.rec_xyz, ax7, fd.nts, par)
    spos = [d.getRegPosUnique() for d in src]
    rpos = [d.getRegPosUnique() for d in rec]
    irr = [np.zeros((1, fd.nts), np.float32) for _ in range(9)]
    for k in (3, 4, 5):
        irr[k][0] = sv.wavelet
    sig = [src[COMP_GRID[k]].adjoint(False, None, irr[k]) for k in range(9)]
    OP.scale_signals(sig, src, fd.planes, fd.dx, fd.dy, fd.dz)

    pr = Propagator(fd.nz, fd.nx, fd.ny, fd.nts, fd.sub, fd.minPad, float(fd.dz), float(fd.dx), float(fd.dy),
                    float(fd.dts), float(fd.alphaCos))
    pr.set_medium(fd.planes)
    pr.nl_forward(sig, spos, rpos)  # warm-up (module load, tensor maps)
    t0 = time.perf_counter()
    got = pr.nl_forward(sig, spos, rpos)
    t_ours = time.perf_counter() - t0

    dims = (ctypes.c_int * 6)(fd.nz, fd.nx, fd.ny, fd.nts, fd.sub, fd.minPad)
    reals = (ctypes.c_double * 5)(float(fd.dz), float(fd.dx), float(fd.dy), float(fd.dts), float(fd.alphaCos))
    # FP64 tree: medium prepared in double from the same parameters (it reads dts as float)
    dtw64 = float(fd.dts) / fd.sub
    med64 = O.medium_planes(sv.elastic.astype(np.float64), dtw64, np.float64)
    sig64 = [src[COMP_GRID[k]].adjoint(False, None, irr[k]).astype(np.float64) for k in range(9)]
    O.scale_signals(sig64, [_Points(d.getRegPosUnique()) for d in src], med64, float(fd.dx), float(fd.dy),
                    float(fd.dz))
    lib64 = ctypes.CDLL(os.path.join(REF, "libref_nl_f64.so"))
    ref64, t64 = _ref_nl_forward(lib64, dims, reals, med64, sig64, spos, rpos, fd.nts, np.float64)
    lib32 = ctypes.CDLL(os.path.join(REF, "libref_nl_f32.so"))
    _ref_nl_forward(lib32, dims, reals, fd.planes, sig, spos, rpos, fd.nts, np.float32)  # warm-up
    ref32, t32 = _ref_nl_forward(lib32, dims, reals, fd.planes, sig, spos, rpos, fd.nts, np.float32)

    def rel(a, b):
        a = np.concatenate([np.asarray(x, np.float64).ravel() for x in a])
        b = np.concatenate([np.asarray(x, np.float64).ravel() for x in b])
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))

    e64, e32 = rel(got, ref64), rel(got, ref32)
    cells = (fd.nz - 8) * (fd.nx - 8) * (fd.ny - 8) * (fd.nts - 1) * fd.sub
    print(json.dumps({"workload": f"plain forward {fd.nz}x{fd.nx}x{fd.ny}, {fd.nts} samples", "cell_updates": cells,
                      "ours_s": t_ours, "reference_fp32_cuda_s": t32, "reference_fp64_cuda_s": t64,
                      "ours_gcell_per_s": cells / t_ours / 1e9, "reference_fp32_gcell_per_s": cells / t32 / 1e9,
                      "rel_l2_vs_ref_fp64": e64, "rel_l2_vs_ref_fp32": e32}), flush=True)
    assert e64 < 1e-5
    assert e32 < 1e-5


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "libref_born_f32.so")),
                    reason="the reference's CUDA drivers were not built (make -C oracle ref)")
def test_born_matches_reference_cuda_fp32_and_times_both():
    """Born forward and adjoint against the reference's FP32 CUDA drivers on an 80^3 interior + 16
    sponge grid (120^3 cells), 400 samples (1596 fine steps), explosive source, 20 x 20 receivers:
    data within 5e-5 and image within 1e-4 relative L2.  Both sides are FP32 with different summation
    orders; over 1596 steps the scattered data differ by 1.4e-5 and the image by 1.3e-5 (measured).
    The reference stores the source wavefield in pinned host memory (3*N*nts floats, 8.3 GB here)
    and streams it back for the adjoint; this library recomputes it from on-device checkpoints.
    With -s the test prints the end-to-end time of each call on both sides."""
    d = 10.0
    axes, pads = S.make_grid(80, 80, 80, 16, d)
    shape = (axes[2].n, axes[1].n, axes[0].n)
    vp, vs, rho = S.gaussian_perturbed_model(shape, 2500.0, 2500.0 / 1.732, 2000.0, 0.10, 4.0, 5)
    el = S.elastic_from_velocity(vp, vs, rho)
    par = S.base_params(axes, pads, 400, 0.002, 2, 40.0)
    fd = H.FdParam(el, axes, par)
    za, xa, ya = axes
    ax7 = H.grid_axes(za.n, xa.n, ya.n, za.o, xa.o, ya.o, za.d, xa.d, ya.d)
    src = H.build_devices(np.array([300.0]), np.array([400.0]), np.array([400.0]), ax7, fd.nts, par)
    g = np.linspace(100.0, 700.0, 20)
    X, Y = np.meshgrid(g, g, indexing="ij")
    rec = H.build_devices(np.full(X.size, 20.0), X.ravel(), Y.ravel(), ax7, fd.nts, par)
    spos = [x.getRegPosUnique() for x in src]
    rpos = [x.getRegPosUnique() for x in rec]
    irr = [np.zeros((1, fd.nts), np.float32) for _ in range(9)]
    for k in (3, 4, 5):
        irr[k][0] = S.ricker(fd.nts, 0.002, 15.0, 1.0 / 15.0)
    sig = [src[COMP_GRID[k]].adjoint(False, None, irr[k]) for k in range(9)]
    OP.scale_signals(sig, src, fd.planes, fd.dx, fd.dy, fd.dz)
    rng = np.random.default_rng(9)
    mask = rng.random(shape) < 0.01
    pert = np.zeros((8,) + shape, np.float32)
    for k in range(8):
        pert[k][mask] = (0.05 * rng.uniform(-1, 1, mask.sum()) * np.abs(fd.planes[k][mask])).astype(np.float32)
    dat = [rng.standard_normal((len(rpos[COMP_GRID[k]]), fd.nts)).astype(np.float32) for k in range(9)]

    pr = Propagator(fd.nz, fd.nx, fd.ny, fd.nts, fd.sub, fd.minPad, float(fd.dz), float(fd.dx), float(fd.dy),
                    float(fd.dts), float(fd.alphaCos))
    pr.set_medium(fd.planes)
    pr.born_forward(sig, pert, spos, rpos)  # warm-up
    t0 = time.perf_counter()
    ours_d = pr.born_forward(sig, pert, spos, rpos)
    t_fwd = time.perf_counter() - t0
    pr.born_adjoint(sig, dat, spos, rpos)  # warm-up
    t0 = time.perf_counter()
    ours_g = pr.born_adjoint(sig, dat, spos, rpos)
    t_adj = time.perf_counter() - t0

    lib = ctypes.CDLL(os.path.join(REF, "libref_born_f32.so"))
    dims = (ctypes.c_int * 6)(fd.nz, fd.nx, fd.ny, fd.nts, fd.sub, fd.minPad)
    reals = (ctypes.c_double * 5)(float(fd.dz), float(fd.dx), float(fd.dy), float(fd.dts), float(fd.alphaCos))
    med = [np.ascontiguousarray(m) for m in fd.planes]
    sp = [np.ascontiguousarray(x, dtype=np.int64) for x in spos]
    rp = [np.ascontiguousarray(x, dtype=np.int64) for x in rpos]
    sn = (ctypes.c_longlong * 7)(*[len(x) for x in sp])
    rn = (ctypes.c_longlong * 7)(*[len(x) for x in rp])
    sg = [np.ascontiguousarray(x) for x in sig]

    def ref(adjoint, data, pp):
        t0 = time.perf_counter()
        st = lib.ref_born_run(adjoint, dims, reals, _pp(med), _pp(sg), _pp(data), _pp(sp), sn, _pp(rp), rn, _pp(pp))
        assert st == 0
        return time.perf_counter() - t0

    ref_d = [np.zeros((len(rpos[COMP_GRID[k]]), fd.nts), np.float32) for k in range(9)]
    pp_in = [np.ascontiguousarray(pert[k]) for k in range(8)]
    r_fwd = ref(0, ref_d, pp_in)
    ref_g = [np.zeros(shape, np.float32) for _ in range(8)]
    r_adj = ref(1, [np.ascontiguousarray(x) for x in dat], ref_g)

    def rel(a, b):
        a = np.concatenate([np.asarray(x, np.float64).ravel() for x in a])
        b = np.concatenate([np.asarray(x, np.float64).ravel() for x in b])
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))

    e_d, e_g = rel(ours_d, ref_d), rel(ours_g, ref_g)
    print(json.dumps({"workload": f"Born {fd.nz}x{fd.nx}x{fd.ny}, {fd.nts} samples", "ours_fwd_s": t_fwd,
                      "ours_adj_s": t_adj, "reference_fp32_fwd_s": r_fwd, "reference_fp32_adj_s": r_adj,
                      "rel_l2_data": e_d, "rel_l2_image": e_g}), flush=True)
    assert e_d < 5e-5
    assert e_g < 1e-4
