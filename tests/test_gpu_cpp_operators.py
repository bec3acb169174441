"""GPU: the C++ shot operators (pyElastic_iso_float_3D) against the Python drop-in operators on
the same two-shot survey (same engine calls and host arithmetic: agreement to 1e-6), and the
C++ Born operator's dot test."""
import numpy as np
import pytest

from operator_case import OperatorCase
from elasticisolib_3d_b200 import hostprep as H
from elasticisolib_3d_b200 import operators as OP
from elasticisolib_3d_b200 import pyElastic_iso_float_3D as P

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _setup():
    c = OperatorCase()
    par = P.paramObj(dict(c.par))
    za, xa, ya = c.axes
    ax7 = H.grid_axes(za.n, xa.n, ya.n, za.o, xa.o, ya.o, za.d, xa.d, ya.d)
    grids = [P.hypercube([P.axis(a.n, a.o, a.d) for a in g]) for g in ax7]
    src = [[P.spaceInterpGpu_3D(*s, grids[g], c.nts, par) for g in range(7)] for s in c.sv.src_xyz]
    rec = [P.spaceInterpGpu_3D(*c.sv.rec_xyz, grids[g], c.nts, par) for g in range(7)]
    dev14 = [[s[g] for s in src] for g in range(7)] + [[rec[g]] for g in range(7)]
    h = P.hypercube([P.axis(za.n), P.axis(xa.n), P.axis(ya.n), P.axis(3)])
    return c, par, dev14, h


def _wavelet_model(c, n=1):
    m = np.zeros((n, 9, c.n_sim, c.nts), np.float32)
    for k in (3, 4, 5):
        m[:, k] = c.sv.wavelet
    m[:, 0] = 0.3 * c.sv.wavelet
    return m


def test_cpp_nonlinear_operator_matches_python_operator():
    c, par, dev14, h = _setup()
    model = _wavelet_model(c)
    ep = P.float4DReg(h, np.ascontiguousarray(c.sv.elastic))
    d_cpp = np.zeros((2, 9, c.n_rec, c.nts), np.float32)
    op = P.nonlinearPropElasticShotsGpu_3D(ep, par, *dev14)
    op.forward(False, P.float4DReg(h, model), P.float4DReg(h, d_cpp))
    d_py = np.zeros_like(d_cpp)
    OP.nonlinearPropElasticShotsGpu_3D(model, d_py, c.sv.elastic, c.par, *c.devices14).forward(False, model, d_py)
    assert np.abs(d_py).max() > 0
    assert _rel(d_cpp, d_py) < 1e-6
    rng = np.random.default_rng(3)
    data = rng.standard_normal(d_cpp.shape).astype(np.float32)
    m_cpp = np.zeros((2, 9, c.n_sim, c.nts), np.float32)
    op.adjoint(False, P.float4DReg(h, m_cpp), P.float4DReg(h, data))
    m_py = np.zeros_like(m_cpp)
    OP.nonlinearPropElasticShotsGpu_3D(m_py, data, c.sv.elastic, c.par, *c.devices14).adjoint(False, m_py, data)
    assert _rel(m_cpp, m_py) < 1e-6


def test_cpp_born_operator_matches_python_operator_and_dot_test():
    c, par, dev14, h = _setup()
    sources = [_wavelet_model(c)[0]]
    rng = np.random.default_rng(6)
    model = (rng.standard_normal((3,) + c.sv.elastic.shape[1:]) *
             np.array([20.0, 1e8, 1e8])[:, None, None, None]).astype(np.float32)
    ep = P.float4DReg(h, np.ascontiguousarray(c.sv.elastic))
    op = P.BornElasticShotsGpu_3D(ep, par, [P.float4DReg(h, np.ascontiguousarray(sources[0]))], *dev14)
    d_cpp = np.zeros((2, 9, c.n_rec, c.nts), np.float32)
    op.forward(False, P.float4DReg(h, model), P.float4DReg(h, d_cpp))
    d_py = np.zeros_like(d_cpp)
    py_op = OP.BornElasticShotsGpu_3D(model, d_py, c.sv.elastic, c.par, sources, *c.devices14)
    py_op.forward(False, model, d_py)
    assert _rel(d_cpp, d_py) < 1e-6
    data = rng.standard_normal(d_cpp.shape).astype(np.float32)
    g_cpp = np.zeros_like(model)
    op.adjoint(False, P.float4DReg(h, g_cpp), P.float4DReg(h, data))
    g_py = np.zeros_like(model)
    py_op.adjoint(False, g_py, data)
    assert _rel(g_cpp, g_py) < 1e-6
    assert op.dotTest(P.float4DReg(h, model), P.float4DReg(h, d_cpp), False, 1e-5)
