"""GPU: the drop-in shot operators (reference class names and layouts) against the oracle
pipeline (interpolation + medium scaling + propagation on the CPU), and their dot tests."""
import numpy as np
import pytest

from operator_case import OperatorCase
from elasticisolib_3d_b200 import operators as OP
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _wavelet_model(c, n_slices=1):
    m = np.zeros((n_slices, 9, c.n_sim, c.nts), np.float32)
    for k in (3, 4, 5):
        m[:, k, :, :] = c.sv.wavelet[None, None, :]
    m[:, 0, :, :] = 0.3 * c.sv.wavelet[None, None, :]
    return m


def test_nonlinear_shots_forward_matches_fp64_oracle():
    c = OperatorCase()
    model = _wavelet_model(c)
    data = np.zeros((2, 9, c.n_rec, c.nts), np.float32)
    op = OP.nonlinearPropElasticShotsGpu_3D(model, data, c.sv.elastic, c.par, *c.devices14)
    op.forward(False, model, data)
    ref = c.nl_forward(c.sv.elastic, model, np.float64)
    assert _rel(data, ref) < 1e-5
    # add accumulates
    op.forward(True, model, data)
    assert _rel(data, 2 * ref) < 1e-5


def test_nonlinear_shots_adjoint_matches_oracle():
    c = OperatorCase()
    rng = np.random.default_rng(5)
    model = np.zeros((2, 9, c.n_sim, c.nts), np.float32)
    data = rng.standard_normal((2, 9, c.n_rec, c.nts)).astype(np.float32)
    op = OP.nonlinearPropElasticShotsGpu_3D(model, data, c.sv.elastic, c.par, *c.devices14)
    op.adjoint(False, model, data)
    med = c.med(c.sv.elastic)
    for i in range(2):
        reg = [c.o_rec[O.COMP_GRID[k]].adjoint(data[i, k]) for k in range(9)]
        O.scale_signals(reg, c.o_rec, med, c.d[1], c.d[2], c.d[0])
        m = O.nl_adjoint_reg(c.p, med, reg, [x.unique for x in c.o_src[i]], [x.unique for x in c.o_rec],
                             np.float32)
        ref = np.stack([c.o_src[i][O.COMP_GRID[k]].forward(m[k]) for k in range(9)])
        assert _rel(model[i], ref) < 1e-5


def test_born_shots_forward_matches_fp64_oracle_and_dot_test():
    c = OperatorCase()
    rng = np.random.default_rng(6)
    sources = [_wavelet_model(c)[0]]
    model = (rng.standard_normal((3,) + c.sv.elastic.shape[1:]) * np.array([20.0, 1e8, 1e8])[:, None, None, None]
             ).astype(np.float32)
    data = np.zeros((2, 9, c.n_rec, c.nts), np.float32)
    op = OP.BornElasticShotsGpu_3D(model, data, c.sv.elastic, c.par, sources, *c.devices14)
    op.forward(False, model, data)
    ref = c.born_forward(c.sv.elastic, sources, model, np.float64)
    assert _rel(data, ref) < 1e-4
    # the Born pair is an exact transpose: the reference's dot test (tolerance 1e-5)
    assert op.dotTest(verb=False, maxError=1e-5)


def test_nonlinear_fwi_operator_models_the_stored_sources():
    c = OperatorCase()
    src = _wavelet_model(c)
    data = np.zeros((2, 9, c.n_rec, c.nts), np.float32)
    op = OP.nonlinearFwiPropElasticShotsGpu_3D(c.sv.elastic, data, src, c.par, *c.devices14)
    op.forward(False, c.sv.elastic, data)
    ref = c.nl_forward(c.sv.elastic, src, np.float64)
    assert _rel(data, ref) < 1e-5
