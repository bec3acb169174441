"""CPU: size-independent properties of the oracle itself, in FP64, on a small heterogeneous survey.

  * the Born forward/adjoint pair is an exact transpose (BornElasticGpuFunctions_3D.cu's two
    phases with stepAdjGpuBorn_3D): dot test to FP64 round-off;
  * the nonlinear forward is linear in the source signals;
  * the reference's nonlinear "adjoint" is the time-reversed forward (quirk Q7,
    nonlinearPropElasticGpuFunctions_3D.cu:765-767), not the transpose: its dot test fails by
    order one, which is why the FWI gradient runs the exact transpose instead.
"""
import numpy as np
import pytest

from cases import prepared, random_signals
from oracle import oracle as O


@pytest.fixture(scope="module")
def case():
    sv, p, med, src, rec, dtw = prepared(seed=21)
    spos = [d.unique for d in src]
    rpos = [d.unique for d in rec]
    return p, [m.astype(np.float64) for m in med], spos, rpos


def _dot(a, b):
    return sum(float(np.sum(np.asarray(x, np.float64) * np.asarray(y, np.float64))) for x, y in zip(a, b))


def test_born_pair_is_an_exact_transpose(case):
    p, med, spos, rpos = case
    rng = np.random.default_rng(4)
    sig = random_signals(spos, p.nts, rng, np.float64)
    dat = random_signals(rpos, p.nts, rng, np.float64)
    pert = [rng.standard_normal(med[0].shape) for _ in range(8)]
    lhs = _dot(O.born_forward_reg(p, med, sig, pert, spos, rpos, np.float64), dat)
    rhs = _dot(pert, O.born_adjoint_reg(p, med, sig, dat, spos, rpos, None, np.float64))
    assert abs(lhs - rhs) / abs(rhs) < 1e-13


def test_nonlinear_forward_is_linear_in_the_source(case):
    p, med, spos, rpos = case
    rng = np.random.default_rng(5)
    m1 = random_signals(spos, p.nts, rng, np.float64)
    m2 = random_signals(spos, p.nts, rng, np.float64)
    f1 = O.nl_forward_reg(p, med, m1, spos, rpos, np.float64)
    f2 = O.nl_forward_reg(p, med, m2, spos, rpos, np.float64)
    f12 = O.nl_forward_reg(p, med, [2 * a - 3 * b for a, b in zip(m1, m2)], spos, rpos, np.float64)
    num = sum(float(np.sum((c - (2 * a - 3 * b)) ** 2)) for a, b, c in zip(f1, f2, f12))
    assert (num / _dot(f12, f12)) ** 0.5 < 1e-13


def test_nonlinear_adjoint_is_time_reversed_not_transposed(case):
    p, med, spos, rpos = case
    rng = np.random.default_rng(6)
    m = random_signals(spos, p.nts, rng, np.float64)
    dat = random_signals(rpos, p.nts, rng, np.float64)
    lhs = _dot(O.nl_forward_reg(p, med, m, spos, rpos, np.float64), dat)
    rhs = _dot(m, O.nl_adjoint_reg(p, med, dat, spos, rpos, np.float64))
    assert abs(lhs - rhs) / max(abs(lhs), abs(rhs)) > 0.1
