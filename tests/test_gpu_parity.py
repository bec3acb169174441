"""GPU parity: the CUDA path (through the C ABI) against the oracle on the same inputs.

Tolerances: relative L2 over all traces.  FP32 CUDA vs FP32 oracle differ
only by summation order/FMA contraction (1e-5); FP32 vs the FP64 oracle is
the accuracy bound of the FP32 path (1e-5 for forward traces, 1e-4 for the Born
image, whose imaging condition multiplies two propagated fields).
"""
import numpy as np
import pytest

from cases import prepared, random_signals, rel_l2
from elasticisolib_3d_b200.engine import Propagator
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _prop(p, **kw):
    pr = Propagator(p.nz, p.nx, p.ny, p.nts, p.sub, p.minPad, p.dz, p.dx, p.dy, p.dts, p.alphaCos, **kw)
    return pr


VARIANTS = [(8, 2, "plain"), (16, 2, "plain"), (8, 2, "cpasync"), (8, 3, "cpasync"), (16, 2, "cpasync"),
            (8, 2, "tma"), (8, 3, "tma"), (16, 2, "tma"), (8, 2, "tma-ring"), (16, 2, "tma-ring"),
            (8, 2, "tma-ring-ldg"), (8, 3, "tma-ring-ldg"), (8, 2, "tma-ring-ldg2"),
            (8, 2, "split"), (8, 3, "split"), (8, 4, "split"),
            (8, 2, "split-pair"), (8, 3, "split-pair"), (8, 4, "split-pair")]


@pytest.mark.parametrize("tx,stages,loader", VARIANTS)
def test_nl_forward_matches_oracle(tx, stages, loader):
    sv, p, med, src, rec, dtw = prepared(seed=1)
    rng = np.random.default_rng(5)
    spos = [d.unique for d in src]
    rpos = [d.unique for d in rec]
    sig = random_signals(spos, p.nts, rng)
    pr = _prop(p)
    pr.set_stepper_variant(tx, stages, loader)
    pr.set_medium(med)
    got = pr.nl_forward(sig, spos, rpos)
    ref32 = O.nl_forward_reg(p, med, sig, spos, rpos, np.float32)
    ref64 = O.nl_forward_reg(p, med.astype(np.float64), [s.astype(np.float64) for s in sig], spos, rpos, np.float64)
    assert rel_l2(got, ref32) < 1e-5
    assert rel_l2(got, ref64) < 1e-5


@pytest.mark.parametrize("loader", ["plain", "tma", "split", "split-pair"])
def test_nl_adjoint_matches_oracle(loader):
    sv, p, med, src, rec, dtw = prepared(seed=2)
    rng = np.random.default_rng(6)
    spos = [d.unique for d in src]
    rpos = [d.unique for d in rec]
    dat = random_signals(rpos, p.nts, rng)
    pr = _prop(p)
    pr.set_stepper_variant(8, 3 if loader.startswith("split") else 2, loader)
    pr.set_medium(med)
    got = pr.nl_adjoint(dat, spos, rpos)
    ref = O.nl_adjoint_reg(p, med, dat, spos, rpos, np.float32)
    assert rel_l2(got, ref) < 1e-5


def test_born_forward_matches_oracle():
    sv, p, med, src, rec, dtw = prepared(seed=3)
    rng = np.random.default_rng(7)
    spos = [d.unique for d in src]
    rpos = [d.unique for d in rec]
    sig = random_signals(spos, p.nts, rng)
    pert = (rng.standard_normal((8,) + med.shape[1:]) * 1e-2).astype(np.float32)
    pr = _prop(p)
    pr.set_medium(med)
    got = pr.born_forward(sig, pert, spos, rpos)
    ref = O.born_forward_reg(p, med, sig, pert, spos, rpos, np.float32)
    assert rel_l2(got, ref) < 1e-5


@pytest.mark.parametrize("segment,loader", [(0, "plain"), (1, "plain"), (3, "plain"), (0, "tma"), (3, "tma"),
                                            (0, "split"), (1, "split"), (3, "split")])
def test_born_adjoint_matches_oracle(segment, loader):
    sv, p, med, src, rec, dtw = prepared(seed=4)
    rng = np.random.default_rng(8)
    spos = [d.unique for d in src]
    rpos = [d.unique for d in rec]
    sig = random_signals(spos, p.nts, rng)
    dat = random_signals(rpos, p.nts, rng)
    pr = _prop(p)
    pr.set_medium(med)
    pr.set_checkpoint_policy("fp32", segment)
    pr.set_stepper_variant(8, 3 if loader.startswith("split") else 2, loader)
    got = pr.born_adjoint(sig, dat, spos, rpos)
    ref = O.born_adjoint_reg(p, med, sig, dat, spos, rpos, None, np.float32)
    assert rel_l2(got, ref) < 1e-5


def test_born_dot_product():
    """<B m, d> = <m, B^T d> for the CUDA Born pair (reference tolerance 1e-5, operator.h:50)."""
    sv, p, med, src, rec, dtw = prepared(seed=5)
    rng = np.random.default_rng(9)
    spos = [d.unique for d in src]
    rpos = [d.unique for d in rec]
    sig = random_signals(spos, p.nts, rng)
    dat = random_signals(rpos, p.nts, rng)
    pert = (rng.standard_normal((8,) + med.shape[1:])).astype(np.float32)
    pr = _prop(p)
    pr.set_medium(med)
    Bm = pr.born_forward(sig, pert, spos, rpos)
    Btd = pr.born_adjoint(sig, dat, spos, rpos)
    lhs = sum(float(np.sum(a.astype(np.float64) * b)) for a, b in zip(Bm, dat))
    rhs = sum(float(np.sum(a.astype(np.float64) * b)) for a, b in zip(pert, Btd))
    assert abs(lhs - rhs) / abs(rhs) < 1e-5


@pytest.mark.parametrize("adjoint,sub", [(False, None), (True, None), (False, 3), (True, 3)])
def test_graph_loop_matches_eager_launches(adjoint, sub):
    """The nonlinear loop replayed as CUDA graphs (one captured coarse block, two for an odd
    internal sub) gives the same bits as launching every kernel from the host."""
    sv, p, med, src, rec, dtw = prepared(seed=6)
    if sub is not None:
        p = O.PropParams(p.nz, p.nx, p.ny, p.nts, sub, p.minPad, p.dz, p.dx, p.dy, p.dts)
    rng = np.random.default_rng(12)
    spos = [d.unique for d in src]
    rpos = [d.unique for d in rec]
    pr = _prop(p)
    pr.set_medium(med)
    out = []
    for graph in (True, False):
        pr.set_graph_loop(graph)
        if adjoint:
            out.append(pr.nl_adjoint(random_signals(rpos, p.nts, np.random.default_rng(3)), spos, rpos))
        else:
            out.append(pr.nl_forward(random_signals(spos, p.nts, np.random.default_rng(3)), spos, rpos))
    for a, b in zip(*out):
        np.testing.assert_array_equal(a, b)
    if sub is not None:
        ref = (O.nl_adjoint_reg(p, med, random_signals(rpos, p.nts, np.random.default_rng(3)), spos, rpos,
                                np.float32) if adjoint else
               O.nl_forward_reg(p, med, random_signals(spos, p.nts, np.random.default_rng(3)), spos, rpos,
                                np.float32))
        assert rel_l2(out[0], ref) < 1e-5
