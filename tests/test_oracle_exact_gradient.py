"""CPU: the FP64 torch restatement of the oracle's nonlinear forward (oracle/exact_gradient.py),
whose autograd gives the exact discrete gradient of the misfit, pinned to the C++ oracle and to
finite differences; and how the shipped Born-adjoint gradient (the reference's imaging on coarse
samples) compares with it.  Test infrastructure for an exact-adjoint gradient mode: no GPU."""
import dataclasses

import numpy as np
import pytest
import torch

from fwi_case import OracleFwi, survey
from oracle import oracle as O
from oracle.exact_gradient import TorchForward, interp_matrix, medium_planes_t, scale_signals_t


@pytest.fixture(scope="module")
def case():
    sv, true = survey(nts=20)
    orc = OracleFwi(sv)
    d_obs, _ = orc.data(true)
    tf = TorchForward(orc.p, orc.spos, orc.rpos)
    src0 = [torch.tensor(orc.src[O.COMP_GRID[k]].adjoint(orc.irr[k])) for k in range(9)]
    R = [interp_matrix(orc.rec[O.COMP_GRID[k]]) for k in range(9)]
    ep0 = torch.tensor(np.asarray(sv.elastic, np.float64))

    def misfit(ep, fixed_sources=None):
        pl = medium_planes_t(ep, orc.dtw)
        src = fixed_sources if fixed_sources is not None else \
            scale_signals_t(src0, orc.spos, pl, orc.d[1], orc.d[2], orc.d[0])
        d = tf.forward(pl, src)
        pred = torch.stack([R[k] @ d[k] for k in range(9)])
        return 0.5 * ((pred - torch.tensor(d_obs)) ** 2).sum()

    return dict(sv=sv, orc=orc, d_obs=d_obs, tf=tf, src0=src0, ep0=ep0, misfit=misfit)


def _rel(a, b):
    a = np.concatenate([np.asarray(x, np.float64).ravel() for x in a])
    b = np.concatenate([np.asarray(x, np.float64).ravel() for x in b])
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_restatement_equals_the_oracle_forward_and_misfit(case):
    orc, sv = case["orc"], case["sv"]
    med = O.medium_planes(np.asarray(sv.elastic, np.float64), orc.dtw, np.float64)
    src = orc.src_reg(med)
    got = case["tf"].forward(torch.tensor(np.stack(med)), [torch.tensor(s) for s in src])
    ref = O.nl_forward_reg(orc.p, med, src, orc.spos, orc.rpos, np.float64)
    assert _rel([g.numpy() for g in got], ref) < 1e-13
    with torch.no_grad():
        j = float(case["misfit"](case["ep0"]))
    assert abs(j - orc.misfit(sv.elastic, case["d_obs"])) <= 1e-12 * abs(j)


def test_autograd_gradient_equals_central_differences(case):
    ep = case["ep0"].clone().requires_grad_(True)
    case["misfit"](ep).backward()
    g = ep.grad.numpy()
    rng = np.random.default_rng(2)
    scale = case["ep0"].numpy().reshape(3, -1).std(axis=1)[:, None, None, None]
    for _ in range(2):
        dl = rng.standard_normal(g.shape) * scale
        dl[:, :8], dl[:, -8:], dl[:, :, :8], dl[:, :, -8:], dl[:, :, :, :8], dl[:, :, :, -8:] = 0, 0, 0, 0, 0, 0
        eps = 1e-6
        with torch.no_grad():
            fd = float(case["misfit"](case["ep0"] + eps * torch.tensor(dl))
                       - case["misfit"](case["ep0"] - eps * torch.tensor(dl))) / (2 * eps)
        an = float((g * dl).sum())
        print(f"central difference {fd:.10g}, exact gradient {an:.10g}")
        assert abs(fd - an) <= 1e-6 * abs(an)


def test_born_gradient_against_the_exact_one(case):
    """The shipped gradient is the reference's Born-adjoint imaging on coarse samples.  With the
    source signals held fixed (no derivative of their medium scaling) and the yz derivative pair
    corrected (q3compat=0) it agrees with the exact gradient to correlation 0.99 for every
    parameter; what is left is the coarse-sample imaging.  At the reference defaults the lambda
    gradient is dominated by the scaling of the explosive source by lambda at the source cells."""
    orc, sv = case["orc"], case["sv"]
    pl0 = medium_planes_t(case["ep0"], orc.dtw)
    fixed = [s.detach() for s in scale_signals_t(case["src0"], orc.spos, pl0, orc.d[1], orc.d[2], orc.d[0])]
    ep = case["ep0"].clone().requires_grad_(True)
    case["misfit"](ep, fixed).backward()
    g_fixed = ep.grad.numpy()
    ep = case["ep0"].clone().requires_grad_(True)
    case["misfit"](ep).backward()
    g_full = ep.grad.numpy()
    stats = {}
    for q3 in (1, 0):
        o = OracleFwi(sv)
        o.p = dataclasses.replace(o.p, q3compat=q3)
        _, gb = o.misfit_and_gradient(sv.elastic, case["d_obs"])
        gb = np.asarray(gb)
        for name, ge in (("fixed sources", g_fixed), ("with source term", g_full)):
            corr = [float(np.dot(gb[k].ravel(), ge[k].ravel()) / np.linalg.norm(gb[k]) / np.linalg.norm(ge[k]))
                    for k in range(3)]
            rel = [float(np.linalg.norm(gb[k] - ge[k]) / np.linalg.norm(ge[k])) for k in range(3)]
            stats[(q3, name)] = corr
            print(f"Born (q3compat={q3}) vs exact, {name}: rho/lambda/mu correlation "
                  f"{corr[0]:+.3f} {corr[1]:+.3f} {corr[2]:+.3f}, relative error {rel[0]:.3f} {rel[1]:.3f} {rel[2]:.3f}")
    assert min(stats[(0, "fixed sources")]) > 0.98
    assert stats[(1, "with source term")][1] < 0.5   # the source term dominates lambda


def test_adjoint_recursion_equals_autograd():
    """The hand-written adjoint recursion (per-fine-step imaging against the adjoint state, the
    oracle's exact-transpose stepper for the transpose) gives autograd's gradient to rounding."""
    from oracle.exact_gradient import exact_gradient_by_adjoint
    sv, _ = survey(nts=10)
    orc = OracleFwi(sv)
    med = O.medium_planes(np.asarray(sv.elastic, np.float64), orc.dtw, np.float64)
    src = orc.src_reg(med)
    tf = TorchForward(orc.p, orc.spos, orc.rpos)
    rng = np.random.default_rng(0)
    w = [rng.standard_normal((len(r), orc.p.nts)) for r in tf.rec]
    pl = torch.tensor(np.stack(med)).requires_grad_(True)
    d = tf.forward(pl, [torch.tensor(s) for s in src])
    sum((torch.tensor(a) * b).sum() for a, b in zip(w, d)).backward()
    g = exact_gradient_by_adjoint(orc.p, med, src, orc.spos, orc.rpos, w)
    e = float(np.linalg.norm(g - pl.grad.numpy()) / np.linalg.norm(pl.grad.numpy()))
    print(f"adjoint recursion vs autograd: {e:.2e}")
    assert e < 1e-12
