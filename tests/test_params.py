"""CPU: parametrisation and mask operators (elasticParamConvertModule_3D.py; efwiMain_3D.py masks)."""
import numpy as np
import torch

from elasticisolib_3d_b200 import params as P


def _model(seed=0, shape=(4, 5, 6)):
    rng = np.random.default_rng(seed)
    vp = 2500.0 + 500.0 * rng.random(shape)
    vs = vp / 1.8
    rho = 2000.0 + 300.0 * rng.random(shape)
    return np.stack([vp, vs, rho])


def test_conversion_round_trip_and_units():
    m = _model()
    out = np.zeros_like(m)
    P.ElasticConv_3D(m, 1).forward(False, m, out)
    back = np.zeros_like(m)
    P.ElasticConv_3D(m, -1).forward(False, out, back)
    np.testing.assert_allclose(back, m, rtol=1e-12)
    km = np.stack([m[0] / 1e3, m[1] / 1e3, m[2] / 1e3])
    out2 = np.zeros_like(m)
    P.ElasticConv_3D(m, 2).forward(False, km, out2)
    np.testing.assert_allclose(out2, out, rtol=1e-12)


def test_jacobian_matches_finite_differences_and_is_an_adjoint_pair():
    m = _model(1)
    rng = np.random.default_rng(2)
    dm = rng.standard_normal(m.shape) * np.array([10.0, 5.0, 3.0])[:, None, None, None]
    J = P.ElasticConvJab_3D(m, m, 1)
    jd = np.zeros_like(m)
    J.forward(False, dm, jd)
    f = P.ElasticConv_3D(m, 1)
    hi, lo = np.zeros_like(m), np.zeros_like(m)
    eps = 1e-4
    f.forward(False, m + eps * dm, hi)
    f.forward(False, m - eps * dm, lo)
    fd = (hi - lo) / (2 * eps)
    assert np.linalg.norm(jd - fd) / np.linalg.norm(fd) < 1e-8
    dd = rng.standard_normal(m.shape)
    jt = np.zeros_like(m)
    J.adjoint(False, jt, dd)
    assert abs(np.vdot(jd, dd) - np.vdot(dm, jt)) / abs(np.vdot(jd, dd)) < 1e-12


def test_torch_conversion_chains_gradients():
    m = torch.tensor(_model(3), requires_grad=True)
    rho, lam, mu = P.vpvsrho_to_rholammu(m[0], m[1], m[2])
    (rho.sum() + 1e-9 * lam.sum() + 1e-9 * mu.sum()).backward()
    vp, vs, r = m.detach()
    np.testing.assert_allclose(m.grad[0].numpy(), (1e-9 * 2 * vp * r).numpy(), rtol=1e-10)
    np.testing.assert_allclose(m.grad[2].numpy(), (1 + 1e-9 * (vp * vp - 2 * vs * vs) + 1e-9 * vs * vs).numpy(),
                               rtol=1e-10)


def test_diagonal_mask_is_self_adjoint():
    rng = np.random.default_rng(4)
    mask = (rng.random((3, 4, 5, 6)) > 0.3).astype(np.float64)
    M = P.DiagonalMask(mask)
    x, y = rng.standard_normal(mask.shape), rng.standard_normal(mask.shape)
    mx, my = np.zeros_like(x), np.zeros_like(y)
    M.forward(False, x, mx)
    M.adjoint(False, my, y)
    assert abs(np.vdot(mx, y) - np.vdot(x, my)) < 1e-9
