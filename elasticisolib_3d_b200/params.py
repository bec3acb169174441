"""Elastic parametrisation and masking operators (seis_utils/python/elasticParamConvertModule_3D.py,
and the diagonal masks of python_float/efwiMain_3D.py:158-233).

Arrays are (3, ny, nx, nz) stacks, numpy or torch (only elementwise arithmetic is used, so torch
tensors keep their autograd graph: FWI in (vp, vs, rho) is `ElasticFwiMisfit` applied to
`vpvsrho_to_rholammu(vp, vs, rho)`).

conv_type (as in the reference):
   1 : (vp, vs, rho) -> (rho, lambda, mu), SI units in and out
   2 : (vp, vs, rho) in km/s, km/s, g/cm^3 -> (rho, lambda, mu) in kg/m^3, Pa, Pa
  -1 : (rho, lambda, mu) -> (vp, vs, rho)
"""
from __future__ import annotations

import numpy as np


def _nd(v):
    return v.getNdArray() if hasattr(v, "getNdArray") else v


def _sqrt(x):
    return x.sqrt() if hasattr(x, "sqrt") and not isinstance(x, np.ndarray) else np.sqrt(x)


def vpvsrho_to_rholammu(vp, vs, rho, scale_km=False):
    """(rho, lambda, mu) = (rho, rho*(vp^2 - 2 vs^2), rho*vs^2); scale_km: inputs in km/s, g/cm^3."""
    if scale_km:
        return rho * 1e3, rho * (vp * vp - 2.0 * vs * vs) * 1e9, rho * vs * vs * 1e9
    return rho, rho * (vp * vp - 2.0 * vs * vs), rho * vs * vs


def rholammu_to_vpvsrho(rho, lam, mu):
    """(vp, vs, rho) = (sqrt((lambda + 2 mu)/rho), sqrt(mu/rho), rho)."""
    return _sqrt((lam + 2.0 * mu) / rho), _sqrt(mu / rho), rho


class ElasticConv_3D:
    """Nonlinear parameter conversion (forward only, like the reference)."""

    def __init__(self, domain, conv_type):
        if conv_type not in (1, 2, -1):
            raise ValueError(f"unsupported conv_type {conv_type}")
        self.conv_type = conv_type
        self.shape = tuple(np.shape(_nd(domain)))

    def forward(self, add, model, data):
        m, d = _nd(model), _nd(data)
        if not add:
            d[...] = 0
        if self.conv_type == -1:
            out = rholammu_to_vpvsrho(m[0], m[1], m[2])
        else:
            out = vpvsrho_to_rholammu(m[0], m[1], m[2], scale_km=self.conv_type == 2)
        for k in range(3):
            d[k] += out[k]


class ElasticConvJab_3D:
    """Jacobian of the (vp, vs, rho) -> (rho, lambda, mu) conversion at a background model:
       d rho    = d rho
       d lambda = (vp^2 - 2 vs^2) d rho - 4 vs rho d vs + 2 vp rho d vp
       d mu     = vs^2 d rho + 2 vs rho d vs
    The reference constructor keeps a clone of the domain instead of the background it is given
    (elasticParamConvertModule_3D.py:57-70) until setBackground is called; here the given
    background is used from the start.  conv_type 2 multiplies the background by 1e3
    (elasticParamConvertModule_3D.py:110-116)."""

    def __init__(self, domain, background, conv_type):
        if conv_type not in (1, 2):
            raise ValueError(f"unsupported conv_type {conv_type}")
        self.conv_type = conv_type
        self.shape = tuple(np.shape(_nd(domain)))
        self.setBackground(background)

    def setBackground(self, background):
        b = _nd(background)
        self.background = b * 1e3 if self.conv_type == 2 else b.copy() if hasattr(b, "copy") else b.clone()

    def forward(self, add, model, data):
        m, d, b = _nd(model), _nd(data), self.background
        if not add:
            d[...] = 0
        vp, vs, rho = b[0], b[1], b[2]
        d[0] += m[2]
        d[1] += (vp * vp - 2.0 * vs * vs) * m[2] - 4.0 * vs * rho * m[1] + 2.0 * vp * rho * m[0]
        d[2] += vs * vs * m[2] + 2.0 * vs * rho * m[1]

    def adjoint(self, add, model, data):
        m, d, b = _nd(model), _nd(data), self.background
        if not add:
            m[...] = 0
        vp, vs, rho = b[0], b[1], b[2]
        m[0] += 2.0 * vp * rho * d[1]
        m[1] += 2.0 * vs * rho * d[2] - 4.0 * vs * rho * d[1]
        m[2] += d[0] + (vp * vp - 2.0 * vs * vs) * d[1] + vs * vs * d[2]


class DiagonalMask:
    """Elementwise mask (pySolver DiagonalOp as efwiMain_3D.py uses it for gradient and data
    masks): forward = adjoint = multiplication by the mask."""

    def __init__(self, mask):
        self.mask = _nd(mask)

    def forward(self, add, model, data):
        m, d = _nd(model), _nd(data)
        if not add:
            d[...] = 0
        d += self.mask * m

    def adjoint(self, add, model, data):
        m, d = _nd(model), _nd(data)
        if not add:
            m[...] = 0
        m += self.mask * d
