"""A homogeneous or smooth half-space whose first updated row is the free surface, for the
free-surface checks on the GPU and on the oracle."""
from __future__ import annotations

import numpy as np

from elasticisolib_3d_b200 import hostprep as H
from elasticisolib_3d_b200 import synthetic as S
from oracle import oracle as O

FAT = 4


def half_space(nzi, nxi, nyi, pad, d=10.0, nts=40, vp=2500.0, vs=2500.0 / np.sqrt(3.0), rho=2000.0,
               smooth=0.0, seed=0):
    """Grid whose first updated row is the free surface (no top pad), sponge elsewhere."""
    # nz-2*FAT and nx-2*FAT multiples of 16 (the reference's block rule, fdParamElastic_3D QC)
    zpp = pad + (-(nzi + pad)) % 16
    xpp = pad + (-(nxi + 2 * pad)) % 16
    nz = FAT + nzi + zpp + FAT
    nx = FAT + pad + nxi + xpp + FAT
    ny = FAT + pad + nyi + pad + FAT
    axes = (H.Axis(nz, -FAT * d, d), H.Axis(nx, -(FAT + pad) * d, d), H.Axis(ny, -(FAT + pad) * d, d))
    pads = dict(zPadMinus=0, zPadPlus=zpp, xPadMinus=pad, xPadPlus=xpp, yPad=pad)
    par = S.base_params(axes, pads, nts, 0.002, 2, 30.0, free_surface=True)
    shape = (ny, nx, nz)
    if smooth:
        vpf, vsf, rhof = S.gaussian_perturbed_model(shape, vp, vs, rho, smooth, 2.0, seed)
    else:
        vpf, vsf, rhof = (np.full(shape, v) for v in (vp, vs, rho))
    return S.elastic_from_velocity(vpf, vsf, rhof), axes, par


def prep(el, axes, par):
    fd = H.FdParam(el, axes, par)
    za, xa, ya = axes
    ax7 = H.grid_axes(za.n, xa.n, ya.n, za.o, xa.o, ya.o, za.d, xa.d, ya.d)
    return fd, ax7


def oracle_params(fd, free_surface):
    return O.PropParams(fd.nz, fd.nx, fd.ny, fd.nts, fd.sub, fd.minPad, float(fd.dz), float(fd.dx), float(fd.dy),
                        float(fd.dts), alphaCos=float(fd.alphaCos), free_surface=free_surface)


def moveout_velocity(vz, dx):
    a, b = vz[0] - vz[0].mean(), vz[1] - vz[1].mean()
    cc = np.correlate(b, a, mode="full")
    lag = int(np.argmax(cc)) - (len(a) - 1)
    # parabolic refinement of the peak
    i = int(np.argmax(cc))
    if 0 < i < len(cc) - 1:
        den = cc[i - 1] - 2 * cc[i] + cc[i + 1]
        if den != 0:
            lag += 0.5 * (cc[i - 1] - cc[i + 1]) / den
    return dx / (lag * 0.002)
