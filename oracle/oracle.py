"""Oracle for the elastic 3D propagation path (test infrastructure only).

This module is the checker: a CPU restatement of elasticIsoLib_3D's host-side
preparation (medium staggering/scaling, trilinear source/receiver mapping,
source/data scaling, component packing) in numpy, plus ctypes bindings to
``elastic_oracle.cpp`` for the time loops.  Only tests, the smoke check and
the CPU-baseline leg of the benchmark import it; the product never does.

Array conventions follow the reference's SEP vectors with the fastest axis
last in numpy: a 3D field is ``(ny, nx, nz)``, the elastic parameter cube is
``(3, ny, nx, nz)`` holding (rho, lambda, mu), a per-shot signal block is
``(9, nDevice, nts)`` in component order vx, vy, vz, sxx, syy, szz, sxz, sxy,
syz.  Citations are to ``elastic_iso_lib_3d/elastic_iso_float/``.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

FAT = 4
NCOMP = 9
GRIDS = ("center", "x", "y", "z", "xz", "xy", "yz")
# grid of each wavefield component (nonlinearPropElasticGpuFunctions_3D.cu:684-742)
COMP_GRID = (1, 2, 3, 0, 0, 0, 4, 5, 6)

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def lib():
    """Load (building if needed, when the sources are present) the oracle library."""
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle_elastic.so")
        if not os.path.exists(path):
            import subprocess
            subprocess.check_call(["make", "-s", "-C", _HERE])
        L = ctypes.CDLL(path)
        P = ctypes.c_void_p
        for suf in ("f32", "f64"):
            for name in ("nl_fwd", "nl_adj"):
                fn = getattr(L, f"oracle_{name}_{suf}")
                fn.argtypes = [P] * 8
                fn.restype = ctypes.c_int
            for name in ("born_fwd", "born_adj"):
                fn = getattr(L, f"oracle_{name}_{suf}")
                fn.argtypes = [P] * 9
                fn.restype = ctypes.c_int
            fn = getattr(L, f"oracle_step_{suf}")
            fn.argtypes = [P, P, P, P, ctypes.c_int, ctypes.c_int]
            fn.restype = ctypes.c_int
            fn = getattr(L, f"oracle_constants_{suf}")
            fn.argtypes = [P] * 5
            fn.restype = ctypes.c_int
        L.oracle_num_threads.argtypes = [ctypes.c_int]
        L.oracle_num_threads.restype = ctypes.c_int
        _LIB = L
    return _LIB


class OracleParams(ctypes.Structure):
    _fields_ = [("nz", ctypes.c_int), ("nx", ctypes.c_int), ("ny", ctypes.c_int),
                ("nts", ctypes.c_int), ("sub", ctypes.c_int), ("minPad", ctypes.c_int),
                ("dz", ctypes.c_double), ("dx", ctypes.c_double), ("dy", ctypes.c_double),
                ("dts", ctypes.c_double), ("alphaCos", ctypes.c_double),
                ("q2compat", ctypes.c_int), ("q3compat", ctypes.c_int), ("fix_q1", ctypes.c_int),
                ("free_surface", ctypes.c_int)]


# ----------------------------------------------------------------------------
# Staggering (stagger_3D.cpp:23-208).  axis: 0=z, 1=x, 2=y of a (ny,nx,nz) cube.
# ----------------------------------------------------------------------------
def _ax(axis):
    return {0: 2, 1: 1, 2: 0}[axis]


def stagger_adjoint(d, axis):
    """m[i] = 0.5(d[i]+d[i-1]); m[0] = 0.5 d[0]; m[n-1] = d[n-1] + 0.5 d[n-2]."""
    a = _ax(axis)
    d = np.moveaxis(np.asarray(d), a, -1)
    m = np.zeros_like(d)
    m[..., 1:-1] = d.dtype.type(0.5) * (d[..., 1:-1] + d[..., :-2])
    m[..., 0] = d.dtype.type(0.5) * d[..., 0]
    m[..., -1] = d[..., -1] + d.dtype.type(0.5) * d[..., -2]
    return np.moveaxis(m, -1, a)


def stagger_forward(m, axis):
    """d[i] = 0.5(m[i]+m[i+1]) for i < n-1; d[n-1] = m[n-1]."""
    a = _ax(axis)
    m = np.moveaxis(np.asarray(m), a, -1)
    d = np.zeros_like(m)
    d[..., :-1] = m.dtype.type(0.5) * (m[..., :-1] + m[..., 1:])
    d[..., -1] = m[..., -1]
    return np.moveaxis(d, -1, a)


# ----------------------------------------------------------------------------
# Medium preparation (fdParamElastic_3D.cpp:13-195)
# ----------------------------------------------------------------------------
def time_axes(nts, dts, sub_par):
    """Internal sub = 2*parfile sub; ntw = (nts-1)*sub+1; dtw = dts/sub in float32."""
    sub = 2 * int(sub_par)
    ntw = (nts - 1) * sub + 1
    dtw = np.float32(np.float32(dts) / np.float32(sub))
    return sub, ntw, dtw


def medium_planes(elastic_param, dtw, dtype=np.float32):
    """Eight scaled planes rhoxDtw, rhoyDtw, rhozDtw, lamb2MuDtw, lambDtw, muxzDtw, muxyDtw, muyzDtw.

    The products/quotients are evaluated in double and rounded once to the
    tree's type, as the reference does (fdParamElastic_3D.cpp:169-183).
    """
    ep = np.asarray(elastic_param, dtype=dtype)
    rho, lam, mu = ep[0], ep[1], ep[2]
    rhox = stagger_adjoint(rho, 1)
    rhoy = stagger_adjoint(rho, 2)
    rhoz = stagger_adjoint(rho, 0)
    muxz = stagger_adjoint(stagger_adjoint(mu, 1), 0)
    muxy = stagger_adjoint(stagger_adjoint(mu, 1), 2)
    muyz = stagger_adjoint(stagger_adjoint(mu, 2), 0)
    two_dtw = 2.0 * float(dtw)
    f64 = np.float64
    out = np.empty((8,) + rho.shape, dtype=dtype)
    with np.errstate(divide="ignore"):
        out[0] = (two_dtw / rhox.astype(f64)).astype(dtype)
        out[1] = (two_dtw / rhoy.astype(f64)).astype(dtype)
        out[2] = (two_dtw / rhoz.astype(f64)).astype(dtype)
    out[3] = (two_dtw * (lam.astype(f64) + 2.0 * mu.astype(f64))).astype(dtype)
    out[4] = (two_dtw * lam.astype(f64)).astype(dtype)
    out[5] = (two_dtw * muxz.astype(f64)).astype(dtype)
    out[6] = (two_dtw * muxy.astype(f64)).astype(dtype)
    out[7] = (two_dtw * muyz.astype(f64)).astype(dtype)
    return out


# ----------------------------------------------------------------------------
# Acquisition devices (spaceInterpGpu_3D.cpp:13-348)
# ----------------------------------------------------------------------------
@dataclass
class SpaceInterp:
    """Linear spatial interpolation of one device set onto one (staggered) grid."""
    index: np.ndarray        # (nIrreg, nFilter) int64 grid-point indices (not unique)
    weight: np.ndarray       # (nIrreg, nFilter) float32
    unique: np.ndarray       # (nReg,) int64 unique indices, first-seen order
    slot: np.ndarray         # (nIrreg, nFilter) position of each index in `unique`
    nt: int = 0

    @property
    def n_reg(self):
        return int(self.unique.shape[0])

    @property
    def n_irreg(self):
        return int(self.index.shape[0])

    def forward(self, reg, add=False, out=None):
        """Regular -> irregular: d[dev,t] += w * m[reg,t] (float32, device then filter order)."""
        reg = np.asarray(reg)
        if out is None or not add:
            out = np.zeros((self.n_irreg, reg.shape[1]), dtype=reg.dtype)
        for k in range(self.index.shape[1]):
            out += self.weight[:, k:k + 1].astype(reg.dtype) * reg[self.slot[:, k]]
        return out

    def adjoint(self, irreg, add=False, out=None):
        """Irregular -> regular: m[reg,t] += w * d[dev,t], accumulated in device/filter order."""
        irreg = np.asarray(irreg)
        if out is None or not add:
            out = np.zeros((self.n_reg, irreg.shape[1]), dtype=irreg.dtype)
        for d in range(self.n_irreg):
            for k in range(self.index.shape[1]):
                out[self.slot[d, k]] += self.weight[d, k].astype(irreg.dtype) * irreg[d]
        return out


@dataclass
class GridAxis:
    n: int
    o: float
    d: float


def _check_inside(z, x, y, axes, pads):
    """checkOutOfBounds (spaceInterpGpu_3D.cpp:178-212): devices inside the model interior,
    float arithmetic with the error tolerance."""
    f32 = np.float32
    za, xa, ya = axes
    oz, dz, ox, dx, oy, dy = (f32(za.o), f32(za.d), f32(xa.o), f32(xa.d), f32(ya.o), f32(ya.d))
    nz, nx, ny = za.n, xa.n, ya.n
    fat = pads["fat"]
    tol = f32(pads.get("errorTolerance", 1e-6))
    nzS = nz - 2 * fat - pads["zPadMinus"] - pads["zPadPlus"]
    nxS = nx - 2 * fat - pads["xPadMinus"] - pads["xPadPlus"]
    nyS = ny - 2 * fat - 2 * pads["yPad"]
    zMin = f32(oz + f32(fat + pads["zPadMinus"]) * dz)
    xMin = f32(ox + f32(fat + pads["xPadMinus"]) * dx)
    yMin = f32(oy + f32(fat + pads["yPad"]) * dy)
    zMax = f32(zMin + f32(nzS - 1) * dz)
    xMax = f32(xMin + f32(nxS - 1) * dx)
    yMax = f32(yMin + f32(nyS - 1) * dy)
    bad = ((z - zMax > tol) | (z - zMin < -tol) | (x - xMax > tol) | (x - xMin < -tol)
           | (y - yMax > tol) | (y - yMin < -tol))
    if np.any(bad):
        raise RuntimeError("spaceInterpGpu_3D: device out of bounds")


def _unique_slots(idx):
    """convertIrregToReg (spaceInterpGpu_3D.cpp:113-138): unique indices in first-seen order,
    keyed as the reference's std::map<int,int> is, by the index converted to int."""
    flat = idx.reshape(-1).astype(np.int32).astype(np.int64)
    seen = {}
    uniq = []
    slots = np.empty(flat.shape, dtype=np.int64)
    for i, v in enumerate(flat.tolist()):
        s = seen.get(v)
        if s is None:
            s = len(uniq)
            seen[v] = s
            uniq.append(v)
        slots[i] = s
    return np.asarray(uniq, dtype=np.int64), slots.reshape(idx.shape)


def space_interp_linear(z, x, y, axes, pads, nt, dipole=0, shifts=(0.0, 0.0, 0.0), compat=True):
    """calcLinearWeights + convertIrregToReg with the reference's float arithmetic.

    axes: (zAxis, xAxis, yAxis) GridAxis of the (possibly shifted) grid.
    pads: dict with fat, zPadMinus, zPadPlus, xPadMinus, xPadPlus, yPad.
    With compat the dipole shifts are truncated to int, as the reference class stores
    them, and the dipole y weight divides by dz (spaceInterpGpu_3D.h:25, .cpp:287);
    without, the shifts stay float and y divides by dy.
    """
    f32, f64 = np.float32, np.float64
    za, xa, ya = axes
    oz, dz, ox, dx, oy, dy = (f32(za.o), f32(za.d), f32(xa.o), f32(xa.d), f32(ya.o), f32(ya.d))
    nz, nx, ny = za.n, xa.n, ya.n
    z = np.asarray(z, dtype=f32); x = np.asarray(x, dtype=f32); y = np.asarray(y, dtype=f32)
    fat = pads["fat"]
    _check_inside(z, x, y, axes, pads)

    def corners(zc, xc, yc, sign):
        wz = (zc - oz) / dz
        wx = (xc - ox) / dx
        wy = (yc - oy) / (dz if sign < 0 and compat else dy)
        zr = wz.astype(np.int64); xr = wx.astype(np.int64); yr = wy.astype(np.int64)
        wz = f32(1.0) - (wz - zr.astype(f32))
        wx = f32(1.0) - (wx - xr.astype(f32))
        wy = f32(1.0) - (wy - yr.astype(f32))
        if (np.any(yr < fat + pads["yPad"]) or np.any(yr + 1 >= ny - fat - pads["yPad"]) or
                np.any(xr < fat + pads["xPadMinus"]) or np.any(xr + 1 >= nx - fat - pads["xPadPlus"]) or
                np.any(zr < fat + pads["zPadMinus"]) or np.any(zr + 1 >= nz - fat - pads["zPadPlus"])):
            raise RuntimeError("spaceInterpGpu_3D: interpolation stencil out of bounds")
        base = yr * nz * nx + xr * nz + zr
        idx = np.stack([base, base + 1, base + nz, base + nz + 1, base + nz * nx, base + nz * nx + 1,
                        base + nz * nx + nz, base + nz * nx + nz + 1], axis=1)
        Z, X, Y = wz.astype(f64), wx.astype(f64), wy.astype(f64)
        w = np.empty(idx.shape, dtype=f32)
        w[:, 0] = wz * wx * wy
        w[:, 1] = ((1.0 - Z) * X * Y).astype(f32)
        w[:, 2] = (Z * (1.0 - X) * Y).astype(f32)
        w[:, 3] = ((1.0 - Z) * (1.0 - X) * Y).astype(f32)
        w[:, 4] = ((wz * wx).astype(f64) * (1.0 - Y)).astype(f32)
        w[:, 5] = ((1.0 - Z) * X * (1.0 - Y)).astype(f32)
        w[:, 6] = (Z * (1.0 - X) * (1.0 - Y)).astype(f32)
        w[:, 7] = ((1.0 - Z) * (1.0 - X) * (1.0 - Y)).astype(f32)
        if sign < 0:
            w = np.stack([
                (-1.0 * Z * X * Y), (-1.0 * (1.0 - Z) * X * Y), (-1.0 * Z * (1.0 - X) * Y),
                (-1.0 * (1.0 - Z) * (1.0 - X) * Y), (-1.0 * Z * X * (1.0 - Y)),
                (-1.0 * (1.0 - Z) * X * (1.0 - Y)), (-1.0 * Z * (1.0 - X) * (1.0 - Y)),
                (-1.0 * (1.0 - Z) * (1.0 - X) * (1.0 - Y))], axis=1).astype(f32)
        return idx, w

    idx, w = corners(z, x, y, +1)
    if dipole:
        sz, sx, sy = (f32(int(s)) if compat else f32(s) for s in shifts)
        idx2, w2 = corners(z + sz, x + sx, y + sy, -1)
        idx = np.concatenate([idx, idx2], axis=1)
        w = np.concatenate([w, w2], axis=1)
    uniq, slots = _unique_slots(idx)
    return SpaceInterp(index=idx, weight=w, unique=uniq, slot=slots, nt=nt)


def _sinc_of_arg(a):
    """sin(a)/a in float64 with its limit 1 at 0: the Taylor series 1 - a^2/6 + a^4/120 below
    |a| = 1.2e-4 (the published small-argument form of boost::math::sinc_pi, the function the
    reference calls, spaceInterpGpu_3D.cpp:409)."""
    a = np.asarray(a, dtype=np.float64)
    small = np.abs(a) < 1.2e-4
    a2 = a * a
    safe = np.where(small, 1.0, a)
    return np.where(small, 1.0 - a2 / 6.0 + a2 * a2 / 120.0, np.sin(safe) / safe)


def space_interp_sinc(z, x, y, axes, pads, nt, h, dipole=0, shifts=(0.0, 0.0, 0.0), compat=True):
    """calcSincWeights + convertIrregToReg (spaceInterpGpu_3D.cpp:351-480).

    Per device, the 2h points r-h+1 .. r+h on each axis around the cell corner r below it,
    y then x then z (z fastest), with weight sinc(pi wz) sinc(pi wx) sinc(pi wy) in float64
    stored as float32, w = (device - point) / d in float32.  The reference's bounds test is
    inverted (it rejects every in-bounds stencil, so its sinc path never returns and no output
    of it exists: parity unpinned); here the stencil must lie inside the array.  Dipole: the
    second pole at the shifted position, shifts truncated to int with compat (as the reference
    class stores them) and with positive weights, as the reference's code has it; without
    compat, float shifts and negative weights, as the linear dipole.
    """
    f32, f64 = np.float32, np.float64
    za, xa, ya = axes
    oz, dz, ox, dx, oy, dy = (f32(za.o), f32(za.d), f32(xa.o), f32(xa.d), f32(ya.o), f32(ya.d))
    nz, nx, ny = za.n, xa.n, ya.n
    z = np.asarray(z, dtype=f32); x = np.asarray(x, dtype=f32); y = np.asarray(y, dtype=f32)
    _check_inside(z, x, y, axes, pads)
    offs = np.arange(2 * h, dtype=np.int64) - h + 1

    def pole(zc, xc, yc):
        rz = ((zc - oz) / dz).astype(np.int64)
        rx = ((xc - ox) / dx).astype(np.int64)
        ry = ((yc - oy) / dy).astype(np.int64)
        for r, n in ((ry, ny), (rx, nx), (rz, nz)):
            if np.any(r - h + 1 < 0) or np.any(r + h >= n):
                raise RuntimeError("spaceInterpGpu_3D: sinc stencil outside the grid")
        pz, px, py = rz[:, None] + offs, rx[:, None] + offs, ry[:, None] + offs   # (n, 2h)
        wz = (zc[:, None] - (pz.astype(f32) * dz + oz)) / dz
        wx = (xc[:, None] - (px.astype(f32) * dx + ox)) / dx
        wy = (yc[:, None] - (py.astype(f32) * dy + oy)) / dy
        sz = _sinc_of_arg(np.pi * wz.astype(f64))
        sx = _sinc_of_arg(np.pi * wx.astype(f64))
        sy = _sinc_of_arg(np.pi * wy.astype(f64))
        w = (sz[:, None, None, :] * sx[:, None, :, None]) * sy[:, :, None, None]
        idx = (nz * nx * py[:, :, None, None] + nz * px[:, None, :, None] + pz[:, None, None, :])
        n = zc.shape[0]
        return idx.reshape(n, -1), w.astype(f32).reshape(n, -1)

    idx, w = pole(z, x, y)
    if dipole:
        sz, sx, sy = (f32(int(s)) if compat else f32(s) for s in shifts)
        idx2, w2 = pole(z + sz, x + sx, y + sy)
        if not compat:
            w2 = -w2
        idx = np.concatenate([idx, idx2], axis=1)
        w = np.concatenate([w, w2], axis=1)
    uniq, slots = _unique_slots(idx)
    return SpaceInterp(index=idx, weight=w, unique=uniq, slot=slots, nt=nt)


def staggered_axes(nz, nx, ny, oz, ox, oy, dz, dx, dy):
    """Seven grid hypercubes (Elastic_iso_float_3D.py:97-110): staggered origins at o - 0.5 d."""
    Z, X, Y = GridAxis(nz, oz, dz), GridAxis(nx, ox, dx), GridAxis(ny, oy, dy)
    Zs, Xs, Ys = GridAxis(nz, oz - 0.5 * dz, dz), GridAxis(nx, ox - 0.5 * dx, dx), GridAxis(ny, oy - 0.5 * dy, dy)
    return {"center": (Z, X, Y), "x": (Z, Xs, Y), "y": (Z, X, Ys), "z": (Zs, X, Y),
            "xz": (Zs, Xs, Y), "xy": (Z, Xs, Ys), "yz": (Zs, X, Ys)}


def build_devices(z, x, y, grid_axes, pads, nt, dipole=0, shifts=(0.0, 0.0, 0.0)):
    return [space_interp_linear(z, x, y, grid_axes[g], pads, nt, dipole, shifts) for g in GRIDS]


# ----------------------------------------------------------------------------
# Signal scaling (nonlinearPropElasticGpu_3D.cpp:200-277, :483-560,
# seismicElasticOperator3D.cpp:147-225)
# ----------------------------------------------------------------------------
def scale_signals(reg, devices, med, dx, dy, dz):
    """Scale 9 regular-grid signal blocks by the medium at their points, in place."""
    flat = [m.reshape(-1) for m in med]
    dt = reg[0].dtype.type
    # forces
    reg[0] *= flat[0][devices[1].unique][:, None]
    reg[1] *= flat[1][devices[2].unique][:, None]
    reg[2] *= flat[2][devices[3].unique][:, None]
    # normal moments / stresses on the center grid
    u = devices[0].unique
    l2m = flat[3][u][:, None]
    lam = flat[4][u][:, None]
    sxx, syy, szz = reg[3].copy(), reg[4].copy(), reg[5].copy()
    reg[3][:] = sxx * l2m + (syy + szz) * lam
    reg[4][:] = syy * l2m + (sxx + szz) * lam
    reg[5][:] = szz * l2m + (sxx + syy) * lam
    reg[6] *= flat[5][devices[4].unique][:, None]
    reg[7] *= flat[6][devices[5].unique][:, None]
    reg[8] *= flat[7][devices[6].unique][:, None]
    area = dt(1.0 / float(np.float32(np.float32(dx) * np.float32(dy)) * np.float32(dz)))
    for k in range(NCOMP):
        reg[k] *= area


# ----------------------------------------------------------------------------
# ctypes glue to the C++ time loops
# ----------------------------------------------------------------------------
def _ptrs(arrs):
    arrs = [np.ascontiguousarray(a) for a in arrs]
    keep = list(arrs)
    P = (ctypes.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
    return P, keep


def _geom(devs_or_pos):
    pos = [np.ascontiguousarray(np.asarray(p, dtype=np.int64)) for p in devs_or_pos]
    P = (ctypes.c_void_p * 7)(*[p.ctypes.data for p in pos])
    N = (ctypes.c_longlong * 7)(*[int(p.shape[0]) for p in pos])
    return P, N, pos


@dataclass
class PropParams:
    nz: int
    nx: int
    ny: int
    nts: int
    sub: int          # internal (2x parfile) value
    minPad: int
    dz: float
    dx: float
    dy: float
    dts: float
    alphaCos: float = 0.99
    q2compat: int = 1
    q3compat: int = 1
    fix_q1: int = 0
    free_surface: int = 0

    def c(self):
        return OracleParams(self.nz, self.nx, self.ny, self.nts, self.sub, self.minPad, self.dz, self.dx,
                            self.dy, self.dts, self.alphaCos, self.q2compat, self.q3compat, self.fix_q1,
                            self.free_surface)


def _suffix(dtype):
    return "f64" if np.dtype(dtype) == np.float64 else "f32"


def nl_forward_reg(p: PropParams, med, model_reg, src_pos, rec_pos, dtype=np.float32):
    """Regular-grid nonlinear forward: model_reg[9] (nReg,nts) -> data_reg[9] (nReg,nts)."""
    L = lib()
    med = [np.asarray(m, dtype=dtype) for m in med]
    model_reg = [np.asarray(m, dtype=dtype) for m in model_reg]
    data = [np.zeros((len(rec_pos[COMP_GRID[k]]), p.nts), dtype=dtype) for k in range(NCOMP)]
    mp, k1 = _ptrs(med); sp, k2 = _ptrs(model_reg); dp, k3 = _ptrs(data)
    SP, SN, k4 = _geom(src_pos); RP, RN, k5 = _geom(rec_pos)
    prm = p.c()
    getattr(L, "oracle_nl_fwd_" + _suffix(dtype))(ctypes.byref(prm), mp, sp, dp, SP, SN, RP, RN)
    return data


def nl_adjoint_reg(p: PropParams, med, data_reg, src_pos, rec_pos, dtype=np.float32):
    L = lib()
    med = [np.asarray(m, dtype=dtype) for m in med]
    data_reg = [np.asarray(d, dtype=dtype) for d in data_reg]
    model = [np.zeros((len(src_pos[COMP_GRID[k]]), p.nts), dtype=dtype) for k in range(NCOMP)]
    mp, k1 = _ptrs(med); sp, k2 = _ptrs(model); dp, k3 = _ptrs(data_reg)
    SP, SN, k4 = _geom(src_pos); RP, RN, k5 = _geom(rec_pos)
    prm = p.c()
    getattr(L, "oracle_nl_adj_" + _suffix(dtype))(ctypes.byref(prm), mp, sp, dp, SP, SN, RP, RN)
    return model


def born_forward_reg(p: PropParams, med, src_reg, pert8, src_pos, rec_pos, dtype=np.float32):
    L = lib()
    med = [np.asarray(m, dtype=dtype) for m in med]
    src_reg = [np.asarray(s, dtype=dtype) for s in src_reg]
    pert8 = [np.asarray(x, dtype=dtype) for x in pert8]
    data = [np.zeros((len(rec_pos[COMP_GRID[k]]), p.nts), dtype=dtype) for k in range(NCOMP)]
    mp, k1 = _ptrs(med); sp, k2 = _ptrs(src_reg); dp, k3 = _ptrs(data); pp, k6 = _ptrs(pert8)
    SP, SN, k4 = _geom(src_pos); RP, RN, k5 = _geom(rec_pos)
    prm = p.c()
    getattr(L, "oracle_born_fwd_" + _suffix(dtype))(ctypes.byref(prm), mp, sp, dp, SP, SN, RP, RN, pp)
    return data


def born_adjoint_reg(p: PropParams, med, src_reg, data_reg, src_pos, rec_pos, pert8_init=None,
                     dtype=np.float32):
    L = lib()
    med = [np.asarray(m, dtype=dtype) for m in med]
    src_reg = [np.asarray(s, dtype=dtype) for s in src_reg]
    data_reg = [np.asarray(d, dtype=dtype) for d in data_reg]
    shape = med[0].shape
    pert8 = [np.zeros(shape, dtype=dtype) if pert8_init is None else np.array(pert8_init[k], dtype=dtype)
             for k in range(8)]
    mp, k1 = _ptrs(med); sp, k2 = _ptrs(src_reg); dp, k3 = _ptrs(data_reg); pp, k6 = _ptrs(pert8)
    SP, SN, k4 = _geom(src_pos); RP, RN, k5 = _geom(rec_pos)
    prm = p.c()
    getattr(L, "oracle_born_adj_" + _suffix(dtype))(ctypes.byref(prm), mp, sp, dp, SP, SN, RP, RN, pp)
    return pert8


def step_once(p: PropParams, p0, p1, med, mode, damp, dtype=np.float32):
    """One stepper application (mode 0 fwd, 1 time-reversed, 2 exact transpose) on copies."""
    L = lib()
    p0 = [np.array(a, dtype=dtype) for a in p0]
    p1 = [np.array(a, dtype=dtype) for a in p1]
    med = [np.asarray(m, dtype=dtype) for m in med]
    a, k1 = _ptrs(p0); b, k2 = _ptrs(p1); m, k3 = _ptrs(med)
    prm = p.c()
    getattr(L, "oracle_step_" + _suffix(dtype))(ctypes.byref(prm), a, b, m, int(mode), int(damp))
    return p0, p1


def constants(p: PropParams, dtype=np.float32):
    L = lib()
    coef = np.zeros(12, dtype=dtype)
    filt = np.zeros(2 * (p.sub + 1), dtype=dtype)
    taper = np.zeros(max(p.minPad, 1), dtype=dtype)
    dinv = np.zeros(1, dtype=dtype)
    prm = p.c()
    getattr(L, "oracle_constants_" + _suffix(dtype))(ctypes.byref(prm), coef.ctypes.data, filt.ctypes.data,
                                                      taper.ctypes.data, dinv.ctypes.data)
    return coef, filt, taper, float(dinv[0])


# ----------------------------------------------------------------------------
# Born model preparation / gradient post-processing (BornElasticShotsGpu_3D.cpp:167-235, :528-605)
# ----------------------------------------------------------------------------
def born_model_to_planes(model3, med_scaling, dtw, dtype=np.float32):
    """(drho, dlame, dmu) -> 8 staggered, scaled perturbation planes."""
    f64 = np.float64
    drho, dlam, dmu = (np.asarray(model3[k], dtype=dtype) for k in range(3))
    planes = np.empty((8,) + drho.shape, dtype=dtype)
    planes[0] = stagger_adjoint(drho, 1)
    planes[1] = stagger_adjoint(drho, 2)
    planes[2] = stagger_adjoint(drho, 0)
    planes[3] = dlam
    planes[4] = dmu
    planes[5] = stagger_adjoint(stagger_adjoint(dmu, 1), 0)
    planes[6] = stagger_adjoint(stagger_adjoint(dmu, 1), 2)
    planes[7] = stagger_adjoint(stagger_adjoint(dmu, 2), 0)
    two_dtw = 2.0 * float(dtw)
    for k in range(3):
        planes[k] = planes[k] * med_scaling[k]
    for k in range(3, 8):
        planes[k] = (planes[k].astype(f64) * two_dtw).astype(dtype)
    return planes


def born_planes_to_model(planes, med_scaling, dtw, model_init=None, dtype=np.float32):
    """Adjoint of born_model_to_planes, accumulated onto model_init."""
    f64 = np.float64
    two_dtw = 2.0 * float(dtw)
    pl = np.array(planes, dtype=dtype)
    for k in range(3):
        pl[k] = pl[k] * med_scaling[k]
    for k in range(3, 8):
        pl[k] = (pl[k].astype(f64) * two_dtw).astype(dtype)
    out = np.zeros((3,) + pl.shape[1:], dtype=dtype) if model_init is None else np.array(model_init, dtype=dtype)
    out[0] = out[0] + stagger_forward(pl[0], 1)
    out[0] = out[0] + stagger_forward(pl[1], 2)
    out[0] = out[0] + stagger_forward(pl[2], 0)
    t2 = stagger_forward(stagger_forward(pl[5], 0), 1)
    t2 = t2 + stagger_forward(stagger_forward(pl[6], 2), 1)
    t2 = t2 + stagger_forward(stagger_forward(pl[7], 0), 2)
    out[1] = out[1] + pl[3]
    out[2] = out[2] + (pl[4] + t2)
    return out
