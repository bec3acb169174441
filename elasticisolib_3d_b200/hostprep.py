"""Host preparation mirroring the reference's C++ host classes.

* ``FdParam``          fdParamElastic_3D (fdParamElastic_3D.cpp:13-327): time axes, QC, medium planes
* ``stagger``          staggerX/Y/Z forward and adjoint (stagger_3D.cpp)
* ``spaceInterpGpu_3D`` trilinear acquisition mapping (spaceInterpGpu_3D.cpp)

The arithmetic-heavy parts run in the native library (host_prep.cpp) so that
indices and weights are bit-identical to the reference's float arithmetic.
Arrays use numpy order with the fastest axis last: a field is (ny, nx, nz).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _native as N

FAT = 4
SUB_MAX = 100


def _as_int(v):
    """int of a parameter value; a decimal string such as "7.5" truncates, as a float does."""
    if isinstance(v, str):
        try:
            return int(v)
        except ValueError:
            return int(float(v))
    return int(v)


class ParamObj(dict):
    """Minimal stand-in for SEP's paramObj: getInt/getFloat/getString with defaults.

    Accepts the reference's parameter keys (nts, dts, sub, nz, nx, ny, zPadMinus,
    zPadPlus, xPadMinus, xPadPlus, yPad, dz, dx, dy, fMax, blockSize, fat,
    alphaCos, freeSurface, mod_par, nExp, ...).
    """

    _missing = object()

    def _get(self, key, default, conv):
        if key in self:
            return conv(self[key])
        if default is ParamObj._missing:
            raise KeyError(f"parameter '{key}' is required")
        return default

    def getInt(self, key, default=_missing):
        return self._get(key, default, _as_int)

    def getFloat(self, key, default=_missing):
        return self._get(key, default, float)

    def getString(self, key, default=_missing):
        return self._get(key, default, str)

    @classmethod
    def from_parfile(cls, text):
        """Parse 'key=value' tokens (SEP parfile / command-line style)."""
        out = cls()
        for tok in text.replace("\n", " ").split():
            if "=" in tok and not tok.startswith("#"):
                k, v = tok.split("=", 1)
                out[k.strip()] = v.strip()
        return out


def stagger(field, axis, adjoint=False, out=None, add=False):
    """staggerX/Y/Z.  axis: 'z', 'x' or 'y'; field (ny, nx, nz) float32."""
    a = np.ascontiguousarray(field, dtype=np.float32)
    ny, nx, nz = a.shape
    if out is None:
        out = np.zeros_like(a)
        add = False
    ax = {"z": 0, "x": 1, "y": 2}[axis]
    N.call("e3d_stagger", nz, nx, ny, ax, int(adjoint), int(add), a.ctypes.data, out.ctypes.data)
    return out


def medium_planes(elastic_param, dtw):
    """Eight scaled planes from (rho, lambda, mu) (3, ny, nx, nz) float32."""
    ep = np.ascontiguousarray(elastic_param, dtype=np.float32)
    _, ny, nx, nz = ep.shape
    out = np.empty((8, ny, nx, nz), dtype=np.float32)
    N.call("e3d_medium_planes", nz, nx, ny, float(np.float32(dtw)), ep.ctypes.data,
           N.ptr_array([out[k] for k in range(8)]))
    return out


@dataclass
class Axis:
    n: int
    o: float
    d: float


class FdParam:
    """fdParamElastic_3D: parameters, QC and the eight scaled medium planes.

    elastic_param: (3, ny, nx, nz) [rho, lambda, mu] in SI units; axes:
    (zAxis, xAxis, yAxis).  mod_par=2 (the C++ default) multiplies the
    spatial samplings and origins by 1000 as a km->m conversion
    (fdParamElastic_3D.cpp:71-79); pass mod_par explicitly.
    """

    def __init__(self, elastic_param, axes, par: ParamObj):
        self.par = par
        self.elastic_param = np.ascontiguousarray(elastic_param, dtype=np.float32)
        self.freeSurface = par.getInt("freeSurface", 0)
        self.nts = par.getInt("nts")
        self.dts = np.float32(par.getFloat("dts", 0.0))
        self.ots = par.getFloat("ots", 0.0)
        self.sub = 2 * par.getInt("sub")
        if self.sub > SUB_MAX:
            raise RuntimeError(f"2*sub={self.sub} exceeds SUB_MAX={SUB_MAX}")
        self.ntw = (self.nts - 1) * self.sub + 1
        self.dtw = np.float32(self.dts / np.float32(self.sub))
        self.nz, self.nx, self.ny = par.getInt("nz"), par.getInt("nx"), par.getInt("ny")
        self.zPadPlus, self.zPadMinus = par.getInt("zPadPlus"), par.getInt("zPadMinus")
        self.zPad = min(self.zPadMinus, self.zPadPlus) if self.freeSurface == 0 else self.zPadPlus
        self.xPadPlus, self.xPadMinus = par.getInt("xPadPlus"), par.getInt("xPadMinus")
        self.xPad = min(self.xPadMinus, self.xPadPlus)
        self.yPad = par.getInt("yPad")
        self.mod_par = par.getInt("mod_par", 2)
        za, xa, ya = axes
        self.dz, self.dx, self.dy = (np.float32(par.getFloat(k, -1.0)) for k in ("dz", "dx", "dy"))
        self.oz, self.ox, self.oy = np.float32(za.o), np.float32(xa.o), np.float32(ya.o)
        if self.mod_par == 2:
            self.dz, self.dx, self.dy = (np.float32(v * 1000.0) for v in (self.dz, self.dx, self.dy))
            self.oz, self.ox, self.oy = (np.float32(v * 1000.0) for v in (self.oz, self.ox, self.oy))
        self.fMax = par.getFloat("fMax", 1000.0)
        self.blockSize = par.getInt("blockSize", 16)
        self.fat = par.getInt("fat", 4)
        self.minPad = min(self.zPad, self.xPad)
        self.alphaCos = np.float32(par.getFloat("alphaCos", 0.99))
        self.errorTolerance = np.float32(par.getFloat("errorTolerance", 0.000001))
        self._qc(axes)
        self.planes = medium_planes(self.elastic_param, self.dtw)

    def _qc(self, axes):
        ep = self.elastic_param
        if ep.shape != (3, self.ny, self.nx, self.nz):
            raise RuntimeError("elastic parameter cube not consistent with nz/nx/ny")
        for ax, n, d in ((axes[0], self.nz, self.dz), (axes[1], self.nx, self.dx), (axes[2], self.ny, self.dy)):
            if ax.n != n or abs(np.float32(ax.d) - d) > self.errorTolerance and self.mod_par != 2:
                raise RuntimeError("axis not consistent with parameters")
        # velocity bounds over the same (odd) window the reference scans (fdParamElastic_3D.cpp:96-114)
        f = self.fat
        sl = (slice(f, self.ny - 2 * f), slice(f, self.nx - 2 * f), slice(f, self.nz - 2 * f))
        rho, lam, mu = ep[0][sl], ep[1][sl], ep[2][sl]
        vp = np.sqrt((lam + 2 * mu) / rho)
        vs = np.sqrt(mu / rho)
        vsn = vs[vs != 0]
        self.minVpVs = float(min(vp.min(), vsn.min() if vsn.size else np.inf, 10000.0))
        self.maxVpVs = float(max(vp.max(), vs.max(), -1.0))
        # stability (fdParamElastic_3D.cpp:288-299)
        self.Courant = self.maxVpVs * float(self.dtw) * 2.0 / float(min(self.dz, self.dx, self.dy))
        if self.Courant > 0.45:
            raise RuntimeError(f"Courant is too big: {self.Courant}")
        # dispersion (fdParamElastic_3D.cpp:301-313)
        self.dispersionRatio = self.minVpVs / (self.fMax * float(max(self.dz, self.dx, self.dy)))
        if self.dispersionRatio < 3.0:
            raise RuntimeError(f"Dispersion is too small: {self.dispersionRatio}")
        if (self.nz - 2 * self.fat) % self.blockSize or (self.nx - 2 * self.fat) % self.blockSize:
            raise RuntimeError("nz-2*FAT and nx-2*FAT must be multiples of blockSize")

    @property
    def rhoxDtw(self):
        return self.planes[0]

    def scaling(self):
        """The three density scalings (rhox/rhoy/rhozDtw) used by the Born operator."""
        return self.planes[0:3]


class spaceInterpGpu_3D:
    """Acquisition devices mapped onto one (possibly staggered) grid.

    Same constructor meaning as the reference (spaceInterpGpu_3D.cpp:13-79):
    coordinates, grid axes, nt, parameters, dipole flag and shifts, method
    ("linear" or "sinc") and half filter length (1 for linear).  The reference's
    sinc path rejects every in-bounds stencil (its bounds test is inverted); here
    that test is written the right way round.  `compat` (not a reference
    argument): True keeps the reference's dipole arithmetic (shifts truncated to
    int, the linear second pole's y offset divided by dz, the sinc second pole
    with positive weights); False corrects it.
    """

    def __init__(self, zCoord, xCoord, yCoord, axes, nt, par: ParamObj, dipole=0, zDipoleShift=0.0,
                 xDipoleShift=0.0, yDipoleShift=0.0, interpMethod="linear", hFilter1d=1, compat=True):
        methods = {"linear": 0, "sinc": 1}
        if interpMethod not in methods:
            raise NotImplementedError(f"spatial interpolation method {interpMethod!r} is not supported")
        if interpMethod == "linear" and hFilter1d != 1:
            raise RuntimeError("linear interpolation requires hFilter1d = 1")
        z = N.as_f32(zCoord).reshape(-1)
        x = N.as_f32(xCoord).reshape(-1)
        y = N.as_f32(yCoord).reshape(-1)
        self.nt = int(nt)
        self.method = interpMethod
        za, xa, ya = axes
        self.shape = (ya.n, xa.n, za.n)
        pads6 = (N.ctypes.c_int * 6)(par.getInt("fat"), par.getInt("zPadMinus"), par.getInt("zPadPlus"),
                                     par.getInt("xPadMinus"), par.getInt("xPadPlus"), par.getInt("yPad"))
        nf = (2 * int(hFilter1d)) ** 3 * (2 if dipole else 1)
        n = z.shape[0]
        self.index = np.empty((n, nf), dtype=np.int64)
        self.weight = np.empty((n, nf), dtype=np.float32)
        uniq = np.empty(max(n * nf, 1), dtype=np.int64)
        self.slot = np.empty((n, nf), dtype=np.int64)
        nu = N.ctypes.c_longlong(0)
        N.call("e3d_space_interp", methods[interpMethod], int(hFilter1d), z.ctypes.data, x.ctypes.data,
               y.ctypes.data, n, za.n, xa.n, ya.n, float(np.float32(za.o)), float(np.float32(xa.o)),
               float(np.float32(ya.o)), float(np.float32(za.d)), float(np.float32(xa.d)), float(np.float32(ya.d)),
               pads6, float(np.float32(par.getFloat("errorTolerance", 1e-6))), int(dipole), float(zDipoleShift),
               float(xDipoleShift), float(yDipoleShift), int(bool(compat)), self.index.ctypes.data,
               self.weight.ctypes.data, uniq.ctypes.data, self.slot.ctypes.data, N.ctypes.byref(nu))
        self.unique = uniq[:nu.value].copy()

    # accessors named after the reference's (spaceInterpGpu_3D.h:54-66)
    def getRegPosUnique(self):
        return self.unique

    def getNDeviceReg(self):
        return int(self.unique.shape[0])

    def getNDeviceIrreg(self):
        return int(self.index.shape[0])

    def getNt(self):
        return self.nt

    def getWeights(self):
        return self.weight

    def forward(self, add, signalReg, signalIrreg=None):
        """Regular (nReg, nt) -> irregular (nIrreg, nt): d[dev] += w * m[reg] in device/filter order."""
        m = np.asarray(signalReg, dtype=np.float32)
        if signalIrreg is None:
            signalIrreg = np.zeros((self.getNDeviceIrreg(), m.shape[1]), dtype=np.float32)
        elif not add:
            signalIrreg[...] = 0
        for k in range(self.index.shape[1]):
            signalIrreg += self.weight[:, k:k + 1] * m[self.slot[:, k]]
        return signalIrreg

    def adjoint(self, add, signalReg, signalIrreg):
        """Irregular -> regular: m[reg] += w * d[dev], accumulated in device then filter order."""
        d = np.asarray(signalIrreg, dtype=np.float32)
        if signalReg is None:
            signalReg = np.zeros((self.getNDeviceReg(), d.shape[1]), dtype=np.float32)
        elif not add:
            signalReg[...] = 0
        # np.add.at applies updates in index order, i.e. device-major then filter,
        # which is the reference's accumulation order
        upd = (self.weight[:, :, None] * d[:, None, :]).reshape(-1, d.shape[1])
        np.add.at(signalReg, self.slot.reshape(-1), upd)
        return signalReg


def grid_axes(nz, nx, ny, oz, ox, oy, dz, dx, dy):
    """Seven grids (Elastic_iso_float_3D.py:97-110): staggered origins at o - 0.5 d,
    in the order center, x, y, z, xz, xy, yz."""
    Z, X, Y = Axis(nz, oz, dz), Axis(nx, ox, dx), Axis(ny, oy, dy)
    Zs, Xs, Ys = Axis(nz, oz - 0.5 * dz, dz), Axis(nx, ox - 0.5 * dx, dx), Axis(ny, oy - 0.5 * dy, dy)
    return [(Z, X, Y), (Z, Xs, Y), (Z, X, Ys), (Zs, X, Y), (Zs, Xs, Y), (Z, Xs, Ys), (Zs, X, Ys)]


def build_devices(z, x, y, axes7, nt, par, dipole=None, shifts=None, method=None, hFilter1d=None, compat=True):
    """The seven spaceInterpGpu_3D objects of one device set (buildSourceGeometry_3D /
    buildReceiversGeometry_3D, Elastic_iso_float_3D.py:21-195).  Unless given, the dipole flag,
    its shifts, the method and the sinc half length come from the parameters as the reference
    reads them: dipole, zDipoleShift, xDipoleShift, yDipoleShift, spaceInterpMethod ("linear"
    by default) and hFilter1d (1 for linear)."""
    if dipole is None:
        dipole = par.getInt("dipole", 0)
    if shifts is None:
        shifts = (par.getFloat("zDipoleShift", 0.0), par.getFloat("xDipoleShift", 0.0),
                  par.getFloat("yDipoleShift", 0.0))
    if method is None:
        method = par.getString("spaceInterpMethod", "linear")
    if hFilter1d is None:
        hFilter1d = 1 if method == "linear" else par.getInt("hFilter1d", 1)
    return [spaceInterpGpu_3D(z, x, y, ax, nt, par, dipole, *shifts, interpMethod=method, hFilter1d=hFilter1d,
                              compat=compat) for ax in axes7]
