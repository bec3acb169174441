"""Seeded synthetic inputs: smooth random media, Ricker sources, acquisition grids.

No public dataset is involved in this path; the benchmark and the tests use
these generators with fixed seeds.  Grid padding follows the reference's
padElasticFileGpuMain_3D.cpp:47-86 rule (z and x padded up to multiples of the
block size, y unconstrained, FAT=4 added on every side, top pad = FAT with a
free surface).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .hostprep import FAT, Axis, ParamObj


def smooth_field(shape, sigma, rng):
    """Unit-variance Gaussian random field smoothed with a Gaussian of sigma cells (FFT)."""
    w = rng.standard_normal(shape)
    if sigma <= 0:
        return w
    k = [np.fft.fftfreq(n) for n in shape]
    g = np.ones(shape)
    for ax, kk in enumerate(k):
        sh = [1] * len(shape)
        sh[ax] = -1
        g = g * np.exp(-2.0 * (np.pi * sigma * kk.reshape(sh)) ** 2)
    f = np.fft.ifftn(np.fft.fftn(w) * g).real
    s = f.std()
    return f / s if s > 0 else f


def ricker(nts, dts, fdom, delay):
    """Ricker wavelet (waveletFloatMain.py:88-110): (1 - 2 a t^2) exp(-a t^2), a = (pi f)^2."""
    t = np.arange(nts) * dts - delay
    a = (np.pi * fdom) ** 2
    return ((1.0 - 2.0 * a * t * t) * np.exp(-a * t * t)).astype(np.float32)


def padded_size(n, pad, block=16, free_surface=False):
    """(n_total, padMinus, padPlus) for z/x per the reference padding program."""
    if free_surface:
        total = pad + n + FAT
        nb = int(np.ceil(total / block))
        pm = FAT
        pp = nb * block - n - pm
    else:
        total = 2 * pad + n
        nb = int(np.ceil(total / block))
        pm = pad
        pp = nb * block - n - pad
    return pm + pp + n + 2 * FAT, pm, pp


def elastic_from_velocity(vp, vs, rho):
    """(rho, lambda, mu) from (vp, vs, rho), as float32 (3, ny, nx, nz)."""
    mu = rho * vs * vs
    lam = rho * vp * vp - 2.0 * mu
    return np.stack([rho, lam, mu]).astype(np.float32)


@dataclass
class Survey:
    """A propagation grid with medium, parameters and acquisition coordinates."""
    elastic: np.ndarray           # (3, ny, nx, nz)
    axes: tuple                   # (zAxis, xAxis, yAxis)
    par: ParamObj
    src_xyz: list = field(default_factory=list)   # per shot: (z, x, y) arrays
    rec_xyz: tuple = None                          # (z, x, y) arrays (same for all shots)
    wavelet: np.ndarray = None                     # (nts,)
    name: str = ""

    @property
    def shape(self):
        return self.elastic.shape[1:]


def make_grid(nzi, nxi, nyi, pad, d, free_surface=False, block=16):
    nz, zpm, zpp = padded_size(nzi, pad, block, free_surface)
    nx, xpm, xpp = padded_size(nxi, pad, block, False)
    ny = nyi + 2 * pad + 2 * FAT
    oz = -(FAT + zpm) * d
    ox = -(FAT + xpm) * d
    oy = -(FAT + pad) * d
    axes = (Axis(nz, oz, d), Axis(nx, ox, d), Axis(ny, oy, d))
    pads = dict(zPadMinus=zpm, zPadPlus=zpp, xPadMinus=xpm, xPadPlus=xpp, yPad=pad)
    return axes, pads


def base_params(axes, pads, nts, dts, sub_par, fmax, free_surface=False):
    za, xa, ya = axes
    par = ParamObj(nts=nts, dts=dts, sub=sub_par, nz=za.n, nx=xa.n, ny=ya.n, dz=za.d, dx=xa.d, dy=ya.d,
                   fMax=fmax, blockSize=16, fat=FAT, alphaCos=0.99, mod_par=0,
                   freeSurface=1 if free_surface else 0, **pads)
    return par


def gaussian_perturbed_model(shape, vp0, vs0, rho0, amp, sigma, seed):
    rng = np.random.default_rng(seed)
    f = smooth_field(shape, sigma, rng)
    f = f / max(np.abs(f).max(), 1e-12)
    return (vp0 * (1 + amp * f), vs0 * (1 + amp * f), rho0 * (1 + amp * f))


def plain_forward_survey(nts=1000, seed=0):
    """Plain forward, single shot: 120^3 interior + 30 sponge, free surface top, dx=10 m,
    vp=2500, vs=vp/1.732, rho=2000 with smooth +-10% perturbations (sigma 5 cells);
    explosive Ricker 15 Hz at the centre, 200 m depth; 40x40 receivers at 20 m depth (30 m spacing)."""
    d = 10.0
    axes, pads = make_grid(120, 120, 120, 30, d, free_surface=True)
    shape = (axes[2].n, axes[1].n, axes[0].n)
    vp, vs, rho = gaussian_perturbed_model(shape, 2500.0, 2500.0 / 1.732, 2000.0, 0.10, 5.0, seed)
    el = elastic_from_velocity(vp, vs, rho)
    dts = 0.002
    par = base_params(axes, pads, nts, dts, 2, 40.0, free_surface=True)
    c = 590.0  # near the centre of the 120-cell interior, keeping every staggered stencil inside
    src = [(np.array([200.0]), np.array([c]), np.array([c]))]
    g = (np.arange(40) - 19.5) * 30.0 + c
    X, Y = np.meshgrid(g, g, indexing="ij")
    rec = (np.full(X.size, 20.0), X.reshape(-1), Y.reshape(-1))
    return Survey(el, axes, par, src, rec, ricker(nts, dts, 15.0, 1.0 / 15.0), "plain-forward-120^3+30")


def gardner_model(shape, seed, vmin=1500.0, vmax=4500.0, sigma=8.0):
    rng = np.random.default_rng(seed)
    f = smooth_field(shape, sigma, rng)
    f = (f - f.min()) / max(f.max() - f.min(), 1e-12)
    vp = vmin + (vmax - vmin) * f
    vs = vp / np.sqrt(3.0)
    rho = 310.0 * vp ** 0.25
    return vp, vs, rho


def batched_forward_survey(nts=2000, seed=1, nshots=16, coarse=8):
    """Batched forward modelling: 400 x 400 (x, y) x 300 (z) interior + 40-cell sponge (392 x 488 x 488
    cells with FAT), Gardner model family (vp smooth random in [1500, 4500] m/s, vs = vp/sqrt(3),
    rho = 310 vp^0.25), explosive Ricker 15 Hz sources on a 4 x 4 surface grid (20 m depth), 200 x 200
    receivers at 10 m spacing (10 m depth), dts 2 ms.  The random field is drawn on a grid `coarse`
    times coarser and repeated, which keeps the set-up cheap on 93 M cells."""
    d = 10.0
    axes, pads = make_grid(300, 400, 400, 40, d)
    shape = (axes[2].n, axes[1].n, axes[0].n)
    cshape = tuple(-(-n // coarse) for n in shape)
    vpc, _, _ = gardner_model(cshape, seed, vmax=4450.0, sigma=2.0)  # Courant 0.45 needs vmax < 4500
    vp = np.repeat(np.repeat(np.repeat(vpc, coarse, 0), coarse, 1), coarse, 2)[:shape[0], :shape[1], :shape[2]]
    vs = vp / np.sqrt(3.0)
    rho = 310.0 * vp ** 0.25
    el = elastic_from_velocity(vp, vs, rho)
    dts = 0.002
    par = base_params(axes, pads, nts, dts, 2, 25.0)
    g4 = np.linspace(800.0, 3200.0, 4)
    src = [(np.array([20.0]), np.array([g4[i % 4]]), np.array([g4[(i // 4) % 4]])) for i in range(nshots)]
    g = 2000.0 + (np.arange(200) - 99.5) * 10.0
    X, Y = np.meshgrid(g, g, indexing="ij")
    rec = (np.full(X.size, 10.0), X.reshape(-1), Y.reshape(-1))
    return Survey(el, axes, par, src, rec, ricker(nts, dts, 15.0, 1.0 / 15.0), "batched-forward-400x400x300+40")


def _with_anomalies(shape, vp, vs, rho):
    """The true model of the FWI survey: two Gaussian anomalies (+-8% vp/vs, +-3% rho) on the background."""
    iy, ix, iz = [np.arange(n, dtype=np.float64) for n in shape]
    for sgn, cz in ((1.0, 0.35), (-1.0, 0.65)):
        cy, cx, czz = shape[0] / 2, shape[1] / 2, shape[2] * cz
        r2 = (((iy - cy) ** 2)[:, None, None] + ((ix - cx) ** 2)[None, :, None] + ((iz - czz) ** 2)[None, None, :]) \
            / (0.08 * min(shape)) ** 2
        g = np.exp(-r2)
        vp = vp * (1 + sgn * 0.08 * g)
        vs = vs * (1 + sgn * 0.08 * g)
        rho = rho * (1 + sgn * 0.03 * g)
    return vp, vs, rho


def fwi_gradient_survey(nzi=300, nxi=300, nyi=300, pad=40, nts=2500, nshots=32, nrec=150, fdom=10.0, seed=3,
               true_model=False, with_true=False):
    """FWI gradient survey (300^3 interior + 40 sponge by default): smooth background (vp 2500, vs vp/1.732, rho 2000 with
    +-10% smooth perturbations) plus, for the true model, two Gaussian anomalies (+-8% vp/vs, +-3% rho).
    with_true=True returns (survey on the background, true (rho, lambda, mu)) from one random field."""
    d = 10.0
    axes, pads = make_grid(nzi, nxi, nyi, pad, d)
    shape = (axes[2].n, axes[1].n, axes[0].n)
    vp, vs, rho = gaussian_perturbed_model(shape, 2500.0, 2500.0 / 1.732, 2000.0, 0.10, 5.0, seed)
    true_el = elastic_from_velocity(*_with_anomalies(shape, vp, vs, rho)) if (true_model or with_true) else None
    el = true_el if true_model else elastic_from_velocity(vp, vs, rho)
    dts = 0.002
    par = base_params(axes, pads, nts, dts, 2, 25.0)
    z0 = (axes[0].n - 2 * FAT - pads["zPadMinus"] - pads["zPadPlus"])
    x_int = (nxi - 2) * d  # the last interior cell cannot hold a trilinear stencil on every staggered grid
    y_int = (nyi - 2) * d
    ns = int(np.ceil(np.sqrt(nshots)))
    sx = np.linspace(0.1, 0.9, ns) * x_int
    src = []
    for i in range(nshots):
        src.append((np.array([20.0]), np.array([sx[i % ns]]), np.array([sx[(i // ns) % ns] * y_int / x_int])))
    gx = np.linspace(0.0, x_int, nrec)
    gy = np.linspace(0.0, y_int, nrec)
    X, Y = np.meshgrid(gx, gy, indexing="ij")
    rec = (np.full(X.size, 10.0), X.reshape(-1), Y.reshape(-1))
    del z0
    sv = Survey(el, axes, par, src, rec, ricker(nts, dts, fdom, 1.0 / fdom), f"fwi-{nzi}x{nxi}x{nyi}")
    return (sv, true_el) if with_true else sv


def small_survey(seed=0, nzi=32, nxi=32, nyi=24, pad=4, nts=20, sub_par=2, d=10.0, nrec=6, nshots=1):
    """A few-second case for parity tests (grid multiple of 16 + 2*FAT on z and x, as the
    reference requires)."""
    axes, pads = make_grid(nzi, nxi, nyi, pad, d)
    shape = (axes[2].n, axes[1].n, axes[0].n)
    vp, vs, rho = gaussian_perturbed_model(shape, 2500.0, 2500.0 / 1.732, 2000.0, 0.10, 2.0, seed)
    el = elastic_from_velocity(vp, vs, rho)
    dts = 0.002
    par = base_params(axes, pads, nts, dts, sub_par, 40.0)
    rng = np.random.default_rng(seed + 100)
    lo = np.array([0.0, 0.0, 0.0])
    hi = np.array([(nzi - 2) * d, (nxi - 2) * d, (nyi - 2) * d])
    src = []
    for _ in range(nshots):
        p = lo + (hi - lo) * (0.3 + 0.4 * rng.random(3))
        src.append((np.array([p[0]]), np.array([p[1]]), np.array([p[2]])))
    r = lo + (hi - lo) * rng.random((nrec, 3))
    rec = (r[:, 0], r[:, 1], r[:, 2])
    return Survey(el, axes, par, src, rec, ricker(nts, dts, 15.0, 0.03), f"small-{nzi}x{nxi}x{nyi}")
