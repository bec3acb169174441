"""Test infrastructure only: the exact discrete gradient of the nonlinear misfit, in FP64 on the CPU.

The oracle's nonlinear forward (elastic_oracle.cpp nlFwd, restating propElasticFwdGpu_3D,
nonlinearPropElasticGpuFunctions_3D.cu:876-975) is restated here with torch tensors, step for
step in the same order -- stepper (stepFwdGpu_3D, kernelsElaGpu_3D.cu:110-460), source injection
(kernelsElaGpu_3D.cu:11-52), the cosine sponge on both levels (dampCosineEdge_3D,
kernelsElaGpu_3D.cu:1182-1226), recording (kernelsElaGpu_3D.cu:61-104) -- so that reverse-mode
autograd gives the exact derivative of a misfit of the recorded traces with respect to the eight
medium planes (and the source signals), for small grids.  The constants (FD coefficients,
time-interpolation filter, taper) come from the oracle library itself.

It pins what an exact-adjoint gradient must return: the shipped gradient is the reference's
Born-adjoint imaging on coarse samples (born_adjoint_reg), which differs from this one.
Nothing in the product imports this module.
"""
from __future__ import annotations

import numpy as np
import torch

from . import oracle as O

FAT = 4
VX, VY, VZ, SXX, SYY, SZZ, SXZ, SXY, SYZ = range(9)
RHOX, RHOY, RHOZ, L2M, LAM, MUXZ, MUXY, MUYZ = range(8)
GZ, GXZ = 3, 4


class TorchForward:
    """FP64 nonlinear forward on regular-grid signals, differentiable with respect to the medium
    planes and the source signals.  Fields are (ny, nx, nz) tensors, z fastest, as the library's.
    No free surface."""

    def __init__(self, p: O.PropParams, src_pos7, rec_pos7):
        if p.free_surface:
            raise ValueError("the restatement has no free surface")
        self.p = p
        coef, filt, taper, _ = O.constants(p, np.float64)
        self.cz, self.cx, self.cy = [torch.tensor(coef[4 * a:4 * a + 4], dtype=torch.float64) for a in range(3)]
        self.filt = [float(f) for f in filt]
        self.h = p.sub + 1
        self.src = [torch.as_tensor(np.asarray(src_pos7[O.COMP_GRID[k]], np.int64)) for k in range(9)]
        rec = [np.asarray(rec_pos7[O.COMP_GRID[k]], np.int64) for k in range(9)]
        if p.q2compat:
            # the reference's sxz receivers read the first n_xz entries of the z-grid table
            rec[SXZ] = np.asarray(rec_pos7[GZ], np.int64)[:len(rec_pos7[GXZ])]
        self.rec = [torch.as_tensor(r) for r in rec]
        # sponge factor per cell: damp[d] where the distance d to the closest non-FAT face is
        # below minPad, 1 elsewhere (and in the FAT ring, which stays zero)
        ny, nx, nz = p.ny, p.nx, p.nz
        iy, ix, iz = np.meshgrid(np.arange(ny), np.arange(nx), np.arange(nz), indexing="ij")
        d = np.minimum.reduce([iz - FAT, ix - FAT, nz - iz - 1 - FAT, nx - ix - 1 - FAT, iy - FAT,
                               ny - iy - 1 - FAT])
        g = np.ones((ny, nx, nz))
        inner = (iz >= FAT) & (iz < nz - FAT) & (ix >= FAT) & (ix < nx - FAT) & (iy >= FAT) & (iy < ny - FAT)
        damp = inner & (d < p.minPad)
        g[damp] = np.asarray(taper, np.float64)[d[damp]]
        self.G = torch.as_tensor(g)

    # shifted interior views: S(a, axis, o)[i] = a[i + o along axis] over the updated cells
    def _S(self, a, axis, o):
        sl = [slice(FAT, a.shape[k] - FAT) for k in range(3)]
        sl[axis] = slice(FAT + o, a.shape[axis] - FAT + o)
        return a[tuple(sl)]

    def _dplus(self, a, axis, c):
        S = lambda o: self._S(a, axis, o)  # noqa: E731
        return c[0] * (S(1) - S(0)) + c[1] * (S(2) - S(-1)) + c[2] * (S(3) - S(-2)) + c[3] * (S(4) - S(-3))

    def _dminus(self, a, axis, c):
        S = lambda o: self._S(a, axis, o)  # noqa: E731
        return c[0] * (S(0) - S(-1)) + c[1] * (S(1) - S(-2)) + c[2] * (S(2) - S(-3)) + c[3] * (S(3) - S(-4))

    def _step(self, p0, p1, m):
        """p0 + M D(p1) on the updated cells (stepFwdGpu_3D); axes (y, x, z) = (0, 1, 2)."""
        cz, cx, cy = self.cz, self.cx, self.cy
        I = lambda a: self._S(a, 0, 0)  # noqa: E731
        dvx_dx = self._dplus(p1[VX], 1, cx)
        dvy_dy = self._dplus(p1[VY], 0, cy)
        dvz_dz = self._dplus(p1[VZ], 2, cz)
        fvx = self._dminus(p1[SXX], 1, cx) + self._dplus(p1[SXY], 0, cy) + self._dplus(p1[SXZ], 2, cz)
        fvy = self._dplus(p1[SXY], 1, cx) + self._dminus(p1[SYY], 0, cy) + self._dplus(p1[SYZ], 2, cz)
        fvz = self._dplus(p1[SXZ], 1, cx) + self._dplus(p1[SYZ], 0, cy) + self._dminus(p1[SZZ], 2, cz)
        fxy = self._dminus(p1[VX], 0, cy) + self._dminus(p1[VY], 1, cx)
        fxz = self._dminus(p1[VX], 2, cz) + self._dminus(p1[VZ], 1, cx)
        fyz = self._dminus(p1[VZ], 0, cy) + self._dminus(p1[VY], 2, cz)
        upd = [I(m[RHOX]) * fvx, I(m[RHOY]) * fvy, I(m[RHOZ]) * fvz,
               I(m[L2M]) * dvx_dx + I(m[LAM]) * (dvy_dy + dvz_dz),
               I(m[L2M]) * dvy_dy + I(m[LAM]) * (dvx_dx + dvz_dz),
               I(m[L2M]) * dvz_dz + I(m[LAM]) * (dvx_dx + dvy_dy),
               I(m[MUXZ]) * fxz, I(m[MUXY]) * fxy, I(m[MUYZ]) * fyz]
        out = []
        for k in range(9):
            f = p0[k].clone()
            f[FAT:-FAT, FAT:-FAT, FAT:-FAT] = I(p0[k]) + upd[k]
            out.append(f)
        return out

    def forward(self, planes8, src_sig9):
        """planes8: (8, ny, nx, nz) FP64 tensor; src_sig9: nine (n_k, nts) FP64 tensors.
        Returns nine (n_rec_k, nts) tensors of recorded regular-grid traces."""
        p = self.p
        shape = (p.ny, p.nx, p.nz)
        zero = torch.zeros(shape, dtype=torch.float64)
        p0 = [zero.clone() for _ in range(9)]
        p1 = [zero.clone() for _ in range(9)]
        cols = [[None] * p.nts for _ in range(9)]
        f, h = self.filt, self.h
        for its in range(p.nts - 1):
            for it2 in range(1, p.sub + 1):
                p0 = self._step(p0, p1, planes8)
                k = it2 - 1
                for c in range(9):
                    if len(self.src[c]):
                        v = src_sig9[c][:, its] * f[k] + src_sig9[c][:, its + 1] * f[h + k]
                        p0[c] = p0[c].reshape(-1).index_add(0, self.src[c], v).reshape(shape)
                p0 = [a * self.G for a in p0]
                p1 = [a * self.G for a in p1]
                for c in range(9):
                    if len(self.rec[c]) == 0:
                        continue
                    v = p0[c].reshape(-1)[self.rec[c]]
                    for t, w in ((its, f[it2]), (its + 1, f[h + it2])):
                        cols[c][t] = v * w if cols[c][t] is None else cols[c][t] + v * w
                p0, p1 = p1, p0
        out = []
        for c in range(9):
            n = len(self.rec[c])
            z = torch.zeros(n, dtype=torch.float64)
            out.append(torch.stack([z if x is None else x for x in cols[c]], dim=1))
        return out


# ---- the medium and the source scaling as functions of (rho, lambda, mu) ------------------------
def _stagger_adjoint_t(d, axis):
    """oracle.stagger_adjoint on torch tensors: m[i] = 0.5(d[i]+d[i-1]), m[0] = 0.5 d[0],
    m[n-1] = d[n-1] + 0.5 d[n-2] along the model axis (0 z, 1 x, 2 y)."""
    a = {0: 2, 1: 1, 2: 0}[axis]
    d = torch.movedim(d, a, -1)
    m = torch.cat([0.5 * d[..., :1], 0.5 * (d[..., 1:-1] + d[..., :-2]), d[..., -1:] + 0.5 * d[..., -2:-1]], dim=-1)
    return torch.movedim(m, -1, a)


def medium_planes_t(ep, dtw):
    """oracle.medium_planes (fdParamElastic_3D.cpp:138-183) in FP64 torch: (3, ny, nx, nz) elastic
    parameters (rho, lambda, mu) -> (8, ny, nx, nz) scaled planes."""
    rho, lam, mu = ep[0], ep[1], ep[2]
    two = 2.0 * float(dtw)
    rhox, rhoy, rhoz = _stagger_adjoint_t(rho, 1), _stagger_adjoint_t(rho, 2), _stagger_adjoint_t(rho, 0)
    muxz = _stagger_adjoint_t(_stagger_adjoint_t(mu, 1), 0)
    muxy = _stagger_adjoint_t(_stagger_adjoint_t(mu, 1), 2)
    muyz = _stagger_adjoint_t(_stagger_adjoint_t(mu, 2), 0)
    return torch.stack([two / rhox, two / rhoy, two / rhoz, two * (lam + 2.0 * mu), two * lam, two * muxz,
                        two * muxy, two * muyz])


def scale_signals_t(reg9, src_pos7, planes, dx, dy, dz):
    """oracle.scale_signals (nonlinearPropElasticGpu_3D.cpp:200-277) in FP64 torch: the medium at
    the source points scales the nine regular-grid source blocks; returns new tensors."""
    flat = planes.reshape(8, -1)
    P = [torch.as_tensor(np.asarray(src_pos7[g], np.int64)) for g in range(7)]
    out = [reg9[0] * flat[0][P[1]][:, None], reg9[1] * flat[1][P[2]][:, None], reg9[2] * flat[2][P[3]][:, None]]
    l2m, lam = flat[3][P[0]][:, None], flat[4][P[0]][:, None]
    sxx, syy, szz = reg9[3], reg9[4], reg9[5]
    out += [sxx * l2m + (syy + szz) * lam, syy * l2m + (sxx + szz) * lam, szz * l2m + (sxx + syy) * lam]
    out += [reg9[6] * flat[5][P[4]][:, None], reg9[7] * flat[6][P[5]][:, None], reg9[8] * flat[7][P[6]][:, None]]
    area = 1.0 / float(np.float32(np.float32(dx) * np.float32(dy)) * np.float32(dz))
    return [o * area for o in out]


def interp_matrix(dev):
    """The regular -> irregular map of an oracle.SpaceInterp as a dense (n_irreg, n_reg) matrix."""
    return torch.as_tensor(dev.forward(np.eye(dev.n_reg, dtype=np.float64)))


# ---- the same gradient by a hand-written adjoint recursion ---------------------------------------
def exact_gradient_by_adjoint(p: O.PropParams, med, src9, src_pos7, rec_pos7, drec9):
    """Exact gradient of a functional of the recorded traces with respect to the eight medium
    planes, by the adjoint recursion a GPU mode would run (FP64 numpy, the oracle's own steppers).

    drec9: nine (n_rec_k, nts) blocks, the derivative of the functional by the recorded traces.
    With (X_j, Y_j) the two levels at the start of fine step j, the forward step is
    X_{j+1} = G Y_j, Y_{j+1} = G (X_j + M D(Y_j) + S_j), and step j records Y_{j+1}.  Backwards,
    with (xi, eta) the derivatives by (X_{j+1}, Y_{j+1}):
      eta~ = eta + the recording weights of step j applied to drec9 (at the receiver positions)
      grad_M += (G eta~) * D(Y_j), term by term (the imaging of every fine step)
      xi, eta <- G eta~, G xi + T(G eta~)
    where T(q) = -D(M q) is the reference's exact-transpose stepper (stepAdjGpuBorn_3D,
    kernelsElaGpu_3D.cu:825-1177) applied to q from zero.  The sources are held fixed."""
    tf = TorchForward(p, src_pos7, rec_pos7)
    shape = (p.ny, p.nx, p.nz)
    f, h = tf.filt, tf.h
    G = tf.G.numpy()
    src_idx = [s.numpy() for s in tf.src]
    rec_idx = [r.numpy() for r in tf.rec]
    steps = [(its, it2) for its in range(p.nts - 1) for it2 in range(1, p.sub + 1)]
    X = [np.zeros(shape) for _ in range(9)]
    Y = [np.zeros(shape) for _ in range(9)]
    ys = []
    for its, it2 in steps:
        ys.append([y.copy() for y in Y])
        Xn, _ = O.step_once(p, X, Y, med, 0, 0, np.float64)
        for c in range(9):
            if len(src_idx[c]):
                v = src9[c][:, its] * f[it2 - 1] + src9[c][:, its + 1] * f[h + it2 - 1]
                np.add.at(Xn[c].reshape(-1), src_idx[c], v)
        X, Y = [G * y for y in Y], [G * x for x in Xn]
    inner = (slice(FAT, -FAT),) * 3
    cz, cx, cy = tf.cz, tf.cx, tf.cy

    def D(a, axis, plus, c):
        return (tf._dplus if plus else tf._dminus)(torch.as_tensor(a), axis, c).numpy()

    grad = np.zeros((8,) + shape)
    xi = [np.zeros(shape) for _ in range(9)]
    eta = [np.zeros(shape) for _ in range(9)]
    for j in range(len(steps) - 1, -1, -1):
        its, it2 = steps[j]
        et = [e.copy() for e in eta]
        for c in range(9):
            if len(rec_idx[c]):
                v = np.asarray(drec9[c])[:, its] * f[it2] + np.asarray(drec9[c])[:, its + 1] * f[h + it2]
                np.add.at(et[c].reshape(-1), rec_idx[c], v)
        ge = [G * e for e in et]
        y = ys[j]
        dvx_dx, dvy_dy, dvz_dz = D(y[VX], 1, True, cx), D(y[VY], 0, True, cy), D(y[VZ], 2, True, cz)
        fvx = D(y[SXX], 1, False, cx) + D(y[SXY], 0, True, cy) + D(y[SXZ], 2, True, cz)
        fvy = D(y[SXY], 1, True, cx) + D(y[SYY], 0, False, cy) + D(y[SYZ], 2, True, cz)
        fvz = D(y[SXZ], 1, True, cx) + D(y[SYZ], 0, True, cy) + D(y[SZZ], 2, False, cz)
        fxy = D(y[VX], 0, False, cy) + D(y[VY], 1, False, cx)
        fxz = D(y[VX], 2, False, cz) + D(y[VZ], 1, False, cx)
        fyz = D(y[VZ], 0, False, cy) + D(y[VY], 2, False, cz)
        e = [x[inner] for x in ge]
        grad[RHOX][inner] += e[VX] * fvx
        grad[RHOY][inner] += e[VY] * fvy
        grad[RHOZ][inner] += e[VZ] * fvz
        grad[L2M][inner] += e[SXX] * dvx_dx + e[SYY] * dvy_dy + e[SZZ] * dvz_dz
        grad[LAM][inner] += e[SXX] * (dvy_dy + dvz_dz) + e[SYY] * (dvx_dx + dvz_dz) + e[SZZ] * (dvx_dx + dvy_dy)
        grad[MUXZ][inner] += e[SXZ] * fxz
        grad[MUXY][inner] += e[SXY] * fxy
        grad[MUYZ][inner] += e[SYZ] * fyz
        t, _ = O.step_once(p, [np.zeros(shape) for _ in range(9)], ge, med, 2, 0, np.float64)
        xi, eta = ge, [G * a + b for a, b in zip(xi, t)]
    return grad
