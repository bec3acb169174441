"""Drop-in operator classes with the reference's Python interface.

Same class names, constructor arguments, vector layouts and methods as the
reference's pyOperator wrappers (python_float/Elastic_iso_float_3D.py:445-770)
and the C++ shot operators they wrap:

  nonlinearPropElasticShotsGpu_3D   (nonlinearPropElasticShotsGpu_3D.cpp:122-420,
                                     nonlinearPropElasticGpu_3D.cpp:66-615)
  nonlinearFwiPropElasticShotsGpu_3D (Elastic_iso_float_3D.py:592-643)
  BornElasticShotsGpu_3D            (BornElasticShotsGpu_3D.cpp:143-605, BornElasticGpu_3D.cpp:70-330,
                                     seismicElasticOperator3D.cpp:74-228)
  ElasticDatComp_3D                 (seis_utils/python/dataCompModule_3D.py)
  buildSourceGeometry_3D, buildReceiversGeometry_3D (Elastic_iso_float_3D.py:21-385), with the
                                     geometry passed as an array instead of a SEP file

Vectors are numpy arrays (or objects with getNdArray(), such as SEP vectors)
in the numpy view of the reference's hypercubes, slowest axis first:
  elastic parameters / Born model  (3, ny, nx, nz)      [rho|lambda|mu] or [drho|dlambda|dmu]
  nonlinear model (source signals) (nExp or 1, 9, nSimSrc, nts)
  data                             (nExp, 9, nRec, nts)  vx,vy,vz,sxx,syy,szz,sxz,sxy,syz
  Born source signals              list of (9, nSimSrc, nts), one per shot or one for all
The 14 acquisition arguments are lists (one entry per shot, or one entry for
all shots on the receiver side) of hostprep.spaceInterpGpu_3D objects in the
order center, x, y, z, xz, xy, yz grid, sources then receivers.

Host work mirrors the reference: spatial interpolation (spaceInterpGpu_3D),
medium scaling of source signals / adjoint data, Born model staggering and
gradient post-processing run on the host; each shot then runs on a GPU
through the C ABI's host-buffer entry points (e3d_nl_forward, e3d_nl_adjoint,
e3d_born_forward, e3d_born_adjoint).  Shots are distributed over the GPUs
named by the parameters `nGpu` / `iGpu` with one host thread per GPU, like
the reference's OpenMP loop (nonlinearPropElasticShotsGpu_3D.cpp:178-204).
Outputs follow the reference's `add` semantics: overwritten unless add.
"""
from __future__ import annotations

import builtins
import threading
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import hostprep as H
from .engine import COMP_GRID, Propagator, SlabPropagator, domain_decomposition


def _nd(v):
    return v.getNdArray() if hasattr(v, "getNdArray") else v


def _axes_of(elastic, par):
    """Grid axes (z, x, y) of an elastic-parameter vector: from its hypercube when it has one,
    else from the parameters nz/nx/ny, dz/dx/dy and oz/ox/oy."""
    if hasattr(elastic, "getHyper"):
        hyp = elastic.getHyper()
        return tuple(H.Axis(hyp.getAxis(i).n, hyp.getAxis(i).o, hyp.getAxis(i).d) for i in (1, 2, 3))
    return (H.Axis(par.getInt("nz"), par.getFloat("oz", 0.0), par.getFloat("dz")),
            H.Axis(par.getInt("nx"), par.getFloat("ox", 0.0), par.getFloat("dx")),
            H.Axis(par.getInt("ny"), par.getFloat("oy", 0.0), par.getFloat("dy")))


def _interp_params(par, receivers):
    """Dipole, shifts, method and sinc half length as the reference's geometry builders read them
    (Elastic_iso_float_3D.py:21-60, 194-240): the receiver builder reads the dipole shifts with
    getInt (truncating them), the source builder with getFloat; sinc sources default hFilter1d
    to 1, sinc receivers require it."""
    get = par.getInt if receivers else par.getFloat
    dipole = par.getInt("dipole", 0)
    shifts = tuple(float(get(k, 0)) for k in ("zDipoleShift", "xDipoleShift", "yDipoleShift"))
    method = par.getString("spaceInterpMethod", "linear")
    if method == "linear":
        h = 1
    elif method == "sinc":
        h = par.getInt("hFilter1d") if receivers else par.getInt("hFilter1d", 1)
    else:
        raise ValueError(f"spatial interpolation method {method!r} is not implemented")
    return dipole, shifts, method, h


def _geometry(par, elastic, geom, receivers):
    za, xa, ya = _axes_of(elastic, par)
    axes7 = H.grid_axes(za.n, xa.n, ya.n, za.o, xa.o, ya.o, za.d, xa.d, ya.d)
    g = np.asarray(_nd(geom), dtype=np.float32)
    if g.ndim != 3 or g.shape[0] != 3:
        raise ValueError("geometry must be (3, nPoints, nExp) in the numpy view: x, y, z rows")
    dipole, shifts, method, h = _interp_params(par, receivers)
    nts = par.getInt("nts")
    vecs = [[] for _ in range(7)]
    for e in builtins.range(g.shape[2]):
        devs = H.build_devices(g[2, :, e], g[0, :, e], g[1, :, e], axes7, nts, par, dipole=dipole, shifts=shifts,
                               method=method, hFilter1d=h)
        for k in builtins.range(7):
            vecs[k].append(devs[k])
    return vecs


def buildSourceGeometry_3D(parObject, elasticParam, sourceGeom):
    """The reference's source-geometry builder (Elastic_iso_float_3D.py:21-191) with the geometry
    passed as an array instead of read from the SEP file `sourceGeomFile` (SEP IO is not part of
    this library): sourceGeom (3, nSimSou, nExp) in the numpy view, rows x, y, z.  Returns the
    seven per-grid lists of spaceInterpGpu_3D objects (center, x, y, z, xz, xy, yz; one per shot)
    and the shot axis."""
    n_exp = parObject.getInt("nExp", -1)
    if n_exp == -1:
        raise ValueError("buildSourceGeometry_3D: the total number of shots (nExp) is required")
    g = np.asarray(_nd(sourceGeom))
    if g.ndim != 3 or g.shape[2] != n_exp:
        raise ValueError(f"nExp ({n_exp}) not consistent with the number of shots in the geometry "
                         f"({g.shape[2] if g.ndim == 3 else 'bad shape'})")
    return (*_geometry(parObject, elasticParam, g, receivers=False), H.Axis(n_exp, 0.0, 1.0))


def buildReceiversGeometry_3D(parObject, elasticParam, receiverGeom):
    """The reference's receiver-geometry builder (Elastic_iso_float_3D.py:194-385) with the geometry
    passed as an array instead of read from `receiverGeomFile`: receiverGeom (3, nReceiverPerShot,
    nExp or 1) in the numpy view, rows x, y, z; one shot-independent set when its last axis is 1.
    Returns the seven per-grid lists and the receiver axis."""
    n_exp = parObject.getInt("nExp", -1)
    if n_exp == -1:
        raise ValueError("buildReceiversGeometry_3D: the total number of shots (nExp) is required")
    n_rec = parObject.getInt("nReceiverPerShot", -1)
    if n_rec == -1:
        raise ValueError("buildReceiversGeometry_3D: the number of receivers per shot (nReceiverPerShot) is "
                         "required")
    g = np.asarray(_nd(receiverGeom))
    if g.ndim != 3:
        raise ValueError("geometry must be (3, nReceiverPerShot, nExp or 1)")
    if g.shape[2] != 1 and g.shape[2] != n_exp:
        raise ValueError(f"number of shots ({n_exp}) not consistent with the receivers' geometry ({g.shape[2]})")
    if g.shape[1] != n_rec:
        raise ValueError(f"nReceiverPerShot ({n_rec}) not consistent with the receivers' geometry ({g.shape[1]})")
    return (*_geometry(parObject, elasticParam, g, receivers=True), H.Axis(n_rec, 0.0, 1.0))


def scale_signals(reg9, devices7, planes, dx, dy, dz):
    """Medium scaling of regular-grid signals in place (nonlinearPropElasticGpu_3D.cpp:200-277 for
    sources, :481-558 for adjoint data; seismicElasticOperator3D.cpp:147-225 for Born sources).
    Each component is read at its own grid's positions; the normal stresses are mixed through
    lambda+2mu and lambda at the center grid; everything is then multiplied by 1/(dx*dy*dz)."""
    flat = planes.reshape(8, -1)
    for k, m in ((0, 0), (1, 1), (2, 2), (6, 5), (7, 6), (8, 7)):
        pos = devices7[COMP_GRID[k]].getRegPosUnique()
        reg9[k] *= flat[m][pos][:, None]
    pos = devices7[0].getRegPosUnique()
    l2m, lam = flat[3][pos][:, None], flat[4][pos][:, None]
    sxx, syy, szz = reg9[3].copy(), reg9[4].copy(), reg9[5].copy()
    reg9[3][...] = sxx * l2m + (syy + szz) * lam
    reg9[4][...] = syy * l2m + (sxx + szz) * lam
    reg9[5][...] = szz * l2m + (sxx + syy) * lam
    area = np.float32(1.0 / float(np.float32(np.float32(dx) * np.float32(dy)) * np.float32(dz)))
    for k in range(9):
        reg9[k] *= area
    return reg9


def born_model_to_planes(model3, scaling3, dtw):
    """Born model preparation (BornElasticShotsGpu_3D.cpp:167-235): (drho, dlambda, dmu) ->
    eight staggered perturbation planes scaled like the medium planes."""
    drho, dlam, dmu = (np.ascontiguousarray(model3[k], dtype=np.float32) for k in range(3))
    out = np.empty((8,) + drho.shape, dtype=np.float32)
    out[0] = H.stagger(drho, "x", adjoint=True)
    out[1] = H.stagger(drho, "y", adjoint=True)
    out[2] = H.stagger(drho, "z", adjoint=True)
    out[3] = dlam
    out[4] = dmu
    out[5] = H.stagger(H.stagger(dmu, "x", adjoint=True), "z", adjoint=True)
    out[6] = H.stagger(H.stagger(dmu, "x", adjoint=True), "y", adjoint=True)
    out[7] = H.stagger(H.stagger(dmu, "y", adjoint=True), "z", adjoint=True)
    two = 2.0 * float(dtw)
    for k in range(3):
        out[k] = out[k] * scaling3[k]
    for k in range(3, 8):
        out[k] = (out[k].astype(np.float64) * two).astype(np.float32)
    return out


def born_planes_to_model(planes8, scaling3, dtw):
    """Adjoint of born_model_to_planes (BornElasticShotsGpu_3D.cpp:528-605)."""
    two = 2.0 * float(dtw)
    g = [np.asarray(planes8[k], dtype=np.float32) * scaling3[k] for k in range(3)]
    g += [(np.asarray(planes8[k], dtype=np.float64) * two).astype(np.float32) for k in range(3, 8)]
    model = np.zeros((3,) + g[0].shape, dtype=np.float32)
    model[0] = H.stagger(g[0], "x")
    model[0] += H.stagger(g[1], "y")
    model[0] += H.stagger(g[2], "z")
    t2 = H.stagger(H.stagger(g[5], "z"), "x")
    t2 += H.stagger(H.stagger(g[6], "y"), "x")
    t2 += H.stagger(H.stagger(g[7], "z"), "y")
    model[1] = g[3]
    model[2] = g[4] + t2
    return model


class _ShotOperatorBase:
    """Shared set-up: finite-difference parameters, per-GPU contexts and acquisition lists."""

    _slab_capable = False  # the operator can run a shot over y-slabs (domDec=1)

    def __init__(self, domain, range, elasticParam, paramP, devices14):
        self.setDomainRange(domain, range)
        self.par = paramP
        self.axes = _axes_of(elasticParam, paramP)
        self.fd = H.FdParam(_nd(elasticParam), self.axes, paramP)
        if len(devices14) != 14:
            raise ValueError("expected 7 source and 7 receiver acquisition lists")
        self.src = [list(devices14[g]) for g in builtins.range(7)]
        self.rec = [list(devices14[7 + g]) for g in builtins.range(7)]
        self.nExp = len(self.src[0])
        if any(len(s) != self.nExp for s in self.src):
            raise ValueError("source acquisition lists differ in length")
        self.constantRecGeom = len(self.rec[0]) == 1
        if not self.constantRecGeom and any(len(r) != self.nExp for r in self.rec):
            raise ValueError("receiver acquisition lists must have one entry or one per shot")
        # domDec=1: every shot runs over y-slabs of the grid, one per listed GPU
        # (nonlinearPropElasticShotsGpu_3D.cpp:43-77); the slabs may share a device
        self.domDec = paramP.getInt("domDec", 0) == 1
        if self.domDec and not self._slab_capable:
            raise ValueError("domain decomposition is built for the nonlinear operators only")
        gpus = str(paramP.getString("iGpu", "-1"))
        ids = [int(t) for t in gpus.split(",") if t.strip() != ""]
        if ids and ids[0] >= 0:
            if len(set(ids)) != len(ids) and not self.domDec:
                raise ValueError("duplicate GPU ids in iGpu")
            self.gpus = ids if self.domDec else sorted(ids)
        else:
            self.gpus = list(builtins.range(paramP.getInt("nGpu", 1)))
        if len(self.gpus) > self.nExp and not self.domDec:
            raise ValueError("more GPUs than shots to model")
        fd = self.fd
        # freeSurface=1 in the parameters runs the free surface (nonlinear operators only: the
        # engine refuses it on the Born path, which has no exact adjoint of it)
        if self.domDec:
            if len(self.gpus) < 2:
                raise ValueError("cannot use domain decomposition on a single card")
            self.props = [SlabPropagator(fd.nz, fd.nx, fd.ny, fd.nts, fd.sub, fd.minPad, float(fd.dz), float(fd.dx),
                                         float(fd.dy), float(fd.dts), float(fd.alphaCos), devices=self.gpus,
                                         ny_domdec=domain_decomposition(fd.ny, len(self.gpus), 4, fd.minPad),
                                         free_surface=int(fd.freeSurface))]
        else:
            self.props = [Propagator(fd.nz, fd.nx, fd.ny, fd.nts, fd.sub, fd.minPad, float(fd.dz), float(fd.dx),
                                     float(fd.dy), float(fd.dts), float(fd.alphaCos), device=g,
                                     free_surface=int(fd.freeSurface)) for g in self.gpus]
        for pr in self.props:
            pr.set_medium(fd.planes)
        self._lock = threading.Lock()

    # pyOperator plumbing
    def setDomainRange(self, domain, range):
        self.domain_shape = tuple(np.shape(_nd(domain)))
        self.range_shape = tuple(np.shape(_nd(range)))

    def _rec(self, iExp):
        i = 0 if self.constantRecGeom else iExp
        return [self.rec[g][i] for g in range(7)]

    def _srcs(self, iExp):
        return [self.src[g][iExp] for g in range(7)]

    def _run_shots(self, fn):
        """fn(prop, iExp) for every shot, one host thread per GPU, shots dealt dynamically."""
        queue = list(range(self.nExp))
        qlock = threading.Lock()

        def worker(prop):
            while True:
                with qlock:
                    if not queue:
                        return
                    iExp = queue.pop(0)
                fn(prop, iExp)

        if len(self.props) == 1:
            worker(self.props[0])
            return
        with ThreadPoolExecutor(len(self.props)) as ex:
            for f in [ex.submit(worker, p) for p in self.props]:
                f.result()

    def setBackground(self, elasticParam):
        """New background model (the reference rebuilds fdParamElastic_3D, with its checks)."""
        self.fd = H.FdParam(_nd(elasticParam), self.axes, self.par)
        for pr in self.props:
            pr.set_medium(self.fd.planes)

    def _scaled_sources(self, iExp, model9):
        src7 = self._srcs(iExp)
        reg = [src7[COMP_GRID[k]].adjoint(False, None, np.asarray(model9[k], dtype=np.float32)) for k in range(9)]
        return scale_signals(reg, src7, self.fd.planes, self.fd.dx, self.fd.dy, self.fd.dz)

    def dotTest(self, verb=False, maxError=1e-5):
        """Dot-product test of forward/adjoint, without and with add (operator.h:50-92)."""
        rng = np.random.default_rng(1234)
        m1 = rng.uniform(-1.0, 1.0, self.domain_shape).astype(np.float32)
        d1 = rng.uniform(-1.0, 1.0, self.range_shape).astype(np.float32)
        m2 = np.zeros(self.domain_shape, np.float32)
        d2 = np.zeros(self.range_shape, np.float32)
        self.adjoint(False, m2, d1)
        self.forward(False, m1, d2)
        dot1, dot2 = float(np.dot(d1.ravel().astype(np.float64), d2.ravel())), float(
            np.dot(m1.ravel().astype(np.float64), m2.ravel()))
        err_no_add = abs((dot1 - dot2) / dot2)
        self.forward(True, m1, d2)
        self.adjoint(True, m2, d1)
        dot3, dot4 = float(np.dot(d1.ravel().astype(np.float64), d2.ravel())), float(
            np.dot(m1.ravel().astype(np.float64), m2.ravel()))
        err_add = abs((dot3 - dot4) / dot4)
        if verb:
            print(f"WITHOUT ADD: dot1 {dot1:.16g} dot2 {dot2:.16g} error {err_no_add:.3e}")
            print(f"WITH ADD:    dot3 {dot3:.16g} dot4 {dot4:.16g} error {err_add:.3e}")
        return bool(err_no_add <= maxError and err_add <= maxError)

    def dotTestCpp(self, verb=False, maxError=1e-5):
        return self.dotTest(verb, maxError)


class nonlinearPropElasticShotsGpu_3D(_ShotOperatorBase):
    """Nonlinear elastic propagation over shots: source signals -> recorded data.

    forward: model (1 or nExp, 9, nSimSrc, nts) -> data (nExp, 9, nRec, nts).  A model with one
    slice uses the same signals for every shot.  adjoint: data -> model, with the reference's
    time-reversed stepper (its quirk Q7: not the exact transpose in heterogeneous media).
    """

    _slab_capable = True

    def __init__(self, domain, range, elasticParam, paramP, *devices14):
        super().__init__(domain, range, elasticParam, paramP, devices14)

    def forward(self, add, model, data):
        m = np.asarray(_nd(model), dtype=np.float32)
        d = _nd(data)
        if m.shape[1] != 9:
            raise ValueError("number of components in source model different than 9")
        constant = m.shape[0] == 1
        if not add:
            d[...] = 0

        def shot(prop, iExp):
            rec7 = self._rec(iExp)
            src7 = self._srcs(iExp)
            reg = self._scaled_sources(iExp, m[0 if constant else iExp])
            out = prop.nl_forward(reg, [x.getRegPosUnique() for x in src7], [x.getRegPosUnique() for x in rec7])
            res = np.stack([rec7[COMP_GRID[k]].forward(False, out[k]) for k in range(9)])
            with self._lock:
                d[iExp] += res

        self._run_shots(shot)

    def adjoint(self, add, model, data):
        m = _nd(model)
        dd = np.asarray(_nd(data), dtype=np.float32)
        constant = m.shape[0] == 1
        if not add:
            m[...] = 0

        def shot(prop, iExp):
            rec7 = self._rec(iExp)
            src7 = self._srcs(iExp)
            reg = [rec7[COMP_GRID[k]].adjoint(False, None, dd[iExp, k]) for k in range(9)]
            scale_signals(reg, rec7, self.fd.planes, self.fd.dx, self.fd.dy, self.fd.dz)
            out = prop.nl_adjoint(reg, [x.getRegPosUnique() for x in src7], [x.getRegPosUnique() for x in rec7])
            res = np.stack([src7[COMP_GRID[k]].forward(False, out[k]) for k in range(9)])
            with self._lock:
                m[0 if constant else iExp] += res

        self._run_shots(shot)


class nonlinearFwiPropElasticShotsGpu_3D(nonlinearPropElasticShotsGpu_3D):
    """Nonlinear modelling as a function of the elastic parameters (the FWI forward operator):
    forward(add, elasticParam, data) sets the background and models the stored sources."""

    def __init__(self, domain, range, sources, paramP, *devices14):
        self.sources = np.array(_nd(sources), dtype=np.float32, copy=True)
        super().__init__(self.sources, range, domain, paramP, *devices14)
        self.setDomainRange(domain, range)

    def __str__(self):
        return " Ela NLOper 3D "

    def forward(self, add, model, data):
        self.setBackground(model)
        super().forward(add, self.sources, data)

    def adjoint(self, add, model, data):
        raise NotImplementedError("the nonlinear FWI operator has no adjoint; use the Born operator or "
                                  "fwi.ElasticFwiMisfit for gradients")


class BornElasticShotsGpu_3D(_ShotOperatorBase):
    """Born (linearised) elastic modelling over shots: (drho, dlambda, dmu) <-> data."""

    def __init__(self, domain, range, elasticParam, paramP, sourcesSignalsVector, *devices14):
        super().__init__(domain, range, elasticParam, paramP, devices14)
        self.sourcesSignals = [np.asarray(_nd(s), dtype=np.float32) for s in sourcesSignalsVector]
        if len(self.sourcesSignals) not in (1, self.nExp):
            raise ValueError("source signals: one for all shots or one per shot")

    def _born_sources(self, iExp):
        sig = self.sourcesSignals[0 if len(self.sourcesSignals) == 1 else iExp]
        return self._scaled_sources(iExp, sig)

    def forward(self, add, model, data):
        pert = born_model_to_planes(_nd(model), self.fd.scaling(), self.fd.dtw)
        d = _nd(data)
        if not add:
            d[...] = 0

        def shot(prop, iExp):
            rec7 = self._rec(iExp)
            src7 = self._srcs(iExp)
            out = prop.born_forward(self._born_sources(iExp), pert, [x.getRegPosUnique() for x in src7],
                                    [x.getRegPosUnique() for x in rec7])
            res = np.stack([rec7[COMP_GRID[k]].forward(False, out[k]) for k in range(9)])
            with self._lock:
                d[iExp] += res

        self._run_shots(shot)

    def adjoint(self, add, model, data):
        dd = np.asarray(_nd(data), dtype=np.float32)
        m = _nd(model)
        acc = np.zeros((8,) + tuple(self.fd.planes.shape[1:]), dtype=np.float32)

        def shot(prop, iExp):
            rec7 = self._rec(iExp)
            src7 = self._srcs(iExp)
            reg = [rec7[COMP_GRID[k]].adjoint(False, None, dd[iExp, k]) for k in range(9)]
            pert = prop.born_adjoint(self._born_sources(iExp), reg, [x.getRegPosUnique() for x in src7],
                                     [x.getRegPosUnique() for x in rec7])
            with self._lock:
                for k in range(8):
                    acc[k] += pert[k]

        self._run_shots(shot)
        res = born_planes_to_model(acc, self.fd.scaling(), self.fd.dtw)
        if add:
            m += res
        else:
            m[...] = res


class ElasticDatComp_3D:
    """Sampling of data components (dataCompModule_3D.py): vx,vy,vz,sxx,syy,szz,sxz,sxy,syz and
    p = (sxx+syy+szz)/3 (the module's code uses 1/3; its doc string says 0.5).
    Domain (nExp, 9, nRec, nts) -> range (nExp, ncomp, nRec, nts)."""

    NAMES = ["vx", "vy", "vz", "sxx", "syy", "szz", "sxz", "sxy", "syz"]
    P_FACTOR = 1.0 / 3.0

    def __init__(self, components, domain):
        self.comp_list = [c.strip().lower() for c in components.split(",")]
        if len(set(self.comp_list)) != len(self.comp_list):
            raise ValueError("a component was provided multiple times")
        for c in self.comp_list:
            if c not in self.NAMES and c != "p":
                raise ValueError(f"unknown data component: {c}")
        shp = np.shape(_nd(domain))
        self.domain_shape = tuple(shp)
        self.range_shape = (shp[0], len(self.comp_list), shp[2], shp[3])

    def forward(self, add, model, data):
        m, d = _nd(model), _nd(data)
        if not add:
            d[...] = 0
        for i, c in enumerate(self.comp_list):
            if c == "p":
                d[:, i] += (m[:, 3] + m[:, 4] + m[:, 5]) * self.P_FACTOR
            else:
                d[:, i] += m[:, self.NAMES.index(c)]

    def adjoint(self, add, model, data):
        m, d = _nd(model), _nd(data)
        if not add:
            m[...] = 0
        for i, c in enumerate(self.comp_list):
            if c == "p":
                for k in (3, 4, 5):
                    m[:, k] += d[:, i] * self.P_FACTOR
            else:
                m[:, self.NAMES.index(c)] += d[:, i]
