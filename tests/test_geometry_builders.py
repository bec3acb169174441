"""CPU: the reference's geometry builders (buildSourceGeometry_3D / buildReceiversGeometry_3D,
Elastic_iso_float_3D.py:21-385), with the geometry passed as an array: per-grid lists equal to
building each shot's devices directly, the reference's consistency checks, and its parameter
reading (sinc, dipole shifts read as int on the receiver side)."""
import numpy as np
import pytest

from operator_case import OperatorCase
from elasticisolib_3d_b200 import hostprep as H
from elasticisolib_3d_b200 import operators as OP


def _geom(points):
    """[(z, x, y) arrays per shot] -> (3, nPoints, nExp), rows x, y, z."""
    return np.stack([np.stack([np.atleast_1d(x), np.atleast_1d(y), np.atleast_1d(z)]) for (z, x, y) in points],
                    axis=-1).astype(np.float32)


def _par(c, **kw):
    # a numpy elastic parameter carries no hypercube: its origins come from oz/ox/oy
    za, xa, ya = c.axes
    p = H.ParamObj(dict(c.par))
    p.update(nExp=2, nReceiverPerShot=c.n_rec, oz=za.o, ox=xa.o, oy=ya.o)
    p.update(kw)
    return p


def test_builders_match_per_shot_devices():
    c = OperatorCase()
    par = _par(c)
    el = c.sv.elastic
    *src7, src_axis = OP.buildSourceGeometry_3D(par, el, _geom(c.sv.src_xyz))
    *rec7, rec_axis = OP.buildReceiversGeometry_3D(par, el, _geom([c.sv.rec_xyz]))
    assert src_axis.n == 2 and rec_axis.n == c.n_rec
    for g in range(7):
        assert len(src7[g]) == 2 and len(rec7[g]) == 1
        for i in range(2):
            np.testing.assert_array_equal(src7[g][i].unique, c.src_dev[i][g].unique)
            np.testing.assert_array_equal(src7[g][i].weight, c.src_dev[i][g].weight)
        np.testing.assert_array_equal(rec7[g][0].unique, c.rec_dev[g].unique)
        np.testing.assert_array_equal(rec7[g][0].slot, c.rec_dev[g].slot)
    # the result is the operators' 14 acquisition arguments
    assert [len(v) for v in src7 + rec7] == [len(v) for v in c.devices14]


def test_builders_check_consistency_like_the_reference():
    c = OperatorCase()
    el = c.sv.elastic
    with pytest.raises(ValueError):
        OP.buildSourceGeometry_3D(_par(c, nExp=3), el, _geom(c.sv.src_xyz))
    with pytest.raises(ValueError):
        OP.buildReceiversGeometry_3D(_par(c, nReceiverPerShot=c.n_rec + 1), el, _geom([c.sv.rec_xyz]))
    with pytest.raises(ValueError):
        OP.buildSourceGeometry_3D(_par(c, spaceInterpMethod="cubic"), el, _geom(c.sv.src_xyz))
    p = _par(c)
    del p["nExp"]
    with pytest.raises(ValueError):
        OP.buildSourceGeometry_3D(p, el, _geom(c.sv.src_xyz))   # nExp missing


def test_builders_read_interpolation_parameters():
    c = OperatorCase()
    el = c.sv.elastic
    par = _par(c, spaceInterpMethod="sinc", hFilter1d=2, dipole=1, zDipoleShift=12.5, xDipoleShift=0.0,
               yDipoleShift=0.0)
    *src7, _ = OP.buildSourceGeometry_3D(par, el, _geom(c.sv.src_xyz))
    *rec7, _ = OP.buildReceiversGeometry_3D(par, el, _geom([c.sv.rec_xyz]))
    assert src7[0][0].method == "sinc" and src7[0][0].index.shape[1] == 2 * 64
    # the receiver builder reads the shifts with getInt: 12.5 -> 12 (then truncated again by the
    # class); the source builder with getFloat, truncated to 12 only by the class
    za, xa, ya = c.axes
    ax7 = H.grid_axes(za.n, xa.n, ya.n, za.o, xa.o, ya.o, za.d, xa.d, ya.d)
    z, x, y = c.sv.rec_xyz
    direct = H.spaceInterpGpu_3D(z, x, y, ax7[0], c.nts, par, 1, 12.0, 0.0, 0.0, interpMethod="sinc", hFilter1d=2)
    np.testing.assert_array_equal(rec7[0][0].index, direct.index)
    # receivers with sinc need hFilter1d
    p = _par(c, spaceInterpMethod="sinc")
    with pytest.raises(KeyError):
        OP.buildReceiversGeometry_3D(p, el, _geom([c.sv.rec_xyz]))
