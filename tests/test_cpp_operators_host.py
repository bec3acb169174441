"""CPU: the C++ operator module loads, and its host parts (parameters, acquisition mapping)
agree with the Python host preparation bit for bit."""
import numpy as np
import pytest

from operator_case import OperatorCase
from elasticisolib_3d_b200 import hostprep as H
from elasticisolib_3d_b200 import pyElastic_iso_float_3D as P


def _cpp_grids(c):
    za, xa, ya = c.axes
    ax7 = H.grid_axes(za.n, xa.n, ya.n, za.o, xa.o, ya.o, za.d, xa.d, ya.d)
    return [P.hypercube([P.axis(a.n, a.o, a.d) for a in g]) for g in ax7]


def test_space_interp_matches_python_host_preparation():
    c = OperatorCase()
    par = P.paramObj(dict(c.par))
    grids = _cpp_grids(c)
    z, x, y = c.sv.rec_xyz
    for g in range(7):
        cpp = P.spaceInterpGpu_3D(z, x, y, grids[g], c.nts, par)
        np.testing.assert_array_equal(np.asarray(cpp.getRegPosUnique()), c.rec_dev[g].getRegPosUnique())
        assert cpp.getNDeviceIrreg() == c.rec_dev[g].getNDeviceIrreg()


@pytest.mark.parametrize("method,h,dipole,compat", [("linear", 1, 1, 1), ("linear", 1, 1, 0), ("sinc", 2, 0, 1),
                                                     ("sinc", 2, 1, 0)])
def test_space_interp_methods_match_python_host_preparation(method, h, dipole, compat):
    c = OperatorCase()
    par = P.paramObj(dict(c.par))
    grids = _cpp_grids(c)
    za, xa, ya = c.axes
    ax7 = H.grid_axes(za.n, xa.n, ya.n, za.o, xa.o, ya.o, za.d, xa.d, ya.d)
    # the receivers line the interior's edges, where a shifted linear pole would leave it: use
    # the sources of every shot
    z, x, y = (np.concatenate([np.atleast_1d(s[k]) for s in c.sv.src_xyz]) for k in range(3))
    shifts = (float(za.d), 0.5 * float(xa.d), float(ya.d))
    for g in (0, 3, 6):
        cpp = P.spaceInterpGpu_3D(z, x, y, grids[g], c.nts, par, dipole, *shifts, method, h, compat)
        py = H.spaceInterpGpu_3D(z, x, y, ax7[g], c.nts, c.par, dipole, *shifts, interpMethod=method,
                                 hFilter1d=h, compat=bool(compat))
        np.testing.assert_array_equal(np.asarray(cpp.getRegPosUnique()), py.getRegPosUnique())
        assert cpp.getNDeviceIrreg() == py.getNDeviceIrreg()


def test_param_object_defaults():
    par = P.paramObj({"nts": 12, "dts": 0.002})
    assert par.getInt("nts") == 12
    assert abs(par.getFloat("dts") - 0.002) < 1e-9
    assert par.getInt("nGpu", 1) == 1
    assert par.getString("iGpu", "-1") == "-1"


def test_cpp_fd_param_matches_python():
    """The C++ operators' fdParamElastic_3D: time axes, minPad and the eight medium planes equal
    the Python host preparation's, bit for bit; the same QC rejects a Courant violation."""
    c = OperatorCase()
    za, xa, ya = c.axes
    h = P.hypercube([P.axis(za.n, za.o, za.d), P.axis(xa.n, xa.o, xa.d), P.axis(ya.n, ya.o, ya.d), P.axis(3)])
    el = np.ascontiguousarray(c.sv.elastic, dtype=np.float32)
    cpp = P.fdParamElastic_3D(P.float4DReg(h, el.copy()), P.paramObj(dict(c.par)))
    py = H.FdParam(el, c.axes, c.par)
    assert (cpp.nz, cpp.nx, cpp.ny, cpp.nts, cpp.sub, cpp.minPad) == (py.nz, py.nx, py.ny, py.nts, py.sub, py.minPad)
    assert np.float32(cpp.dtw) == py.dtw
    np.testing.assert_array_equal(cpp.getPlanes().view(np.int32), py.planes.view(np.int32))
    bad = dict(c.par)
    bad["dts"] = 0.05
    with pytest.raises(RuntimeError, match="Courant"):
        P.fdParamElastic_3D(P.float4DReg(h, el.copy()), P.paramObj(bad))
