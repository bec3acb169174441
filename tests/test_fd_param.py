"""CPU: fdParamElastic_3D's parameter handling and QC (fdParamElastic_3D.cpp:13-195, 271-313):
internal sub = 2 x the parfile value, ntw and dtw; minPad and the free surface's top pad; the
mod_par = 2 km->m scaling; and the rejections (Courant > 0.45, dispersion < 3 points per
wavelength, grids off the block size, inconsistent cubes)."""
import numpy as np
import pytest

from elasticisolib_3d_b200 import hostprep as H
from elasticisolib_3d_b200 import synthetic as S


def _case(nts=21, dts=0.002, sub=2, fmax=30.0, vp=2500.0, free_surface=False, d=10.0):
    axes, pads = S.make_grid(16, 16, 8, 6, d, free_surface=free_surface)
    shape = (axes[2].n, axes[1].n, axes[0].n)
    el = S.elastic_from_velocity(np.full(shape, vp), np.full(shape, vp / 1.732), np.full(shape, 2000.0))
    par = S.base_params(axes, pads, nts, dts, sub, fmax, free_surface=free_surface)
    return el, axes, par, pads


def test_time_axes_and_pads():
    el, axes, par, pads = _case(nts=21, sub=3)
    fd = H.FdParam(el, axes, par)
    assert fd.sub == 6 and fd.ntw == 20 * 6 + 1
    assert fd.dtw == np.float32(np.float32(0.002) / np.float32(6))
    assert fd.minPad == min(pads["zPadMinus"], pads["zPadPlus"], pads["xPadMinus"], pads["xPadPlus"])
    np.testing.assert_array_equal(fd.planes, H.medium_planes(el, fd.dtw))


def test_free_surface_takes_the_bottom_pad():
    el, axes, par, pads = _case(free_surface=True)
    fd = H.FdParam(el, axes, par)
    assert fd.freeSurface == 1 and fd.zPad == pads["zPadPlus"]


def test_mod_par_2_scales_samplings_by_1000():
    el, axes, par, _ = _case(d=0.01)   # km
    par["mod_par"] = 2
    par["fMax"] = 30.0
    fd = H.FdParam(el, axes, par)
    assert abs(float(fd.dz) - 10.0) < 1e-4 and abs(float(fd.ox) - 1000.0 * np.float32(axes[1].o)) < 1e-2


def test_rejections():
    el, axes, par, _ = _case(dts=0.02)            # Courant far above 0.45
    with pytest.raises(RuntimeError, match="Courant"):
        H.FdParam(el, axes, par)
    el, axes, par, _ = _case(fmax=200.0)           # a few cells per shortest wavelength
    with pytest.raises(RuntimeError, match="Dispersion"):
        H.FdParam(el, axes, par)
    el, axes, par, _ = _case()
    par["blockSize"] = 12
    with pytest.raises(RuntimeError, match="blockSize"):
        H.FdParam(el, axes, par)
    el, axes, par, _ = _case()
    with pytest.raises(RuntimeError, match="consistent"):
        H.FdParam(el[:, :-1], axes, par)
    el, axes, par, _ = _case(sub=60)               # internal 120 > SUB_MAX
    with pytest.raises(RuntimeError, match="SUB_MAX"):
        H.FdParam(el, axes, par)


def test_parfile_parsing():
    """SEP parfile / command-line style 'key=value' tokens, with the getters' conversions."""
    par = H.ParamObj.from_parfile("nts=1000 dts=0.002 sub=2\n# a comment line\nspaceInterpMethod=sinc "
                                  "zDipoleShift=7.5 fMax=40")
    assert par.getInt("nts") == 1000 and abs(par.getFloat("dts") - 0.002) < 1e-12
    assert par.getString("spaceInterpMethod") == "sinc"
    assert par.getInt("zDipoleShift") == 7 and par.getFloat("zDipoleShift") == 7.5
    assert par.getInt("fMax") == 40 and par.getFloat("fMax") == 40.0
    assert par.getInt("nExp", -1) == -1
    with pytest.raises(KeyError):
        par.getInt("nExp")
