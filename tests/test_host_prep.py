"""CPU: native host preparation against the oracle's restatements.

  * trilinear acquisition mapping (spaceInterpGpu_3D.cpp:216-348): grid indices, unique points and
    slots bit-exact, weights bit-exact, monopole and dipole, with the reference's dipole
    arithmetic (int-truncated shifts, y offset over dz) and with it corrected;
  * sinc mapping (spaceInterpGpu_3D.cpp:351-480) with the bounds test the reference inverts
    written the right way round: indices exact, weights within one float ulp (the two sides call
    different sin implementations), and properties (a device on a grid point gets weight 1 there
    and ~0 elsewhere; smooth fields are interpolated accurately; stencils outside the array are
    refused);
  * the medium planes and the staggering operators (fdParamElastic_3D.cpp:130-193,
    stagger_3D.cpp:23-208) bit-exact.
"""
import numpy as np
import pytest

from elasticisolib_3d_b200 import hostprep as H
from oracle import oracle as O

PADS = dict(fat=4, zPadMinus=6, zPadPlus=6, xPadMinus=6, xPadPlus=6, yPad=6)


def _par(**kw):
    d = {"fat": 4, "zPadMinus": PADS["zPadMinus"], "zPadPlus": PADS["zPadPlus"], "xPadMinus": PADS["xPadMinus"],
         "xPadPlus": PADS["xPadPlus"], "yPad": PADS["yPad"]}
    d.update(kw)
    return H.ParamObj(d)


def _grid(dz=10.0, dx=10.0, dy=12.5, nz=44, nx=40, ny=36, oz=-3.0, ox=5.0, oy=0.0):
    return [H.Axis(nz, oz, dz), H.Axis(nx, ox, dx), H.Axis(ny, oy, dy)], \
           (O.GridAxis(nz, oz, dz), O.GridAxis(nx, ox, dx), O.GridAxis(ny, oy, dy))


def _devices(axes_o, n, rng, margin):
    """Random devices inside the model interior, `margin` cells away from its faces."""
    out = []
    for a, lo_pad, hi_pad in zip(axes_o, ("zPadMinus", "xPadMinus", "yPad"), ("zPadPlus", "xPadPlus", "yPad")):
        lo = a.o + (PADS["fat"] + PADS[lo_pad] + margin) * a.d
        hi = a.o + (a.n - 1 - PADS["fat"] - PADS[hi_pad] - margin) * a.d
        out.append(rng.uniform(lo, hi, n).astype(np.float32))
    return out


def _same(native, ref, weights_exact=True):
    np.testing.assert_array_equal(native.index, ref.index)
    np.testing.assert_array_equal(native.unique, ref.unique)
    np.testing.assert_array_equal(native.slot, ref.slot)
    if weights_exact:
        np.testing.assert_array_equal(native.weight.view(np.int32), ref.weight.view(np.int32))
    else:
        np.testing.assert_array_max_ulp(native.weight, ref.weight, maxulp=1)


@pytest.mark.parametrize("dipole,shifts,compat", [
    (0, (0.0, 0.0, 0.0), True),
    (1, (20.0, -10.0, 30.0), True),
    (1, (7.5, -3.25, 12.9), True),     # fractional shifts: truncated to int by the reference class
    (1, (7.5, -3.25, 12.9), False),    # corrected: float shifts, y over dy
])
def test_linear_mapping_matches_oracle_bitwise(dipole, shifts, compat):
    rng = np.random.default_rng(11)
    axes_h, axes_o = _grid()
    z, x, y = _devices(axes_o, 200, rng, margin=5)
    if dipole and compat:
        # the reference's second pole divides its y offset by dz (12.5 / 10 here): keep the devices
        # in the lower y cells so that the stretched pole stays inside the model
        ya = axes_o[2]
        y0 = ya.o + (PADS["fat"] + PADS["yPad"]) * ya.d
        y = rng.uniform(y0, y0 + 4 * ya.d, y.shape[0]).astype(np.float32)
    nat = H.spaceInterpGpu_3D(z, x, y, axes_h, 17, _par(), dipole, *shifts, compat=compat)
    ref = O.space_interp_linear(z, x, y, axes_o, PADS, 17, dipole, shifts, compat=compat)
    _same(nat, ref)


def test_linear_compat_and_corrected_agree_where_the_quirks_vanish():
    """Integer shifts with dy == dz: the reference's dipole arithmetic and the corrected one agree."""
    rng = np.random.default_rng(12)
    axes_h, axes_o = _grid(dy=10.0)
    z, x, y = _devices(axes_o, 50, rng, margin=5)
    a = H.spaceInterpGpu_3D(z, x, y, axes_h, 5, _par(), 1, 20.0, -10.0, 30.0, compat=True)
    b = H.spaceInterpGpu_3D(z, x, y, axes_h, 5, _par(), 1, 20.0, -10.0, 30.0, compat=False)
    np.testing.assert_array_equal(a.index, b.index)
    np.testing.assert_array_equal(a.weight, b.weight)


@pytest.mark.parametrize("h,dipole,compat", [(1, 0, True), (2, 0, True), (4, 0, True), (3, 1, True),
                                             (3, 1, False)])
def test_sinc_mapping_matches_oracle(h, dipole, compat):
    rng = np.random.default_rng(13 + h)
    axes_h, axes_o = _grid()
    z, x, y = _devices(axes_o, 60, rng, margin=0)
    shifts = (12.5, -7.0, 5.5)
    nat = H.spaceInterpGpu_3D(z, x, y, axes_h, 9, _par(), dipole, *shifts, interpMethod="sinc", hFilter1d=h,
                              compat=compat)
    ref = O.space_interp_sinc(z, x, y, axes_o, PADS, 9, h, dipole, shifts, compat=compat)
    assert nat.index.shape == (60, (2 * h) ** 3 * (2 if dipole else 1))
    _same(nat, ref, weights_exact=False)
    if dipole:
        half = (2 * h) ** 3
        s1 = nat.weight[:, :half].sum(axis=1)
        s2 = nat.weight[:, half:].sum(axis=1)
        assert np.all(np.sign(s2) == (np.sign(s1) if compat else -np.sign(s1)))


def test_sinc_device_on_a_grid_point():
    axes_h, axes_o = _grid()
    za, xa, ya = axes_o
    iz, ix, iy = 20, 17, 15
    z = np.array([za.o + iz * za.d], np.float32)
    x = np.array([xa.o + ix * xa.d], np.float32)
    y = np.array([ya.o + iy * ya.d], np.float32)
    d = H.spaceInterpGpu_3D(z, x, y, axes_h, 3, _par(), interpMethod="sinc", hFilter1d=4)
    target = (iy * xa.n + ix) * za.n + iz
    k = int(np.nonzero(d.index[0] == target)[0][0])
    assert d.weight[0, k] == np.float32(1.0)
    others = np.delete(d.weight[0], k)
    assert np.max(np.abs(others)) < 1e-6


def test_sinc_interpolates_a_smooth_field():
    """Forward interpolation (regular -> irregular) of a low-wavenumber field sampled on the grid
    recovers its value at the devices; error shrinks as the half length grows."""
    rng = np.random.default_rng(14)
    axes_h, axes_o = _grid(dy=10.0)
    za, xa, ya = axes_o
    z, x, y = _devices(axes_o, 40, rng, margin=0)

    def field(zz, xx, yy):
        return (np.cos(2 * np.pi * zz / 170.0 + 0.3) * np.cos(2 * np.pi * xx / 230.0) *
                np.cos(2 * np.pi * yy / 190.0 - 0.7))

    errs = []
    for h in (2, 4):
        d = H.spaceInterpGpu_3D(z, x, y, axes_h, 1, _par(), interpMethod="sinc", hFilter1d=h)
        iz = d.unique % za.n
        ix = (d.unique // za.n) % xa.n
        iy = d.unique // (za.n * xa.n)
        reg = field(za.o + iz * za.d, xa.o + ix * xa.d, ya.o + iy * ya.d).astype(np.float32)[:, None]
        got = d.forward(False, reg)[:, 0]
        errs.append(float(np.max(np.abs(got - field(z, x, y)))))
    assert errs[1] < errs[0] and errs[1] < 0.05, errs


def test_sinc_stencil_outside_the_array_is_refused():
    axes_h, axes_o = _grid()
    za, xa, ya = axes_o
    # on the first interior row, fat + zPadMinus = 10 cells from the edge: the stencil spans rows
    # 10-h+1 .. 10+h, inside the array up to h = 11
    z = np.array([za.o + 10 * za.d], np.float32)
    x = np.array([xa.o + 20 * xa.d], np.float32)
    y = np.array([ya.o + 18 * ya.d], np.float32)
    d = H.spaceInterpGpu_3D(z, x, y, axes_h, 1, _par(), interpMethod="sinc", hFilter1d=11)
    assert int((d.index % za.n).min()) == 0
    with pytest.raises(Exception):
        H.spaceInterpGpu_3D(z, x, y, axes_h, 1, _par(), interpMethod="sinc", hFilter1d=12)
    with pytest.raises(RuntimeError):
        O.space_interp_sinc(z, x, y, axes_o, PADS, 1, 12)


def test_build_devices_reads_the_interpolation_parameters():
    rng = np.random.default_rng(15)
    axes_h, axes_o = _grid()
    z, x, y = _devices(axes_o, 10, rng, margin=2)
    ax7 = [axes_h] * 7
    par = _par(spaceInterpMethod="sinc", hFilter1d=2, dipole=1, zDipoleShift=10.0, xDipoleShift=0.0,
               yDipoleShift=12.5)
    devs = H.build_devices(z, x, y, ax7, 4, par)
    assert all(d.method == "sinc" and d.index.shape == (10, 2 * 64) for d in devs)
    lin = H.build_devices(z, x, y, ax7, 4, _par())
    assert all(d.method == "linear" and d.index.shape == (10, 8) for d in lin)


def test_medium_planes_match_oracle_bitwise():
    rng = np.random.default_rng(16)
    ny, nx, nz = 14, 12, 16
    vp = rng.uniform(2000, 4000, (ny, nx, nz))
    vs = vp / 1.8
    rho = rng.uniform(1800, 2600, (ny, nx, nz))
    elastic = np.stack([rho, rho * (vp ** 2 - 2 * vs ** 2), rho * vs ** 2]).astype(np.float32)
    dtw = np.float32(0.25e-3)
    got = H.medium_planes(elastic, dtw)
    ref = O.medium_planes(elastic, dtw, np.float32)
    for k in range(8):
        np.testing.assert_array_equal(np.asarray(got[k]).view(np.int32), np.asarray(ref[k]).view(np.int32))


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_stagger_operators_match_oracle_bitwise(axis):
    rng = np.random.default_rng(17 + axis)
    f = rng.standard_normal((9, 11, 13)).astype(np.float32)
    name = "zxy"[axis]
    np.testing.assert_array_equal(H.stagger(f, name), O.stagger_forward(f, axis))
    np.testing.assert_array_equal(H.stagger(f, name, adjoint=True), O.stagger_adjoint(f, axis))


def test_coinciding_devices_share_grid_points():
    """Two devices at one position (and a third sharing a cell corner): unique points appear once,
    in first-seen order, both devices' taps point at the same slots, and the adjoint accumulates
    both signals there -- as the reference's std::map-keyed convertIrregToReg does."""
    axes_h, axes_o = _grid()
    za, xa, ya = axes_o
    z0 = za.o + 20.5 * za.d
    x0 = xa.o + 17.25 * xa.d
    y0 = ya.o + 15.75 * ya.d
    z = np.array([z0, z0, z0 + za.d], np.float32)
    x = np.array([x0, x0, x0], np.float32)
    y = np.array([y0, y0, y0], np.float32)
    nat = H.spaceInterpGpu_3D(z, x, y, axes_h, 4, _par())
    ref = O.space_interp_linear(z, x, y, axes_o, PADS, 4)
    _same(nat, ref)
    assert len(set(nat.unique.tolist())) == len(nat.unique) == 12     # 8 + 4 new corners
    np.testing.assert_array_equal(nat.slot[0], nat.slot[1])
    sig = np.ones((3, 4), np.float32)
    reg = nat.adjoint(False, None, sig)
    np.testing.assert_allclose(reg.sum(axis=0), np.full(4, 3.0), rtol=1e-6)   # weights sum to 1 per device


def test_torch_medium_planes_and_gradient_post_processing_on_the_cpu():
    """The FWI path's torch restatements (fwi.medium_planes, fwi.planes_to_model), run on CPU
    tensors, equal the native medium planes and the oracle's Born gradient post-processing bit
    for bit (on the GPU they are compared through the gradient's FP64 parity)."""
    import torch
    from elasticisolib_3d_b200 import fwi as F
    rng = np.random.default_rng(3)
    ny, nx, nz = 10, 12, 14
    vp = rng.uniform(2000, 4000, (ny, nx, nz))
    vs = vp / 1.8
    rho = rng.uniform(1800, 2600, (ny, nx, nz))
    el = np.stack([rho, rho * (vp ** 2 - 2 * vs ** 2), rho * vs ** 2]).astype(np.float32)
    dtw = np.float32(0.25e-3)
    tp = F.medium_planes(*[torch.from_numpy(el[k]) for k in range(3)], dtw)
    hp = H.medium_planes(el, dtw)
    for k in range(8):
        np.testing.assert_array_equal(tp[k].numpy().view(np.int32), hp[k].view(np.int32))
    g8 = rng.standard_normal((8, ny, nx, nz)).astype(np.float32)
    tm = F.planes_to_model(torch.from_numpy(g8), torch.from_numpy(hp), dtw)
    om = O.born_planes_to_model(g8, hp[0:3], dtw)
    for k in range(3):
        np.testing.assert_array_equal(tm[k].numpy().view(np.int32), np.asarray(om[k]).view(np.int32))


def test_torch_source_scaling_on_the_cpu():
    """fwi.scale_sources (the FWI path's device-side medium scaling of the regular-grid source
    signals, nonlinearPropElasticGpu_3D.cpp:200-277) on CPU tensors equals the oracle's bit for bit."""
    import torch
    from operator_case import OperatorCase
    from elasticisolib_3d_b200 import fwi as F
    from elasticisolib_3d_b200.engine import COMP_GRID
    c = OperatorCase()
    src7 = c.src_dev[0]
    rng = np.random.default_rng(2)
    reg = [rng.standard_normal((len(src7[COMP_GRID[k]].unique), c.nts)).astype(np.float32) for k in range(9)]
    planes = H.medium_planes(c.sv.elastic, np.float32(c.dtw))
    dz, dx, dy = c.d
    got = F.scale_sources(torch.from_numpy(np.concatenate(reg, axis=0).T.copy()), F.DeviceSet.from_devices(src7, "cpu"),
                          torch.from_numpy(planes), np.float32(dx), np.float32(dy), np.float32(dz))
    ref = [r.copy() for r in reg]
    O.scale_signals(ref, c.o_src[0], planes, dx, dy, dz)
    np.testing.assert_array_equal(got.numpy().view(np.int32), np.concatenate(ref, axis=0).T.view(np.int32))
