"""GPU: the device-pointer entry points check their position tables before anything is written.

A table entry inside the FAT ring or outside the grid returns E3D_ERR_BOUNDS (as the host-buffer
calls do for host tables); the check only reads the table, so no kernel touches the bad address,
the output signals keep their contents and the context stays usable for a correct call.
"""
import dataclasses

import numpy as np
import pytest
import torch

from cases import prepared, random_signals, rel_l2
from elasticisolib_3d_b200 import _native as N
from elasticisolib_3d_b200.engine import COMP_GRID, Propagator
from oracle import oracle as O

pytestmark = pytest.mark.gpu
E3D_ERR_BOUNDS = 5


def _device_set(pos7):
    pos = [np.asarray(pos7[COMP_GRID[k]], dtype=np.int64) for k in range(9)]
    off = [0]
    for a in pos:
        off.append(off[-1] + len(a))
    return np.concatenate(pos), off


def _time_major(sig9):
    return torch.from_numpy(np.ascontiguousarray(np.concatenate(sig9, axis=0).T)).cuda()


def _bad_tables(p, pos):
    """The table with one entry moved into the FAT ring (z = 2), and with one beyond the grid."""
    fat = pos.copy()
    iy, ix = pos[3] // (p.nz * p.nx), (pos[3] // p.nz) % p.nx
    fat[3] = iy * p.nz * p.nx + ix * p.nz + 2
    out = pos.copy()
    out[-1] = p.nz * p.nx * p.ny + 17
    return [fat, out]


@pytest.mark.parametrize("which", ["source", "receiver"])
def test_nl_propagate_device_rejects_bad_positions(which):
    sv, p, med, src, rec, dtw = prepared(seed=3)
    rng = np.random.default_rng(4)
    spos7 = [d.unique for d in src]
    rpos7 = [d.unique for d in rec]
    sp, soff = _device_set(spos7)
    rp, roff = _device_set(rpos7)
    ssig = _time_major(random_signals(spos7, p.nts, rng))
    pr = Propagator(p.nz, p.nx, p.ny, p.nts, p.sub, p.minPad, p.dz, p.dx, p.dy, p.dts, p.alphaCos)
    pr.set_medium(med)
    pr.set_stream(torch.cuda.current_stream())
    for bad in _bad_tables(p, sp if which == "source" else rp):
        s_dev = torch.from_numpy(bad if which == "source" else sp).cuda()
        r_dev = torch.from_numpy(bad if which == "receiver" else rp).cuda()
        rsig = torch.full((p.nts, roff[9]), 5.0, device="cuda")
        with pytest.raises(N.E3DError) as err:
            pr.nl_propagate_device(False, s_dev, soff, r_dev, roff, ssig, rsig)
        assert err.value.status == E3D_ERR_BOUNDS
        torch.cuda.synchronize()
        assert bool((rsig == 5.0).all())   # nothing was written
    # the context still propagates a correct call, to the oracle's traces
    rsig = torch.zeros((p.nts, roff[9]), device="cuda")
    pr.nl_propagate_device(False, torch.from_numpy(sp).cuda(), soff, torch.from_numpy(rp).cuda(), roff, ssig, rsig)
    torch.cuda.synchronize()
    got = rsig.double().cpu().numpy().T
    # the device tables give every component its own grid's points; the host-buffer calls and the
    # oracle's default also apply the reference's sxz-receiver quirk (Q2), which is off here
    ref = O.nl_forward_reg(dataclasses.replace(p, q2compat=0), med,
                           [ssig.cpu().numpy().T[soff[k]:soff[k + 1]] for k in range(9)], spos7, rpos7, np.float32)
    assert rel_l2([got[roff[k]:roff[k + 1]] for k in range(9)], ref) < 1e-5
    pr.close()


def test_fwi_forward_device_rejects_bad_positions():
    sv, p, med, src, rec, dtw = prepared(seed=5)
    rng = np.random.default_rng(6)
    spos7 = [d.unique for d in src]
    rpos7 = [d.unique for d in rec]
    sp, soff = _device_set(spos7)
    rp, roff = _device_set(rpos7)
    ssig = _time_major(random_signals(spos7, p.nts, rng))
    pr = Propagator(p.nz, p.nx, p.ny, p.nts, p.sub, p.minPad, p.dz, p.dx, p.dy, p.dts, p.alphaCos)
    pr.set_medium(med)
    pr.set_stream(torch.cuda.current_stream())
    bad = _bad_tables(p, rp)[0]
    rsig = torch.full((p.nts, roff[9]), 5.0, device="cuda")
    with pytest.raises(N.E3DError) as err:
        pr.fwi_forward_device(torch.from_numpy(sp).cuda(), soff, torch.from_numpy(bad).cuda(), roff, ssig, rsig)
    assert err.value.status == E3D_ERR_BOUNDS
    torch.cuda.synchronize()
    assert bool((rsig == 5.0).all())
    pr.close()
