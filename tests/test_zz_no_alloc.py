"""GPU: the allocation-free propagation entry point against the context-based one.

e3d_nl_propagate_device_noalloc is for callers that cannot allocate device
memory while they propagate: a host framework that already holds most of the
device's memory in its own pool, or a loop that must not call cudaMalloc or
cudaFree (which can synchronize the whole device).  It keeps both wavefield
levels in one fixed device array that every call reuses, so each check below
makes two calls in a row and compares both with e3d_nl_propagate_device, which
allocates its wavefields per context.  Both run the "plain" stepper, so the
results agree to the parity tolerance (1e-5 relative L2) and in practice
bit for bit.

The file name sorts last, so a run that stops at the first failure has run
every other test before this one.
"""
import ctypes

import numpy as np
import pytest
import torch

from cases import prepared, random_signals, rel_l2
from elasticisolib_3d_b200 import _native as N
from elasticisolib_3d_b200.engine import COMP_GRID, Propagator

pytestmark = pytest.mark.gpu


def _device_set(pos7):
    pos = [np.asarray(pos7[COMP_GRID[k]], dtype=np.int64) for k in range(9)]
    off = [0]
    for a in pos:
        off.append(off[-1] + len(a))
    return torch.from_numpy(np.concatenate(pos)).cuda(), off


def _time_major(sig9):
    return torch.from_numpy(np.ascontiguousarray(np.concatenate(sig9, axis=0).T)).cuda()


def _noalloc(p, planes, adjoint, spos, soff, rpos, roff, ssig, rsig):
    desc = N.E3DDesc(0, p.nz, p.nx, p.ny, p.nts, p.sub, p.minPad, p.dz, p.dx, p.dy, p.dts, p.alphaCos, 0, 1, 1)
    so = (ctypes.c_int * 10)(*soff)
    ro = (ctypes.c_int * 10)(*roff)
    stream = torch.cuda.current_stream().cuda_stream
    N.call("e3d_nl_propagate_device_noalloc", ctypes.byref(desc), N.ptr_array([planes[k] for k in range(8)]),
           int(adjoint), spos.data_ptr(), so, rpos.data_ptr(), ro, ssig.data_ptr(), rsig.data_ptr(), stream)
    torch.cuda.current_stream().synchronize()


@pytest.mark.parametrize("adjoint", [False, True])
def test_noalloc_matches_context_entry_point_twice(adjoint):
    sv, p, med, src, rec, dtw = prepared(seed=7)
    rng = np.random.default_rng(11)
    spos7 = [d.unique for d in src]
    rpos7 = [d.unique for d in rec]
    spos, soff = _device_set(spos7)
    rpos, roff = _device_set(rpos7)
    planes = torch.from_numpy(np.ascontiguousarray(med)).cuda()

    pr = Propagator(p.nz, p.nx, p.ny, p.nts, p.sub, p.minPad, p.dz, p.dx, p.dy, p.dts, p.alphaCos)
    pr.set_stepper_variant(8, 2, "plain")
    pr.set_medium(planes)
    pr.set_stream(torch.cuda.current_stream())

    for call in range(2):
        # fresh inputs on each call: the second call must not see the first call's wavefields
        if adjoint:
            rsig = _time_major(random_signals(rpos7, p.nts, rng))
            ref_s = torch.full((p.nts, soff[9]), 7.0, device="cuda")
            got_s = torch.full((p.nts, soff[9]), -3.0, device="cuda")
            pr.nl_propagate_device(True, spos, soff, rpos, roff, ref_s, rsig)
            torch.cuda.synchronize()
            _noalloc(p, planes, True, spos, soff, rpos, roff, got_s, rsig)
            ref, got = ref_s, got_s
        else:
            ssig = _time_major(random_signals(spos7, p.nts, rng))
            ref_r = torch.full((p.nts, roff[9]), 7.0, device="cuda")
            got_r = torch.full((p.nts, roff[9]), -3.0, device="cuda")
            pr.nl_propagate_device(False, spos, soff, rpos, roff, ssig, ref_r)
            torch.cuda.synchronize()
            _noalloc(p, planes, False, spos, soff, rpos, roff, ssig, got_r)
            ref, got = ref_r, got_r
        r = ref.double().cpu().numpy()
        g = got.double().cpu().numpy()
        assert np.abs(r).max() > 0, call
        assert rel_l2([g], [r]) < 1e-5, (call, rel_l2([g], [r]))


def test_noalloc_rejects_oversized_grid():
    limit = int(N.lib().e3d_noalloc_work_bytes())
    assert limit == 64 << 20
    n = 112  # 112^3 cells need 18 * 4 * 112^3 bytes, above the 64 MiB array
    assert 18 * 4 * n ** 3 > limit
    desc = N.E3DDesc(0, n, n, n, 10, 4, 8, 10.0, 10.0, 10.0, 0.002, 0.99, 0, 1, 1)
    dummy = torch.zeros(1, device="cuda")
    off = (ctypes.c_int * 10)(*([0] * 10))
    st = N.lib().e3d_nl_propagate_device_noalloc(ctypes.byref(desc), N.ptr_array([dummy] * 8), 0, None, off, None,
                                                 off, None, None, None)
    assert st == 1  # E3D_ERR_ARG
    assert b"static work memory" in N.lib().e3d_last_error()


def test_noalloc_rejects_positions_in_the_fat_ring():
    """A position table with an entry inside the FAT ring returns E3D_ERR_BOUNDS before anything is
    written: the output signals keep their contents, and the next correct call still agrees with the
    context entry point."""
    sv, p, med, src, rec, dtw = prepared(seed=8)
    rng = np.random.default_rng(12)
    spos7 = [d.unique for d in src]
    rpos7 = [d.unique for d in rec]
    spos, soff = _device_set(spos7)
    rpos, roff = _device_set(rpos7)
    planes = torch.from_numpy(np.ascontiguousarray(med)).cuda()
    ssig = _time_major(random_signals(spos7, p.nts, rng))
    bad = rpos.clone()
    q = int(bad[0])
    bad[0] = (q // (p.nz * p.nx)) * p.nz * p.nx + ((q // p.nz) % p.nx) * p.nz + 1   # z = 1: the FAT ring
    out = torch.full((p.nts, roff[9]), 5.0, device="cuda")
    desc = N.E3DDesc(0, p.nz, p.nx, p.ny, p.nts, p.sub, p.minPad, p.dz, p.dx, p.dy, p.dts, p.alphaCos, 0, 1, 1)
    so = (ctypes.c_int * 10)(*soff)
    ro = (ctypes.c_int * 10)(*roff)
    stream = torch.cuda.current_stream().cuda_stream
    st = N.lib().e3d_nl_propagate_device_noalloc(ctypes.byref(desc), N.ptr_array([planes[k] for k in range(8)]), 0,
                                                 spos.data_ptr(), so, bad.data_ptr(), ro, ssig.data_ptr(),
                                                 out.data_ptr(), stream)
    torch.cuda.synchronize()
    assert st == 5  # E3D_ERR_BOUNDS
    assert bool((out == 5.0).all())
    pr = Propagator(p.nz, p.nx, p.ny, p.nts, p.sub, p.minPad, p.dz, p.dx, p.dy, p.dts, p.alphaCos)
    pr.set_stepper_variant(8, 2, "plain")
    pr.set_medium(planes)
    pr.set_stream(torch.cuda.current_stream())
    ref = torch.zeros((p.nts, roff[9]), device="cuda")
    pr.nl_propagate_device(False, spos, soff, rpos, roff, ssig, ref)
    torch.cuda.synchronize()
    _noalloc(p, planes, False, spos, soff, rpos, roff, ssig, out)
    assert rel_l2([out.double().cpu().numpy()], [ref.double().cpu().numpy()]) < 1e-5
    pr.close()
