"""GPU: several shots advanced by one stepper launch per fine step (e3d_nl_forward_batch_device)
equal the same shots propagated one at a time, and every shot matches the FP64 oracle.

The batched stepper runs each shot's cells with the single-shot arithmetic, so the traces agree to
FP32 rounding (1e-6 relative L2); against the FP64 oracle the bound is the parity tests' 1e-5.
"""
import dataclasses

import numpy as np
import pytest

from cases import prepared, random_signals, rel_l2
from elasticisolib_3d_b200.engine import Propagator
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _shots(nshots, seed):
    sv, p, med, src, rec, dtw = prepared(seed=seed, nshots=nshots)
    par = sv.par
    za, xa, ya = sv.axes
    ax7 = O.staggered_axes(za.n, xa.n, ya.n, za.o, xa.o, ya.o, za.d, xa.d, ya.d)
    pads = dict(fat=4, zPadMinus=par.getInt("zPadMinus"), zPadPlus=par.getInt("zPadPlus"),
                xPadMinus=par.getInt("xPadMinus"), xPadPlus=par.getInt("xPadPlus"), yPad=par.getInt("yPad"))
    spos = [[d.unique for d in O.build_devices(*sv.src_xyz[s], ax7, pads, p.nts)] for s in range(nshots)]
    return p, med, spos, [d.unique for d in rec]


@pytest.mark.parametrize("nshots,q2", [(1, 1), (3, 1), (3, 0), (5, 0)])
def test_batched_forward_equals_single_shots(nshots, q2):
    p, med, spos, rpos = _shots(nshots, seed=6)
    rng = np.random.default_rng(7)
    models = [random_signals(sp, p.nts, rng) for sp in spos]
    pr = Propagator(p.nz, p.nx, p.ny, p.nts, p.sub, p.minPad, p.dz, p.dx, p.dy, p.dts, p.alphaCos, q2compat=q2)
    pr.set_stepper_variant(8, 3, "split-fwd")
    pr.set_medium(med)
    batched = pr.nl_forward_batch(models, spos, rpos)
    for s in range(nshots):
        single = pr.nl_forward(models[s], spos[s], rpos)
        e = rel_l2(batched[s], single)
        print(f"{nshots} shots (q2compat {q2}), shot {s}: batched vs single {e:.2e}")
        assert max(float(np.abs(x).max()) for x in single) > 0
        assert e < 1e-6, (s, e)
    if q2 == 0:
        for s in range(nshots):
            # the oracle with the same receiver rule (sxz receivers on their own table)
            p0 = dataclasses.replace(p, q2compat=0)
            ref = O.nl_forward_reg(p0, med.astype(np.float64), [m.astype(np.float64) for m in models[s]], spos[s],
                                   rpos, np.float64)
            assert rel_l2(batched[s], ref) < 1e-5
    pr.close()


def test_batched_forward_rejects_a_position_outside_its_shot():
    """A stacked table whose entry leaves the stacked fields is refused before any write
    (device validation), and the context stays usable."""
    import torch
    from elasticisolib_3d_b200 import _native as N
    p, med, spos, rpos = _shots(2, seed=8)
    rng = np.random.default_rng(9)
    models = [random_signals(sp, p.nts, rng) for sp in spos]
    pr = Propagator(p.nz, p.nx, p.ny, p.nts, p.sub, p.minPad, p.dz, p.dx, p.dy, p.dts, p.alphaCos, q2compat=0)
    pr.set_medium(med)
    bt = pr.batch_tables(models, spos, rpos)
    good = bt.src_pos.clone()
    bt.src_pos[-1] = 2 * p.nz * p.nx * p.ny + 5
    with pytest.raises(N.E3DError):
        pr.nl_forward_batch_device(bt)
    bt.src_pos.copy_(good)
    pr.nl_forward_batch_device(bt)
    N.call("e3d_synchronize", pr.handle)
    got = bt.split(bt.rec_sig.cpu().numpy().T)
    assert rel_l2(got[1], pr.nl_forward(models[1], spos[1], rpos)) < 1e-6
    del torch
    pr.close()


def test_batched_forward_with_different_record_lengths():
    """Shots of one batch may have different record lengths (the widths of their source blocks):
    a shorter shot's traces are the first samples of the same shot propagated on the context's
    time axis with zero sources after its end."""
    p, med, spos, rpos = _shots(3, seed=12)
    rng = np.random.default_rng(13)
    lengths = [p.nts, p.nts - 5, p.nts - 9]
    models = [[m[:, :L].copy() for m in random_signals(sp, p.nts, rng)] for sp, L in zip(spos, lengths)]
    pr = Propagator(p.nz, p.nx, p.ny, p.nts, p.sub, p.minPad, p.dz, p.dx, p.dy, p.dts, p.alphaCos, q2compat=0)
    pr.set_medium(med)
    batched = pr.nl_forward_batch(models, spos, rpos)
    for s, L in enumerate(lengths):
        padded = [np.pad(m, ((0, 0), (0, p.nts - L))) for m in models[s]]
        single = pr.nl_forward(padded, spos[s], rpos)
        assert all(b.shape[1] == L for b in batched[s])
        e = rel_l2(batched[s], [x[:, :L] for x in single])
        print(f"record length {L} of {p.nts}: batched vs single {e:.2e}")
        assert e < 1e-6
    pr.close()


def test_shots_admitted_by_memory_budget_equal_one_batch():
    """nl_forward_shots deals the shots into batched launches by a memory budget; with a budget
    that admits two shots per launch, three shots run as two launches and give the traces of one
    batch of three."""
    from elasticisolib_3d_b200.engine import forward_batch_plan
    p, med, spos, rpos = _shots(3, seed=14)
    rng = np.random.default_rng(15)
    models = [random_signals(sp, p.nts, rng) for sp in spos]
    pr = Propagator(p.nz, p.nx, p.ny, p.nts, p.sub, p.minPad, p.dz, p.dx, p.dy, p.dts, p.alphaCos, q2compat=0)
    pr.set_medium(med)
    n = p.nz * p.nx * p.ny
    sp = max(sum(len(s[O.COMP_GRID[k]]) for k in range(9)) for s in spos)
    rp = sum(len(rpos[O.COMP_GRID[k]]) for k in range(9))
    per_shot = 18 * n * 4 + p.nts * (sp + rp) * 4 + 8 * (sp + rp)
    budget = 2.5 * per_shot / 0.9
    assert [len(b) for b in forward_batch_plan(3, n, p.nts, sp, rp, budget)] == [2, 1]
    dealt = pr.nl_forward_shots(models, spos, rpos, free_bytes=budget)
    whole = pr.nl_forward_batch(models, spos, rpos)
    for s in range(3):
        assert rel_l2(dealt[s], whole[s]) < 1e-6
    pr.close()
