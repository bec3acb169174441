"""CPU: the checkpoint schedule the engine runs (e3d_checkpoint_schedule), checked against what
the imaging condition needs, and the velocity-slot windows against the slot counts the memory
plan allocates (FP32: L+3 slots per segment window, FP16: L+2)."""
import pytest

from elasticisolib_3d_b200.engine import checkpoint_schedule


def _needed_blocks(b0, b1, blocks):
    """Source blocks whose decimation completes V[b0 .. min(b1+1, blocks)], the velocities the
    imaging of adjoint blocks [b0, b1) reads (V[its..its+2] for its in [b0, b1)): V[t] takes the
    right weights of block t-1 and the left weights of block t (when t < blocks)."""
    need = set()
    for t in range(b0, min(b1 + 1, blocks) + 1):
        if t - 1 >= 0:
            need.add(t - 1)
        if t < blocks:
            need.add(t)
    return need


CASES = [(1, 1), (2, 1), (2, 5), (3, 1), (10, 3), (31, 4), (31, 5), (31, 31), (39, 7), (999, 572),
         (999, 999), (999, 993), (2499, 170), (2499, 1), (100, 99), (100, 50), (7, 2)]


@pytest.mark.parametrize("blocks,seg", CASES)
def test_schedule_covers_the_imaging_and_fits_the_slots(blocks, seg):
    starts, recomputed = checkpoint_schedule(blocks, seg)
    L = min(seg, blocks)
    nseg = -(-blocks // L)
    assert len(starts) == nseg + 1 and starts[0] == 0 and starts[-1] == blocks
    lengths = [b - a for a, b in zip(starts, starts[1:])]
    assert all(n == L for n in lengths[1:]) and 1 <= lengths[0] <= L
    # every segment but the last is recomputed; the forward pass decimates the last one from
    # the block before it
    total = 0
    for s in range(nseg - 1):
        b0, b1 = starts[s], starts[s + 1]
        need = _needed_blocks(b0, b1, blocks)
        run = set(range(b0 - 1 if s else 0, min(b1 + 1, blocks - 1) + 1))
        assert need <= run
        total += len(run)
        # checkpoint s >= 1 is the state at the start of block b0 - 1
        assert s == 0 or b0 - 1 >= 0
        # FP32 window V[b0 .. b1+2] (the recompute's last block accumulates V[b1+2]) in L+3 slots;
        # FP16 stores V[b0 .. b1+1] in L+2 slots
        last_acc = min(b1 + 1, blocks - 1) + 1
        assert last_acc - b0 < L + 3
        assert min(b1 + 1, blocks) - b0 < L + 2
    assert recomputed == total
    tail = starts[nseg - 1]
    assert _needed_blocks(tail, blocks, blocks) <= set(range(max(tail - 1, 0), blocks))
    assert blocks - tail < L + 2  # V[tail .. blocks] in the slots (both storages)


def test_schedule_rejects_bad_arguments():
    with pytest.raises(ValueError):
        checkpoint_schedule(0, 3)
    with pytest.raises(ValueError):
        checkpoint_schedule(10, 0)


def test_recompute_shrinks_with_the_segment():
    """Longer segments recompute fewer blocks; one segment recomputes none."""
    counts = [checkpoint_schedule(999, L)[1] for L in (50, 100, 200, 500, 998, 999)]
    assert counts == sorted(counts, reverse=True) and counts[-1] == 0


# ---- memory plan (e3d_checkpoint_plan: the choice the checkpointed passes make) -------------
from elasticisolib_3d_b200.engine import checkpoint_plan  # noqa: E402

N288, NY288 = 288 ** 3, 288


def test_plan_fits_its_budget_and_prefers_full_precision_when_all_fits():
    plan = checkpoint_plan(N288, NY288, 1000, 1e13)
    assert plan[:3] == ("fp32", "fp32", 999)
    for budget in (3e10, 6e10, 1.0e11, 1.4e11):
        ck, vt, L, b = checkpoint_plan(N288, NY288, 1000, budget)
        assert b <= budget


def test_plan_takes_16_bit_slots_where_they_cut_recomputation():
    # 288^3 cells, 1000 samples, 143.6 GB: FP32 slots hold about half the record, FP16 slots
    # nearly all of it -- the FP16 plan removes ~490 recomputed blocks and wins
    ck, vt, L, _ = checkpoint_plan(N288, NY288, 1000, 143.6e9)
    assert (ck, vt) == ("fp16", "fp16") and L > 900
    assert checkpoint_schedule(999, L)[1] < 50
    # the all-FP32 plan for the same budget recomputes ~half the record
    ck, vt, L32, _ = checkpoint_plan(N288, NY288, 1000, 143.6e9, "fp32", "fp32")
    assert (ck, vt) == ("fp32", "fp32") and checkpoint_schedule(999, L32)[1] > 400
    # 392^3, 2500 samples: FP16 slots double the segment (about 330 blocks against 160 with FP32
    # slots), which removes about 190 recomputed blocks, more than their 5 % margin of 125
    ck, vt, L, _ = checkpoint_plan(392 * 392 * 388, 388, 2500, 150e9)
    assert (ck, vt) == ("fp16", "fp16") and 300 < L < 450
    ck, vt, L32, _ = checkpoint_plan(392 * 392 * 388, 388, 2500, 150e9, velocity="fp32")
    assert (ck, vt) == ("fp16", "fp32") and 100 < L32 < 250
    assert checkpoint_schedule(2499, L32)[1] - checkpoint_schedule(2499, L)[1] > 0.05 * 2499


def test_plan_respects_explicit_types_and_segment():
    for ckpt in ("fp32", "fp16", "bf16"):
        assert checkpoint_plan(N288, NY288, 1000, 1e11, ckpt)[0] == ckpt
    for vel in ("fp32", "fp16"):
        assert checkpoint_plan(N288, NY288, 1000, 1e11, velocity=vel)[1] == vel
    assert checkpoint_plan(N288, NY288, 1000, 1e11, "fp32", "fp32", segment=7)[2] == 7
    assert checkpoint_plan(N288, NY288, 1000, 1e9) is None


def test_plan_cost_falls_with_more_memory():
    """The chosen plan's cost -- recomputed blocks plus the precision margins (5 % of the blocks
    for 16-bit states, 5 % for 16-bit slots) -- never rises with the budget, and with enough
    memory the all-FP32 plan recomputes nothing."""
    prev = None
    for budget in (3e10, 5e10, 8e10, 1.2e11, 1.6e11, 2.5e11, 3.5e11):
        ck, vt, L, _ = checkpoint_plan(N288, NY288, 1000, budget)
        cost = checkpoint_schedule(999, L)[1] + 999 * (0.05 * (ck != "fp32") + 0.05 * (vt == "fp16"))
        assert prev is None or cost <= prev + 1e-9
        prev = cost
    assert prev == 0
