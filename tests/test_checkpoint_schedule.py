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
