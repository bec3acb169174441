"""CPU, two gloo ranks: shot sharding and the misfit/gradient all-reduce of the multi-GPU FWI
path, checked against the serial sum (the per-shot gradient is replaced by a CPU stand-in)."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from elasticisolib_3d_b200.fwi import reduce_misfit, shard_shots


def _fake_shot(i, shape):
    g = torch.Generator().manual_seed(100 + i)
    # misfits with digits below FP32 resolution: the reduced total must keep them
    return (torch.tensor(1e8 + float(i + 1) ** 2 + 0.125 * (i + 1), dtype=torch.float64),
            [torch.randn(shape, generator=g) for _ in range(3)])


def _worker(rank, world, port, n_shots, shape, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        total = torch.zeros((), dtype=torch.float64)
        grads = [torch.zeros(shape) for _ in range(3)]
        for i in shard_shots(n_shots, rank, world):
            l, g = _fake_shot(i, shape)
            total += l
            for a, b in zip(grads, g):
                a += b
        total, grads = reduce_misfit(total, grads)
        out[rank] = (float(total), [g.clone() for g in grads])
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_shards_cover_every_shot_once():
    for n in (1, 5, 32):
        for w in (1, 2, 3, 8):
            got = sorted(sum((shard_shots(n, r, w) for r in range(w)), []))
            assert got == list(range(n))


@pytest.mark.timeout(120)
def test_two_rank_reduction_matches_serial_sum():
    n_shots, shape = 5, (3, 4, 6)
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(2, _free_port(), n_shots, shape, out), nprocs=2, join=True,
                       start_method="spawn")
    serial_loss = 0.0
    serial = [torch.zeros(shape) for _ in range(3)]
    for i in range(n_shots):
        l, g = _fake_shot(i, shape)
        serial_loss += float(l)
        for a, b in zip(serial, g):
            a += b
    for r in range(2):
        loss, grads = out[r]
        assert abs(loss - serial_loss) < 1e-3   # an FP32 misfit would be off by ~10 at 5e8
        for a, b in zip(grads, serial):
            assert torch.allclose(a, b, atol=1e-5)


def _dynamic_worker(rank, world, port, n_shots, shape, out):
    import time
    from elasticisolib_3d_b200.fwi import ShotQueue, rendezvous_store
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        store = rendezvous_store(timeout_s=60.0)
        results = []
        for evaluation in range(2):  # two evaluations: distinct counters, every shot dealt in each
            total = torch.zeros((), dtype=torch.float64)
            grads = [torch.zeros(shape) for _ in range(3)]
            mine = []
            for i in ShotQueue(n_shots, f"e3d/shots/test/{evaluation}", store):
                time.sleep(0.02 if rank == 0 else 0.12)  # rank 1's shots are six times as costly
                l, g = _fake_shot(i, shape)
                total += l
                for a, b in zip(grads, g):
                    a += b
                mine.append(i)
            total, grads = reduce_misfit(total, grads)
            results.append((mine, float(total), [g.clone() for g in grads]))
        out[rank] = results
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_dynamic_dealing_covers_every_shot_once_and_balances():
    n_shots, shape = 12, (3, 4, 5)
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_dynamic_worker, args=(2, _free_port(), n_shots, shape, out), nprocs=2, join=True,
                       start_method="spawn")
    serial_loss = sum(float(_fake_shot(i, shape)[0]) for i in range(n_shots))
    for evaluation in range(2):
        m0, m1 = out[0][evaluation][0], out[1][evaluation][0]
        assert sorted(m0 + m1) == list(range(n_shots))
        assert len(m0) > len(m1)  # the faster rank took more shots
        for r in range(2):
            assert abs(out[r][evaluation][1] - serial_loss) < 1e-3


def _broadcast_worker(rank, world, port, out):
    from elasticisolib_3d_b200.fwi import broadcast_model
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g = torch.Generator().manual_seed(7 + rank)   # every rank starts from a different medium
        model = [torch.rand((3, 4, 5), generator=g) + 1.0 for _ in range(3)]
        out[rank] = [t.clone() for t in broadcast_model(model)]
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_model_broadcast_makes_every_rank_use_the_first_ranks_medium():
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_broadcast_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    g = torch.Generator().manual_seed(7)
    ref = [torch.rand((3, 4, 5), generator=g) + 1.0 for _ in range(3)]
    for r in range(2):
        for a, b in zip(out[r], ref):
            assert torch.equal(a, b)
