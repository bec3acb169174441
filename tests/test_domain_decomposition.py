"""CPU: y-slab sizes of the domain decomposition (the reference's rule,
nonlinearPropElasticShotsGpu_3D.cpp:48-76) and the seam's argument checks of the decomposed
propagation (no GPU work: the checks fail before any CUDA call)."""
import ctypes

import pytest

from elasticisolib_3d_b200 import _native as N
from elasticisolib_3d_b200.engine import domain_decomposition

FAT = 4


@pytest.mark.parametrize("ny,n", [(120, 2), (120, 3), (388, 2), (388, 4), (97, 3), (1000, 8)])
def test_slabs_cover_the_grid_with_2fat_overlaps(ny, n):
    sizes = domain_decomposition(ny, n, FAT)
    assert len(sizes) == n
    # slab s covers global planes [Y_s, Y_s + ny_s), Y_{s+1} = Y_s + ny_s - 2 FAT, and the last ends at ny
    y0 = 0
    owned = []
    for sz in sizes:
        assert sz >= 3 * FAT
        owned.append((y0 + FAT, y0 + sz - FAT))
        y0 += sz - 2 * FAT
    assert y0 + 2 * FAT == ny
    # the updated planes [FAT, ny - FAT) are dealt once each
    assert owned[0][0] == FAT and owned[-1][1] == ny - FAT
    assert all(a[1] == b[0] for a, b in zip(owned, owned[1:]))


def test_infeasible_splits_are_refused():
    with pytest.raises(ValueError):
        domain_decomposition(120, 1)
    with pytest.raises(ValueError):
        domain_decomposition(24, 3)
    with pytest.raises(ValueError):
        domain_decomposition(60, 2, FAT, min_pad=30)


def _call(name, ny_domdec, gpus):
    lib = N.lib()
    fn = getattr(lib, name)
    null = ctypes.c_void_p()
    args = [null] * 18 + [null, ctypes.c_longlong(0)] * 14 + [64, 64, 64]
    nd = (ctypes.c_int * max(len(ny_domdec), 1))(*ny_domdec)
    gl = (ctypes.c_int * max(len(gpus), 1))(*gpus)
    return fn(*args, nd, len(ny_domdec), gl, len(gpus))


@pytest.mark.parametrize("name", ["propElasticFwdGpudomDec_3D", "propElasticAdjGpudomDec_3D"])
def test_seam_refuses_bad_decompositions_before_any_gpu_work(name):
    # one slab, mismatched list lengths, slots never allocated
    E3D_ERR_ARG, E3D_ERR_STATE = 1, 3
    assert _call(name, [64], [0]) == E3D_ERR_ARG
    assert _call(name, [36, 36], [0]) == E3D_ERR_ARG
    assert _call(name, [36, 36], [0, 0]) == E3D_ERR_STATE


# ---- admission of shots into batched forward launches (host arithmetic) ----------------------
from elasticisolib_3d_b200.engine import forward_batch_plan  # noqa: E402


def test_batches_fit_the_budget_and_keep_every_shot_once():
    n_cells, nts, sp, rp = 392 * 488 * 488, 2000, 27, 9 * 40000
    per_shot = 18 * n_cells * 4 + nts * (sp + rp) * 4 + 8 * (sp + rp)
    for n_shots in (1, 3, 16, 17):
        for free in (1.2 * per_shot, 3.3 * per_shot, 180e9):
            plan = forward_batch_plan(n_shots, n_cells, nts, sp, rp, free)
            assert sorted(i for b in plan for i in b) == list(range(n_shots))
            assert all(len(b) * per_shot <= 0.9 * free for b in plan)
            sizes = [len(b) for b in plan]
            assert max(sizes) - min(sizes) <= 1          # as even as the budget allows
    # 180 GB: 16 shots of the 93 M-cell grid (2000 samples, 200 x 200 receivers) per launch
    assert len(forward_batch_plan(16, n_cells, nts, sp, rp, 180e9)) == 1
    assert forward_batch_plan(0, n_cells, nts, sp, rp, 180e9) == []


def test_a_shot_that_does_not_fit_is_refused():
    with pytest.raises(ValueError):
        forward_batch_plan(4, 392 * 488 * 488, 2000, 27, 360000, 1e9)
