"""CPU: bench.py's host-side bookkeeping for every stepper and imaging choice it accepts -- the
kernel labels, the ncu summaries whose DRAM bytes it reports and the algorithmic bytes per cell
(no GPU work)."""
import itertools
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402

KINDS = (0, 1, 2, 3, 5, 6, 7)


@pytest.mark.parametrize("variant,imaging", list(itertools.product(
    ["split", "split-pair", "tma", "plain", "auto"], ["auto", "cells", "tma", "tma-levels", "tma-levels-4"])))
def test_labels_profiles_and_bytes_for_every_choice(variant, imaging):
    args = bench.parse(["--variant", variant, "--imaging", imaging])
    names = bench.kind_names(args)
    assert set(KINDS) <= set(names)
    for kind in KINDS:
        prof = bench.profiled(kind, args)
        if prof is not None:
            assert os.path.exists(prof), prof
            assert any(line.startswith("dram_bytes_per_cell:") for line in open(prof))
        for prem in (False, True):
            assert bench.kind_bytes(kind, 4, prem, dual=variant != "plain") > 0


def test_default_command_reports_the_paired_stepper_profile():
    args = bench.parse([])
    assert args.variant == "split-pair" and args.imaging == "auto"
    assert bench.profiled(0, args).endswith("kStepSplitPair_forward_392x392x104.txt")
    assert bench.profiled(6, args).endswith("kImagingTma_280x280x280.txt")
