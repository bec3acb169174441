"""Pin the oracle to the reference: outputs of the reference's own CUDA build
(elastic_iso_float and elastic_iso_double trees, compiled from the reference
sources by oracle/Makefile and run by tests/golden/make_golden.py on a GPU)
against the oracle's CPU restatement on the same inputs.

Bounds: the FP64 restatement against the FP64 reference differs only in
summation order (1e-12 relative L2); the FP32 restatement against the FP32
reference accumulates float rounding over 60 fine steps (1e-6).
"""
import os

import numpy as np
import pytest

from golden_case import SUBSAMPLE, golden_inputs
from oracle import oracle as O

FIX = os.path.join(os.path.dirname(__file__), "golden", "ref_small.npz")


@pytest.fixture(scope="module")
def golden():
    if not os.path.exists(FIX):
        pytest.skip("golden fixture missing")
    return np.load(FIX), golden_inputs()


def _flat(xs):
    return np.concatenate([np.asarray(x, dtype=np.float64).ravel() for x in xs])


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


TOL = {"f64": 1e-12, "f32": 1e-6}


def test_inputs_unchanged(golden):
    fx, case = golden
    assert bytes(fx["digest"].tobytes()) == case["digest"], "input generation drifted from the fixture"


@pytest.mark.parametrize("suf", ["f64", "f32"])
def test_nl_forward_pinned(golden, suf):
    fx, c = golden
    dt = np.float64 if suf == "f64" else np.float32
    med = c["med64"] if suf == "f64" else c["med32"]
    got = O.nl_forward_reg(c["params"], med, [s.astype(dt) for s in c["sig"]], c["spos"], c["rpos"], dt)
    assert _rel(_flat(got), fx[f"nl_fwd_{suf}"]) < TOL[suf]


@pytest.mark.parametrize("suf", ["f64", "f32"])
def test_nl_adjoint_pinned(golden, suf):
    fx, c = golden
    dt = np.float64 if suf == "f64" else np.float32
    med = c["med64"] if suf == "f64" else c["med32"]
    got = O.nl_adjoint_reg(c["params"], med, [d.astype(dt) for d in c["dat"]], c["spos"], c["rpos"], dt)
    assert _rel(_flat(got), fx[f"nl_adj_{suf}"]) < TOL[suf]


@pytest.mark.parametrize("suf", ["f64", "f32"])
def test_born_forward_pinned(golden, suf):
    fx, c = golden
    dt = np.float64 if suf == "f64" else np.float32
    med = c["med64"] if suf == "f64" else c["med32"]
    pert = c["pert64"] if suf == "f64" else c["pert32"]
    got = O.born_forward_reg(c["params"], med, [s.astype(dt) for s in c["sig"]], pert, c["spos"], c["rpos"], dt)
    assert _rel(_flat(got), fx[f"born_fwd_{suf}"]) < TOL[suf]


@pytest.mark.parametrize("suf", ["f64", "f32"])
def test_born_adjoint_pinned(golden, suf):
    fx, c = golden
    dt = np.float64 if suf == "f64" else np.float32
    med = c["med64"] if suf == "f64" else c["med32"]
    got = O.born_adjoint_reg(c["params"], med, [s.astype(dt) for s in c["sig"]], [d.astype(dt) for d in c["dat"]],
                             c["spos"], c["rpos"], None, dt)
    s = SUBSAMPLE
    got = np.stack([g[::s, ::s, ::s] for g in got])
    assert _rel(got.astype(np.float64).ravel(), fx[f"born_adj_{suf}"].astype(np.float64).ravel()) < TOL[suf]


def test_fp32_reference_within_1e5_of_fp64(golden):
    """The reference's own FP32 traces against its FP64 traces (relative L2 <= 1e-5)."""
    fx, _ = golden
    for k in ("nl_fwd", "born_fwd"):
        assert _rel(fx[f"{k}_f32"], fx[f"{k}_f64"]) < 1e-5
