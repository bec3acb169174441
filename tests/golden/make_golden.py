"""Generate golden vectors by running the reference's own CUDA drivers.

The reference (elastic_iso_lib_3d, FP32 tree and FP64 tree) is compiled from
its sources by ``oracle/Makefile`` (target ``ref``) into ``oracle/_ref/``;
this script loads those libraries, feeds them one small seeded survey and
stores what they return in ``tests/golden/ref_small.npz``.  It needs a GPU
and runs once; the committed .npz is then read by the CPU tests to pin the
oracle (tests/test_oracle_golden.py).

Inputs are not stored: they are regenerated from the seeds below by the same
code (synthetic.small_survey + the oracle's host preparation), and a digest
of them is stored so a drift in input generation is detected.

Usage (on a machine with a GPU):  python tests/golden/make_golden.py [COPY_DIR]
COPY_DIR, when given and present, receives a second copy of the .npz (for
runs whose working tree does not persist).
"""
from __future__ import annotations

import ctypes
import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from golden_case import golden_inputs, SUBSAMPLE  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")


def _load(name):
    L = ctypes.CDLL(os.path.join(REF, name))
    return L


def _pp(arrs):
    return (ctypes.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])


def run_ref(lib, fn, adjoint, case, dtype, pert=None):
    p = case["params"]
    dims = (ctypes.c_int * 6)(p.nz, p.nx, p.ny, p.nts, p.sub, p.minPad)
    reals = (ctypes.c_double * 5)(p.dz, p.dx, p.dy, p.dts, p.alphaCos)
    med = [np.ascontiguousarray(m, dtype=dtype) for m in case["med64" if dtype == np.float64 else "med32"]]
    spos = [np.ascontiguousarray(x, dtype=np.int64) for x in case["spos"]]
    rpos = [np.ascontiguousarray(x, dtype=np.int64) for x in case["rpos"]]
    sn = (ctypes.c_longlong * 7)(*[len(x) for x in spos])
    rn = (ctypes.c_longlong * 7)(*[len(x) for x in rpos])
    if fn == "nl":
        if not adjoint:
            sig = [np.ascontiguousarray(x, dtype=dtype) for x in case["sig"]]
            dat = [np.zeros_like(x, dtype=dtype) for x in case["dat"]]
        else:
            sig = [np.zeros_like(x, dtype=dtype) for x in case["sig"]]
            dat = [np.ascontiguousarray(x, dtype=dtype) for x in case["dat"]]
        st = lib.ref_nl_run(int(adjoint), dims, reals, _pp(med), _pp(sig), _pp(dat), _pp(spos), sn, _pp(rpos), rn)
        assert st == 0
        return sig if adjoint else dat
    sig = [np.ascontiguousarray(x, dtype=dtype) for x in case["sig"]]
    if not adjoint:
        dat = [np.zeros_like(x, dtype=dtype) for x in case["dat"]]
        pp = [np.ascontiguousarray(x, dtype=dtype) for x in pert]
    else:
        dat = [np.ascontiguousarray(x, dtype=dtype) for x in case["dat"]]
        pp = [np.zeros(case["med32"].shape[1:], dtype=dtype) for _ in range(8)]
    st = lib.ref_born_run(int(adjoint), dims, reals, _pp(med), _pp(sig), _pp(dat), _pp(spos), sn, _pp(rpos), rn,
                          _pp(pp))
    assert st == 0
    return pp if adjoint else dat


def main():
    case = golden_inputs()
    out = {"digest": np.frombuffer(case["digest"], dtype=np.uint8)}
    for dtype, suf in ((np.float32, "f32"), (np.float64, "f64")):
        nl = _load(f"libref_nl_{suf}.so")
        born = _load(f"libref_born_{suf}.so")
        d = run_ref(nl, "nl", False, case, dtype)
        out[f"nl_fwd_{suf}"] = np.concatenate([x.ravel() for x in d]).astype(np.float64)
        m = run_ref(nl, "nl", True, case, dtype)
        out[f"nl_adj_{suf}"] = np.concatenate([x.ravel() for x in m]).astype(np.float64)
        pert = case["pert64"] if dtype == np.float64 else case["pert32"]
        d = run_ref(born, "born", False, case, dtype, pert)
        out[f"born_fwd_{suf}"] = np.concatenate([x.ravel() for x in d]).astype(np.float64)
        g = run_ref(born, "born", True, case, dtype)
        s = SUBSAMPLE
        out[f"born_adj_{suf}"] = np.stack([x[::s, ::s, ::s] for x in g]).astype(np.float32 if suf == "f32"
                                                                                   else np.float64)
        print(suf, {k: float(np.abs(v).max()) for k, v in out.items() if k.endswith(suf)})
    path = os.path.join(ROOT, "tests", "golden", "ref_small.npz")
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.savez_compressed(path, **out)
    if len(sys.argv) > 1 and os.path.isdir(sys.argv[1]):
        np.savez_compressed(os.path.join(sys.argv[1], "ref_small.npz"), **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
