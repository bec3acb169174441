"""ctypes binding of libelastic3d_b200.so (the C ABI in include/elastic3d_b200.h).

The library is built in-tree by ``elasticisolib_3d_b200.build``.  There is no
fallback: if the shared object is missing or fails to load, every entry point
raises, so a silent CPU path can never stand in for the CUDA one.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libelastic3d_b200.so")

E3D_OK = 0
E3D_ERR_OOM = 4
STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "call out of order", 4: "out of device memory",
          5: "acquisition device out of bounds"}

P = ctypes.c_void_p
I = ctypes.c_int
LL = ctypes.c_longlong
F = ctypes.c_float
D = ctypes.c_double

# exported symbol -> (argtypes, restype); every declaration of the header is listed
_SEAM_SIG = [P] * 18 + [P, LL] * 14 + [I] * 5
SIGNATURES = {
    "e3d_last_error": ([], ctypes.c_char_p),
    "e3d_version": ([], ctypes.c_char_p),
    "getGpuInfo_3D": ([P, I, I, I], I),
    "setGpuP2P": ([I, I, P], I),
    "initNonlinearElasticGpu_3D": ([F, F, F, I, I, I, I, F, I, I, I, F, I, I, I], I),
    "allocateNonlinearElasticGpu_3D": ([P] * 8 + [I] * 5, I),
    "deallocateNonlinearElasticGpu_3D": ([I, I], I),
    "propElasticFwdGpu_3D": (_SEAM_SIG, I),
    "propElasticAdjGpu_3D": (_SEAM_SIG, I),
    "propElasticFwdGpudomDec_3D": (_SEAM_SIG[:-2] + [P, I, P, I], I),
    "propElasticAdjGpudomDec_3D": (_SEAM_SIG[:-2] + [P, I, P, I], I),
    "initBornElasticGpu_3D": ([F, F, F, I, I, I, I, F, I, I, I, F, I, I, I], I),
    "allocateBornElasticGpu_3D": ([P] * 8 + [I] * 5, I),
    "deallocateBornElasticGpu_3D": ([I, I], I),
    "allocatePinBornElasticGpu_3D": ([I] * 8, I),
    "deallocatePinBornElasticGpu_3D": ([I, I], I),
    "BornElasticFwdGpu_3D": ([P] * 18 + [P, LL] * 14 + [P] * 8 + [I] * 5, I),
    "BornElasticAdjGpu_3D": ([P] * 18 + [P, LL] * 14 + [P] * 8 + [I] * 5, I),
    "e3d_context_create": ([P, P], I),
    "e3d_context_destroy": ([P], I),
    "e3d_set_medium": ([P, P, I], I),
    "e3d_set_stepper_variant": ([P, I, I, I], I),
    "e3d_set_checkpoint_policy": ([P, I, I, D], I),
    "e3d_synchronize": ([P], I),
    "e3d_stream": ([P], P),
    "e3d_set_stream": ([P, P, I], I),
    "e3d_cells_per_step": ([P], LL),
    "e3d_checkpoint_segment": ([P], I),
    "e3d_nl_forward": ([P] * 7, I),
    "e3d_nl_adjoint": ([P] * 7, I),
    "e3d_nl_propagate_slabs": ([P, I, I, I] + [P] * 6, I),
    "e3d_born_forward": ([P] * 8, I),
    "e3d_born_adjoint": ([P] * 8, I),
    "e3d_nl_propagate_device": ([P, I, P, P, P, P, P, P], I),
    "e3d_fwi_forward_device": ([P] * 8, I),
    "e3d_fwi_gradient_device": ([P] * 10, I),
    "e3d_set_velocity_storage": ([P, I], I),
    "e3d_set_stepper_chunks": ([P, I], I),
    "e3d_set_graph_loop": ([P, I], I),
    "e3d_nl_propagate_device_noalloc": ([P, P, I, P, P, P, P, P, P, P], I),
    "e3d_noalloc_work_bytes": ([], ctypes.c_size_t),
    "e3d_velocity_storage": ([P], I),
    "e3d_set_decimation_ring": ([P, I], I),
    "e3d_set_imaging_chunks": ([P, I], I),
    "e3d_set_imaging_variant": ([P, I], I),
    "e3d_set_premultiplied_adjoint": ([P, I], I),
    "e3d_nl_forward_batch_device": ([P, I, P, P, P, P, P, P], I),
    "e3d_checkpoint_type": ([P], I),
    "e3d_checkpoint_schedule": ([I, I, P, I, P], I),
    "e3d_checkpoint_plan": ([LL, I, I, D, I, I, I, P, P, P, P], I),
    "e3d_step_only": ([P, I, I], I),
    "e3d_kernel_timing": ([P, I], I),
    "e3d_kernel_timing_read": ([P, I, P, P], I),
    "e3d_launch_count": ([P], LL),
    "e3d_medium_planes": ([I, I, I, F, P, P], I),
    "e3d_stagger": ([I, I, I, I, I, I, P, P], I),
    "e3d_space_interp_linear": ([P, P, P, LL, I, I, I, F, F, F, F, F, F, P, F, I, F, F, F, P, P, P, P, P], I),
    "e3d_space_interp": ([I, I, P, P, P, LL, I, I, I, F, F, F, F, F, F, P, F, I, F, F, F, I, P, P, P, P, P], I),
}

_lib = None


class E3DError(RuntimeError):
    """A non-zero status from the native library."""

    def __init__(self, fn, status):
        msg = _lib.e3d_last_error().decode() if _lib is not None else ""
        super().__init__(f"{fn}: {STATUS.get(status, status)}: {msg}")
        self.status = status


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"native library {LIB_PATH} is missing; run python -m elasticisolib_3d_b200.build")
        L = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def call(name, *args):
    """Call a status-returning entry point and raise E3DError on failure."""
    st = getattr(lib(), name)(*args)
    if st != E3D_OK:
        raise E3DError(name, st)
    return st


class E3DDesc(ctypes.Structure):
    _fields_ = [("device", I), ("nz", I), ("nx", I), ("ny", I), ("nts", I), ("sub", I), ("minPad", I),
                ("dz", F), ("dx", F), ("dy", F), ("dts", F), ("alphaCos", F), ("fix_q1", I), ("q2compat", I),
                ("q3compat", I), ("free_surface", I)]


class E3DTraceMap(ctypes.Structure):
    _fields_ = [("n_irreg", I), ("n_taps", I), ("slot", P), ("weight", P), ("row_ptr", P), ("idx", P), ("w", P)]


def ptr_array(arrays, ctype=P):
    """C array of pointers to numpy arrays or torch tensors (data_ptr)."""
    vals = []
    for a in arrays:
        if a is None:
            vals.append(None)
        elif hasattr(a, "data_ptr"):
            vals.append(a.data_ptr())
        else:
            vals.append(a.ctypes.data)
    return (ctype * len(vals))(*vals)


def as_f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def as_i64(a):
    return np.ascontiguousarray(a, dtype=np.int64)
