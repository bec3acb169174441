"""CPU: the C-ABI library loads (no GPU needed) and exports every function that
include/elastic3d_b200.h declares; the Python bindings declare a signature for each."""
import ctypes
import os
import re

from elasticisolib_3d_b200 import _native as N

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "elastic3d_b200.h")


def _declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(", text, flags=re.M)
    return sorted(set(n for n in names if n not in ("if", "while", "for", "return", "sizeof")))


def test_header_declares_the_seam_and_the_explicit_api():
    names = _declared()
    for n in ("propElasticFwdGpu_3D", "propElasticAdjGpu_3D", "BornElasticFwdGpu_3D", "BornElasticAdjGpu_3D",
              "initNonlinearElasticGpu_3D", "allocateBornElasticGpu_3D", "e3d_fwi_gradient_device",
              "e3d_nl_propagate_device_noalloc"):
        assert n in names, n


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(N.LIB_PATH)
    missing = [n for n in _declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_bindings_cover_every_declared_symbol():
    missing = [n for n in _declared() if n not in N.SIGNATURES]
    assert not missing, missing


# ---- the seam's host-side argument and state checks (no device work reached) ----------------
E3D_ERR_ARG, E3D_ERR_STATE = 1, 3
SPARE_SLOT = 15   # the last slot: no other test uses it


def _init(lib, **kw):
    a = dict(dz=10.0, dx=10.0, dy=10.0, nz=40, nx=40, ny=32, nts=20, dts=0.002, sub=4, minPad=6, blockSize=16,
             alphaCos=0.99, nGpu=1, iGpuId=0, iGpuAlloc=0)
    a.update(kw)
    return lib.initNonlinearElasticGpu_3D(*a.values())


def test_seam_rejects_bad_arguments_without_a_gpu():
    lib = N.lib()
    assert _init(lib, nGpu=0) == E3D_ERR_ARG
    assert _init(lib, nGpu=17) == E3D_ERR_ARG
    assert _init(lib, sub=100) == E3D_ERR_ARG           # SUB_MAX
    assert b"SUB_MAX" in lib.e3d_last_error()
    assert lib.deallocateNonlinearElasticGpu_3D(16, 0) == E3D_ERR_ARG                  # slots 0..15
    assert lib.allocatePinBornElasticGpu_3D(40, 32, 40, 2, 1, 0, 0, 0) == E3D_ERR_ARG   # nts < 3
    assert lib.allocatePinBornElasticGpu_3D(40, 32, 40, 20, 1, 0, 0, 0) == 0


def test_seam_refuses_propagation_on_an_unallocated_slot():
    lib = N.lib()
    nulls = [None] * 18
    geom = []
    for _ in range(14):
        geom += [None, 0]
    st = lib.propElasticFwdGpu_3D(*nulls, *geom, 40, 32, 40, SPARE_SLOT, 0)
    assert st == E3D_ERR_STATE
    assert b"not allocated" in lib.e3d_last_error()
