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
