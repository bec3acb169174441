"""B200-native elastic isotropic 3D propagation (drop-in for elasticIsoLib_3D's propagation path).

Layers:
  * ``_native``   ctypes binding of libelastic3d_b200.so (CUDA kernels + C ABI)
  * ``engine``    Propagator: one device context, reference-driver semantics
  * ``hostprep``  fdParamElastic_3D / stagger / spaceInterpGpu_3D (native host code)
  * ``operators`` reference-compatible operator classes (nonlinear and Born, per shot and shots)
  * ``fwi``       torch.autograd.Function FWI gradient with on-device checkpoints
  * ``synthetic`` seeded synthetic models, sources and acquisition geometries
"""
__version__ = "0.1.0"

from .engine import Propagator  # noqa: F401
