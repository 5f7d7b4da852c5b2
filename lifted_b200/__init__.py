"""B200-native lifting-scheme DWT: the hot path of jcapriot/lifted (the
multi-level lifting transform and its adjoint, separable and non-separable
nD) as hand-written sm_100a CUDA kernels behind the reference's own API.

Submodules:
  pylifted   the reference's Python entry points (lwt_forward, ...)
  autograd   torch.autograd.Function forms (backward = adjoint kernel)
  build      builds liblifted_b200.so in-tree (nvcc, sm_100a)
"""
from .pylifted import (  # noqa: F401
    BoundaryCondition,
    Transform,
    Wavelet,
    lwt_forward,
    lwt_forward_adjoint,
    lwt_inverse,
    lwt_inverse_adjoint,
    lwt_program,
)

__all__ = [
    "lwt_forward",
    "lwt_inverse",
    "lwt_forward_adjoint",
    "lwt_inverse_adjoint",
    "lwt_program",
    "Transform",
    "Wavelet",
    "BoundaryCondition",
]
