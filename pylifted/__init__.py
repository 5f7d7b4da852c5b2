"""Drop-in for the reference's `pylifted` package: the same names,
re-exported from lifted_b200 (GPU-backed)."""
from lifted_b200.pylifted import (  # noqa: F401
    BoundaryCondition,
    Transform,
    Wavelet,
    lwt_forward,
    lwt_forward_adjoint,
    lwt_inverse,
    lwt_inverse_adjoint,
)
