"""pyheat3d_b200: a B200-native (sm_100a) stencil backend for pyheat3d.

Hand-written CUDA kernels for the FTCS heat update and the Jacobi sweep
``u' = c0*u + c1*S (+ b)`` (5-point 2D, 7-point 3D, Dirichlet and periodic), bit-identical to
pyheat3d's NumPy reference, reached through the ``libph3b200.so`` C ABI (``include/ph3b200.h``)
and registered as backend ``b200`` in pyheat3d's variant registry.

Importing this package never loads the CUDA library; the first stepper does, and fails loudly
if it is missing.
"""

from .contract import (  # noqa: F401
    HAVE_PYHEAT3D,
    Stencil,
    heat_stencil,
    jacobi_stencil,
    stability_limit,
)
from .registry import VARIANTS, availability, make_stepper, register  # noqa: F401

__version__ = "1.0.0"
