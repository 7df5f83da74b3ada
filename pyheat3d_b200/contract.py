"""The pyheat3d plug-in contract this backend implements.

When pyheat3d is importable its own classes are used, so a ``B200Stepper`` *is* a
``pyheat3d.backends.base.Stepper`` and the variants enter ``pyheat3d.registry.VARIANTS``
unchanged. Without pyheat3d (on a machine where only this package is installed) this module
provides same-named mirrors with the same fields, argument meaning and errors:

- ``Stencil``, ``heat_stencil``, ``jacobi_stencil``, ``stability_limit``:
  pyheat3d ``src/pyheat3d/problem.py:33-69``
- ``Stepper``: ``src/pyheat3d/backends/base.py:12-74``
- ``Variant``: ``src/pyheat3d/registry.py:33-54``
"""

from __future__ import annotations

from abc import ABC, abstractmethod
from collections.abc import Callable
from dataclasses import dataclass, field

import numpy as np

BCS = ("dirichlet", "periodic")

try:  # the real plug-in point
    from pyheat3d.backends.base import Stepper as _RefStepper  # type: ignore
    from pyheat3d.problem import Stencil as _RefStencil  # type: ignore
    from pyheat3d.problem import heat_stencil as _ref_heat  # type: ignore
    from pyheat3d.problem import jacobi_stencil as _ref_jacobi  # type: ignore
    from pyheat3d.problem import stability_limit as _ref_limit  # type: ignore
    from pyheat3d.registry import Variant as _RefVariant  # type: ignore

    HAVE_PYHEAT3D = True
except ImportError:  # pragma: no cover - exercised when pyheat3d is absent
    HAVE_PYHEAT3D = False


if HAVE_PYHEAT3D:
    Stencil = _RefStencil
    heat_stencil = _ref_heat
    jacobi_stencil = _ref_jacobi
    stability_limit = _ref_limit
    Stepper = _RefStepper
    Variant = _RefVariant
else:

    @dataclass(frozen=True)
    class Stencil:  # type: ignore[no-redef]
        """Coefficients and boundary condition of ``u' = c0 u + c1 S`` (problem.py:33-43)."""

        c0: float
        c1: float
        bc: str = "dirichlet"

        def __post_init__(self) -> None:
            if self.bc not in BCS:
                raise ValueError(f"bc must be one of {BCS}, got {self.bc!r}")

    def stability_limit(dims: int) -> float:  # type: ignore[no-redef]
        """Largest stable FTCS mesh Fourier number, ``1/(2d)`` (problem.py:46-48)."""
        return 1.0 / (2.0 * dims)

    def heat_stencil(dims: int, r: float, bc: str = "dirichlet",  # type: ignore[no-redef]
                     check: bool = True) -> Stencil:
        """FTCS heat stencil ``c0 = 1 - 2 d r``, ``c1 = r`` (problem.py:51-62)."""
        if dims not in (2, 3):
            raise ValueError("dims must be 2 or 3")
        if check and not (0.0 < r <= stability_limit(dims) + 1e-15):
            raise ValueError(
                f"r = {r:g} violates the FTCS stability limit r <= 1/(2d) = "
                f"{stability_limit(dims):g}")
        return Stencil(c0=1.0 - 2.0 * dims * r, c1=r, bc=bc)

    def jacobi_stencil(dims: int, bc: str = "dirichlet") -> Stencil:  # type: ignore[no-redef]
        """Jacobi stencil ``c0 = 0``, ``c1 = 1/(2d)`` (problem.py:65-69)."""
        if dims not in (2, 3):
            raise ValueError("dims must be 2 or 3")
        return Stencil(c0=0.0, c1=1.0 / (2.0 * dims), bc=bc)

    class Stepper(ABC):  # type: ignore[no-redef]
        """Owns a ping-pong pair of buffers and advances the update (base.py:12-74)."""

        storage: str = "float32"
        steps_per_pass: int = 1

        def __init__(self, u0: np.ndarray, stencil, source: np.ndarray | None = None):
            if u0.ndim not in (2, 3):
                raise ValueError("u0 must be 2D or 3D")
            if min(u0.shape) < 3:
                raise ValueError("every axis needs at least 3 points")
            self.shape = tuple(int(s) for s in u0.shape)
            self.dims = u0.ndim
            self.stencil = stencil
            self.c0 = float(stencil.c0)
            self.c1 = float(stencil.c1)
            self.bc = stencil.bc
            self.periodic = stencil.bc == "periodic"
            self.has_source = source is not None
            self.steps_done = 0

        @property
        def ncells(self) -> int:
            """Sites updated per step: interior only for Dirichlet (base.py:50-55)."""
            if self.periodic:
                return int(np.prod(self.shape))
            return int(np.prod([s - 2 for s in self.shape]))

        def step(self, n: int = 1) -> None:
            for _ in range(n):
                self._step_once()
            self.steps_done += n

        def _step_once(self) -> None:  # pragma: no cover - overridden
            raise NotImplementedError

        @abstractmethod
        def get(self) -> np.ndarray:
            """Current state as a host float32/float64 array."""

        def synchronize(self) -> None:  # noqa: B027
            """Block until queued device work has finished."""

        def close(self) -> None:  # noqa: B027
            """Release device memory."""

    @dataclass(frozen=True)
    class Variant:  # type: ignore[no-redef]
        """One registry entry (registry.py:33-54)."""

        backend: str
        name: str
        factory: Callable[[], type] = field(repr=False, compare=False)
        dims: tuple[int, ...] = (2, 3)
        storage: str = "float32"
        steps_per_pass: int = 1
        gpu: bool = True
        source: bool = False
        rung: int = 0
        description: str = ""

        @property
        def key(self) -> str:
            return f"{self.backend}/{self.name}"

        @property
        def bytes_per_value(self) -> int:
            return {"float32": 4, "float16": 2, "bfloat16": 2, "float64": 8}.get(self.storage, 4)
