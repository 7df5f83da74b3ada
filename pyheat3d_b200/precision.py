"""Mixed-precision Jacobi for lap(u) = f: FP64 defect correction around 16-bit inner sweeps.

The reference solves the Poisson problem with plain Jacobi and the source b = -h^2 f / (2d)
(pyheat3d ``src/pyheat3d/validation.py:135-147``) in a single precision, which cannot reach a
1e-10 relative residual in fp32, let alone with 16-bit storage. Here:

* the solution u and the residual r = f - A u live in FP64 on the GPU (``ph3_dc_residual``,
  ``ph3_dc_correct``: the only FP64 steps);
* each outer iteration solves the scaled correction equation A e = r / s (s: a power of two at
  or below the residual's RMS, so e stays inside the 16-bit exponent range) approximately with
  ``m`` Jacobi sweeps on a 16-bit (or fp32) field with fp32 arithmetic — the library's stencil
  kernels with the source b = -h^2 (r / s) / (2d) — starting from e = 0;
* u <- u + s e, and the loop stops when ||r||_2 / ||f||_2 <= tol.

``m`` is chosen from the Jacobi spectral radius rho = cos(pi h) so that one inner solve damps
the smoothest error mode by the storage type's resolution (``REDUCTION``), but never more than
``MAX_INNER`` sweeps: past that many sweeps from e = 0, one sweep's change of the smooth part of
e is below half an ulp of the storage type and rounds away.
"""

from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib

#: per-outer-iteration damping target of the inner solve, by storage type
REDUCTION = {"bfloat16": 2.0**-6, "float16": 2.0**-9, "float32": 2.0**-18}

#: inner sweeps per outer iteration at most, by storage type. Starting from e = 0, sweep k
#: changes the smooth part of the correction by about e / k; once that falls below half a unit
#: in the last place of the storage type (k ~ 2^(significand bits)) every further update rounds
#: away and the inner solve stalls (bf16 stalls after ~256 sweeps on any large grid).
MAX_INNER = {"bfloat16": 128, "float16": 1024, "float32": 1 << 20}


def _torch():
    import torch

    return torch


def inner_sweeps(n: int, storage: str, k: int = 1) -> int:
    """Sweeps per inner solve: enough to damp the smoothest mode by REDUCTION[storage], at most
    MAX_INNER[storage] (a multiple of k)."""
    rho = math.cos(math.pi / (n - 1))
    m = int(math.ceil(math.log(REDUCTION[storage]) / math.log(rho)))
    m = min(m, MAX_INNER[storage])
    return max(k, int(math.ceil(m / k)) * k)


def jacobi_sweeps(n: int, tol: float) -> int:
    """Sweeps plain Jacobi needs to damp the smoothest mode by tol (validation.py:89-93)."""
    return int(math.ceil(math.log(tol) / math.log(math.cos(math.pi / (n - 1)))))


@dataclass
class DCResult:
    """Outcome of :meth:`DefectCorrection.solve`."""

    u: object                      # FP64 device tensor (torch)
    history: list[float]           # relative residual before each outer iteration and at exit
    outer: int
    sweeps: int                    # inner Jacobi sweeps in total
    seconds: float
    storage: str
    variant: str
    converged: bool
    extra: dict = field(default_factory=dict)

    def host(self) -> np.ndarray:
        return self.u.cpu().numpy()


class DefectCorrection:
    """FP64 defect correction for lap(u) = f on a Dirichlet grid with zero boundary values.

    ``f``: FP64 array (ny, nx) or (nz, ny, nx) including the boundary layer (ignored there);
    ``h``: grid spacing; ``storage``: storage type of the inner correction field;
    ``variant``: "march" (single-step: TMA z-march / y-march) or "tb" with ``k`` steps per pass.
    """

    def __init__(self, f: np.ndarray, h: float, storage: str = "bfloat16", variant: str = "march",
                 k: int = 1, device=None):
        torch = _torch()
        if not torch.cuda.is_available():
            raise RuntimeError("no CUDA device")
        self.lib = _lib.lib()
        if f.ndim not in (2, 3) or min(f.shape) < 3:
            raise ValueError("f must be 2D or 3D with at least 3 points per axis")
        if storage not in _lib.STORAGE:
            raise ValueError(f"unknown storage {storage!r}")
        if variant not in ("march", "tb"):
            raise ValueError("variant must be 'march' or 'tb'")
        self.dims = f.ndim
        self.shape = tuple(int(s) for s in f.shape)
        self.h = float(h)
        self.storage = storage
        self.variant = variant
        self.k = k if variant == "tb" else 1
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        td = getattr(torch, storage)
        self.f = torch.from_numpy(np.ascontiguousarray(f, dtype=np.float64)).to(self.device)
        self.u = torch.zeros(self.shape, dtype=torch.float64, device=self.device)
        self.b = torch.zeros(self.shape, dtype=torch.float32, device=self.device)
        self.ea = torch.zeros(self.shape, dtype=td, device=self.device)
        self.eb = torch.zeros(self.shape, dtype=td, device=self.device)
        self.scratch = torch.empty(int(self.lib.ph3_reduction_scratch_len()),
                                   dtype=torch.float64, device=self.device)
        self.rn2 = torch.zeros(1, dtype=torch.float64, device=self.device)
        core = (slice(1, -1),) * self.dims
        self.fnorm = float(np.sqrt(np.sum(np.asarray(f, np.float64)[core] ** 2)))
        if self.dims == 2:
            self.nz, self.ny, self.nx = 1, self.shape[0], self.shape[1]
        else:
            self.nz, self.ny, self.nx = self.shape
        self.c1 = float(np.float32(1.0 / (2 * self.dims)))
        self.use_graph = True
        self._graphs: dict[int, tuple] = {}

    def _stream(self):
        return _torch().cuda.current_stream(self.device).cuda_stream

    def _residual(self, b_scale: float, with_b: bool) -> float:
        _lib.check(self.lib.ph3_dc_residual(
            self.dims, self.nz, self.ny, self.nx, self.u.data_ptr(), self.f.data_ptr(), self.h,
            b_scale, self.b.data_ptr() if with_b else None, self.rn2.data_ptr(),
            self.scratch.data_ptr(), self.scratch.numel(), self._stream()))
        return max(float(self.rn2.item()), 0.0)

    def residual(self) -> float:
        """Relative residual ||f - A u|| / ||f|| of the current u. The same pass also leaves
        the unscaled correction source b = -h^2 r / (2d) in ``self.b`` for the next inner solve
        (``self._b_scale`` = 1), so an outer iteration needs one FP64 residual pass."""
        self._rn2 = self._residual(1.0, True)
        self._b_scale = 1.0
        return math.sqrt(self._rn2) / self.fnorm

    def inner(self, m: int, rn2: float | None = None) -> None:
        """m Jacobi sweeps on the scaled correction equation A e = r / s from e = 0, u += s e.

        s is a power of two at or below the residual's RMS: the correction then stays inside
        the storage type's exponent range (fp16 would flush a small correction to zero).
        ``rn2``: sum(r^2) of the current u if already known (saves one residual pass).
        """
        ncore = int(np.prod([x - 2 for x in self.shape]))
        if rn2 is None or getattr(self, "_b_scale", None) != 1.0:
            rn2 = self._residual(1.0, True)
        rms = math.sqrt(rn2 / ncore)
        sc = math.ldexp(1.0, math.floor(math.log2(rms))) if rms > 0 and math.isfinite(rms) \
            else 1.0
        # b of the scaled equation: the unscaled source times 1/sc, a power of two, so the
        # product is exact wherever b stays a normal fp32 number
        self.b.mul_(1.0 / sc)
        self._b_scale = 1.0 / sc
        # the inner solve starts from e = 0; the other buffer's boundary layer is zero from the
        # start and never written, its interior is overwritten by the first sweep
        self.ea.zero_()
        e = self._sweeps(int(m))
        _lib.check(self.lib.ph3_dc_correct(self.u.data_ptr(), e.data_ptr(),
                                           _lib.STORAGE[self.storage], sc, e.numel(),
                                           self._stream()))

    def _advance(self, m: int) -> bool:
        in_b = ctypes.c_int(0)
        _lib.check(self.lib.ph3_advance(
            self.dims, self.nz, self.ny, self.nx, _lib.STORAGE[self.storage], _lib.BC["dirichlet"],
            0.0, self.c1, _lib.VARIANT[self.variant], self.k, self.ea.data_ptr(),
            self.eb.data_ptr(), self.b.data_ptr(), int(m), self._stream(), ctypes.byref(in_b)))
        return bool(in_b.value)

    def _sweeps(self, m: int):
        """m inner sweeps from ea (buffers and source fixed for the whole solve); returns the
        buffer holding the result. With ``use_graph`` the launch sequence of m sweeps is
        captured once in a CUDA graph and replayed by later outer iterations: the inner
        kernels are short (about 15 us at 256^3), so host-side launch work would otherwise
        leave the GPU waiting between them."""
        if not self.use_graph:
            return self.eb if self._advance(m) else self.ea
        torch = _torch()
        g = self._graphs.get(m)
        if g is None:
            in_b = self._advance(m)  # warm-up outside capture (one-time kernel attributes)
            self.ea.zero_()
            side = torch.cuda.Stream(self.device)
            side.wait_stream(torch.cuda.current_stream(self.device))
            graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(graph, stream=side):
                in_b = self._advance(m)
            torch.cuda.current_stream(self.device).wait_stream(side)
            g = self._graphs[m] = (graph, in_b)
        g[0].replay()
        return self.eb if g[1] else self.ea

    def solve(self, tol: float = 1e-10, max_outer: int | None = None,
              sweeps: int | list[int] | None = None, max_sweeps: int | None = None) -> DCResult:
        """Outer iterations until the relative residual is <= tol.

        ``sweeps``: inner sweeps per outer iteration (int), an explicit schedule (list; the loop
        then runs exactly len(schedule) outer iterations), or None for :func:`inner_sweeps`.
        The loop also stops after ``max_outer`` outer iterations or ``max_sweeps`` inner sweeps
        (default: three times what plain Jacobi needs for ``tol``).
        """
        torch = _torch()
        n = min(self.shape)
        schedule = sweeps if isinstance(sweeps, list) else None
        m = sweeps if isinstance(sweeps, int) else inner_sweeps(n, self.storage, self.k)
        if max_sweeps is None:
            max_sweeps = 3 * jacobi_sweeps(n, tol)
        torch.cuda.synchronize(self.device)
        t0 = time.perf_counter()
        hist = [self.residual()]
        total = 0
        outer = 0
        limit = len(schedule) if schedule is not None else (max_outer or 1 << 30)
        while outer < limit:
            if schedule is None and (hist[-1] <= tol or total >= max_sweeps):
                break
            mm = schedule[outer] if schedule is not None else m
            self.inner(mm, self._rn2)
            total += mm
            outer += 1
            hist.append(self.residual())
        torch.cuda.synchronize(self.device)
        secs = time.perf_counter() - t0
        return DCResult(self.u, hist, outer, total, secs, self.storage,
                        self.variant if self.k == 1 else f"tb{self.k}", hist[-1] <= tol)
