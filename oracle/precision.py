"""NumPy restatement of the mixed-precision defect-correction solver (oracle; test infrastructure).

The reference solves lap(u) = f by plain Jacobi with the source b = -h^2 f / (2d)
(``src/pyheat3d/validation.py:135-147``, ``src/pyheat3d/problem.py:15-16``) on the manufactured
problem of ``src/pyheat3d/analytic.py:101-108``. The GPU solver adds an FP64 outer loop; this
module states, operation by operation, what the GPU computes, so small cases match bit for bit:

- :func:`residual_f64` — r = f - A u with A u = (S(u) - 2d u) / h^2 (S in the canonical x, y, z
  order), r = 0 on the boundary, b = float32(-h^2 r / (2d)), and sum(r^2);
- :func:`defect_correction` — the outer loop: a power-of-two scale s near the residual's RMS,
  the scaled correction equation A e = r / s solved by Jacobi sweeps emulated by
  :func:`oracle.stencil.emulated_reference` (16-bit storage rounding, source b added last), and
  u <- u + s e;
- :func:`manufactured` / :func:`discrete_solution` — the manufactured problem and its exact
  discrete (FP64) solution: f is an eigenfunction of the discrete Laplacian, so the converged
  FP64 Jacobi iterate is known in closed form.
"""

from __future__ import annotations

import math

import numpy as np

from .stencil import _neighbour_pairs, emulated_reference


def grid_axis(n: int) -> np.ndarray:
    """Dirichlet unit-interval axis with n points including both walls (analytic.py:14-22)."""
    return np.arange(n, dtype=np.float64) / (n - 1)


def sine_mode(n: int, dims: int) -> np.ndarray:
    """prod_i sin(pi x_i) with exact zeros on the walls (analytic.py:42-54, m = 1)."""
    s = np.sin(math.pi * grid_axis(n))
    s[0] = 0.0
    s[-1] = 0.0
    out = s
    for _ in range(dims - 1):
        out = np.multiply.outer(out, s)
    return out


def manufactured(n: int, dims: int) -> tuple[np.ndarray, np.ndarray]:
    """(u_exact, f) with lap(u) = f, u = prod sin(pi x_i) (analytic.py:101-108)."""
    u = sine_mode(n, dims)
    return u, -dims * math.pi**2 * u


def discrete_solution(n: int, dims: int) -> np.ndarray:
    """Exact solution of the 2d+1-point discrete problem L_h u = f for the manufactured f.

    L_h sin-mode = lambda_h sin-mode with lambda_h = -(4 d / h^2) sin^2(pi h / 2).
    """
    h = 1.0 / (n - 1)
    lam = -(4.0 * dims / (h * h)) * math.sin(0.5 * math.pi * h) ** 2
    _, f = manufactured(n, dims)
    return f / lam


def pow2_scale(rn2: float, ncells: int) -> float:
    """Power of two at or below the residual's RMS (1.0 for a zero residual)."""
    rms = math.sqrt(rn2 / max(ncells, 1))
    if not rms > 0.0 or not math.isfinite(rms):
        return 1.0
    return math.ldexp(1.0, math.floor(math.log2(rms)))


def residual_f64(u: np.ndarray, f: np.ndarray, h: float, b_scale: float = 1.0):
    """(r, b, sum(r^2)) exactly as the GPU's FP64 residual kernel computes r and b."""
    d = u.ndim
    core = (slice(1, -1),) * d
    p = _neighbour_pairs(u, periodic=False)
    s = p[0][0] + p[0][1]
    s = s + (p[1][0] + p[1][1])
    if d == 3:
        s = s + (p[2][0] + p[2][1])
    inv_h2 = 1.0 / (h * h)
    au = (s - (2.0 * d) * u[core]) * inv_h2
    r = np.zeros_like(u)
    r[core] = f[core] - au
    bscale = (-(h * h) / (2.0 * d)) * b_scale
    b = (bscale * r).astype(np.float32)
    return r, b, float(np.sum(r * r))


def jacobi_rho(n: int) -> float:
    """Spectral radius cos(pi h) of Jacobi on an n-point Dirichlet grid (validation.py:89-93)."""
    return math.cos(math.pi / (n - 1))


def defect_correction(f: np.ndarray, h: float, storage: str, k: int, sweeps: list[int]):
    """Outer FP64 loop with len(sweeps) inner solves; returns (u, relative residuals)."""
    d = f.ndim
    c0, c1 = 0.0, 1.0 / (2 * d)
    u = np.zeros_like(f, dtype=np.float64)
    fn = math.sqrt(float(np.sum(f[(slice(1, -1),) * d] ** 2)))
    hist = []
    ncore = int(np.prod([s - 2 for s in f.shape]))
    for m in sweeps:
        _, _, rn2 = residual_f64(u, f, h)
        hist.append(math.sqrt(rn2) / fn)
        sc = pow2_scale(rn2, ncore)
        _, b, _ = residual_f64(u, f, h, 1.0 / sc)
        e = emulated_reference(np.zeros(f.shape, np.float32), c0, c1, "dirichlet", m, storage,
                               k, b)
        u = u + sc * e.astype(np.float64)
    _, _, rn2 = residual_f64(u, f, h)
    hist.append(math.sqrt(rn2) / fn)
    return u, hist
