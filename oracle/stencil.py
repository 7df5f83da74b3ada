"""NumPy restatement of the pyheat3d stencil update (oracle; test infrastructure only).

The update, for a C-ordered ``(y, x)`` or ``(z, y, x)`` array with x contiguous::

    u'[c] = c0 * u[c] + c1 * S[c]  (+ b[c], added last)
    S     = ((u[x-1] + u[x+1]) + (u[y-1] + u[y+1])) + (u[z-1] + u[z+1])

Every operation rounds in the array dtype (float32 or float64) with no fused multiply-add,
exactly like NumPy ufuncs. Dirichlet problems update the interior only (the outer layer keeps
its boundary values); periodic problems update every cell with wrap-around neighbours.

Sources restated (paths relative to the pyheat3d project):
- ``reference_step``: ``src/pyheat3d/backends/numpy_ref.py:11-47``
- ``round_storage``: ``src/pyheat3d/validation.py:157-165``
- ``emulated_reference``: ``src/pyheat3d/validation.py:168-183``
- ``to_bf16_bits`` / ``from_bf16_bits``: ``src/pyheat3d/backends/cupy_backend.py:103-112``
- ``TOLERANCE``: ``src/pyheat3d/validation.py:153-154``
"""

from __future__ import annotations

import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np

#: max relative deviation per storage type accepted by the reference (validation.py:153).
#: This project's own fp32 bar is stricter (1e-6; the kernels are bit-exact in practice).
TOLERANCE = {"float32": 2e-6, "float16": 4e-3, "bfloat16": 3e-2, "native": 0.0,
             "float64": 1e-12}


def _neighbour_pairs(u: np.ndarray, periodic: bool) -> list[tuple[np.ndarray, np.ndarray]]:
    """(minus, plus) neighbour arrays for each axis in the order x, y, z.

    Periodic: whole rolled arrays. Dirichlet: views aligned with the interior.
    (numpy_ref.py:11-27)
    """
    nd = u.ndim
    out = []
    for ax in reversed(range(nd)):
        if periodic:
            out.append((np.roll(u, 1, axis=ax), np.roll(u, -1, axis=ax)))
            continue
        lo = [slice(1, -1)] * nd
        hi = [slice(1, -1)] * nd
        lo[ax] = slice(None, -2)
        hi[ax] = slice(2, None)
        out.append((u[tuple(lo)], u[tuple(hi)]))
    return out


def reference_step(u: np.ndarray, c0: float, c1: float, bc: str,
                   b: np.ndarray | None = None) -> np.ndarray:
    """One update in the canonical summation order; returns a new array (numpy_ref.py:30-47)."""
    periodic = bc == "periodic"
    cast = u.dtype.type
    p = _neighbour_pairs(u, periodic)
    s = p[0][0] + p[0][1]
    s = s + (p[1][0] + p[1][1])
    if u.ndim == 3:
        s = s + (p[2][0] + p[2][1])
    core = (slice(None),) * u.ndim if periodic else (slice(1, -1),) * u.ndim
    new = cast(c0) * u[core] + cast(c1) * s
    if b is not None:
        new = new + b[core]
    out = u.copy()
    out[core] = new
    return out


def to_bf16_bits(x: np.ndarray) -> np.ndarray:
    """float32 -> bfloat16 bit pattern (uint16), round to nearest even (cupy_backend.py:103-107)."""
    w = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    w = (w + 0x7FFF + ((w >> 16) & 1)) >> 16
    return w.astype(np.uint16)


def from_bf16_bits(bits: np.ndarray) -> np.ndarray:
    """bfloat16 bit pattern (uint16) -> float32 (cupy_backend.py:110-112)."""
    return (np.asarray(bits).astype(np.uint32) << 16).view(np.float32)


def round_storage(u: np.ndarray, storage: str) -> np.ndarray:
    """Round float32 values to the storage precision and back (validation.py:157-165)."""
    if storage == "float16":
        return u.astype(np.float16).astype(np.float32)
    if storage == "bfloat16":
        return from_bf16_bits(to_bf16_bits(u)).reshape(np.shape(u))
    return u


def emulated_reference(u0: np.ndarray, c0: float, c1: float, bc: str, steps: int,
                       storage: str = "float32", k: int = 1,
                       b: np.ndarray | None = None) -> np.ndarray:
    """fp32 reference with the storage rounding of a variant (validation.py:168-183).

    Rounds to ``storage`` after every pass of ``k`` fused steps, then rounds each of the
    ``steps % k`` leftover single steps. ``b`` (optional, float32) is the Jacobi source; the
    reference's emulation has no source argument, so with ``b`` this follows the same rounding
    schedule with ``reference_step(..., b)`` (numpy_ref.py:44-45: b is added last).
    """
    u = round_storage(np.asarray(u0, dtype=np.float32), storage)
    passes, rem = divmod(steps, k)
    for _ in range(passes):
        for _ in range(k):
            u = reference_step(u, c0, c1, bc, b)
        u = round_storage(u, storage)
    for _ in range(rem):
        u = round_storage(reference_step(u, c0, c1, bc, b), storage)
    return u


def run_reference(u0: np.ndarray, c0: float, c1: float, bc: str, steps: int,
                  b: np.ndarray | None = None) -> np.ndarray:
    """``steps`` plain updates in the dtype of ``u0`` (float32 or float64)."""
    u = np.array(u0, copy=True)
    for _ in range(steps):
        u = reference_step(u, c0, c1, bc, b)
    return u


# ---------------------------------------------------------------------------------------------
# Multi-threaded CPU baseline: the same ufunc sequence applied to z-slabs (y-slabs in 2D) by a
# thread pool. NumPy releases the GIL inside ufuncs, so slabs run in parallel. Each output value
# goes through exactly the operations of ``reference_step``, so the result is bit-identical.
# ---------------------------------------------------------------------------------------------

def _slab_update(u: np.ndarray, out: np.ndarray, c0, c1, periodic: bool,
                 b: np.ndarray | None, lo: int, hi: int) -> None:
    """Write ``out[lo:hi]`` (planes along axis 0) from ``u``; bit-identical to reference_step."""
    n0 = u.shape[0]
    idx = np.arange(lo, hi)
    if periodic:
        im, ip = (idx - 1) % n0, (idx + 1) % n0
    else:
        im, ip = idx - 1, idx + 1
    ctr = u[lo:hi]
    # axis 0 neighbours: a contiguous block unless it wraps
    zm = u[im] if (periodic and (lo == 0 or hi == n0)) else u[lo - 1:hi - 1]
    zp = u[ip] if (periodic and (lo == 0 or hi == n0)) else u[lo + 1:hi + 1]
    if u.ndim == 3:
        if periodic:
            xm, xp = np.roll(ctr, 1, axis=2), np.roll(ctr, -1, axis=2)
            ym, yp = np.roll(ctr, 1, axis=1), np.roll(ctr, -1, axis=1)
            s = xm + xp
            s = s + (ym + yp)
            s = s + (zm + zp)
            new = c0 * ctr + c1 * s
            if b is not None:
                new = new + b[lo:hi]
            out[lo:hi] = new
        else:
            c = ctr[:, 1:-1, 1:-1]
            s = ctr[:, 1:-1, :-2] + ctr[:, 1:-1, 2:]
            s = s + (ctr[:, :-2, 1:-1] + ctr[:, 2:, 1:-1])
            s = s + (zm[:, 1:-1, 1:-1] + zp[:, 1:-1, 1:-1])
            new = c0 * c + c1 * s
            if b is not None:
                new = new + b[lo:hi, 1:-1, 1:-1]
            out[lo:hi, 1:-1, 1:-1] = new
    else:
        if periodic:
            xm, xp = np.roll(ctr, 1, axis=1), np.roll(ctr, -1, axis=1)
            s = xm + xp
            s = s + (zm + zp)
            new = c0 * ctr + c1 * s
            if b is not None:
                new = new + b[lo:hi]
            out[lo:hi] = new
        else:
            c = ctr[:, 1:-1]
            s = ctr[:, :-2] + ctr[:, 2:]
            s = s + (zm[:, 1:-1] + zp[:, 1:-1])
            new = c0 * c + c1 * s
            if b is not None:
                new = new + b[lo:hi, 1:-1]
            out[lo:hi, 1:-1] = new


def threaded_step(u: np.ndarray, out: np.ndarray, c0: float, c1: float, bc: str,
                  b: np.ndarray | None = None, threads: int | None = None,
                  pool: ThreadPoolExecutor | None = None) -> None:
    """``out = reference_step(u, ...)`` computed by ``threads`` workers over slabs of axis 0.

    ``out`` must already hold the Dirichlet boundary values (as both ping-pong buffers do).
    """
    periodic = bc == "periodic"
    cast = u.dtype.type
    c0, c1 = cast(c0), cast(c1)
    n0 = u.shape[0]
    lo0, hi0 = (0, n0) if periodic else (1, n0 - 1)
    threads = max(1, threads or os.cpu_count() or 1)
    nchunks = min(threads * 2, max(1, hi0 - lo0))
    edges = np.linspace(lo0, hi0, nchunks + 1).astype(int)
    jobs = [(int(a), int(e)) for a, e in zip(edges[:-1], edges[1:]) if e > a]
    if pool is None or threads == 1:
        for a, e in jobs:
            _slab_update(u, out, c0, c1, periodic, b, a, e)
        return
    list(pool.map(lambda ae: _slab_update(u, out, c0, c1, periodic, b, *ae), jobs))


def threaded_emulated(u0: np.ndarray, c0: float, c1: float, bc: str, steps: int,
                      storage: str = "float32", k: int = 1, b: np.ndarray | None = None,
                      threads: int | None = None, snapshots: tuple[int, ...] = ()
                      ) -> np.ndarray | dict[int, np.ndarray]:
    """:func:`emulated_reference` computed with :func:`threaded_step` (bit-identical result).

    For full-size grids: every update runs thread-chunked over slabs of axis 0, and the storage
    rounding follows the same schedule (after every pass of ``k`` updates, then after every
    leftover single update). With ``snapshots`` (step counts), returns ``{step: state}`` for
    each requested step reached on the way to ``steps`` (fp32 only, ``k`` = 1), so one
    trajectory serves several checks.
    """
    threads = max(1, threads or os.cpu_count() or 1)
    u = round_storage(np.array(u0, dtype=np.float32, copy=True), storage)
    out = u.copy()  # carries the Dirichlet boundary values
    passes, rem = divmod(steps, k)
    schedule = [k] * passes + [1] * rem
    want = set(snapshots)
    snaps: dict[int, np.ndarray] = {}
    done = 0
    with ThreadPoolExecutor(threads) as pool:
        for n in schedule:
            for _ in range(n):
                threaded_step(u, out, c0, c1, bc, b, threads=threads, pool=pool)
                u, out = out, u
                done += 1
                if done in want:
                    snaps[done] = u.copy()
            if storage != "float32":
                u[...] = round_storage(u, storage)
    if want:
        return snaps
    return u
