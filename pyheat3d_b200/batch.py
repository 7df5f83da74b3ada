"""Batched solves: many uneven grids advanced in one persistent launch (optionally a CUDA graph).

Host side of ``ph3_batch_*`` (``include/ph3b200.h``). No counterpart in pyheat3d, which advances
one grid at a time with one launch per step (``src/pyheat3d/backends/cupy_backend.py:183-194``);
the per-problem results are bit-identical to the single-grid steppers.

    batch = Batch([Problem(u0, heat_stencil(3, 0.15), steps=500, storage="bfloat16"), ...])
    batch.run()                  # one launch
    g = batch.graph()            # or: capture launch (+ state reset) in a CUDA graph
    g.replay()
    outs = batch.results()       # host float32 arrays

:func:`synthetic_batch` draws the problem mix of the batching benchmark (half 2D, half 3D,
log-uniform sizes, random r, boundary, storage and step counts, one seed).
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np

from . import _lib


def _torch():
    import torch

    return torch


class ProblemDesc(ctypes.Structure):
    """ctypes mirror of ``ph3_problem``."""

    _fields_ = [("a", ctypes.c_void_p), ("b", ctypes.c_void_p), ("src", ctypes.c_void_p),
                ("dims", ctypes.c_int32), ("nz", ctypes.c_int32), ("ny", ctypes.c_int32),
                ("nx", ctypes.c_int32), ("bc", ctypes.c_int32), ("storage", ctypes.c_int32),
                ("c0", ctypes.c_float), ("c1", ctypes.c_float), ("steps", ctypes.c_int32),
                ("k", ctypes.c_int32)]


@dataclass
class Problem:
    """One grid: initial state, coefficients (``stencil`` with c0, c1, bc), steps, storage."""

    u0: np.ndarray
    stencil: object
    steps: int
    storage: str = "float32"
    source: np.ndarray | None = None
    k: int = 1  # fused steps per pass: 1, or 2 / 4 for 2D grids

    @property
    def passes(self) -> int:
        """Passes over the grid: steps, or steps // k fused passes and steps % k single steps."""
        return self.steps // self.k + self.steps % self.k if self.k > 1 else self.steps

    @property
    def cells(self) -> int:
        """Site updates per step (interior for Dirichlet, all cells for periodic)."""
        if self.stencil.bc == "periodic":
            return int(np.prod(self.u0.shape))
        return int(np.prod([s - 2 for s in self.u0.shape]))


class Batch:
    """Device-resident fields of a problem list plus the prepared persistent-launch plan."""

    def __init__(self, problems: list[Problem], device=None):
        torch = _torch()
        if not torch.cuda.is_available():
            raise RuntimeError("no CUDA device")
        self.lib = _lib.lib()
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self.problems = list(problems)
        n = len(self.problems)
        self.descs = (ProblemDesc * max(n, 1))()
        self.a, self.b, self.init, self.src = [], [], [], []
        for i, p in enumerate(self.problems):
            if p.u0.ndim not in (2, 3):
                raise ValueError(f"problem {i}: u0 must be 2D or 3D")
            dt = getattr(torch, p.storage)
            host = torch.from_numpy(np.ascontiguousarray(p.u0, dtype=np.float32))
            a = host.to(self.device).to(dt).contiguous()
            self.init.append(a.clone())
            self.a.append(a)
            self.b.append(a.clone())
            s = None
            if p.source is not None:
                s = torch.from_numpy(np.ascontiguousarray(p.source, np.float32)).to(self.device)
            self.src.append(s)
            d = self.descs[i]
            d.a, d.b = a.data_ptr(), self.b[i].data_ptr()
            d.src = s.data_ptr() if s is not None else None
            d.dims = p.u0.ndim
            d.nz, d.ny, d.nx = (1, *p.u0.shape) if p.u0.ndim == 2 else p.u0.shape
            d.bc = _lib.BC[p.stencil.bc]
            d.storage = _lib.STORAGE[p.storage]
            d.c0 = float(np.float32(p.stencil.c0))
            d.c1 = float(np.float32(p.stencil.c1))
            d.steps = int(p.steps)
            d.k = int(p.k)
        self.n = n
        from .tune import configure_batch

        configure_batch(self.lib)  # tile configuration from the tuning table, if one is active
        descs = ctypes.addressof(self.descs)
        nbytes = int(self.lib.ph3_batch_workspace_bytes(descs, n))
        if nbytes < 0:
            _lib.check(1)
        self.ws = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=self.device)
        _lib.check(self.lib.ph3_batch_prepare(descs, n, self.ws.data_ptr(), self.ws.numel(),
                                              self._stream()))

    def _stream(self):
        return _torch().cuda.current_stream(self.device).cuda_stream

    @property
    def updates(self) -> int:
        """Total site updates of one run."""
        return sum(p.cells * p.steps for p in self.problems)

    def reset(self) -> None:
        """Restore every problem's initial state (both buffers) on the current stream."""
        for a, b, x in zip(self.a, self.b, self.init):
            a.copy_(x)
            b.copy_(x)

    def run(self) -> None:
        """One persistent launch advancing every problem by its step count (asynchronous)."""
        _lib.check(self.lib.ph3_batch_launch(self.ws.data_ptr(), self.n, self._stream()))

    def graph(self, with_reset: bool = True):
        """A CUDA graph of (state reset +) the persistent launch; call ``.replay()``."""
        torch = _torch()
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):  # warm-up on the capture stream
            if with_reset:
                self.reset()
            self.run()
        torch.cuda.current_stream(self.device).wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            if with_reset:
                self.reset()
            self.run()
        return g

    def result_tensor(self, i: int):
        """Device tensor holding problem i's final state."""
        return self.b[i] if self.problems[i].passes % 2 else self.a[i]

    def results(self) -> list[np.ndarray]:
        return [self.result_tensor(i).float().cpu().numpy() for i in range(self.n)]


def synthetic_batch(n: int = 512, seed: int = 0, n2d: tuple[int, int] = (64, 2048),
                    n3d: tuple[int, int] = (32, 256), steps: tuple[int, int] = (50, 2000),
                    storages: tuple[str, ...] = ("float32", "bfloat16")) -> list[Problem]:
    """The batching benchmark's problem mix (all draws from one seed).

    Half 2D with N log-uniform in n2d, half 3D with N log-uniform in n3d; r uniform in
    [0.05, 0.95/(2d)]; Dirichlet or periodic at random; storage drawn from ``storages``; steps
    uniform in ``steps``; fields uniform random [0, 1).
    """
    from .contract import heat_stencil

    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        dims = 2 if i < n // 2 else 3
        lo, hi = n2d if dims == 2 else n3d
        size = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
        r = float(rng.uniform(0.05, 0.95 / (2 * dims)))
        bc = "dirichlet" if rng.random() < 0.5 else "periodic"
        storage = storages[int(rng.integers(len(storages)))]
        nsteps = int(rng.integers(steps[0], steps[1] + 1))
        u0 = rng.random((size,) * dims, dtype=np.float32)
        out.append(Problem(u0, heat_stencil(dims, r, bc), nsteps, storage))
    return out
