"""``B200Stepper``: the pyheat3d ``Stepper`` of this backend.

Same contract as pyheat3d's CuPy stepper (``src/pyheat3d/backends/cupy_backend.py:115-213``):
two device buffers hold the ping-pong pair, ``step(n)`` runs ``n // k`` fused passes and
``n % k`` single steps and is asynchronous, ``get()`` returns a host float32 array. Differences:
the buffers are torch CUDA tensors, the kernels are called through the ``libph3b200`` C ABI on
torch's current stream, and a Jacobi source term is supported (``source=``).

Small grids (fewer than ``GRAPH_CELLS`` sites) are bound by kernel launches, not by memory: a
repeated ``step(n)`` of the same n from the same buffer replays a CUDA graph of that advance
(captured on its second occurrence, after one plain run has set up every launch), with the same
kernels and results. ``PH3_STEP_GRAPHS=0`` turns this off.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _lib
from .contract import Stepper
from .tune import configure

_TORCH_DTYPE_NAMES = {"float32": "float32", "float16": "float16", "bfloat16": "bfloat16"}


def _torch():
    import torch

    return torch


class B200Stepper(Stepper):
    """sm_100a stencil stepper. Subclasses fix ``kind`` ("naive", "march", "tb"), K, storage."""

    kind = "march"
    K = 1
    storage = "float32"
    GRAPH_CELLS = 1 << 22  # grids below this size replay repeated advances as CUDA graphs
    GRAPH_MIN_STEPS = 8

    def __init__(self, u0: np.ndarray, stencil, source: np.ndarray | None = None):
        super().__init__(u0, stencil, source)
        torch = _torch()
        if not torch.cuda.is_available():
            raise RuntimeError("no CUDA device")
        self._lib = _lib.lib()  # fails loudly when the extension is missing
        if self.kind == "auto":  # kernel family and temporal-block depth from the tuning table
            from .tune import active_table

            t = active_table()
            best = t.best_for(self.dims, self.storage, self.ncells) if t is not None else None
            self.kind, self.K = (best["variant"], int(best["k"])) if best else ("march", 1)
        if self.kind == "march" and self.dims not in (2, 3):  # pragma: no cover
            raise ValueError("march needs a 2D or 3D grid")
        self.steps_per_pass = self.K if self.kind == "tb" else 1
        self.device = torch.device("cuda", torch.cuda.current_device())
        dt = getattr(torch, _TORCH_DTYPE_NAMES[self.storage])
        host = torch.from_numpy(np.ascontiguousarray(u0, dtype=np.float32))
        # float32 -> storage on the device: round to nearest even, as cupy_backend.py:103-107
        self.a = host.to(self.device).to(dt).contiguous()
        self.b = self.a.clone()
        self.src = None
        if source is not None:
            if tuple(source.shape) != self.shape:
                raise ValueError(f"source shape {source.shape} != field shape {self.shape}")
            self.src = torch.from_numpy(
                np.ascontiguousarray(source, dtype=np.float32)).to(self.device)
        self._c0 = float(np.float32(self.c0))
        self._c1 = float(np.float32(self.c1))
        sh = self.shape
        self._nz, self._ny, self._nx = (1, sh[0], sh[1]) if self.dims == 2 else sh
        self._variant = _lib.VARIANT[self.kind]
        self._k = self.K if self.kind == "tb" else 1
        self.tile = {"kind": self.kind, "k": self._k}
        if self.kind == "tb":  # the tile of the tb<k> pass, for pyheat3d's halo-traffic model
            configure(self.dims, self.storage, self._k, self.ncells, self._lib)
            tx, ty, ch = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
            _lib.check(self._lib.ph3_tb_tile(
                self.dims, self._nz, self._ny, self._nx, _lib.STORAGE[self.storage],
                _lib.BC[self.bc], self._k, ctypes.byref(tx), ctypes.byref(ty), ctypes.byref(ch)))
            self.tile.update({"tx": tx.value, "ty": ty.value, "zch": ch.value})
        self._in_b = ctypes.c_int(0)
        self._graphs: dict = {}  # (n, start buffer) -> (CUDA graph, ends in the other buffer)
        self._seen: set = set()  # (n, start buffer) advances run once plainly
        self._use_graphs = (self.ncells < self.GRAPH_CELLS
                            and os.environ.get("PH3_STEP_GRAPHS", "1") != "0")

    # -- stepping ------------------------------------------------------------------------
    def _advance(self, n: int, stream: int) -> bool:
        src = self.src.data_ptr() if self.src is not None else None
        _lib.check(self._lib.ph3_advance(
            self.dims, self._nz, self._ny, self._nx, _lib.STORAGE[self.storage],
            _lib.BC[self.bc], self._c0, self._c1, self._variant, self._k,
            self.a.data_ptr(), self.b.data_ptr(), src, int(n), stream,
            ctypes.byref(self._in_b)))
        return bool(self._in_b.value)

    def step(self, n: int = 1) -> None:
        if n < 0:
            raise ValueError("n must be >= 0")
        torch = _torch()
        cur = torch.cuda.current_stream(self.device)
        configure(self.dims, self.storage, self._k, self.ncells, self._lib)
        key = (int(n), self.a.data_ptr())
        if self._use_graphs and n >= self.GRAPH_MIN_STEPS and not torch.cuda.is_current_stream_capturing():
            g = self._graphs.get(key)
            if g is None and key in self._seen:  # second occurrence: capture, then replay
                side = torch.cuda.Stream(self.device)
                side.wait_stream(cur)
                graph = torch.cuda.CUDAGraph()
                with torch.cuda.graph(graph, stream=side):
                    swap = self._advance(n, side.cuda_stream)
                cur.wait_stream(side)
                g = self._graphs[key] = (graph, swap)
            if g is not None:
                g[0].replay()
                if g[1]:
                    self.a, self.b = self.b, self.a
                self.steps_done += n
                return
            self._seen.add(key)
        if self._advance(n, cur.cuda_stream):
            self.a, self.b = self.b, self.a
        self.steps_done += n

    def get(self, out=None) -> np.ndarray:
        """Current state as a host float32 array.

        ``out`` (optional): a host float32 torch tensor of the field's shape, typically pinned;
        the device-to-host copy then lands there (asynchronously for pinned memory, followed by
        a stream synchronisation) and its NumPy view is returned.
        """
        if out is None:
            return self.a.float().cpu().numpy()
        torch = _torch()
        src = self.a if self.a.dtype == torch.float32 else self.a.float()
        out.copy_(src, non_blocking=True)
        torch.cuda.current_stream(self.device).synchronize()
        return out.numpy()

    def set_state(self, u) -> None:
        """Replace the state by ``u`` (NumPy array or host / device torch tensor of the shape).

        Host tensors in pinned memory are copied asynchronously on the current stream. With
        Dirichlet boundaries both ping-pong buffers receive the new boundary values.
        """
        torch = _torch()
        t = torch.from_numpy(np.ascontiguousarray(u, dtype=np.float32)) if isinstance(
            u, np.ndarray) else u
        if tuple(t.shape) != self.shape:
            raise ValueError(f"state shape {tuple(t.shape)} != field shape {self.shape}")
        if self.a.dtype == t.dtype:
            self.a.copy_(t, non_blocking=True)
        else:
            self.a.copy_(t.to(self.device, non_blocking=True).to(self.a.dtype))
        if not self.periodic:
            self.b.copy_(self.a)

    def get_tensor(self):
        """Current state as the device tensor (storage dtype); no copy."""
        return self.a

    def synchronize(self) -> None:
        _torch().cuda.synchronize(self.device)

    def close(self) -> None:
        self._graphs.clear()
        self.a = self.b = self.src = None


def make(kind: str, storage: str = "float32", K: int = 1) -> type[B200Stepper]:
    """A ``B200Stepper`` subclass for a kernel family, storage type and K (cupy_backend.py:207).

    ``kind="auto"`` picks family and K per grid from the tuning table (pyheat3d_b200.tune).
    """
    if kind not in _lib.VARIANT and kind != "auto":
        raise ValueError(f"unknown kind {kind!r}")
    if storage not in _lib.STORAGE:
        raise ValueError(f"unknown storage {storage!r}")
    _lib.lib()  # availability probe: raises if the extension cannot be loaded
    return type(f"B200_{kind}{K}_{storage}", (B200Stepper,),
                {"kind": kind, "storage": storage, "K": K})
