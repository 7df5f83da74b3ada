"""Z-slab split of one 3D grid over several GPUs, one process per GPU.

No counterpart in pyheat3d, which runs one grid on one GPU (``cupy_backend.py:188-194``). The
grid's planes are dealt out in contiguous slabs, one per rank. Each rank keeps its slab between
two halo planes, ``(n + 2, ny, nx)`` per ping-pong buffer on its own GPU, and per time step:

1. posts the halo exchange of the current buffer: its first owned plane goes to the previous
   rank (which stores it as its upper halo), its last owned plane to the next rank (its lower
   halo); ``torch.distributed`` point-to-point over NCCL (NVLink / NVSwitch), landing in the
   receiver's own memory, so every kernel reads local memory only;
2. updates the planes that need no halo (``ph3_zmarch3d_planes`` on planes 2 .. n-1) while the
   exchange is in flight;
3. waits for the exchange and updates the first and last owned planes.

Periodic grids wrap the ring of ranks (and x / y inside each slab); Dirichlet grids keep the
global boundary planes fixed, so the end ranks neither send nor receive past them. With one
rank the periodic halos are two local plane copies. The results are bit-identical to the
single-GPU z-march of the whole grid, whatever the split.

The arithmetic of every rank is the single-step z-march, so the split covers the single-step
variant only; fused temporal blocks would need k halo planes per pass and are not split.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _lib
from .tune import configure


@dataclass(frozen=True)
class SlabSplit:
    """Planes [0, nz) of a grid dealt to ``world`` ranks in contiguous, near-equal slabs."""

    nz: int
    world: int
    periodic: bool

    def __post_init__(self):
        if self.world < 1:
            raise ValueError("world must be >= 1")
        if self.nz < max(3, self.world):
            raise ValueError(f"{self.nz} planes cannot be split over {self.world} ranks "
                             "(at least 3 planes and one per rank)")

    def bounds(self, rank: int) -> tuple[int, int]:
        """Global planes [zb, ze) owned by ``rank`` (the first nz % world ranks own one more)."""
        if not 0 <= rank < self.world:
            raise ValueError(f"rank {rank} outside [0, {self.world})")
        q, r = divmod(self.nz, self.world)
        zb = rank * q + min(rank, r)
        return zb, zb + q + (1 if rank < r else 0)

    def planes(self, rank: int) -> int:
        zb, ze = self.bounds(rank)
        return ze - zb

    def prev(self, rank: int) -> int | None:
        """Rank owning the plane below this slab (None at a Dirichlet end)."""
        if rank > 0:
            return rank - 1
        return self.world - 1 if self.periodic else None

    def next(self, rank: int) -> int | None:
        """Rank owning the plane above this slab (None at a Dirichlet end)."""
        if rank < self.world - 1:
            return rank + 1
        return 0 if self.periodic else None

    def update_range(self, rank: int) -> tuple[int, int]:
        """Local planes [z0, z1) a step updates in the (n + 2)-plane buffer: every owned plane,
        except the global boundary planes of a Dirichlet grid (kept fixed)."""
        zb, ze = self.bounds(rank)
        n = ze - zb
        z0 = 1 + (1 if not self.periodic and zb == 0 else 0)
        z1 = n + 1 - (1 if not self.periodic and ze == self.nz else 0)
        return z0, max(z0, z1)

    def halo_plan(self, rank: int) -> list[tuple[str, int, int]]:
        """Point-to-point transfers of one exchange, in the order every rank posts them:
        ``("send", peer, local plane)`` then ``("recv", peer, local plane)``.

        Sends go to the previous rank first, then the next; receives come from the next rank
        first, then the previous. With two ranks on a periodic ring the same peer is both, and
        this order pairs each rank's first send with the other's first receive (messages between
        a pair of ranks are matched in posting order).
        """
        n = self.planes(rank)
        p, q = self.prev(rank), self.next(rank)
        plan = []
        if p is not None:
            plan.append(("send", p, 1))
        if q is not None:
            plan.append(("send", q, n))
        if q is not None:
            plan.append(("recv", q, n + 1))
        if p is not None:
            plan.append(("recv", p, 0))
        return plan

    def slab_of(self, u: np.ndarray, rank: int) -> np.ndarray:
        """The (n + 2)-plane local array of ``rank`` cut from a global array: owned planes and
        their halos (wrapped for a periodic grid; zero planes beyond a Dirichlet end, never
        read)."""
        zb, ze = self.bounds(rank)
        out = np.zeros((ze - zb + 2,) + u.shape[1:], dtype=u.dtype)
        out[1:-1] = u[zb:ze]
        lo, hi = zb - 1, ze
        if self.periodic:
            out[0] = u[lo % self.nz]
            out[-1] = u[hi % self.nz]
        else:
            if lo >= 0:
                out[0] = u[lo]
            if hi < self.nz:
                out[-1] = u[hi]
        return out


def exchange_halos(buf, split: SlabSplit, rank: int, group=None, async_op: bool = False):
    """Refresh the two halo planes of ``buf`` (``(n + 2, ny, nx)``, any device) from the
    neighbouring ranks through ``torch.distributed``; with one rank, the periodic wrap is two
    local copies. Returns the pending requests when ``async_op`` (wait on each before reading
    the halos), else waits and returns an empty list."""
    if split.world == 1:
        if split.periodic:
            n = split.planes(0)
            buf[0].copy_(buf[n])
            buf[n + 1].copy_(buf[1])
        return []
    import torch.distributed as dist

    ops = []
    for kind, peer, plane in split.halo_plan(rank):
        fn = dist.isend if kind == "send" else dist.irecv
        ops.append(dist.P2POp(fn, buf[plane], peer, group))
    reqs = dist.batch_isend_irecv(ops) if ops else []
    if async_op:
        return reqs
    for r in reqs:
        r.wait()
    return []


class SlabStepper:
    """One rank's slab of a z-split 3D grid on this process's current GPU.

    ``slab``: the rank's ``(n + 2, ny, nx)`` local array (``SlabSplit.slab_of``), host NumPy.
    ``stencil``: coefficients and boundary condition of the whole grid (``contract.Stencil``);
    its boundary must match ``split.periodic``. ``source``: optional Jacobi source of the same
    local shape (fp32). ``overlap``: update the halo-free planes while the exchange is in flight.
    """

    def __init__(self, slab: np.ndarray, stencil, split: SlabSplit, rank: int,
                 storage: str = "float32", source: np.ndarray | None = None, group=None,
                 overlap: bool = True):
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError("no CUDA device")
        self._lib = _lib.lib()  # fails loudly when the extension is missing
        if slab.ndim != 3:
            raise ValueError("the slab split is for 3D grids")
        if (stencil.bc == "periodic") != split.periodic:
            raise ValueError("stencil boundary and split disagree")
        n = split.planes(rank)
        if slab.shape[0] != n + 2:
            raise ValueError(f"rank {rank} owns {n} planes: slab needs {n + 2}, got {slab.shape[0]}")
        # nothing to overlap with one rank: its halos are two local copies
        self.split, self.rank, self.group = split, rank, group
        self.overlap = overlap and split.world > 1
        self.storage = storage
        self.device = torch.device("cuda", torch.cuda.current_device())
        dt = getattr(torch, storage)
        host = torch.from_numpy(np.ascontiguousarray(slab, dtype=np.float32))
        self.a = host.to(self.device).to(dt).contiguous()
        self.b = self.a.clone()  # fixed planes (Dirichlet) must be in both buffers
        self.src = None
        if source is not None:
            if source.shape != slab.shape:
                raise ValueError(f"source shape {source.shape} != slab shape {slab.shape}")
            self.src = torch.from_numpy(np.ascontiguousarray(source, dtype=np.float32)).to(
                self.device)
        self.c0 = float(np.float32(stencil.c0))
        self.c1 = float(np.float32(stencil.c1))
        self.bc = _lib.BC[stencil.bc]
        self.z0, self.z1 = split.update_range(rank)
        self.nz, self.ny, self.nx = self.a.shape
        self.steps_done = 0
        self.ncells = (self.z1 - self.z0) * self.ny * self.nx  # site updates per step

    def _planes(self, z0: int, z1: int, stream: int) -> None:
        if z1 <= z0:
            return
        src = self.src.data_ptr() if self.src is not None else None
        _lib.check(self._lib.ph3_zmarch3d_planes(
            self.a.data_ptr(), self.b.data_ptr(), src, self.nz, self.ny, self.nx, z0, z1,
            self.c0, self.c1, _lib.STORAGE[self.storage], self.bc, 0, stream))

    def step(self, n: int = 1) -> None:
        """n steps: per step one halo exchange and the update of the owned planes."""
        import torch

        if n < 0:
            raise ValueError("n must be >= 0")
        stream = torch.cuda.current_stream(self.device).cuda_stream
        configure(3, self.storage, 1, self.split.nz * self.ny * self.nx, self._lib)
        z0, z1 = self.z0, self.z1
        for _ in range(n):
            if self.overlap and z1 - z0 >= 3:
                # the exchange is posted first, so it waits only for the previous step
                reqs = exchange_halos(self.a, self.split, self.rank, self.group, async_op=True)
                self._planes(z0 + 1, z1 - 1, stream)
                for r in reqs:
                    r.wait()
                self._planes(z0, z0 + 1, stream)
                self._planes(z1 - 1, z1, stream)
            else:
                exchange_halos(self.a, self.split, self.rank, self.group)
                self._planes(z0, z1, stream)
            self.a, self.b = self.b, self.a
        self.steps_done += n

    def owned(self):
        """The owned planes of the current state (a device tensor view, storage dtype)."""
        return self.a[1:-1]

    def get(self) -> np.ndarray:
        """Owned planes of the current state as a host float32 array."""
        return self.owned().float().cpu().numpy()


def gather_planes(owned, split: SlabSplit, rank: int, group=None):
    """Assemble the global grid on rank 0 from every rank's owned planes (``owned``: a tensor of
    ``split.planes(rank)`` planes on the device the process group communicates from). Returns a
    float32 NumPy array on rank 0, None elsewhere."""
    import torch
    import torch.distributed as dist

    nmax = max(split.planes(r) for r in range(split.world))
    pad = torch.zeros((nmax,) + tuple(owned.shape[1:]), dtype=owned.dtype, device=owned.device)
    pad[:owned.shape[0]] = owned
    parts = [torch.empty_like(pad) for _ in range(split.world)] if rank == 0 else None
    dist.gather(pad, parts, dst=0, group=group)
    if rank != 0:
        return None
    return np.concatenate([parts[r][:split.planes(r)].float().cpu().numpy()
                           for r in range(split.world)], axis=0)
