"""Serving: a continuous-batching request loop for heat and Jacobi solves.

No counterpart in pyheat3d (one solve at a time from the CLI, ``src/pyheat3d/cli.py:28-51``).

Requests arrive over time (a Poisson stream in the benchmark). The engine keeps every admitted
request's fields resident on the device and advances all of them together: each *round* is one
persistent batch launch (``ph3_batch_run_static``, falling back to a workspace launch for large
plans) that moves every active request forward by up to ``quantum`` steps. Between rounds,
finished requests leave (result copied to the host, memory released) and newly arrived requests
are admitted while a slot and the HBM budget allow. Requests that arrive while others are on the
GPU therefore join the very next round, and their work overlaps on the device.

* heat request: ``steps`` FTCS updates; done when they are all applied;
* Jacobi request for A u = f (A the 2d+1-point Laplacian over h^2, Dirichlet zero walls): sweeps
  ``u' = S(u)/(2d) + b`` with ``b = -h^2 f / (2d)`` until the relative residual
  ``||f - A u|| / ||f||`` is at most ``tol`` or ``max_sweeps`` is reached. One sweep's change is
  the scaled residual of the iterate it started from, ``u_k+1 - u_k = -(h^2/(2d)) (f - A u_k)``,
  so the relative residual of u_k is ``||u_k+1 - u_k|| / ||b||``: the two ping-pong buffers hold
  both iterates after each round and the norms are taken on the device (one synchronisation per
  round for all Jacobi requests). With 16-bit storage the iterates are the stored (rounded)
  values, whose residual stalls near the storage resolution; such requests end at the cap.

Each result equals the same request run alone with the same step / sweep count, bit for bit: a
problem's arithmetic does not depend on what else is in the batch.

:class:`PlainServer` is the baseline: first come, first served, one solve at a time, each solve
one call of the single-grid launch loop (``ph3_advance``).

The engine is written against a small executor interface (``alloc``, ``advance``, ``converged``,
``fetch``, ``free``) so its scheduling can run on CPU with a fake executor in tests.
"""

from __future__ import annotations

import ctypes
import heapq
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib

ES = {"float32": 4, "float16": 2, "bfloat16": 2}


@dataclass
class Request:
    """One solve request. Fields are generated on the device from ``seed``."""

    rid: int
    arrival: float                 # seconds after the stream starts
    kind: str                      # "heat" | "jacobi"
    dims: int
    n: int                         # grid edge
    bc: str
    storage: str
    r: float = 0.0                 # heat: mesh Fourier number
    steps: int = 0                 # heat: updates
    tol: float = 0.0               # jacobi: relative-residual tolerance
    max_sweeps: int = 20000        # jacobi: cap
    seed: int = 0

    @property
    def shape(self) -> tuple[int, ...]:
        return (self.n,) * self.dims

    @property
    def cells(self) -> int:
        if self.bc == "periodic":
            return self.n ** self.dims
        return (self.n - 2) ** self.dims

    @property
    def device_bytes(self) -> int:
        """HBM the request holds while resident: two field buffers (+ fp32 source)."""
        nb = 2 * ES[self.storage] * self.n ** self.dims
        if self.kind == "jacobi":
            nb += 4 * self.n ** self.dims
        return nb

    def coefficients(self) -> tuple[float, float]:
        if self.kind == "heat":
            return 1.0 - 2.0 * self.dims * self.r, self.r
        return 0.0, 1.0 / (2 * self.dims)


@dataclass
class Outcome:
    rid: int
    kind: str
    arrival: float
    admitted: float
    finished: float
    steps_done: int
    converged: bool
    result: np.ndarray | None = None

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def poisson_stream(rate: float, duration: float, seed: int = 0, n2d=(64, 2048), n3d=(32, 256),
                   steps=(50, 2000), tol=(1e-10, 1e-6), jacobi_fraction: float = 0.5,
                   storages=("float32", "bfloat16"), max_sweeps: int = 20000) -> list[Request]:
    """Requests of the serving benchmark: Poisson arrivals, sizes as in the batching mix."""
    rng = np.random.default_rng(seed)
    out, t, rid = [], 0.0, 0
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t >= duration:
            break
        dims = 2 if rng.random() < 0.5 else 3
        lo, hi = n2d if dims == 2 else n3d
        n = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
        storage = storages[int(rng.integers(len(storages)))]
        if rng.random() < jacobi_fraction:
            req = Request(rid, t, "jacobi", dims, n, "dirichlet", storage,
                          tol=float(math.exp(rng.uniform(math.log(tol[0]), math.log(tol[1])))),
                          max_sweeps=max_sweeps, seed=int(rng.integers(1 << 31)))
        else:
            req = Request(rid, t, "heat", dims, n,
                          "dirichlet" if rng.random() < 0.5 else "periodic", storage,
                          r=float(rng.uniform(0.05, 0.95 / (2 * dims))),
                          steps=int(rng.integers(steps[0], steps[1] + 1)),
                          seed=int(rng.integers(1 << 31)))
        out.append(req)
        rid += 1
    return out


# ------------------------------------------------------------------------------------------
# GPU executor
# ------------------------------------------------------------------------------------------
class _Slot:
    __slots__ = ("req", "a", "b", "src", "in_b", "done", "last_change", "src_norm")

    def __init__(self, req, a, b, src):
        self.req, self.a, self.b, self.src = req, a, b, src
        self.in_b = False      # current state in b
        self.done = 0          # steps / sweeps applied
        self.last_change = math.inf  # Jacobi: relative residual of the previous iterate
        self.src_norm = None   # Jacobi: ||b||, a device scalar (set at allocation)


class GpuExecutor:
    """Device side of the engine: fields in torch tensors, rounds as batch launches."""

    def __init__(self, device=None):
        import torch

        from .batch import ProblemDesc

        if not torch.cuda.is_available():
            raise RuntimeError("no CUDA device")
        self.torch = torch
        self.lib = _lib.lib()
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self.Desc = ProblemDesc
        self._ws = None

    def init_fields(self, req: Request):
        """Initial field (and source) of a request, generated on the device from its seed."""
        torch = self.torch
        g = torch.Generator(device=self.device)
        g.manual_seed(req.seed)
        u = torch.rand(req.shape, generator=g, device=self.device, dtype=torch.float32)
        src = None
        if req.kind == "jacobi":
            u.zero_()
            h = 1.0 / (req.n - 1)
            f = torch.rand(req.shape, generator=g, device=self.device, dtype=torch.float32) - 0.5
            src = (-(h * h) / (2 * req.dims)) * f
        return u, src

    def alloc(self, req: Request) -> _Slot:
        u, src = self.init_fields(req)
        a = u.to(getattr(self.torch, req.storage)).contiguous()
        slot = _Slot(req, a, a.clone(), src)
        if src is not None:
            slot.src_norm = src.norm()
        return slot

    def advance(self, slots: list[_Slot], counts: list[int]) -> None:
        """One round: every slot advances by its count, in one persistent launch."""
        n = len(slots)
        descs = (self.Desc * max(n, 1))()
        for i, (s, c) in enumerate(zip(slots, counts)):
            d = descs[i]
            cur, nxt = (s.b, s.a) if s.in_b else (s.a, s.b)
            d.a, d.b = cur.data_ptr(), nxt.data_ptr()
            d.src = s.src.data_ptr() if s.src is not None else None
            d.dims = s.req.dims
            d.nz, d.ny, d.nx = (1, s.req.n, s.req.n) if s.req.dims == 2 else s.req.shape
            d.bc = _lib.BC[s.req.bc]
            d.storage = _lib.STORAGE[s.req.storage]
            c0, c1 = s.req.coefficients()
            d.c0, d.c1 = float(np.float32(c0)), float(np.float32(c1))
            d.steps = int(c)
            d.k = 1
        addr = ctypes.addressof(descs)
        need = int(self.lib.ph3_batch_workspace_bytes(addr, n))
        # the library's fixed workspace belongs to the current device: make it this one
        with self.torch.cuda.device(self.device):
            stream = self.torch.cuda.current_stream(self.device).cuda_stream
            if need <= _lib.STATIC_BATCH_BYTES:
                _lib.check(self.lib.ph3_batch_run_static(addr, n, stream))
            else:  # plan larger than the fixed workspace: use an allocated one
                if self._ws is None or self._ws.numel() < need:
                    self._ws = self.torch.empty(need, dtype=self.torch.uint8, device=self.device)
                _lib.check(self.lib.ph3_batch_prepare(addr, n, self._ws.data_ptr(),
                                                      self._ws.numel(), stream))
                _lib.check(self.lib.ph3_batch_launch(self._ws.data_ptr(), n, stream))
        for s, c in zip(slots, counts):
            if c % 2:
                s.in_b = not s.in_b
            s.done += c

    def converged(self, s: _Slot) -> bool:
        """Jacobi: relative residual ||f - A u|| / ||f|| of the previous iterate within tol."""
        return self.converged_many([s])[0]

    def converged_many(self, slots: list[_Slot]) -> list[bool]:
        """:meth:`converged` for several slots with a single device synchronisation."""
        torch = self.torch
        if not slots:
            return []
        pairs = []
        for s in slots:
            cur, prev = (s.b, s.a) if s.in_b else (s.a, s.b)
            pairs.append(torch.stack([(cur.float() - prev.float()).norm(), s.src_norm]))
        vals = torch.stack(pairs).cpu().tolist()
        out = []
        for s, (diff, bn) in zip(slots, vals):
            s.last_change = diff / bn if bn > 0 else 0.0
            out.append(s.done > 0 and s.last_change <= s.req.tol)
        return out

    def fetch(self, s: _Slot) -> np.ndarray:
        return ((s.b if s.in_b else s.a).float()).cpu().numpy()

    def free(self, s: _Slot) -> None:
        s.a = s.b = s.src = None

    def synchronize(self) -> None:
        self.torch.cuda.synchronize(self.device)

    def advance_alone(self, s: _Slot, count: int) -> None:
        """Plain path: one ph3_advance call (the single-grid launch loop) of `count` steps."""
        req = s.req
        c0, c1 = req.coefficients()
        nz, ny, nx = (1, req.n, req.n) if req.dims == 2 else req.shape
        cur, nxt = (s.b, s.a) if s.in_b else (s.a, s.b)
        ib = ctypes.c_int(0)
        _lib.check(self.lib.ph3_advance(
            req.dims, nz, ny, nx, _lib.STORAGE[req.storage], _lib.BC[req.bc],
            float(np.float32(c0)), float(np.float32(c1)), _lib.VARIANT["march"], 1,
            cur.data_ptr(), nxt.data_ptr(), s.src.data_ptr() if s.src is not None else None,
            int(count), self.torch.cuda.current_stream(self.device).cuda_stream,
            ctypes.byref(ib)))
        if ib.value:
            s.in_b = not s.in_b
        s.done += count

    def solve_alone(self, req: Request, count: int) -> _Slot:
        """Fresh fields for `req`, advanced by `count` steps in one ph3_advance call."""
        s = self.alloc(req)
        self.advance_alone(s, count)
        return s


# ------------------------------------------------------------------------------------------
# engines
# ------------------------------------------------------------------------------------------
@dataclass
class ServeStats:
    outcomes: list[Outcome]
    wall: float
    rounds: int
    submitted: int
    peak_bytes: int
    backlog: int
    updates: int
    extra: dict = field(default_factory=dict)
    #: arrival times of the requests that had arrived but not finished when the run ended
    open_arrivals: list[float] = field(default_factory=list)

    def latencies_all(self) -> list[float]:
        """Latency of every arrived request: completed ones by latency, unfinished ones by
        their age when the run ended (right-censored: a lower bound of their latency)."""
        return [o.latency for o in self.outcomes] + [max(0.0, self.wall - a)
                                                      for a in self.open_arrivals]

    def summary(self) -> dict:
        lat_done = (np.array([o.latency for o in self.outcomes]) if self.outcomes
                    else np.array([np.nan]))
        lat_all = np.array(self.latencies_all() or [np.nan])
        return {
            "completed": len(self.outcomes), "submitted": self.submitted,
            "backlog": self.backlog, "wall_s": round(self.wall, 3),
            "solves_per_s": round(len(self.outcomes) / self.wall, 2) if self.wall > 0 else 0.0,
            # over every arrived request; unfinished ones count with their age at the end
            "p50_ms": round(float(np.percentile(lat_all, 50)) * 1e3, 2),
            "p99_ms": round(float(np.percentile(lat_all, 99)) * 1e3, 2),
            "censored": len(self.open_arrivals),
            "completed_p50_ms": round(float(np.percentile(lat_done, 50)) * 1e3, 2),
            "completed_p99_ms": round(float(np.percentile(lat_done, 99)) * 1e3, 2),
            "glups": round(self.updates / self.wall / 1e9, 2) if self.wall > 0 else 0.0,
            "rounds": self.rounds, "peak_hbm_gb": round(self.peak_bytes / 1e9, 2),
            "jacobi_converged": sum(o.converged for o in self.outcomes if o.kind == "jacobi"),
            "jacobi_capped": sum((not o.converged) for o in self.outcomes if o.kind == "jacobi"),
            **self.extra,
        }


class Server:
    """Continuous-batching engine.

    ``budget_bytes``: HBM the resident requests may hold together; ``max_active``: slots;
    ``quantum``: steps / sweeps per request per round; ``duration``: stop admitting at this time
    (seconds after start; requests already admitted run to completion unless ``drain`` is False);
    ``keep_results``: copy every result to the host.
    """

    def __init__(self, executor, budget_bytes: float = 150e9, max_active: int = 1024,
                 quantum: int = 64, keep_results: bool = False, clock=time.perf_counter,
                 sleep=time.sleep, keep_ids=()):
        self.ex = executor
        self.budget = float(budget_bytes)
        self.max_active = max_active
        self.quantum = quantum
        self.keep = keep_results
        self.keep_ids = set(keep_ids)  # requests whose results are copied back in any case
        self.clock = clock
        self.sleep = sleep

    def run(self, requests: list[Request], duration: float | None = None,
            drain: bool = True) -> ServeStats:
        pending = sorted(requests, key=lambda r: r.arrival)
        arrived: list[tuple[float, int, Request]] = []
        active: list[tuple[_Slot, float]] = []
        used = 0
        peak = 0
        outcomes = []
        rounds = 0
        updates = 0
        horizon = duration if duration is not None else math.inf
        t0 = self.clock()
        i = 0
        while True:
            now = self.clock() - t0
            while i < len(pending) and pending[i].arrival <= min(now, horizon):
                heapq.heappush(arrived, (pending[i].arrival, pending[i].rid, pending[i]))
                i += 1
            # admit in arrival order while a slot and the budget allow
            while arrived and len(active) < self.max_active:
                req = arrived[0][2]
                if used + req.device_bytes > self.budget:
                    if not active and req.device_bytes > self.budget:
                        heapq.heappop(arrived)  # can never fit: reject
                        continue
                    break
                heapq.heappop(arrived)
                slot = self.ex.alloc(req)
                used += req.device_bytes
                peak = max(peak, used)
                active.append((slot, self.clock() - t0))
            if not active:
                if i >= len(pending) or now >= horizon:
                    break
                nxt = pending[i].arrival
                if nxt > now:
                    self.sleep(min(nxt - now, 0.01))
                continue
            if now >= horizon and not drain:
                break
            counts = []
            for slot, _ in active:
                req = slot.req
                left = (req.steps if req.kind == "heat" else req.max_sweeps) - slot.done
                counts.append(max(0, min(self.quantum, left)))
            self.ex.advance([s for s, _ in active], counts)
            self.ex.synchronize()
            rounds += 1
            for (slot, _), c in zip(active, counts):
                updates += slot.req.cells * c
            still = []
            tnow = None
            jac = [s for s, _ in active if s.req.kind == "jacobi"]
            many = getattr(self.ex, "converged_many", None)
            conv_of = dict(zip(map(id, jac), many(jac) if many else
                               [self.ex.converged(s) for s in jac]))
            for slot, adm in active:
                req = slot.req
                if req.kind == "heat":
                    fin, conv = slot.done >= req.steps, True
                else:
                    conv = conv_of[id(slot)]
                    fin = conv or slot.done >= req.max_sweeps
                if fin:
                    res = self.ex.fetch(slot) if self.keep or req.rid in self.keep_ids else None
                    tnow = self.clock() - t0
                    outcomes.append(Outcome(req.rid, req.kind, req.arrival, adm, tnow, slot.done,
                                            conv, res))
                    self.ex.free(slot)
                    used -= req.device_bytes
                else:
                    still.append((slot, adm))
            active = still
        wall = self.clock() - t0
        backlog = len(arrived) + len(active) + (len(pending) - i)
        open_arr = [a for a, _, _ in arrived] + [s.req.arrival for s, _ in active] + [
            r.arrival for r in pending[i:] if r.arrival <= wall]
        return ServeStats(outcomes, wall, rounds, len(requests), peak, backlog, updates,
                          open_arrivals=open_arr)


class PlainServer:
    """Baseline: first come, first served, one solve at a time, one ``ph3_advance`` per solve.

    Jacobi solves advance ``quantum`` sweeps per call and check convergence in between (the same
    schedule as the engine, so results are comparable bit for bit).
    """

    def __init__(self, executor, quantum: int = 64, keep_results: bool = False,
                 clock=time.perf_counter, sleep=time.sleep, keep_ids=()):
        self.ex = executor
        self.quantum = quantum
        self.keep = keep_results
        self.keep_ids = set(keep_ids)
        self.clock = clock
        self.sleep = sleep

    def run(self, requests: list[Request], duration: float | None = None) -> ServeStats:
        pending = sorted(requests, key=lambda r: r.arrival)
        outcomes, updates = [], 0
        horizon = duration if duration is not None else math.inf
        t0 = self.clock()
        i = 0
        peak = 0
        while i < len(pending):
            now = self.clock() - t0
            if now >= horizon:
                break
            req = pending[i]
            if req.arrival > now:
                self.sleep(min(req.arrival - now, 0.01))
                continue
            i += 1
            adm = self.clock() - t0
            peak = max(peak, req.device_bytes)
            if req.kind == "heat":
                slot = self.ex.solve_alone(req, req.steps)
                conv = True
            else:
                slot = self.ex.alloc(req)
                conv = False
                while slot.done < req.max_sweeps:
                    c = min(self.quantum, req.max_sweeps - slot.done)
                    self.ex.advance_alone(slot, c)
                    if self.ex.converged(slot):
                        conv = True
                        break
            self.ex.synchronize()
            res = self.ex.fetch(slot) if self.keep or req.rid in self.keep_ids else None
            updates += req.cells * slot.done
            outcomes.append(Outcome(req.rid, req.kind, req.arrival, adm, self.clock() - t0,
                                    slot.done, conv, res))
            self.ex.free(slot)
        wall = self.clock() - t0
        open_arr = [r.arrival for r in pending[len(outcomes):] if r.arrival <= wall]
        return ServeStats(outcomes, wall, len(outcomes), len(requests), peak,
                          len(pending) - len(outcomes), updates, open_arrivals=open_arr)


# ------------------------------------------------------------------------------------------
# replicas: one engine per GPU, requests split by id, statistics merged
# ------------------------------------------------------------------------------------------
def shard(requests: list[Request], rank: int, world: int) -> list[Request]:
    """The requests replica `rank` of `world` serves (round-robin by request id)."""
    return [r for r in requests if r.rid % world == rank]


def merge(stats: list[dict], latencies: list[list[float]]) -> dict:
    """Whole-job summary from per-replica summaries and raw latencies (seconds; unfinished
    requests by their age at the end, as :meth:`ServeStats.latencies_all`)."""
    lat = np.array([x for part in latencies for x in part]) if any(latencies) else np.array([0.0])
    wall = max(s["wall_s"] for s in stats)
    done = sum(s["completed"] for s in stats)
    return {
        "replicas": len(stats), "completed": done,
        "submitted": sum(s["submitted"] for s in stats),
        "backlog": sum(s["backlog"] for s in stats), "wall_s": wall,
        "solves_per_s": round(done / wall, 2) if wall > 0 else 0.0,
        "p50_ms": round(float(np.percentile(lat, 50)) * 1e3, 2),
        "p99_ms": round(float(np.percentile(lat, 99)) * 1e3, 2),
        "glups": round(sum(s["glups"] for s in stats), 2),
    }


def gather_summary(local: ServeStats, group=None) -> dict:
    """Merge the replicas' statistics over a torch.distributed group (any backend)."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    parts: list = [None] * world
    dist.all_gather_object(parts, (local.summary(), local.latencies_all()), group=group)
    return merge([p[0] for p in parts], [p[1] for p in parts])
