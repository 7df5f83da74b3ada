"""Serving engine: scheduling on CPU (fake executor, virtual clock), replicas over gloo, and on
the GPU the continuous-batching result of every request equals the request run alone.
"""

from __future__ import annotations

import os

import numpy as np
import pytest

from pyheat3d_b200.serve import (
    PlainServer,
    Request,
    Server,
    gather_summary,
    merge,
    poisson_stream,
    shard,
)


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, dt):
        self.t += dt


class FakeSlot:
    def __init__(self, req):
        self.req, self.done, self.in_b = req, 0, False


class FakeExecutor:
    """Time advances by the work: 1 ns per site update, 50 us per batch round, and 10 us per
    step for the single-grid path (one kernel launch per step)."""

    def __init__(self, clock):
        self.clock = clock
        self.alive = 0
        self.max_alive = 0
        self.rounds = []

    def alloc(self, req):
        self.alive += 1
        self.max_alive = max(self.max_alive, self.alive)
        return FakeSlot(req)

    def advance(self, slots, counts):
        self.rounds.append(sorted(s.req.rid for s in slots))
        work = sum(s.req.cells * c for s, c in zip(slots, counts))
        self.clock.t += 50e-6 + work * 1e-9
        for s, c in zip(slots, counts):
            s.done += c

    def advance_alone(self, s, c):
        self.clock.t += 10e-6 * c + s.req.cells * c * 1e-9
        s.done += c

    def solve_alone(self, req, c):
        s = self.alloc(req)
        self.advance_alone(s, c)
        return s

    def converged(self, s):
        return s.done >= 3 * 64

    def fetch(self, s):
        return None

    def free(self, s):
        self.alive -= 1

    def synchronize(self):
        pass


def test_poisson_stream_statistics():
    reqs = poisson_stream(2000.0, 2.0, seed=1)
    assert 3600 < len(reqs) < 4400
    gaps = np.diff([r.arrival for r in reqs])
    assert abs(gaps.mean() - 1 / 2000) < 1e-4
    kinds = [r.kind for r in reqs]
    assert 0.4 < kinds.count("jacobi") / len(kinds) < 0.6
    for r in reqs:
        if r.kind == "jacobi":
            assert 1e-10 <= r.tol <= 1e-6 and r.bc == "dirichlet"
        else:
            assert 50 <= r.steps <= 2000 and 0.05 <= r.r <= 0.95 / (2 * r.dims)
    assert [r.rid for r in reqs] == list(range(len(reqs)))


def test_engine_admits_continuously_and_respects_budget():
    clock = FakeClock()
    ex = FakeExecutor(clock)
    reqs = [Request(i, 0.0002 * i, "heat", 2, 64, "periodic", "float32", r=0.1, steps=200)
            for i in range(40)]
    budget = 5 * reqs[0].device_bytes  # at most five resident requests
    stats = Server(ex, budget_bytes=budget, quantum=64, clock=clock, sleep=clock.sleep).run(reqs)
    assert len(stats.outcomes) == 40 and stats.backlog == 0
    assert ex.max_alive == 5 and stats.peak_bytes == budget
    # a request admitted mid-flight shares rounds with requests admitted earlier
    assert any(len(r) > 1 and r[0] != r[-1] for r in ex.rounds)
    assert all(o.steps_done == 200 for o in stats.outcomes)
    s = stats.summary()
    assert s["completed"] == 40 and s["p99_ms"] >= s["p50_ms"] > 0


def test_engine_beats_plain_when_overloaded():
    reqs = poisson_stream(500.0, 0.2, seed=3, n2d=(32, 96), n3d=(16, 32), steps=(50, 200))
    c1, c2 = FakeClock(), FakeClock()
    eng = Server(FakeExecutor(c1), quantum=64, clock=c1, sleep=c1.sleep).run(reqs)
    plain = PlainServer(FakeExecutor(c2), quantum=64, clock=c2, sleep=c2.sleep).run(reqs)
    assert len(eng.outcomes) == len(plain.outcomes) == len(reqs)
    assert eng.wall < plain.wall
    assert eng.summary()["solves_per_s"] > plain.summary()["solves_per_s"]


def test_shard_and_merge():
    reqs = poisson_stream(1000.0, 0.1, seed=4)
    parts = [shard(reqs, r, 3) for r in range(3)]
    assert sorted(x.rid for p in parts for x in p) == [r.rid for r in reqs]
    m = merge([{"completed": 2, "submitted": 3, "backlog": 1, "wall_s": 1.0, "glups": 1.0},
               {"completed": 4, "submitted": 4, "backlog": 0, "wall_s": 2.0, "glups": 2.0}],
              [[0.1, 0.2], [0.3, 0.4, 0.5, 0.6]])
    assert m["completed"] == 6 and m["solves_per_s"] == 3.0 and m["glups"] == 3.0


def _replica(rank, world, port, out):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    reqs = shard(poisson_stream(400.0, 0.1, seed=6, n2d=(32, 64), n3d=(16, 24), steps=(50, 100)),
                 rank, world)
    clock = FakeClock()
    stats = Server(FakeExecutor(clock), quantum=64, clock=clock, sleep=clock.sleep).run(reqs)
    m = gather_summary(stats)
    if rank == 0:
        out.put(m)
    dist.destroy_process_group()


def test_replicas_gloo_world_size_2():
    import socket

    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_replica, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    m = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    total = len(poisson_stream(400.0, 0.1, seed=6))
    assert m["replicas"] == 2 and m["completed"] == total and m["backlog"] == 0


# ------------------------------------------------------------------------------------ GPU
@pytest.mark.gpu
def test_gpu_each_result_same_alone_and_in_the_mix():
    from pyheat3d_b200.serve import GpuExecutor

    ex = GpuExecutor()
    reqs = poisson_stream(400.0, 0.05, seed=9, n2d=(16, 200), n3d=(8, 40), steps=(5, 150),
                          tol=(1e-6, 1e-4), max_sweeps=640,
                          storages=("float32", "bfloat16", "float16"))
    assert len(reqs) >= 10
    stats = Server(ex, quantum=32, keep_results=True).run(reqs)
    assert len(stats.outcomes) == len(reqs)
    for o in stats.outcomes:
        req = reqs[o.rid]
        alone = ex.solve_alone(req, o.steps_done)
        ex.synchronize()
        assert np.array_equal(ex.fetch(alone), o.result), (req, o.steps_done)
        ex.free(alone)
    s = stats.summary()
    assert s["completed"] == len(reqs) and s["rounds"] >= 1


@pytest.mark.gpu
def test_gpu_engine_and_plain_agree_on_a_stream():
    from pyheat3d_b200.serve import GpuExecutor

    ex = GpuExecutor()
    reqs = poisson_stream(200.0, 0.05, seed=10, n2d=(32, 128), n3d=(16, 32), steps=(10, 80),
                          tol=(1e-5, 1e-4), max_sweeps=256)
    eng = Server(ex, quantum=32, keep_results=True).run(reqs)
    plain = PlainServer(ex, quantum=32, keep_results=True).run(reqs)
    a = {o.rid: o for o in eng.outcomes}
    b = {o.rid: o for o in plain.outcomes}
    assert set(a) == set(b) == {r.rid for r in reqs}
    for rid in a:
        assert a[rid].steps_done == b[rid].steps_done
        assert np.array_equal(a[rid].result, b[rid].result)


def test_censored_latencies_count_the_backlog():
    """Requests still open at the end of a run count with their age (a lower bound)."""
    clock = FakeClock()
    ex = FakeExecutor(clock)
    reqs = poisson_stream(2000.0, 0.05, seed=11)
    stats = Server(ex, quantum=64, clock=clock, sleep=clock.sleep, max_active=4).run(
        reqs, duration=0.05, drain=False)
    s = stats.summary()
    assert s["backlog"] > 0 and s["censored"] == len(stats.open_arrivals) > 0
    lat = stats.latencies_all()
    assert len(lat) == len(stats.outcomes) + s["censored"]
    assert all(x >= 0 for x in lat)


@pytest.mark.gpu
def test_gpu_served_results_match_the_oracle():
    """Every served result equals the oracle run on the same initial field for the same number
    of steps / sweeps, with the storage rounding of a single-step kernel (emulated_reference,
    k = 1): fp32 bit for bit, 16-bit storage bit for bit with its per-step rounding."""
    import torch

    from oracle import emulated_reference
    from pyheat3d_b200.serve import GpuExecutor

    ex = GpuExecutor()
    reqs = poisson_stream(400.0, 0.05, seed=12, n2d=(16, 96), n3d=(8, 24), steps=(5, 90),
                          tol=(1e-6, 1e-4), max_sweeps=320,
                          storages=("float32", "bfloat16", "float16"))
    assert len(reqs) >= 10
    stats = Server(ex, quantum=32, keep_results=True).run(reqs)
    assert len(stats.outcomes) == len(reqs)
    for o in stats.outcomes:
        req = reqs[o.rid]
        u, src = ex.init_fields(req)  # regenerated from the request's seed on the device
        u0 = u.cpu().numpy()
        b = src.cpu().numpy() if src is not None else None
        c0, c1 = req.coefficients()
        want = emulated_reference(u0, c0, c1, req.bc, o.steps_done, req.storage, 1, b)
        assert np.array_equal(o.result, want), (req, o.steps_done)
    torch.cuda.synchronize()
