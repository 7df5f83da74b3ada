"""Batched persistent launch: every problem bit-identical to the oracle and to the single-grid
steppers, through plain launches and a CUDA graph.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import emulated_reference
from pyheat3d_b200.batch import synthetic_batch


def test_synthetic_batch_distribution():
    probs = synthetic_batch(64, seed=3, n2d=(64, 2048), n3d=(32, 256))
    dims = [p.u0.ndim for p in probs]
    assert dims.count(2) == 32 and dims.count(3) == 32
    for p in probs:
        n = p.u0.shape[0]
        d = p.u0.ndim
        assert (64 <= n <= 2048) if d == 2 else (32 <= n <= 256)
        assert 0.05 <= p.stencil.c1 <= 0.95 / (2 * d) + 1e-12
        assert 50 <= p.steps <= 2000 and p.storage in ("float32", "bfloat16")
    again = synthetic_batch(64, seed=3)
    assert all(np.array_equal(a.u0, b.u0) and a.steps == b.steps for a, b in zip(probs, again))


def _oracle(p):
    k = 1
    return emulated_reference(p.u0, p.stencil.c0, p.stencil.c1, p.stencil.bc, p.steps, p.storage,
                              k, p.source)


@pytest.mark.gpu
def test_small_batch_matches_oracle_bitwise():
    from pyheat3d_b200 import heat_stencil, jacobi_stencil
    from pyheat3d_b200.batch import Batch, Problem

    rng = np.random.default_rng(12)
    probs = synthetic_batch(24, seed=5, n2d=(5, 150), n3d=(5, 40), steps=(0, 40),
                            storages=("float32", "bfloat16", "float16"))
    # odd shapes, a Jacobi problem with a source, a zero-step problem
    u = rng.random((7, 9, 11), dtype=np.float32)
    b = (rng.random(u.shape, dtype=np.float32) - np.float32(0.5)) * np.float32(1e-2)
    probs.append(Problem(u, jacobi_stencil(3, "dirichlet"), 13, "float32", b))
    probs.append(Problem(rng.random((33, 130), dtype=np.float32), heat_stencil(2, 0.2, "periodic"),
                         0, "bfloat16"))
    batch = Batch(probs)
    batch.run()
    outs = batch.results()
    for i, (p, got) in enumerate(zip(probs, outs)):
        want = _oracle(p)
        assert np.array_equal(got, want), (i, p.u0.shape, p.storage, p.stencil.bc, p.steps)


@pytest.mark.gpu
def test_graph_replay_and_plain_steppers_agree():
    import torch

    from pyheat3d_b200.batch import Batch
    from pyheat3d_b200.registry import make_stepper

    probs = synthetic_batch(16, seed=8, n2d=(64, 700), n3d=(32, 96), steps=(50, 300))
    batch = Batch(probs)
    g = batch.graph(with_reset=True)
    for _ in range(2):
        g.replay()
    torch.cuda.synchronize()
    outs = batch.results()
    for p, got in zip(probs, outs):
        suf = {"float32": "", "bfloat16": "-bf16"}[p.storage]
        key = ("b200/zmarch" if p.u0.ndim == 3 else "b200/ymarch") + suf
        s = make_stepper(key, p.u0, p.stencil)
        s.step(p.steps)
        s.synchronize()
        assert np.array_equal(got, s.get())


@pytest.mark.gpu
@pytest.mark.parametrize("cfg", [0, 1, 3, 10])
def test_long_plan_with_few_tiles_per_step(cfg):
    """Long dependency chains (7000 and 3001 steps of grids that are one or two tiles each)
    beside a short problem stay bit-exact, for four tile configurations."""
    from pyheat3d_b200 import _lib, heat_stencil, tune
    from pyheat3d_b200.batch import Batch, Problem

    rng = np.random.default_rng(21)
    probs = [Problem(rng.random((5, 6, 7), dtype=np.float32), heat_stencil(3, 0.1, "periodic"),
                     7000, "float32"),
             Problem(rng.random((9, 40), dtype=np.float32), heat_stencil(2, 0.2, "dirichlet"),
                     3001, "bfloat16"),
             Problem(rng.random((6, 17, 33), dtype=np.float32), heat_stencil(3, 0.15, "dirichlet"),
                     57, "float32")]
    L = _lib.lib()
    prev = tune.active_table()
    tune.use(None)
    try:
        _lib.check(L.ph3_tune_set(_lib.KERNEL["batch"], 3, 0, 1, cfg, 0))
        batch = Batch(probs)
        batch.run()
        outs = batch.results()
    finally:
        L.ph3_tune_set(_lib.KERNEL["batch"], 3, 0, 1, -1, 0)
        tune.use(prev)
    for i, (p, got) in enumerate(zip(probs, outs)):
        assert np.array_equal(got, _oracle(p)), (i, p.u0.shape, p.steps)


def _tb_mix(seed: int):
    """2D problems with k = 2 / 4 fused steps per pass (odd and tiny shapes, all storages, both
    boundaries, a Jacobi source) beside single-step 2D and 3D problems."""
    from pyheat3d_b200 import heat_stencil, jacobi_stencil
    from pyheat3d_b200.batch import Problem

    rng = np.random.default_rng(seed)
    out = []
    shapes = [(5, 7), (9, 40), (64, 64), (150, 333), (257, 1000), (700, 129), (1030, 2050)]
    storages = ("float32", "bfloat16", "float16")
    for i, shape in enumerate(shapes):
        for k in (2, 4):
            bc = ("periodic", "dirichlet")[(i + k) % 2]
            st = storages[(i + k // 2) % 3]
            r = float(rng.uniform(0.05, 0.95 / 4))
            steps = k * int(rng.integers(1, 40)) + int(rng.integers(0, k))  # with remainders
            out.append(Problem(rng.random(shape, dtype=np.float32), heat_stencil(2, r, bc), steps,
                               st, k=k))
    u = rng.random((96, 200), dtype=np.float32)
    b = (rng.random(u.shape, dtype=np.float32) - np.float32(0.5)) * np.float32(1e-2)
    out.append(Problem(u, jacobi_stencil(2, "dirichlet"), 27, "float32", b, k=4))
    out.append(Problem(u, jacobi_stencil(2, "periodic"), 18, "bfloat16", b, k=2))
    out.append(Problem(u, heat_stencil(2, 0.2, "dirichlet"), 3, "float16", k=4))  # remainder only
    out.append(Problem(rng.random((40, 50), dtype=np.float32), heat_stencil(2, 0.2, "periodic"), 0,
                       "float32", k=2))
    out.append(Problem(rng.random((130, 77), dtype=np.float32), heat_stencil(2, 0.2, "dirichlet"),
                       37, "float32"))
    out.append(Problem(rng.random((20, 33, 45), dtype=np.float32), heat_stencil(3, 0.1, "periodic"),
                       29, "bfloat16"))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("cfg", [0, 2, 3, 5, 6, 9])
def test_temporal_blocking_problems_match_oracle_and_tb_steppers(cfg):
    """Per-problem k: a 2D problem with k = 2 or 4 advances by steps // k passes of k fused steps
    and steps % k single steps, rounded to its storage type once per pass — bit-identical to the
    oracle's per-pass rounding and to the single-grid tb<k> stepper, in six batch kernel
    configurations (lean and shared-memory plane tile sets, compiled for three and for two blocks
    per SM)."""
    from pyheat3d_b200 import _lib, tune
    from pyheat3d_b200.batch import Batch
    from pyheat3d_b200.registry import make_stepper

    probs = _tb_mix(31)
    L = _lib.lib()
    prev = tune.active_table()
    tune.use(None)
    try:
        _lib.check(L.ph3_tune_set(_lib.KERNEL["batch"], 3, 0, 1, cfg, 0))
        batch = Batch(probs)
        batch.run()
        outs = batch.results()
    finally:
        L.ph3_tune_set(_lib.KERNEL["batch"], 3, 0, 1, -1, 0)
        tune.use(prev)
    suf = {"float32": "", "bfloat16": "-bf16", "float16": "-fp16"}
    for i, (p, got) in enumerate(zip(probs, outs)):
        want = emulated_reference(p.u0, p.stencil.c0, p.stencil.c1, p.stencil.bc, p.steps,
                                  p.storage, p.k, p.source)
        assert np.array_equal(got, want), (i, p.u0.shape, p.storage, p.stencil.bc, p.steps, p.k)
        if p.k > 1 and p.source is None:
            s = make_stepper(f"b200/tb{p.k}{suf[p.storage]}", p.u0, p.stencil)
            s.step(p.steps)
            s.synchronize()
            assert np.array_equal(got, s.get()), (i, "differs from the tb stepper")
            s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("dims,k,steps", [(2, 3, 6), (3, 2, 4), (3, 4, 9), (2, 8, 8)])
def test_batch_rejects_bad_temporal_depth(dims, k, steps):
    import ctypes

    import torch

    from pyheat3d_b200 import _lib
    from pyheat3d_b200.batch import ProblemDesc

    L = _lib.lib()
    shape = (16, 16) if dims == 2 else (8, 8, 8)
    a = torch.zeros(shape, device="cuda")
    b = torch.zeros_like(a)
    descs = (ProblemDesc * 1)()
    d = descs[0]
    d.a, d.b, d.src = a.data_ptr(), b.data_ptr(), None
    d.dims = dims
    d.nz, d.ny, d.nx = (1, *shape) if dims == 2 else shape
    d.bc, d.storage, d.c0, d.c1, d.steps, d.k = 1, 0, 0.5, 0.125, steps, k
    ws = torch.empty(1 << 16, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    addr = ctypes.addressof(descs)
    einval = 1  # PH3_EINVAL
    assert L.ph3_batch_prepare(addr, 1, ws.data_ptr(), ws.numel(), stream) == einval
    assert L.ph3_batch_run_static(addr, 1, stream) == einval
