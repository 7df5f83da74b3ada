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
@pytest.mark.parametrize("cfg", [0, 1])
def test_long_plan_with_few_tiles_per_step(cfg):
    """Long dependency chains (7000 and 3001 steps of grids that are one or two tiles each)
    beside a short problem stay bit-exact, for two tile configurations."""
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
