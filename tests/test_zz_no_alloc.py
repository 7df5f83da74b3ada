"""The allocation-free batch entry point, ``ph3_batch_run_static``.

Some hosts cannot allocate device memory where they run a batch — a serving loop that must not
allocate once it is in steady state, or a foreign host (Go, Java, a plugin) that hands over field
buffers but owns no CUDA allocator. For them the library keeps the batch plan and counters in a
fixed 1 MiB device array. This test calls the entry point through the C ABI twice in a row and
checks every problem's result against the workspace entry points (ph3_batch_prepare +
ph3_batch_launch), bit for bit — the tolerance of every parity test in this suite — and that a
plan larger than the array is refused with a clear error.

It lives in its own file, collected last, so that a failure here does not stop the other tests.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_static_batch_equals_workspace_batch_two_calls():
    import torch

    from pyheat3d_b200 import _lib, heat_stencil
    from pyheat3d_b200.batch import Batch, Problem, synthetic_batch

    probs = synthetic_batch(20, seed=21, n2d=(9, 300), n3d=(6, 48), steps=(1, 60),
                            storages=("float32", "bfloat16", "float16"))
    rng = np.random.default_rng(2)
    probs.append(Problem(rng.random((5, 6, 7), dtype=np.float32), heat_stencil(3, 0.1, "periodic"),
                         9, "float32"))
    batch = Batch(probs)
    batch.run()
    torch.cuda.synchronize()
    want = batch.results()

    lib = _lib.lib()
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        batch.reset()
        rc = lib.ph3_batch_run_static(ctypes.addressof(batch.descs), batch.n, stream)
        assert rc == 0, _lib.last_error()
        torch.cuda.synchronize()
        got = batch.results()
        for i, (g, w) in enumerate(zip(got, want)):
            assert np.array_equal(g, w), (call, i)
    assert _lib.device_status(clear=True) == 0


def test_static_batch_rejects_plans_beyond_its_array():
    import torch

    from pyheat3d_b200 import _lib
    from pyheat3d_b200.batch import ProblemDesc

    a = torch.zeros((8, 8), device="cuda")
    b = torch.zeros((8, 8), device="cuda")
    descs = (ProblemDesc * 1)()
    d = descs[0]
    d.a, d.b, d.src = a.data_ptr(), b.data_ptr(), None
    d.dims, d.nz, d.ny, d.nx = 2, 1, 8, 8
    d.bc, d.storage, d.c0, d.c1, d.steps, d.k = 1, 0, 0.5, 0.125, 400000, 1
    lib = _lib.lib()
    rc = lib.ph3_batch_run_static(ctypes.addressof(descs), 1, None)
    assert rc == 1
    assert "static workspace holds" in _lib.last_error()
