"""Full-size cases (the largest configured grid, 3D 1024^3 fp32: 4 GiB per field).

At this size the oracle is still affordable for a couple of updates when it runs thread-chunked
over z-slabs, so the single-step z-march is compared with it bit for bit; the other kernel
families are checked through size-independent properties: every fp32 kernel computes the same
update sequence, so the naive kernel and tb4 (four fused updates per pass) must equal the z-march
bit for bit after the same number of steps, also for a step count that is not a multiple of 4.
"""

from __future__ import annotations

import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from oracle import threaded_step
from pyheat3d_b200 import heat_stencil
from pyheat3d_b200.registry import make_stepper

pytestmark = pytest.mark.gpu

N = 1024


@pytest.fixture(scope="module")
def field():
    return np.random.default_rng(17).random((N, N, N), dtype=np.float32)


def _run(key, u0, st, steps):
    s = make_stepper(key, u0, st)
    s.step(steps)
    s.synchronize()
    return s


def test_zmarch_matches_oracle_at_1024_cubed(field):
    st = heat_stencil(3, 0.95 / 6, "periodic")
    s = _run("b200/zmarch", field, st, 2)
    got = s.get()
    s.close()
    u, out = field.copy(), np.empty_like(field)
    threads = max(1, os.cpu_count() or 1)
    with ThreadPoolExecutor(threads) as pool:
        for _ in range(2):
            threaded_step(u, out, st.c0, st.c1, "periodic", threads=threads, pool=pool)
            u, out = out, u
    assert np.array_equal(got, u)


@pytest.mark.parametrize("bc", ["periodic", "dirichlet"])
def test_kernel_families_agree_at_1024_cubed(field, bc):
    import torch

    st = heat_stencil(3, 0.95 / 6, bc)
    ref = _run("b200/zmarch", field, st, 9)
    want = ref.get_tensor().clone()
    ref.close()
    for key in ("b200/naive", "b200/tb4", "b200/auto"):  # auto: tb4 from the table at 1024^3
        s = _run(key, field, st, 9)
        same = torch.equal(s.get_tensor(), want)
        s.close()
        assert same, key
    del want
    torch.cuda.empty_cache()
