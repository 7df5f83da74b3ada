"""The bounded-wait watchdog on the GPU, without a fault.

Every spin-wait of the library (mbarrier rings, the batch kernel's dependency counters) gives up
after a limited number of polls, records a code in the per-device status word and returns.
``ph3_wait_flag`` runs that same wait alone, so a test can make it run out: it polls a device
flag that nothing sets, with a short poll limit (a few milliseconds). The test then reads the
code, checks that the context still runs kernels correctly, and that a flag that is already set
passes without any code. No kernel here traps, faults or waits without a bound.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import run_reference
from pyheat3d_b200 import _lib, heat_stencil
from pyheat3d_b200.registry import make_stepper

pytestmark = pytest.mark.gpu

LIMIT = 1 << 12  # polls of at most ~0.25 us each: the wait gives up within a few milliseconds


@pytest.fixture
def torch_cuda():
    import torch

    _lib.device_status(clear=True)
    yield torch
    _lib.device_status(clear=True)


def _stream(torch):
    return torch.cuda.current_stream().cuda_stream


def test_wait_on_a_flag_nothing_sets_times_out_into_the_status_word(torch_cuda):
    torch = torch_cuda
    flag = torch.zeros(4, dtype=torch.int32, device="cuda")
    _lib.check(_lib.lib().ph3_wait_flag(flag.data_ptr(), 1, LIMIT, _stream(torch)))
    assert _lib.device_status(clear=True) == _lib.STATUS["dependency_timeout"]
    assert _lib.device_status(clear=False) == 0  # cleared

    # the context is still usable: a stencil run right after matches the oracle bit for bit
    u0 = np.random.default_rng(3).random((9, 20, 32), dtype=np.float32)
    st = heat_stencil(3, 0.15, "periodic")
    s = make_stepper("b200/zmarch", u0, st)
    s.step(7)
    s.synchronize()
    got = s.get()
    s.close()
    assert np.array_equal(got, run_reference(u0, st.c0, st.c1, "periodic", 7))
    assert _lib.device_status(clear=True) == 0


def test_wait_on_a_set_flag_passes_without_a_code(torch_cuda):
    torch = torch_cuda
    flag = torch.full((1,), 5, dtype=torch.int32, device="cuda")
    for target in (0, 5, -3):
        _lib.check(_lib.lib().ph3_wait_flag(flag.data_ptr(), target, LIMIT, _stream(torch)))
    assert _lib.device_status(clear=True) == 0


def test_status_word_keeps_the_first_code(torch_cuda):
    torch = torch_cuda
    flag = torch.zeros(1, dtype=torch.int32, device="cuda")
    for _ in range(3):
        _lib.check(_lib.lib().ph3_wait_flag(flag.data_ptr(), 1, 64, _stream(torch)))
    assert _lib.device_status(clear=True) == _lib.STATUS["dependency_timeout"]
    assert _lib.device_status(clear=True) == 0
