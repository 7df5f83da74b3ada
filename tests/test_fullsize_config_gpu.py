"""Parity at the roofline sizes of the plain GPU workload: 3D 512^3 and 2D 16384^2, fp32 fields,
r = 0.95/(2d), uniform [0, 1) from seed 0 — the grids the bench measures.

Every kernel family the bench times is run here at that size and compared with the oracle bit
for bit: the single step, tb2 / tb3 / tb4 / tb8 with step counts that are not multiples of k
(2k + 1: two passes and a single-step remainder), and the 16-bit storage variants against the
oracle with the same per-pass storage rounding. At these sizes the TMA boxes, the periodic
seams, the partial tiles and the chunk edges of the production launch geometry are all
exercised, which small shapes do not do. The oracle runs thread-chunked over slabs
(``oracle.threaded_emulated``), bit-identical to ``reference_step`` / ``emulated_reference``.

Bar: bit-identical (relative error 0; the stated fp32 bound is 1e-6, asserted as well).
"""

from __future__ import annotations

import os

import numpy as np
import pytest

from oracle import threaded_emulated
from pyheat3d_b200 import heat_stencil
from pyheat3d_b200.registry import VARIANTS, make_stepper

pytestmark = pytest.mark.gpu

N3, N2 = 512, 16384
FP32_TOL = 1e-6
THREADS = max(1, os.cpu_count() or 1)


def _field(dims: int, n: int, bc: str) -> np.ndarray:
    u = np.random.default_rng(0).random((n,) * dims, dtype=np.float32)
    if bc == "dirichlet":  # pyheat3d's Dirichlet problems: fixed zero boundary layer
        u[0] = u[-1] = 0
        u[:, 0] = u[:, -1] = 0
        if dims == 3:
            u[:, :, 0] = u[:, :, -1] = 0
    return u


def _gpu(key: str, u0: np.ndarray, st, steps: int) -> np.ndarray:
    s = make_stepper(key, u0, st)
    s.step(steps)
    s.synchronize()
    out = s.get()
    s.close()
    return out


def _assert_same(got: np.ndarray, ref: np.ndarray, what: str) -> None:
    g = np.asarray(got, np.float64)
    r = np.asarray(ref, np.float64)
    err = float(np.abs(g - r).max() / np.abs(r).max())
    assert err <= FP32_TOL, (what, err)
    assert np.array_equal(got, ref), (what, "not bit-identical", err,
                                      int(np.count_nonzero(got != ref)))


def _steps(key: str) -> int:
    k = VARIANTS[key].steps_per_pass
    return 2 * k + 1 if k > 1 else 3


# ------------------------------------------------------------------------------------- fixtures
_FP32_KEYS3 = ("b200/zmarch", "b200/naive", "b200/tb2", "b200/tb3", "b200/tb4", "b200/tb8",
               "b200/auto")
_FP32_KEYS2 = ("b200/ymarch", "b200/naive", "b200/tb2", "b200/tb3", "b200/tb4", "b200/tb8",
               "b200/auto")


@pytest.fixture(scope="module")
def case3():
    st = heat_stencil(3, 0.95 / 6, "periodic")
    u0 = _field(3, N3, "periodic")
    want = sorted({_steps(k) for k in _FP32_KEYS3})
    snaps = threaded_emulated(u0, st.c0, st.c1, "periodic", max(want), threads=THREADS,
                              snapshots=tuple(want))
    return u0, st, snaps


@pytest.fixture(scope="module")
def case2():
    st = heat_stencil(2, 0.95 / 4, "periodic")
    u0 = _field(2, N2, "periodic")
    want = sorted({_steps(k) for k in _FP32_KEYS2})
    snaps = threaded_emulated(u0, st.c0, st.c1, "periodic", max(want), threads=THREADS,
                              snapshots=tuple(want))
    return u0, st, snaps


# ---------------------------------------------------------------------------------- fp32 parity
@pytest.mark.parametrize("key", _FP32_KEYS3)
def test_3d_512_fp32_periodic(case3, key):
    u0, st, snaps = case3
    n = _steps(key)
    _assert_same(_gpu(key, u0, st, n), snaps[n], f"{key} 512^3 periodic {n} steps")


@pytest.mark.parametrize("key", _FP32_KEYS2)
def test_2d_16384_fp32_periodic(case2, key):
    u0, st, snaps = case2
    n = _steps(key)
    _assert_same(_gpu(key, u0, st, n), snaps[n], f"{key} 16384^2 periodic {n} steps")


@pytest.mark.parametrize("key", ["b200/zmarch", "b200/tb4"])
def test_3d_512_fp32_dirichlet(key):
    st = heat_stencil(3, 0.95 / 6, "dirichlet")
    u0 = _field(3, N3, "dirichlet")
    n = _steps(key)
    ref = threaded_emulated(u0, st.c0, st.c1, "dirichlet", n, threads=THREADS)
    _assert_same(_gpu(key, u0, st, n), ref, f"{key} 512^3 dirichlet {n} steps")


@pytest.mark.parametrize("key", ["b200/ymarch", "b200/tb4"])
def test_2d_16384_fp32_dirichlet(key):
    st = heat_stencil(2, 0.95 / 4, "dirichlet")
    u0 = _field(2, N2, "dirichlet")
    n = _steps(key)
    ref = threaded_emulated(u0, st.c0, st.c1, "dirichlet", n, threads=THREADS)
    _assert_same(_gpu(key, u0, st, n), ref, f"{key} 16384^2 dirichlet {n} steps")


# -------------------------------------------------------------------------------- 16-bit parity
@pytest.mark.parametrize("key", ["b200/zmarch-bf16", "b200/zmarch-fp16", "b200/tb4-bf16",
                                 "b200/tb8-fp16"])
def test_3d_512_16bit_periodic(case3, key):
    u0, st, _ = case3
    var = VARIANTS[key]
    n = _steps(key)
    ref = threaded_emulated(u0, st.c0, st.c1, "periodic", n, var.storage, var.steps_per_pass,
                            threads=THREADS)
    _assert_same(_gpu(key, u0, st, n), ref, f"{key} 512^3 periodic {n} steps")


@pytest.mark.parametrize("key", ["b200/ymarch-bf16", "b200/tb4-fp16", "b200/tb8-bf16"])
def test_2d_16384_16bit_periodic(case2, key):
    u0, st, _ = case2
    var = VARIANTS[key]
    n = _steps(key)
    ref = threaded_emulated(u0, st.c0, st.c1, "periodic", n, var.storage, var.steps_per_pass,
                            threads=THREADS)
    _assert_same(_gpu(key, u0, st, n), ref, f"{key} 16384^2 periodic {n} steps")


# ------------------------------------------------------------ unaligned rows, tuned defaults
@pytest.mark.parametrize("n,bc,key", [(255, "periodic", "b200/zmarch"),
                                      (255, "dirichlet", "b200/zmarch-bf16"),
                                      (127, "periodic", "b200/zmarch-fp16")])
def test_3d_unaligned_rows_tuned_defaults(n, bc, key):
    """Rows without 16-byte vectors take the march family's tuned configuration (shared-memory
    plane tiles with overlapped edge tiles from 255^3 up, the lean march below)."""
    st = heat_stencil(3, 0.95 / 6, bc)
    u0 = _field(3, n, bc)
    var = VARIANTS[key]
    ref = threaded_emulated(u0, st.c0, st.c1, bc, 5, var.storage, 1, threads=THREADS)
    _assert_same(_gpu(key, u0, st, 5), ref, f"{key} {n}^3 {bc} 5 steps")
