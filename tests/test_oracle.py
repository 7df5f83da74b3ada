"""The oracle is pinned bit for bit to golden vectors made by the reference itself.

Fixtures: ``tests/golden/make_golden.py`` (runs pyheat3d's own ``reference_step``,
``emulated_reference`` and ``NumpyStepper``). CPU only.
"""

from __future__ import annotations

import hashlib
import json
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

import numpy as np
import pytest

from oracle import (
    emulated_reference,
    from_bf16_bits,
    reference_step,
    round_storage,
    run_reference,
    threaded_emulated,
    threaded_step,
    to_bf16_bits,
)

GOLD = Path(__file__).resolve().parent / "golden"
G = np.load(GOLD / "stencil_small.npz")
META = json.loads((GOLD / "dirichlet128.json").read_text())
STEPS = META["steps"]
SCHEDULES = [tuple(x) for x in META["schedules"]]


def heat(dims, bc, r=None):
    r = 0.9 / (2 * dims) if r is None else r
    return np.float64(1.0 - 2.0 * dims * r), np.float64(r)


@pytest.mark.parametrize("storage,k", SCHEDULES)
@pytest.mark.parametrize("bc", ["dirichlet", "periodic"])
@pytest.mark.parametrize("dims", [2, 3])
def test_emulated_reference_matches_golden(dims, bc, storage, k):
    c0, c1 = heat(dims, bc)
    out = emulated_reference(G[f"u0_{dims}d"], c0, c1, bc, STEPS, storage, k)
    assert np.array_equal(out, G[f"heat_{dims}d_{bc}_{storage}_k{k}"])


@pytest.mark.parametrize("bc", ["dirichlet", "periodic"])
@pytest.mark.parametrize("dims", [2, 3])
def test_jacobi_with_and_without_source_matches_golden(dims, bc):
    c0, c1 = 0.0, 1.0 / (2 * dims)
    u0 = G[f"u0_{dims}d"]
    assert np.array_equal(run_reference(u0, c0, c1, bc, 24), G[f"jacobi_{dims}d_{bc}"])
    b = G[f"src_{dims}d_{bc}"]
    assert np.array_equal(run_reference(u0, c0, c1, bc, 24, b), G[f"jacobi_src_{dims}d_{bc}"])


@pytest.mark.parametrize("bc", ["dirichlet", "periodic"])
@pytest.mark.parametrize("dims", [2, 3])
def test_float64_matches_golden(dims, bc):
    c0, c1 = heat(dims, bc)
    out = run_reference(G[f"u0_{dims}d"].astype(np.float64), c0, c1, bc, 24)
    assert out.dtype == np.float64
    assert np.array_equal(out, G[f"heat64_{dims}d_{bc}"])


@pytest.mark.parametrize("bc", ["dirichlet", "periodic"])
@pytest.mark.parametrize("dims", [2, 3])
def test_in_place_stepper_equals_reference_step(dims, bc):
    c0, c1 = heat(dims, bc)
    assert np.array_equal(run_reference(G[f"u0_{dims}d"], c0, c1, bc, 5),
                          G[f"stepper5_{dims}d_{bc}"])


@pytest.mark.parametrize("storage,k", SCHEDULES)
@pytest.mark.parametrize("bc", ["dirichlet", "periodic"])
@pytest.mark.parametrize("dims", [2, 3])
def test_tiny_grids_match_golden(dims, bc, storage, k):
    c0, c1 = heat(dims, bc, 0.1)
    out = emulated_reference(G[f"tiny_u0_{dims}d"], c0, c1, bc, 9, storage, k)
    assert np.array_equal(out, G[f"tiny_{dims}d_{bc}_{storage}_k{k}"])


def test_storage_rounding_matches_golden():
    x = G["round_in"]
    assert np.array_equal(round_storage(x, "bfloat16"), G["round_bf16"])
    with np.errstate(over="ignore"):
        f16 = round_storage(x, "float16")
    assert np.array_equal(f16, G["round_f16"], equal_nan=True)
    bits = to_bf16_bits(x)
    assert np.array_equal(from_bf16_bits(bits), G["round_bf16"])


def test_torch_rounding_equals_oracle():
    """The stepper converts float32 -> 16-bit with torch; it must round exactly like the oracle."""
    torch = pytest.importorskip("torch")
    x = G["round_in"]
    t = torch.from_numpy(x)
    assert np.array_equal(t.to(torch.bfloat16).float().numpy(), G["round_bf16"])
    assert np.array_equal(t.to(torch.float16).float().numpy(), G["round_f16"])


@pytest.mark.parametrize("src", [False, True])
@pytest.mark.parametrize("bc", ["dirichlet", "periodic"])
@pytest.mark.parametrize("dims", [2, 3])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_threaded_step_is_bitwise_reference_step(dims, bc, src, dtype):
    rng = np.random.default_rng(5)
    shape = (17, 23, 29)[:dims] if dims == 3 else (37, 41)
    u = rng.random(shape).astype(dtype)
    b = (rng.random(shape).astype(dtype) - dtype(0.5)) * dtype(1e-3) if src else None
    c0, c1 = heat(dims, bc)
    ref = reference_step(u, c0, c1, bc, b)
    out = u.copy()
    with ThreadPoolExecutor(4) as pool:
        threaded_step(u, out, c0, c1, bc, b, threads=4, pool=pool)
    assert np.array_equal(out, ref)


def test_dirichlet128_hash_matches_reference_run():
    """3D 128^3 Dirichlet, zero walls, r = 0.15, seed 0, 100 steps: SHA-256 of the result."""
    cfg = META["dirichlet128"]
    u0 = np.random.default_rng(0).random((128,) * 3, dtype=np.float32)
    u0[0] = u0[-1] = 0
    u0[:, 0] = u0[:, -1] = 0
    u0[:, :, 0] = u0[:, :, -1] = 0
    u = u0
    out = u0.copy()
    with ThreadPoolExecutor(8) as pool:
        for _ in range(cfg["steps"]):
            threaded_step(u, out, cfg["c0"], cfg["c1"], "dirichlet", threads=8, pool=pool)
            u, out = out, u
    assert hashlib.sha256(np.ascontiguousarray(u).tobytes()).hexdigest() == cfg["sha256"]


@pytest.mark.parametrize("storage,k,bc", [("float32", 1, "periodic"), ("bfloat16", 4, "periodic"),
                                          ("float16", 3, "dirichlet"), ("bfloat16", 1, "dirichlet"),
                                          ("float16", 8, "periodic")])
@pytest.mark.parametrize("dims", [2, 3])
def test_threaded_emulated_is_bitwise_emulated_reference(dims, storage, k, bc):
    """The full-size GPU tests check 16-bit and tb<k> variants against this threaded form."""
    shape = (13, 17, 19) if dims == 3 else (37, 41)
    u0 = np.random.default_rng(2).random(shape, dtype=np.float32)
    c0, c1 = heat(dims, bc)
    got = threaded_emulated(u0, c0, c1, bc, 2 * k + 1, storage, k, threads=4)
    assert np.array_equal(got, emulated_reference(u0, c0, c1, bc, 2 * k + 1, storage, k))


def test_threaded_emulated_snapshots():
    u0 = np.random.default_rng(3).random((29, 31), dtype=np.float32)
    c0, c1 = heat(2, "periodic")
    snaps = threaded_emulated(u0, c0, c1, "periodic", 9, snapshots=(3, 5, 9), threads=3)
    for n in (3, 5, 9):
        assert np.array_equal(snaps[n], run_reference(u0, c0, c1, "periodic", n))
