"""Mixed-precision defect correction: oracle pinning (CPU) and GPU parity.

The oracle restates the GPU's FP64 residual / update and emulates the 16-bit inner sweeps, so a
fixed schedule must match bit for bit; the converged solution is checked against the exact
discrete FP64 solution and the continuum solution.
"""

from __future__ import annotations

import math

import numpy as np
import pytest

from oracle import run_reference
from oracle.precision import (
    defect_correction,
    discrete_solution,
    jacobi_rho,
    manufactured,
    residual_f64,
)


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("dims", [2, 3])
def test_discrete_solution_is_the_fp64_jacobi_fixed_point(dims):
    """FP64 Jacobi (the reference's solve, validation.py:96-113) converges to the closed form."""
    n = 9 if dims == 3 else 17
    h = 1.0 / (n - 1)
    _, f = manufactured(n, dims)
    b = -h * h * f / (2 * dims)
    iters = int(math.ceil(math.log(1e-13) / math.log(jacobi_rho(n))))
    u = run_reference(np.zeros_like(f), 0.0, 1.0 / (2 * dims), "dirichlet", iters, b)
    assert _rel(u, discrete_solution(n, dims)) < 1e-11


@pytest.mark.parametrize("dims", [2, 3])
def test_residual_of_discrete_solution_is_roundoff(dims):
    n = 17
    h = 1.0 / (n - 1)
    _, f = manufactured(n, dims)
    r, b, rn2 = residual_f64(discrete_solution(n, dims), f, h)
    assert math.sqrt(rn2) / np.linalg.norm(f) < 1e-13
    assert b.dtype == np.float32 and np.all(b[0] == 0)


def test_oracle_defect_correction_converges_bf16():
    n, dims = 17, 3
    h = 1.0 / (n - 1)
    _, f = manufactured(n, dims)
    u, hist = defect_correction(f, h, "bfloat16", 1, [180] * 8)
    assert hist[-1] < 1e-9 < hist[0]
    assert _rel(u, discrete_solution(n, dims)) < 1e-8


# ---------------------------------------------------------------------------------- GPU
@pytest.mark.gpu
@pytest.mark.parametrize("storage,variant,k", [("bfloat16", "march", 1), ("float16", "tb", 4),
                                               ("bfloat16", "tb", 2), ("float32", "march", 1)])
@pytest.mark.parametrize("n", [17, 32])
@pytest.mark.parametrize("dims", [2, 3])
def test_gpu_fixed_schedule_is_bit_exact(dims, n, storage, variant, k):
    """n = 17: plain-load kernels; n = 32: rows of whole 16-byte vectors (TMA / bulk paths)."""
    from pyheat3d_b200.precision import DefectCorrection

    n = n if dims == 3 else 2 * n
    h = 1.0 / (n - 1)
    _, f = manufactured(n, dims)
    sched = [8 * k, 12 * k, 4 * k + (1 if variant == "tb" else 0)]
    want_u, want_hist = defect_correction(f, h, storage, k, sched)
    dc = DefectCorrection(f, h, storage, variant, k)
    res = dc.solve(sweeps=sched)
    got = res.host()
    assert np.array_equal(got, want_u)
    assert np.allclose(res.history, want_hist, rtol=1e-12, atol=0)


@pytest.mark.gpu
@pytest.mark.parametrize("storage", ["bfloat16", "float16"])
def test_gpu_converges_to_1e10(storage):
    from pyheat3d_b200.precision import DefectCorrection

    n, dims = 33, 3
    h = 1.0 / (n - 1)
    u_exact, f = manufactured(n, dims)
    res = DefectCorrection(f, h, storage, "march").solve(tol=1e-10)
    assert res.converged and res.history[-1] <= 1e-10
    u = res.host()
    assert _rel(u, discrete_solution(n, dims)) < 1e-9       # FP64 oracle
    assert _rel(u, u_exact) < 2e-3                           # O(h^2) discretisation error


@pytest.mark.gpu
def test_gpu_residual_and_dot_kernels_match_numpy():
    import ctypes

    import torch

    from pyheat3d_b200 import _lib

    L = _lib.lib()
    rng = np.random.default_rng(4)
    for shape in ((9, 11, 13), (20, 31)):
        u = rng.standard_normal(shape)
        f = rng.standard_normal(shape)
        h = 0.03
        r, b, rn2 = residual_f64(u, f, h)
        U, F = (torch.from_numpy(x).cuda() for x in (u, f))
        B = torch.empty(shape, dtype=torch.float32, device="cuda")
        out = torch.zeros(1, dtype=torch.float64, device="cuda")
        scr = torch.empty(int(L.ph3_reduction_scratch_len()), dtype=torch.float64, device="cuda")
        nz, ny, nx = (1, *shape) if len(shape) == 2 else shape
        _lib.check(L.ph3_dc_residual(len(shape), nz, ny, nx, U.data_ptr(), F.data_ptr(), h, 1.0,
                                     B.data_ptr(), out.data_ptr(), scr.data_ptr(), scr.numel(),
                                     None))
        torch.cuda.synchronize()
        assert np.array_equal(B.cpu().numpy(), b)
        assert out.item() == pytest.approx(rn2, rel=1e-12)
        _lib.check(L.ph3_dot_f64(U.data_ptr(), F.data_ptr(), U.numel(), out.data_ptr(),
                                 scr.data_ptr(), scr.numel(), None))
        torch.cuda.synchronize()
        assert out.item() == pytest.approx(float(np.sum(u * f)), rel=1e-12, abs=1e-12)
        assert L.ph3_dot_f64(U.data_ptr(), F.data_ptr(), 5, out.data_ptr(), scr.data_ptr(), 3,
                             None) == 1
        assert ctypes is not None
