"""Generate the golden fixtures from the reference pyheat3d itself.

Run in a checkout where the pyheat3d sources are importable, e.g.::

    PYTHONPATH=<pyheat3d checkout>/src python tests/golden/make_golden.py

It imports the reference's own ``reference_step`` (``src/pyheat3d/backends/numpy_ref.py:30``),
``emulated_reference`` / ``round_storage`` (``src/pyheat3d/validation.py:157-183``),
``to_bf16_bits`` is restated there too (``cupy_backend.py:103`` needs CuPy to import, so the bf16
vectors come from ``validation.round_storage``) and the problem constructors
(``src/pyheat3d/problem.py:51-69``), runs them on small seeded inputs and writes:

- ``stencil_small.npz``: initial fields and outputs for 2D/3D x Dirichlet/periodic x
  (storage, k) rounding schedules, 197 steps (every k of 2, 3, 4, 8 plus a remainder, as in the
  reference's ``tests/test_backends.py:40``), plus Jacobi sweeps with and without a source,
  float64 runs and the tiny-grid cases of ``tests/test_backends.py:86-103``;
- ``dirichlet128.json``: SHA-256 and summary statistics of the 3D 128^3 Dirichlet heat run
  (r = 0.15, seed 0, zero boundary layer, 100 steps), too large to store as an array.
"""

from __future__ import annotations

import hashlib
import json
import pathlib

import numpy as np
from pyheat3d import validation as val
from pyheat3d.backends.numpy_ref import NumpyStepper, reference_step
from pyheat3d.problem import heat_stencil, jacobi_stencil

HERE = pathlib.Path(__file__).resolve().parent
SHAPES = {2: (33, 47), 3: (13, 17, 19)}
STEPS = 2 * 3 * 4 * 8 + 5
SCHEDULES = [("float32", 1), ("float16", 1), ("bfloat16", 1), ("float16", 2), ("bfloat16", 3),
             ("float16", 4), ("bfloat16", 8)]


def main() -> None:
    arrays: dict[str, np.ndarray] = {}
    meta: dict[str, object] = {"steps": STEPS, "schedules": SCHEDULES, "shapes": SHAPES}
    rng = np.random.default_rng(7)
    for dims, shape in SHAPES.items():
        u0 = rng.random(shape, dtype=np.float32)
        arrays[f"u0_{dims}d"] = u0
        for bc in ("dirichlet", "periodic"):
            st = heat_stencil(dims, 0.9 / (2 * dims), bc)
            for storage, k in SCHEDULES:
                out = val.emulated_reference(u0, st.c0, st.c1, bc, STEPS, storage, k)
                arrays[f"heat_{dims}d_{bc}_{storage}_k{k}"] = out.astype(np.float32)
            # Jacobi sweeps with a source (b added last, numpy_ref.py:44-45)
            js = jacobi_stencil(dims, bc)
            b = (rng.random(shape, dtype=np.float32) - np.float32(0.5)) * np.float32(1e-2)
            arrays[f"src_{dims}d_{bc}"] = b
            u = u0.copy()
            for _ in range(24):
                u = reference_step(u, js.c0, js.c1, bc, b)
            arrays[f"jacobi_src_{dims}d_{bc}"] = u
            u = u0.copy()
            for _ in range(24):
                u = reference_step(u, js.c0, js.c1, bc)
            arrays[f"jacobi_{dims}d_{bc}"] = u
            # float64 oracle runs (the FP64 error statements of the precision path)
            u = u0.astype(np.float64)
            for _ in range(24):
                u = reference_step(u, st.c0, st.c1, bc)
            arrays[f"heat64_{dims}d_{bc}"] = u
            # in-place stepper must agree bitwise with reference_step (test_reference.py:13-24)
            s = NumpyStepper(u0, st)
            s.step(5)
            arrays[f"stepper5_{dims}d_{bc}"] = s.get()
    # tiny grids smaller than one tile (test_backends.py:86-103)
    rng = np.random.default_rng(9)
    for dims, shape in ((2, (5, 7)), (3, (5, 6, 7))):
        u0 = rng.random(shape, dtype=np.float32)
        arrays[f"tiny_u0_{dims}d"] = u0
        for bc in ("dirichlet", "periodic"):
            st = heat_stencil(dims, 0.1, bc)
            for storage, k in SCHEDULES:
                out = val.emulated_reference(u0, st.c0, st.c1, bc, 9, storage, k)
                arrays[f"tiny_{dims}d_{bc}_{storage}_k{k}"] = out.astype(np.float32)
    # bf16 / fp16 rounding of edge values (ties, subnormals, overflow)
    special = np.array([0.0, -0.0, 1.0, 1.00390625, 1.01171875, 1.0 + 2**-9, 1.0 + 3 * 2**-9,
                        3.4e38, 6.6e4, 65519.0, 65520.0, 1e-8, 6e-8, 2**-24, 2**-25, -2.5,
                        0.1, 1 / 3, 2**-126, 2**-130], dtype=np.float32)
    special = np.concatenate([special, np.random.default_rng(11).standard_normal(
        4096).astype(np.float32) * np.float32(100)])
    arrays["round_in"] = special
    arrays["round_bf16"] = val.round_storage(special, "bfloat16")
    with np.errstate(over="ignore"):
        arrays["round_f16"] = val.round_storage(special, "float16")
    np.savez_compressed(HERE / "stencil_small.npz", **arrays)

    # the 128^3 fp32 Dirichlet case: zero walls, r = 0.15, seed 0, 100 steps
    u0 = np.random.default_rng(0).random((128,) * 3, dtype=np.float32)
    u0[0] = u0[-1] = 0
    u0[:, 0] = u0[:, -1] = 0
    u0[:, :, 0] = u0[:, :, -1] = 0
    st = heat_stencil(3, 0.15, "dirichlet")
    s = NumpyStepper(u0, st)
    s.step(100)
    u = s.get()
    meta["dirichlet128"] = {
        "shape": [128, 128, 128], "r": 0.15, "steps": 100, "seed": 0, "bc": "dirichlet",
        "c0": st.c0, "c1": st.c1,
        "sha256": hashlib.sha256(np.ascontiguousarray(u).tobytes()).hexdigest(),
        "sum64": float(u.astype(np.float64).sum()), "max": float(u.max()),
        "probe": [float(u[64, 64, 64]), float(u[1, 1, 1]), float(u[100, 7, 33])],
    }
    (HERE / "dirichlet128.json").write_text(json.dumps(meta, indent=1, default=list))
    print("wrote", HERE / "stencil_small.npz", "and", HERE / "dirichlet128.json")


if __name__ == "__main__":
    main()
