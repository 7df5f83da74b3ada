"""Traffic models of pyheat3d (``src/pyheat3d/traffic.py:23-50``), for this backend's records.

``minimal_bytes`` is the roofline denominator every figure uses (one read and one write of each
value per pass). ``tb_model_bytes`` is pyheat3d's second, halo-aware estimate for overlapped
temporal blocking; pyheat3d computes it only for its CuPy kernels (``benchmark.py:219-230``),
from the stepper's tile. ``B200Stepper.tile`` carries the same three numbers for the b200 tb<k>
variants (from ``ph3_tb_tile``), so the b200 rows get the same column.
"""

from __future__ import annotations


def minimal_bytes(bytes_per_value: int, steps_per_pass: int = 1) -> float:
    """Minimal DRAM bytes per site update: 2 * bytes_per_value / k (traffic.py:23-25)."""
    return 2.0 * bytes_per_value / steps_per_pass


def tb_model_bytes(dims: int, k: int, bytes_per_value: int, tx: int, ty: int, zch: int) -> float:
    """Bytes per update of overlapped tiling with a k-deep halo on every tiled side and k extra
    planes (rows in 2D) at each end of a chunk, no L2 reuse assumed (traffic.py:38-50)."""
    if dims == 3:
        over_xy = (tx * ty) / ((tx - 2 * k) * (ty - 2 * k))
    else:
        over_xy = tx / (tx - 2 * k)
    over_z = (zch + 2 * k) / zch
    return bytes_per_value * (over_xy * over_z + 1.0) / k
