"""Autotuner: sweep the compiled tile configurations, march chunks and temporal-block depths,
persist the winners in a JSON table, and apply the table to the launches.

Extends pyheat3d's ``bench/tune.py`` (which sweeps the CuPy kernels' tile constants by
monkey-patching module globals, ``bench/tune.py:47-96``): here every kernel family exposes its
compiled configurations through the C ABI (``ph3_tune_count`` / ``ph3_tune_name``), a table entry
(``ph3_tune_set``) selects configuration and chunk per (family, dims, storage, k), and the
results are stored per shape class so that one table serves every grid size:

    python -m pyheat3d_b200.tune b200-zmarch --n 512           # like `tune.py cuda-zmarch`
    python -m pyheat3d_b200.tune b200-tb3d --n 512 --K 2 4     # like `tune.py cuda-tb3d`
    python -m pyheat3d_b200.tune b200-ymarch --n 16384         # 2D single step
    python -m pyheat3d_b200.tune b200-tb2d --n 16384 --K 2 4 8
    python -m pyheat3d_b200.tune b200-batch                    # batch tile configurations
    python -m pyheat3d_b200.tune all --quick                   # every target, small sizes

The table also records, per (dims, storage, shape class), the fastest kernel family and k
(``best``), which the ``b200/auto`` variant uses: that is how the temporal-block depth is chosen.
Timing: CUDA events around a calibrated number of steps, best of ``repeats`` (on a shared GPU
contention only ever slows a repeat down, as bench/tune.py notes).

Tables load from ``$PH3_TUNING`` or ``pyheat3d_b200/tuning.json``; :func:`configure` applies the
entries that match a stepper's grid before its launches.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import sys
import time
from pathlib import Path

import numpy as np

from . import _lib

DEFAULT_TABLE = Path(__file__).resolve().with_name("tuning.json")
CLASSES = ((1 << 22, "small"), (1 << 26, "medium"), (1 << 29, "large"), (None, "xlarge"))


def shape_class(cells: int) -> str:
    """'small' (< 4 Mi sites), 'medium' (< 64 Mi), 'large' (< 512 Mi, e.g. 512^3) or 'xlarge'
    (e.g. 1024^3)."""
    for bound, name in CLASSES:
        if bound is None or cells < bound:
            return name
    return "xlarge"


def _nearest_classes(cls: str) -> list[str]:
    """`cls` first, then the other classes by distance (the larger one first on a tie)."""
    names = [name for _, name in CLASSES]
    i = names.index(cls)
    return sorted(names, key=lambda c: (abs(names.index(c) - i), -names.index(c)))


def _key(kernel: str, dims: int, storage: str, k: int, cls: str) -> str:
    return f"{kernel}:{dims}:{storage}:{k}:{cls}"


class Table:
    """Winning configurations: entries keyed 'kernel:dims:storage:k:class' -> {cfg, chunk, ...},
    best kernels keyed 'dims:storage:class' -> {variant, k, glups}."""

    def __init__(self, data: dict | None = None):
        data = data or {}
        self.gpu = data.get("gpu", "")
        self.entries: dict[str, dict] = dict(data.get("entries", {}))
        self.best: dict[str, dict] = dict(data.get("best", {}))

    def to_json(self) -> dict:
        return {"gpu": self.gpu, "entries": self.entries, "best": self.best}

    def save(self, path: str | Path) -> None:
        Path(path).write_text(json.dumps(self.to_json(), indent=1, sort_keys=True))

    @classmethod
    def load(cls, path: str | Path) -> Table:
        return cls(json.loads(Path(path).read_text()))

    def entry(self, kernel: str, dims: int, storage: str, k: int, cells: int) -> dict | None:
        for c in _nearest_classes(shape_class(cells)):  # nearest available class
            e = self.entries.get(_key(kernel, dims, storage, k, c))
            if e is not None:
                return e
        return None

    def best_for(self, dims: int, storage: str, cells: int) -> dict | None:
        for c in _nearest_classes(shape_class(cells)):
            b = self.best.get(f"{dims}:{storage}:{c}")
            if b is not None:
                return b
        return None


_ACTIVE: Table | None = None
_LOADED = False


def active_table() -> Table | None:
    """The table in use: $PH3_TUNING, else pyheat3d_b200/tuning.json, else None."""
    global _ACTIVE, _LOADED
    if not _LOADED:
        _LOADED = True
        path = os.environ.get("PH3_TUNING") or (DEFAULT_TABLE if DEFAULT_TABLE.exists() else None)
        if path:
            try:
                _ACTIVE = Table.load(path)
            except (OSError, ValueError):
                _ACTIVE = None
    return _ACTIVE


def use(table: Table | None) -> None:
    """Make `table` the active one (None: built-in defaults)."""
    global _ACTIVE, _LOADED
    _ACTIVE, _LOADED = table, True


def configure(dims: int, storage: str, k: int, cells: int, lib=None) -> None:
    """Write the active table's entries for this grid into the library's tuning table.

    Without an active table nothing is written (explicit ``ph3_tune_set`` calls stay in force).
    """
    t = active_table()
    if t is None:
        return
    lib = lib or _lib.lib()
    S = _lib.STORAGE[storage]
    for kernel in ("zmarch", "march", "tb"):
        kk = k if kernel == "tb" else 1
        if kernel == "zmarch" and dims != 3:
            continue
        if kernel == "tb" and k < 2:
            continue
        e = t.entry(kernel, dims, storage, kk, cells)
        if e is not None:
            lib.ph3_tune_set(_lib.KERNEL[kernel], dims, S, kk, int(e["cfg"]), int(e["chunk"]))


def configure_batch(lib=None) -> None:
    """Apply the active table's batch tile configuration (if any)."""
    t = active_table()
    e = t.entries.get(_key("batch", 3, "float32", 1, "large")) if t is not None else None
    if e is not None:
        (lib or _lib.lib()).ph3_tune_set(_lib.KERNEL["batch"], 3, 0, 1, int(e["cfg"]), 0)


def batch_k2d() -> int:
    """Temporal-block depth the active table picked for the 2D problems of a batch (1: none)."""
    t = active_table()
    e = t.entries.get(_key("batch", 3, "float32", 1, "large")) if t is not None else None
    return int(e.get("k2d", 1)) if e is not None else 1


def with_batch_k(problems: list) -> list:
    """The problems with the table's 2D temporal-block depth set on every 2D problem."""
    import dataclasses

    k = batch_k2d()
    return [dataclasses.replace(p, k=k) if p.u0.ndim == 2 else p for p in problems]


# ------------------------------------------------------------------------------------------
# measurement
# ------------------------------------------------------------------------------------------
def time_key(key: str, u0: np.ndarray, stencil, min_time: float = 0.1, repeats: int = 3) -> float:
    """Best GLUPS of a registered variant on u0 (calibrated steps, CUDA events)."""
    import torch

    from .registry import make_stepper

    st = make_stepper(key, u0, stencil)
    k = st.steps_per_pass
    st.step(2 * k)
    torch.cuda.synchronize()
    n = k
    while True:
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        st.step(n)
        b.record()
        b.synchronize()
        dt = a.elapsed_time(b) * 1e-3
        if dt >= 0.2 * min_time or n >= 1 << 20:
            break
        n *= 2
    n = max(k, int(math.ceil(min_time / (dt / n) / k)) * k)
    best = 0.0
    for _ in range(repeats):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        st.step(n)
        b.record()
        b.synchronize()
        best = max(best, st.ncells * n / (a.elapsed_time(b) * 1e-3) / 1e9)
    st.close()
    return best


def _suffix(storage: str) -> str:
    return {"float32": "", "float16": "-fp16", "bfloat16": "-bf16"}[storage]


def sweep_family(table: Table, kernel: str, dims: int, storage: str, k: int, n: int,
                 chunks=(0, 8, 16, 32, 64), min_time: float = 0.1, verbose: bool = True) -> dict:
    """Time every (configuration, chunk) of one family on an n^dims periodic field; record the
    winner in `table` and return it."""
    from .contract import heat_stencil

    lib = _lib.lib()
    S = _lib.STORAGE[storage]
    kid = _lib.KERNEL[kernel]
    u0 = np.random.default_rng(0).random((n,) * dims, dtype=np.float32)
    st = heat_stencil(dims, 0.95 / (2 * dims), "periodic")
    if kernel == "tb":
        key = f"b200/tb{k}" + _suffix(storage)
    else:
        key = ("b200/zmarch" if dims == 3 else "b200/ymarch") + _suffix(storage)
    ncfg = lib.ph3_tune_count(kid, dims, k)
    best = None
    prev = active_table()
    use(None)  # the steppers must not overwrite the configuration under test
    try:
        for cfg in range(ncfg):
            name = lib.ph3_tune_name(kid, dims, k, cfg).decode()
            for chunk in chunks:
                _lib.check(lib.ph3_tune_set(kid, dims, S, k, cfg, chunk))
                g = time_key(key, u0, st, min_time)
                if verbose:
                    print(f"{kernel:6s} {dims}D {storage:8s} k={k} n={n} {name:22s} chunk={chunk:3d}"
                          f" {g:9.1f} GLUPS", flush=True)
                if best is None or g > best["glups"]:
                    best = {"cfg": cfg, "cfg_name": name, "chunk": chunk, "glups": round(g, 2),
                            "n": n}
    finally:
        lib.ph3_tune_set(kid, dims, S, k, -1, 0)
        use(prev)
    if best is not None:
        table.entries[_key(kernel, dims, storage, k, shape_class(n ** dims))] = best
    return best or {}


def sweep_batch(table: Table, quick: bool = False, verbose: bool = True) -> dict:
    """Time every batch tile configuration with each 2D temporal-block depth (1, 2, 4) on a
    problem mix of the batching workload's distribution (another seed; quick: a scaled-down mix);
    record the fastest pair."""
    import dataclasses

    import torch

    from .batch import Batch, synthetic_batch

    lib = _lib.lib()
    kid = _lib.KERNEL["batch"]
    if quick:
        base = synthetic_batch(64, seed=1, n2d=(64, 1024), n3d=(32, 128), steps=(20, 100))
    else:
        base = synthetic_batch(512, seed=1)
    best = None
    prev = active_table()
    use(None)
    try:
        for k2d in (1, 2, 4):
            probs = [dataclasses.replace(p, k=k2d) if p.u0.ndim == 2 else p for p in base]
            for cfg in range(lib.ph3_tune_count(kid, 3, 1)):
                _lib.check(lib.ph3_tune_set(kid, 3, 0, 1, cfg, 0))
                b = Batch(probs)
                b.run()
                torch.cuda.synchronize()
                b.reset()
                t0 = time.perf_counter()
                b.run()
                torch.cuda.synchronize()
                dt = time.perf_counter() - t0
                g = b.updates / dt / 1e9
                name = lib.ph3_tune_name(kid, 3, 1, cfg).decode()
                if verbose:
                    print(f"batch  {name:22s} k2d={k2d} {g:9.1f} GLUPS ({dt:.3f} s)", flush=True)
                if best is None or g > best["glups"]:
                    best = {"cfg": cfg, "cfg_name": name, "chunk": 0, "k2d": k2d,
                            "glups": round(g, 2)}
                del b
    finally:
        lib.ph3_tune_set(kid, 3, 0, 1, -1, 0)
        use(prev)
    if best is not None:
        table.entries[_key("batch", 3, "float32", 1, "large")] = best
    return best or {}


def pick_best(table: Table, dims: int, storage: str, n: int, ks=(1, 2, 3, 4, 8),
              min_time: float = 0.1, verbose: bool = True) -> dict:
    """With the table applied, time the single-step kernel and every tb<k>; record the fastest
    (the temporal-block depth) for this (dims, storage, shape class)."""
    from .contract import heat_stencil

    u0 = np.random.default_rng(0).random((n,) * dims, dtype=np.float32)
    st = heat_stencil(dims, 0.95 / (2 * dims), "periodic")
    prev = active_table()
    use(table)
    out = {}
    try:
        for k in ks:
            key = (("b200/zmarch" if dims == 3 else "b200/ymarch") if k == 1 else f"b200/tb{k}") \
                + _suffix(storage)
            configure(dims, storage, k, n ** dims)
            out[k] = time_key(key, u0, st, min_time)
            if verbose:
                print(f"best?  {dims}D {storage:8s} n={n} k={k}: {out[k]:9.1f} GLUPS", flush=True)
    finally:
        use(prev)
    k = max(out, key=out.get)
    rec = {"k": k, "variant": "march" if k == 1 else "tb", "glups": round(out[k], 2),
           "all": {str(a): round(b, 2) for a, b in out.items()}, "n": n}
    table.best[f"{dims}:{storage}:{shape_class(n ** dims)}"] = rec
    return rec


def report(table: Table) -> str:
    """Markdown view of a table: the winning configuration per entry and the fastest kernel
    (single step or tb<k>) per (dims, storage, shape class)."""
    out = ["| family:dims:storage:k:class | winning config | chunk | GLUPS |", "|---|---|---:|---:|"]
    for key in sorted(table.entries):
        e = table.entries[key]
        out.append(f"| `{key}` | {e.get('cfg_name', e.get('cfg'))} | {e.get('chunk', 0)} | "
                   f"{e.get('glups', '')} |")
    out += ["", "| dims:storage:class | k=1 | k=2 | k=3 | k=4 | k=8 | chosen |",
            "|---|---:|---:|---:|---:|---:|---|"]
    for key in sorted(table.best):
        b = table.best[key]
        cells = " | ".join(str(b.get("all", {}).get(str(k), "-")) for k in (1, 2, 3, 4, 8))
        chosen = "single step" if b["k"] == 1 else f"tb k={b['k']}"
        out.append(f"| `{key}` (n={b.get('n')}) | {cells} | {chosen} |")
    return "\n".join(out)


# ------------------------------------------------------------------------------------------
# CLI
# ------------------------------------------------------------------------------------------
def main(argv: list[str] | None = None) -> int:
    ap = argparse.ArgumentParser(description=__doc__,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("what", choices=("b200-zmarch", "b200-ymarch", "b200-tb3d", "b200-tb2d",
                                     "b200-batch", "all", "report"))
    ap.add_argument("--n", type=int, default=None)
    ap.add_argument("--K", type=int, nargs="*", default=None)
    ap.add_argument("--storage", nargs="*", default=["float32", "bfloat16"])
    ap.add_argument("--min-time", type=float, default=0.1)
    ap.add_argument("--quick", action="store_true", help="small sizes and few chunks")
    ap.add_argument("--out", default=None, help="table to update (default: the active table "
                                                "path, pyheat3d_b200/tuning.json)")
    a = ap.parse_args(argv)
    if a.what == "report":  # the table as Markdown (no GPU needed)
        path = Path(a.out or os.environ.get("PH3_TUNING") or DEFAULT_TABLE)
        print(report(Table.load(path)))
        return 0
    import torch

    if not torch.cuda.is_available():
        print("no CUDA device", file=sys.stderr)
        return 2
    out = Path(a.out or os.environ.get("PH3_TUNING") or DEFAULT_TABLE)
    table = Table.load(out) if out.exists() else Table()
    table.gpu = torch.cuda.get_device_name(0)
    chunks = (0, 16, 32) if a.quick else (0, 8, 16, 32, 64)
    n3 = a.n or (128 if a.quick else 512)
    n2 = a.n or (2048 if a.quick else 16384)
    for storage in a.storage:
        if a.what in ("b200-zmarch", "all"):
            sweep_family(table, "zmarch", 3, storage, 1, n3, chunks, a.min_time)
            sweep_family(table, "march", 3, storage, 1, n3 - 1, chunks, a.min_time)
        if a.what in ("b200-ymarch", "all"):
            sweep_family(table, "march", 2, storage, 1, n2, (0, 64, 256, 1024), a.min_time)
        if a.what in ("b200-tb3d", "all"):
            for k in a.K or (2, 3, 4, 8):
                sweep_family(table, "tb", 3, storage, k, n3, (0, 32, 64, 128), a.min_time)
        if a.what in ("b200-tb2d", "all"):
            for k in a.K or (2, 4, 8):
                sweep_family(table, "tb", 2, storage, k, n2, (0, 256, 1024), a.min_time)
        if a.what == "all":
            pick_best(table, 3, storage, n3, min_time=a.min_time)
            pick_best(table, 2, storage, n2, (1, 2, 4, 8), min_time=a.min_time)
    if a.what in ("b200-batch", "all"):
        sweep_batch(table, a.quick)
    table.save(out)
    print(f"wrote {out}")
    return 0


if __name__ == "__main__":
    # Run the package's own module object: the steppers consult `pyheat3d_b200.tune` for the
    # active table, so `use(None)` during a sweep must act on that module, not on __main__.
    from pyheat3d_b200 import tune as _package_module

    sys.exit(_package_module.main())
