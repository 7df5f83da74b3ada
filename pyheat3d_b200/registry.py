"""The ``b200`` variants and their registration into pyheat3d's registry.

Variant table in the shape of pyheat3d's ``_build()`` ladder (``src/pyheat3d/registry.py:114-158``);
keys are ``"b200/<name>"``. :func:`register` inserts them into ``pyheat3d.registry.VARIANTS`` (the
dict the CLI, ``validation.cross_backend``, ``benchmark.run`` and the reference tests iterate), so
``pyheat3d run --variant b200/zmarch``, ``pyheat3d validate`` and ``bench/run.py`` drive the new
kernels unchanged. Without pyheat3d, :data:`VARIANTS` and :func:`make_stepper` mirror
``registry.py:161`` and ``:198-209``.
"""

from __future__ import annotations

import numpy as np

from .contract import HAVE_PYHEAT3D, Variant

BACKEND = "b200"
COLOR = "#17becf"
_SHORT = {"float32": "", "float16": "-fp16", "bfloat16": "-bf16"}
STORAGES = ("float32", "float16", "bfloat16")
TB_KS = (2, 3, 4, 8)


def _factory(kind: str, storage: str, K: int):
    def f():
        from .stepper import make

        return make(kind, storage, K)

    return f


def _build(variant_cls=Variant) -> dict[str, Variant]:
    v = []
    for st in STORAGES:
        v.append(variant_cls(BACKEND, "naive" + _SHORT[st], _factory("naive", st, 1), storage=st,
                             source=True, rung=3,
                             description=f"B200 CUDA, one site per thread, {st} storage"))
    for st in STORAGES:
        v.append(variant_cls(BACKEND, "zmarch" + _SHORT[st], _factory("march", st, 1), dims=(3,),
                             storage=st, source=True, rung=4,
                             description=f"B200 CUDA 2.5D z-march: TMA plane ring + mbarrier "
                                         f"pipeline, register z-queue, {st} storage"))
    for st in STORAGES:
        v.append(variant_cls(BACKEND, "ymarch" + _SHORT[st], _factory("march", st, 1), dims=(2,),
                             storage=st, source=True, rung=4,
                             description=f"B200 CUDA 2D y-march with register row window, "
                                         f"{st} storage"))
    for K in TB_KS:
        for st in STORAGES:
            v.append(variant_cls(BACKEND, f"tb{K}" + _SHORT[st], _factory("tb", st, K),
                                 dims=(2, 3), storage=st, steps_per_pass=K, source=True,
                                 rung=5 if st == "float32" else 6,
                                 description=f"B200 CUDA temporal blocking, {K} steps per DRAM "
                                             f"pass, {st} storage"))
    v.append(variant_cls(BACKEND, "auto", _factory("auto", "float32", 1), storage="float32",
                         source=True, rung=7,
                         description="B200 CUDA, kernel family and temporal-block depth chosen "
                                     "per grid size by the autotuner's table"))
    return {x.key: x for x in v}


#: the b200 variants (local Variant class when pyheat3d is absent)
VARIANTS: dict[str, Variant] = _build()


def register() -> list[str]:
    """Insert the b200 variants into ``pyheat3d.registry.VARIANTS``; returns the keys added.

    Idempotent. Returns ``[]`` when pyheat3d is not importable.
    """
    if not HAVE_PYHEAT3D:
        return []
    import pyheat3d.registry as reg  # type: ignore

    added = []
    for key, var in _build(reg.Variant).items():
        if key not in reg.VARIANTS:
            reg.VARIANTS[key] = var
            added.append(key)
    if BACKEND not in reg.BACKENDS:
        reg.BACKENDS = tuple(reg.BACKENDS) + (BACKEND,)
    reg.COLORS.setdefault(BACKEND, COLOR)
    return added


def availability(key: str) -> tuple[bool, str]:
    """``(ok, reason)`` like ``registry.availability`` (registry.py:179-189)."""
    if key not in VARIANTS:
        return False, f"unknown variant {key!r}"
    try:
        import torch

        if not torch.cuda.is_available():
            return False, "no CUDA GPU"
        VARIANTS[key].factory()
    except Exception as e:  # missing extension, broken install, ...
        return False, f"{type(e).__name__}: {e}".splitlines()[0][:120]
    return True, ""


def make_stepper(key: str, u0: np.ndarray, stencil, source: np.ndarray | None = None):
    """Instantiate a b200 variant on an initial state (registry.py:198-209)."""
    var = VARIANTS[key]
    if u0.ndim not in var.dims:
        raise ValueError(f"{key} supports dims {var.dims}, got {u0.ndim}")
    if source is not None and not var.source:
        raise ValueError(f"{key} does not support a source term")
    cls = var.factory()
    st = cls(u0, stencil, source)
    st.steps_per_pass = var.steps_per_pass
    return st
