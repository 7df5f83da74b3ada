"""ctypes binding of ``libph3b200.so`` (declarations: ``include/ph3b200.h``).

The library is loaded on first use. There is no fallback: if it is missing or cannot be loaded,
:func:`lib` raises, so no caller can silently run something else.
"""

from __future__ import annotations

import ctypes
import threading
from pathlib import Path

LIB_PATH = Path(__file__).resolve().with_name("libph3b200.so")

STORAGE = {"float32": 0, "float16": 1, "bfloat16": 2}
BC = {"dirichlet": 0, "periodic": 1}
VARIANT = {"naive": 0, "march": 1, "tb": 2}

#: every symbol include/ph3b200.h declares, with (restype, argtypes)
_i, _f, _p, _i64 = ctypes.c_int, ctypes.c_float, ctypes.c_void_p, ctypes.c_int64
SIGNATURES: dict[str, tuple[object, list[object]]] = {
    "ph3_version": (_i, []),
    "ph3_last_error": (ctypes.c_char_p, []),
    "ph3_sm_count": (_i, []),
    "ph3_device_status": (_i, [ctypes.POINTER(_i), _i]),
    "ph3_naive2d": (_i, [_p, _p, _p, _i, _i, _f, _f, _i, _i, _p]),
    "ph3_naive3d": (_i, [_p, _p, _p, _i, _i, _i, _f, _f, _i, _i, _p]),
    "ph3_zmarch3d": (_i, [_p, _p, _p, _i, _i, _i, _f, _f, _i, _i, _i, _p]),
    "ph3_zmarch3d_planes": (_i, [_p, _p, _p, _i, _i, _i, _i, _i, _f, _f, _i, _i, _i, _p]),
    "ph3_ymarch2d": (_i, [_p, _p, _p, _i, _i, _f, _f, _i, _i, _i, _p]),
    "ph3_tb3d": (_i, [_p, _p, _p, _i, _i, _i, _i, _f, _f, _i, _i, _i, _p]),
    "ph3_tb2d": (_i, [_p, _p, _p, _i, _i, _i, _f, _f, _i, _i, _i, _p]),
    "ph3_tb_tile": (_i, [_i, _i, _i, _i, _i, _i, _i, ctypes.POINTER(_i), ctypes.POINTER(_i),
                         ctypes.POINTER(_i)]),
    "ph3_advance": (_i, [_i, _i, _i, _i, _i, _i, _f, _f, _i, _i, _p, _p, _p, _i64, _p,
                         ctypes.POINTER(_i)]),
    "ph3_reduction_scratch_len": (_i64, []),
    "ph3_dc_residual": (_i, [_i, _i, _i, _i, _p, _p, ctypes.c_double, ctypes.c_double, _p, _p,
                             _p, _i64, _p]),
    "ph3_dot_f64": (_i, [_p, _p, _i64, _p, _p, _i64, _p]),
    "ph3_dc_correct": (_i, [_p, _p, _i, ctypes.c_double, _i64, _p]),
    "ph3_batch_workspace_bytes": (_i64, [_p, _i]),
    "ph3_batch_prepare": (_i, [_p, _i, _p, _i64, _p]),
    "ph3_batch_launch": (_i, [_p, _i, _p]),
    "ph3_batch_run_static": (_i, [_p, _i, _p]),
    "ph3_wait_flag": (_i, [_p, _i, ctypes.c_uint, _p]),
    "ph3_tune_count": (_i, [_i, _i, _i]),
    "ph3_tune_name": (ctypes.c_char_p, [_i, _i, _i, _i]),
    "ph3_tune_set": (_i, [_i, _i, _i, _i, _i, _i]),
    "ph3_tune_get": (_i, [_i, _i, _i, _i, ctypes.POINTER(_i), ctypes.POINTER(_i)]),
}

#: size of the fixed device workspace behind ph3_batch_run_static (include/ph3b200.h)
STATIC_BATCH_BYTES = 1 << 20

#: tuning-table kernel families (include/ph3b200.h PH3_KERNEL_*)
KERNEL = {"zmarch": 0, "march": 1, "tb": 2, "naive": 3, "batch": 4}

_lock = threading.Lock()
_lib: ctypes.CDLL | None = None


class Ph3Error(RuntimeError):
    """A libph3b200 entry point returned a nonzero code."""

    def __init__(self, code: int, message: str):
        super().__init__(f"libph3b200 error {code}: {message}")
        self.code = code


def lib() -> ctypes.CDLL:
    """The loaded library (loads and binds it on first call; raises if unavailable)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.exists():
                raise RuntimeError(
                    f"{LIB_PATH.name} is not built; run `python -m pyheat3d_b200.build` "
                    "(needs nvcc with sm_100a support)")
            handle = ctypes.CDLL(str(LIB_PATH))
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(handle, name)
                fn.restype = res
                fn.argtypes = args
            _lib = handle
    return _lib


def last_error() -> str:
    msg = lib().ph3_last_error()
    return msg.decode() if msg else ""


def check(rc: int) -> None:
    """Raise :class:`Ph3Error` for a nonzero return code."""
    if rc != 0:
        raise Ph3Error(rc, last_error())


#: status-word codes (ph3_common.cuh DeviceError)
STATUS = {"ok": 0, "mbarrier_timeout": 1, "dependency_timeout": 2, "stop_requested": 3}


def device_status(clear: bool = True) -> int:
    """Kernel status word of the current device (0 = no expired bounded wait). Synchronises."""
    code = ctypes.c_int(0)
    check(lib().ph3_device_status(ctypes.byref(code), int(clear)))
    return code.value
