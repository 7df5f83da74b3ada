"""The C-ABI library: built, loadable, exports every declared symbol, rejects bad arguments.

CPU only: no call here launches a kernel (argument checks run before any CUDA call).
"""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

from pyheat3d_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols() -> set[str]:
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(ph3_\w+)\s*\(", text))
    return names


@pytest.fixture(scope="module")
def lib():
    if not _lib.LIB_PATH.exists():
        from pyheat3d_b200.build import build

        build()
    return _lib.lib()


def test_every_declared_symbol_is_exported_and_bound(lib):
    decl = declared_symbols()
    assert "ph3_advance" in decl and len(decl) >= 10
    for name in decl:
        assert hasattr(lib, name), name
    assert decl == set(_lib.SIGNATURES), decl ^ set(_lib.SIGNATURES)


def test_version(lib):
    assert lib.ph3_version() >= 10000


P = ctypes.c_void_p


@pytest.mark.parametrize("args,msg", [
    ((P(16), P(32), None, 0, 5, 5, 0.1, 0.1, 0, 0, None), "every axis"),
    ((P(16), P(32), None, 5, 5, 5, 0.1, 0.1, 7, 0, None), "storage"),
    ((P(16), P(32), None, 5, 5, 5, 0.1, 0.1, 0, 3, None), "bc must"),
    ((P(16), P(16), None, 5, 5, 5, 0.1, 0.1, 0, 0, None), "distinct"),
    ((None, P(16), None, 5, 5, 5, 0.1, 0.1, 0, 0, None), "non-null"),
])
def test_naive3d_rejects_bad_arguments(lib, args, msg):
    rc = lib.ph3_naive3d(*args)
    assert rc == 1
    assert msg in _lib.last_error()


def test_tb_rejects_unsupported_k(lib):
    rc = lib.ph3_tb3d(P(16), P(32), None, 5, 5, 5, 5, 0.1, 0.1, 0, 0, 0, None)
    assert rc == 1 and "k must be" in _lib.last_error()


def test_advance_rejects_bad_variant_and_steps(lib):
    ib = ctypes.c_int(0)
    rc = lib.ph3_advance(3, 5, 5, 5, 0, 0, 0.1, 0.1, 9, 1, P(16), P(32), None, 1, None,
                         ctypes.byref(ib))
    assert rc == 1 and "unknown variant" in _lib.last_error()
    rc = lib.ph3_advance(3, 5, 5, 5, 0, 0, 0.1, 0.1, 1, 2, P(16), P(32), None, 1, None,
                         ctypes.byref(ib))
    assert rc == 1 and "k must be 1" in _lib.last_error()
    rc = lib.ph3_advance(2, 5, 5, 5, 0, 0, 0.1, 0.1, 1, 1, P(16), P(32), None, 1, None,
                         ctypes.byref(ib))
    assert rc == 1 and "nz == 1" in _lib.last_error()
    rc = lib.ph3_advance(3, 5, 5, 5, 0, 0, 0.1, 0.1, 1, 1, P(16), P(32), None, -1, None,
                         ctypes.byref(ib))
    assert rc == 1 and "nsteps" in _lib.last_error()


def test_check_raises_with_message(lib):
    rc = lib.ph3_naive2d(P(16), P(16), None, 5, 5, 0.1, 0.1, 0, 0, None)
    with pytest.raises(_lib.Ph3Error, match="distinct"):
        _lib.check(rc)


def test_product_path_does_not_import_the_oracle():
    """The package never imports the CPU oracle (no CPU fallback on the product path)."""
    pkg = ROOT / "pyheat3d_b200"
    for py in pkg.rglob("*.py"):
        text = py.read_text()
        assert not re.search(r"^\s*(from|import)\s+oracle\b", text, flags=re.M), py


def test_tuning_table_roundtrip(lib):
    K = _lib.KERNEL
    assert lib.ph3_tune_count(K["zmarch"], 3, 1) >= 2
    assert lib.ph3_tune_count(K["zmarch"], 2, 1) == 0
    for k in (2, 3, 4, 8):
        n = lib.ph3_tune_count(K["tb"], 3, k)
        assert n >= 1
        names = {lib.ph3_tune_name(K["tb"], 3, k, c).decode() for c in range(n)}
        assert len(names) == n and all(names)
    assert lib.ph3_tune_name(K["tb"], 3, 2, 99) == b""
    cfg, chunk = ctypes.c_int(7), ctypes.c_int(7)
    _lib.check(lib.ph3_tune_get(K["tb"], 3, 0, 4, ctypes.byref(cfg), ctypes.byref(chunk)))
    assert (cfg.value, chunk.value) == (-1, 0)
    _lib.check(lib.ph3_tune_set(K["tb"], 3, 0, 4, 1, 48))
    _lib.check(lib.ph3_tune_get(K["tb"], 3, 0, 4, ctypes.byref(cfg), ctypes.byref(chunk)))
    assert (cfg.value, chunk.value) == (1, 48)
    _lib.check(lib.ph3_tune_set(K["tb"], 3, 0, 4, -1, 0))
    assert lib.ph3_tune_set(K["tb"], 3, 0, 4, 99, 0) == 1
    assert lib.ph3_tune_set(K["tb"], 4, 0, 4, 0, 0) == 1
    assert lib.ph3_tune_set(K["tb"], 3, 0, 4, 0, -5) == 1


def test_wait_flag_rejects_bad_arguments(lib):
    assert lib.ph3_wait_flag(None, 1, 16, None) == 1 and "non-null" in _lib.last_error()
    assert lib.ph3_wait_flag(P(18), 1, 16, None) == 1 and "aligned" in _lib.last_error()
    assert lib.ph3_wait_flag(P(16), 1, 0, None) == 1 and "spin_limit" in _lib.last_error()
    assert lib.ph3_wait_flag(P(16), 1, (1 << 22) + 1, None) == 1
    assert "spin_limit" in _lib.last_error()
