"""Autotuner table: shape classes, persistence, nearest-class lookup, application (CPU)."""

from __future__ import annotations

import ctypes

import pytest

from pyheat3d_b200 import _lib, tune


def test_shape_classes():
    assert tune.shape_class(64 ** 3) == "small"
    assert tune.shape_class(256 ** 3) == "medium"
    assert tune.shape_class(512 ** 3) == "large"
    assert tune.shape_class(1024 ** 3) == "xlarge"


def test_nearest_class_order():
    assert tune._nearest_classes("large") == ["large", "xlarge", "medium", "small"]
    assert tune._nearest_classes("xlarge") == ["xlarge", "large", "medium", "small"]
    assert tune._nearest_classes("small") == ["small", "medium", "large", "xlarge"]
    t = tune.Table({})
    t.entries["tb:3:float32:4:large"] = {"cfg": 0, "chunk": 0, "glups": 1.0}
    t.entries["tb:3:float32:4:xlarge"] = {"cfg": 1, "chunk": 64, "glups": 1.0}
    assert t.entry("tb", 3, "float32", 4, 1024 ** 3)["cfg"] == 1
    assert t.entry("tb", 3, "float32", 4, 512 ** 3)["cfg"] == 0
    assert t.entry("tb", 3, "float32", 4, 128 ** 3)["cfg"] == 0  # medium: nearest is large


def test_table_roundtrip_and_lookup(tmp_path):
    t = tune.Table({"gpu": "x"})
    t.entries["zmarch:3:float32:1:large"] = {"cfg": 3, "chunk": 16, "glups": 1.0}
    t.best["3:float32:large"] = {"k": 4, "variant": "tb", "glups": 2.0}
    p = tmp_path / "t.json"
    t.save(p)
    u = tune.Table.load(p)
    assert u.entry("zmarch", 3, "float32", 1, 512 ** 3)["cfg"] == 3
    # nearest class: a small grid falls back to the large entry
    assert u.entry("zmarch", 3, "float32", 1, 32 ** 3)["chunk"] == 16
    assert u.entry("tb", 3, "float32", 4, 512 ** 3) is None
    assert u.best_for(3, "float32", 100 ** 3)["k"] == 4


def test_configure_writes_only_with_an_active_table():
    L = _lib.lib()
    K = _lib.KERNEL
    cfg, chunk = ctypes.c_int(), ctypes.c_int()
    prev = tune.active_table()
    try:
        _lib.check(L.ph3_tune_set(K["zmarch"], 3, 0, 1, 2, 24))
        tune.use(None)
        tune.configure(3, "float32", 1, 512 ** 3, L)
        _lib.check(L.ph3_tune_get(K["zmarch"], 3, 0, 1, ctypes.byref(cfg), ctypes.byref(chunk)))
        assert (cfg.value, chunk.value) == (2, 24)
        t = tune.Table()
        t.entries["zmarch:3:float32:1:large"] = {"cfg": 5, "chunk": 32, "glups": 1.0}
        tune.use(t)
        tune.configure(3, "float32", 1, 512 ** 3, L)
        _lib.check(L.ph3_tune_get(K["zmarch"], 3, 0, 1, ctypes.byref(cfg), ctypes.byref(chunk)))
        assert (cfg.value, chunk.value) == (5, 32)
    finally:
        L.ph3_tune_set(K["zmarch"], 3, 0, 1, -1, 0)
        tune.use(prev)


def test_batch_family_has_configurations():
    L = _lib.lib()
    n = L.ph3_tune_count(_lib.KERNEL["batch"], 3, 1)
    assert n >= 2
    assert all(L.ph3_tune_name(_lib.KERNEL["batch"], 3, 1, i) for i in range(n))


def test_module_entry_point_runs_the_package_module(monkeypatch):
    """`python -m pyheat3d_b200.tune` must act on the module the steppers read the table from
    (a sweep's `use(None)` on a separate __main__ copy would leave the table in force)."""
    import runpy

    import pyheat3d_b200.tune as t

    called = []
    monkeypatch.setattr(t, "main", lambda argv=None: called.append(argv) or 0)
    with pytest.raises(SystemExit) as e:
        runpy.run_module("pyheat3d_b200.tune", run_name="__main__")
    assert e.value.code == 0 and called == [None]


def test_report_lists_entries_and_choices():
    t = tune.Table({})
    t.entries["tb:3:float32:4:xlarge"] = {"cfg": 0, "cfg_name": "V4_R2_W16_S4", "chunk": 0,
                                          "glups": 782.5}
    t.best["3:float32:xlarge"] = {"k": 4, "variant": "tb", "glups": 782.5, "n": 1024,
                                  "all": {"1": 717.4, "4": 782.5}}
    md = tune.report(t)
    assert "| `tb:3:float32:4:xlarge` | V4_R2_W16_S4 | 0 | 782.5 |" in md
    assert "| `3:float32:xlarge` (n=1024) | 717.4 | - | - | 782.5 | - | tb k=4 |" in md


def test_committed_table_picks_tb4_for_1024_cubed_fp32():
    """The committed table's b200/auto choice depends on the grid size (measured on a B200)."""
    t = tune.Table.load(tune.DEFAULT_TABLE)
    assert t.best_for(3, "float32", 1024 ** 3)["k"] == 4
    assert t.best_for(3, "float32", 512 ** 3)["k"] == 4
    assert t.best_for(3, "float32", 256 ** 3)["k"] == 1  # tiles too few to fill the GPU
    assert t.best_for(3, "bfloat16", 512 ** 3)["k"] == 1
    assert t.best_for(2, "float32", 16384 ** 2)["k"] == 8
