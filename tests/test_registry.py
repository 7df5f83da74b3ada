"""The b200 variants and their registration into pyheat3d (CPU only)."""

from __future__ import annotations

import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

import pyheat3d_b200 as pb
from pyheat3d_b200.registry import STORAGES, TB_KS, VARIANTS, make_stepper

ROOT = Path(__file__).resolve().parents[1]


def test_variant_table():
    keys = set(VARIANTS)
    for st, suf in zip(STORAGES, ("", "-fp16", "-bf16")):
        assert f"b200/naive{suf}" in keys
        assert f"b200/zmarch{suf}" in keys and VARIANTS[f"b200/zmarch{suf}"].dims == (3,)
        assert f"b200/ymarch{suf}" in keys and VARIANTS[f"b200/ymarch{suf}"].dims == (2,)
        for k in TB_KS:
            v = VARIANTS[f"b200/tb{k}{suf}"]
            assert v.steps_per_pass == k and v.storage == st and v.dims == (2, 3)
    assert all(v.gpu and v.source and v.backend == "b200" for v in VARIANTS.values())
    assert len(VARIANTS) == 3 * (3 + len(TB_KS)) + 1
    assert VARIANTS["b200/auto"].storage == "float32" and VARIANTS["b200/auto"].dims == (2, 3)


def test_make_stepper_checks_dims_before_touching_the_gpu():
    u0 = np.zeros((5, 6), np.float32)
    with pytest.raises(ValueError, match="supports dims"):
        make_stepper("b200/zmarch", u0, pb.heat_stencil(2, 0.1))


def test_heat_and_jacobi_coefficients():
    st = pb.heat_stencil(3, 0.15)
    assert st.c0 == pytest.approx(0.1) and st.c1 == 0.15
    with pytest.raises(ValueError):
        pb.heat_stencil(3, 0.17)
    assert pb.jacobi_stencil(2).c1 == 0.25 and pb.jacobi_stencil(3).c0 == 0.0


def test_local_contract_mirror_without_pyheat3d():
    """With pyheat3d absent the package still imports and its mirrors behave like pyheat3d."""
    code = (
        "import sys; sys.modules['pyheat3d'] = None\n"
        "import numpy as np, pytest\n"
        "import pyheat3d_b200 as pb\n"
        "assert not pb.HAVE_PYHEAT3D\n"
        "st = pb.heat_stencil(2, 0.2, 'periodic'); assert abs(st.c0 - 0.2) < 1e-15\n"
        "try:\n    pb.heat_stencil(2, 0.3)\nexcept ValueError as e:\n    assert 'stability' in str(e)\n"
        "else:\n    raise SystemExit('no error')\n"
        "try:\n    pb.Stencil(0.1, 0.1, 'neumann')\nexcept ValueError:\n    pass\n"
        "else:\n    raise SystemExit('no error')\n"
        "v = pb.VARIANTS['b200/tb4-bf16']; assert v.key == 'b200/tb4-bf16' and v.bytes_per_value == 2\n"
        "assert pb.register() == []\n"
        "print('ok')\n"
    )
    res = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    assert res.stdout.strip() == "ok"


pyheat3d = pytest.importorskip("pyheat3d", reason="pyheat3d checkout not available")


def test_register_into_pyheat3d_registry():
    import pyheat3d.registry as reg

    pb.register()
    for key in VARIANTS:
        assert key in reg.VARIANTS
        assert reg.VARIANTS[key].key == key
    assert "b200" in reg.BACKENDS and "b200" in reg.COLORS
    assert pb.register() == []  # idempotent
    # the B200 stepper is a pyheat3d Stepper
    from pyheat3d.backends.base import Stepper

    from pyheat3d_b200.stepper import B200Stepper

    assert issubclass(B200Stepper, Stepper)


def test_pyheat3d_cli_lists_b200_variants_unchanged(capsys):
    from pyheat3d.cli import main

    pb.register()
    assert main(["list"]) == 0
    out = capsys.readouterr().out
    assert "b200/zmarch" in out and "b200/tb8-bf16" in out


def test_module_entry_point_runs_pyheat3d_cli():
    import os

    env = dict(os.environ)
    src = str(Path(pyheat3d.__file__).resolve().parents[1])
    env["PYTHONPATH"] = os.pathsep.join([str(ROOT), src])
    res = subprocess.run([sys.executable, "-m", "pyheat3d_b200", "list"], cwd=ROOT, env=env,
                         capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    assert "b200/ymarch-bf16" in res.stdout


def test_sitecustomize_hook_registers_at_startup():
    import os

    env = dict(os.environ)
    src = str(Path(pyheat3d.__file__).resolve().parents[1])
    env["PYTHONPATH"] = os.pathsep.join([str(ROOT / "pyheat3d_b200" / "site"), str(ROOT), src])
    code = "from pyheat3d.registry import VARIANTS; print(sum(k.startswith('b200/') for k in VARIANTS))"
    res = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True,
                         text=True)
    assert res.returncode == 0, res.stderr
    assert int(res.stdout.strip()) == len(VARIANTS)
