"""Test configuration: markers, GPU auto-skip, import paths.

``gpu`` tests need a CUDA device and the built ``libph3b200.so``; without a device they are
skipped (the reference's ``tests/conftest.py:6-12`` does the same).

If ``PYHEAT3D_SRC`` names a pyheat3d source tree (the directory holding the ``pyheat3d``
package), or a pyheat3d checkout sits beside this repository (``<sibling>/src/pyheat3d``), it is
put on ``sys.path`` so the CPU tests can check the registry plug-in against the real pyheat3d.
GPU tests never need it.
"""

from __future__ import annotations

import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

def _pyheat3d_src() -> str | None:
    env = os.environ.get("PYHEAT3D_SRC")
    if env and (Path(env) / "pyheat3d" / "__init__.py").exists():
        return env
    try:
        for sib in sorted(ROOT.parent.iterdir()):
            if sib != ROOT and (sib / "src" / "pyheat3d" / "__init__.py").is_file():
                return str(sib / "src")
    except OSError:
        pass
    return None


_src = _pyheat3d_src()
if _src and _src not in sys.path:
    sys.path.append(_src)


def _cuda_ok() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU and libph3b200.so")
    config.addinivalue_line("markers", "slow: long-running")


def pytest_collection_modifyitems(config, items):
    if _cuda_ok():
        return
    skip = pytest.mark.skip(reason="no CUDA GPU")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)
