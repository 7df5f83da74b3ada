"""Interpreter-start hook: registers the b200 variants in pyheat3d's registry.

Put this directory on ``PYTHONPATH`` (``PYTHONPATH=<repo>/pyheat3d_b200/site:<repo>``) and every
``pyheat3d`` command, ``bench/run.py`` and the reference test-suite see ``b200/*`` variants
without any change to pyheat3d. Registration is skipped silently if pyheat3d is not installed.
"""

try:
    from pyheat3d_b200.registry import register as _register

    _register()
except Exception:  # pragma: no cover - never break interpreter start-up
    pass
