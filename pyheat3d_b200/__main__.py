"""``python -m pyheat3d_b200 <pyheat3d CLI arguments>``: pyheat3d's own CLI with b200 registered.

Equivalent to running ``pyheat3d ...`` with the ``sitecustomize`` hook of
``pyheat3d_b200/site`` on ``PYTHONPATH``.
"""

from __future__ import annotations

import sys


def main(argv: list[str] | None = None) -> int:
    from .registry import register

    try:
        from pyheat3d.cli import main as cli_main  # type: ignore
    except ImportError:
        print("pyheat3d is not installed; nothing to drive", file=sys.stderr)
        return 2
    register()
    return cli_main(argv)


if __name__ == "__main__":
    sys.exit(main())
