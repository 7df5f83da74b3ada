"""CPU oracle for the pyheat3d stencil path (TEST INFRASTRUCTURE ONLY).

This package restates, in NumPy, the reference algorithm that every GPU kernel of
``pyheat3d_b200`` must reproduce. Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import it, and only as the
checker or as the timed CPU baseline. The product path (``pyheat3d_b200``) never imports it and
has no CPU fallback.

Parity is pinned: ``tests/test_oracle.py`` checks this restatement bit for bit against golden
vectors generated by the reference's own ``reference_step`` / ``emulated_reference``
(``tests/golden/make_golden.py``).
"""

from .stencil import (  # noqa: F401
    TOLERANCE,
    emulated_reference,
    from_bf16_bits,
    reference_step,
    round_storage,
    run_reference,
    threaded_emulated,
    threaded_step,
    to_bf16_bits,
)
