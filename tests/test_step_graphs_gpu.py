"""Repeated small-grid advances replayed as CUDA graphs give the plain launches' results.

A stepper of a grid below ``B200Stepper.GRAPH_CELLS`` sites runs the first ``step(n)`` from a
buffer plainly, captures the second one into a CUDA graph and replays it afterwards. Every
intermediate state must equal, bit for bit, a stepper with graphs switched off and the oracle.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import emulated_reference
from pyheat3d_b200 import heat_stencil, jacobi_stencil
from pyheat3d_b200.registry import VARIANTS, make_stepper

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("key,shape,bc,calls", [
    ("b200/zmarch", (40, 48, 64), "periodic", (10, 10, 10, 11, 11, 11, 10)),
    ("b200/zmarch", (21, 33, 45), "dirichlet", (9, 9, 9, 12, 12, 12)),
    ("b200/tb4-bf16", (130, 257), "dirichlet", (9, 9, 9, 9, 8, 8, 8)),
    ("b200/ymarch-fp16", (64, 96), "periodic", (16, 16, 16, 17, 17)),
    ("b200/auto", (128, 128, 128), "dirichlet", (100, 100, 100)),
])
def test_graph_replay_matches_plain_and_oracle(key, shape, bc, calls):
    rng = np.random.default_rng(3)
    u0 = rng.random(shape, dtype=np.float32)
    dims = len(shape)
    st = heat_stencil(dims, 0.9 / (2 * dims), bc)
    g = make_stepper(key, u0, st)
    p = make_stepper(key, u0, st)
    p._use_graphs = False
    var = VARIANTS[key]
    done = 0
    for n in calls:
        g.step(n)
        p.step(n)
        done += n
        got, want = g.get(), p.get()
        assert np.array_equal(got, want), (key, n, done)
    assert g._graphs, "no advance was replayed as a graph"
    k = getattr(g, "steps_per_pass", var.steps_per_pass)
    ref = u0
    # the same advances on the oracle, call by call (each call rounds per pass of its own)
    for n in calls:
        ref = emulated_reference(ref, st.c0, st.c1, bc, n, g.storage, k)
    assert np.array_equal(g.get(), ref)
    g.close()
    p.close()


def test_graph_replay_with_source():
    rng = np.random.default_rng(4)
    u0 = rng.random((24, 40, 56), dtype=np.float32)
    b = (rng.random(u0.shape, dtype=np.float32) - np.float32(0.5)) * np.float32(1e-2)
    st = jacobi_stencil(3, "periodic")
    g = make_stepper("b200/zmarch", u0, st, source=b)
    p = make_stepper("b200/zmarch", u0, st, source=b)
    p._use_graphs = False
    for n in (12, 12, 12, 12):
        g.step(n)
        p.step(n)
        assert np.array_equal(g.get(), p.get())
    assert g._graphs
