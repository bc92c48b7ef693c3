"""Captured KKT solves (CUDA graphs) against eager launches.

With graphs on, every refined KKT solve is one graph whose two refinement loops are WHILE nodes
driven on the device; with SDPX_B200_GRAPHS=0 the host drives the loops and launches eagerly.
Both run the same kernels in the same order on the same stream and apply the same stopping
rules, so the solves must be bitwise identical, take the same refinement steps, and repeated
solves on one handle (graph replays) must stay bitwise identical too.
"""
import os

import numpy as np
import pytest

from sdpx_b200 import problems as P
from sdpx_b200.solver import DefaultSettings, DefaultSolver

pytestmark = pytest.mark.gpu


def _make(prob, graphs):
    old = os.environ.get("SDPX_B200_GRAPHS")
    os.environ["SDPX_B200_GRAPHS"] = "1" if graphs else "0"
    try:
        return DefaultSolver(prob.P, prob.q, prob.A, prob.b, prob.cones,
                             DefaultSettings(kkt_form="condensed"))
    finally:
        if old is None:
            del os.environ["SDPX_B200_GRAPHS"]
        else:
            os.environ["SDPX_B200_GRAPHS"] = old


@pytest.mark.parametrize("maker", [lambda: P.rank1_sdp(8, 200, seed=4, nmin=6, nmax=24),
                                   lambda: P.dense_sdp(20, 60, seed=5),
                                   lambda: P.conic_qp(6, n=40, n_nn=30, psd=6, rank=8)])
def test_graphs_bitwise_equal_eager(maker):
    prob = maker()
    eager = _make(prob, False)
    a = eager.solve()
    assert eager.kkt_paths()["device"] == 0
    g = _make(prob, True)
    b = g.solve()
    paths = g.kkt_paths()
    assert paths["host"] == 0 and paths["device"] == g.info.counts["kkt_solves"] > 0
    assert g.info.counts == eager.info.counts  # same refinement steps at both levels
    c = g.solve()  # second solve replays the cached graphs
    for s in (b, c):
        assert s.status == a.status and s.iterations == a.iterations
        assert np.array_equal(s.x, a.x) and np.array_equal(s.z, a.z) and np.array_equal(s.s, a.s)


def test_graphs_survive_update():
    prob = P.rank1_sdp(6, 120, seed=8, nmin=6, nmax=20)
    g = _make(prob, True)
    g.solve()
    g.update(prob.q * 1.5, prob.b)
    s1 = g.solve()
    eager = _make(prob, False)
    eager.update(prob.q * 1.5, prob.b)
    s2 = eager.solve()
    assert s1.iterations == s2.iterations and np.array_equal(s1.x, s2.x)
