"""Batches of independent small SDPs (the batching workload: one PSD block, n in [8, 64],
m in [20, 300], data as the dense generator, instance b from seed + b).

BatchSolver runs instances concurrently, one handle and stream per worker thread, re-preparing
each handle in place (sdpx_b200_reprepare).  Bars: every instance bitwise equal to a fresh
handle's solve of the same instance (re-preparation leaves no state behind), and equal to the
oracle in status, iterations within 1 and objective within 1e-8 relative.
"""
import numpy as np
import pytest

from oracle import ipm
from sdpx_b200 import problems as P
from sdpx_b200.solver import BatchSolver, DefaultSettings, solve_problem

pytestmark = pytest.mark.gpu


def test_batch_matches_fresh_handles_and_oracle():
    probs = P.batch_sdps(12, seed=40, nrange=(8, 24), mrange=(20, 90))
    st = DefaultSettings(kkt_form="condensed")
    batch = BatchSolver(workers=4, settings=st).solve(probs)
    for p, b in zip(probs, batch):
        f = solve_problem(p, st).solution
        assert b.status == f.status and b.iterations == f.iterations
        assert np.array_equal(b.x, f.x) and np.array_equal(b.z, f.z)
        n, m = p.cones[0][1], p.n
        if m > n * (n + 1) // 2:  # dependent constraints: statuses may legitimately differ
            continue
        o = ipm.solve(p)
        assert b.status_code == o.status, (p.name, b.status, o.status)
        assert abs(b.iterations - o.iterations) <= 1
        assert abs(b.obj_val - o.objective) <= 1e-8 * max(1.0, abs(o.objective))


def test_batch_reprepare_grows_and_shrinks():
    """One worker handle takes instances of growing then shrinking size in turn."""
    sizes = [(8, 20), (40, 200), (12, 30), (64, 300), (9, 25)]
    probs = [P.dense_sdp(n, m, seed=3 + k) for k, (n, m) in enumerate(sizes)]
    st = DefaultSettings(kkt_form="condensed")
    batch = BatchSolver(workers=1, settings=st).solve(probs)
    for p, b in zip(probs, batch):
        f = solve_problem(p, st).solution
        assert b.iterations == f.iterations and np.array_equal(b.x, f.x)
        o = ipm.solve(p)  # every size here has m <= tri(n): independent constraints
        assert b.status_code == o.status
        assert abs(b.iterations - o.iterations) <= 1
        assert abs(b.obj_val - o.objective) <= 1e-8 * max(1.0, abs(o.objective))
