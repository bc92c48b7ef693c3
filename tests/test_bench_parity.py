"""GPU parity on the benchmarked workloads, at their full sizes.

The bench times the bootstrap-shaped Float64 SDPs (32 blocks, m = 2000; 64 blocks, m = 4000).
These tests solve the same seeded instances through the C ABI and compare with the oracle's
solve of them, committed as fixtures (tests/golden/make_solve_fixtures.py writes them; the
oracle needs minutes of CPU per instance, so the GPU run reads the files instead):

  * status equal, iteration count within 1, primal and dual objective within 1e-8 relative
    (the reference's Float64 bar), x within 1e-6 relative;
  * the factorisation and refined solve at m = 2000 (32 x 32 tiles of 64, the bench's own
    schedule) against numpy's LU solve of the same Schur complement, 1e-9 relative;
  * the Schur complement of the 32 blocks at a random interior point against the oracle's
    ordinary per-block Schur (kkt/condensed/psd.rs restated), 1e-11 relative.
"""
from pathlib import Path

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import ipm
from sdpx_b200 import problems as P
from sdpx_b200.solver import DefaultSettings, KernelContext, solve_problem

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
WORKLOADS = {"rank1_b32_m2000_s0": (32, 2000, 0), "rank1_b64_m4000_s0": (64, 4000, 0)}


def _rel(a, b):
    return abs(a - b) / max(1.0, abs(b))


@pytest.mark.parametrize("name", sorted(WORKLOADS))
def test_bench_workload_matches_oracle_fixture(name):
    fx = np.load(GOLDEN / f"solve_{name}.npz")
    blocks, m, seed = WORKLOADS[name]
    prob = P.rank1_sdp(blocks, m, seed=seed)
    g = solve_problem(prob, DefaultSettings(kkt_form="condensed")).solution
    assert g.status_code == int(fx["status"]), (g.status, int(fx["status"]))
    assert abs(g.iterations - int(fx["iterations"])) <= 1, (g.iterations, int(fx["iterations"]))
    assert _rel(g.obj_val, float(fx["objective"])) <= 1e-8
    assert _rel(g.obj_val_dual, float(fx["dual_objective"])) <= 1e-8
    xo = fx["x"]
    assert np.max(np.abs(g.x - xo)) <= 1e-6 * max(1.0, float(np.max(np.abs(xo))))


def _interior_point(prob, seed):
    rng = np.random.default_rng(seed)
    s, z = [], []
    for _, d in prob.cones:
        for out in (s, z):
            B = rng.standard_normal((d, d))
            out.append(P.svec(B @ B.T / d + 0.1 * np.eye(d)))
    return np.concatenate(s), np.concatenate(z)


@pytest.fixture(scope="module")
def bench_ctx():
    prob = P.rank1_sdp(32, 2000, seed=0)
    ctx = KernelContext()
    ctx.upload(prob.A, [d for _, d in prob.cones])
    s, z = _interior_point(prob, 11)
    lam, st = ctx.nt_scale(s, z)
    assert st == 0
    return prob, ctx, s, z


def test_schur_m2000_matches_oracle(bench_ctx):
    prob, ctx, s, z = bench_ctx
    H = ctx.schur()
    A = sp.csc_matrix(prob.A)
    Ho = np.zeros((prob.n, prob.n))
    r = 0
    for _, d in prob.cones:
        c = ipm.PsdCone(d)
        sl = slice(r, r + c.numel)
        assert c.update_scaling(s[sl], z[sl])
        sub = A[sl, :]
        cols = np.flatnonzero(sub.getnnz(axis=0))
        Ho[np.ix_(cols, cols)] += c.schur_block(sub[:, cols].toarray())
        r += c.numel
    assert np.max(np.abs(H - Ho)) <= 1e-11 * np.max(np.abs(Ho))


@pytest.mark.parametrize("shift", [1e-8, 1e-3])
def test_factor_and_refined_solve_m2000(bench_ctx, shift):
    prob, ctx, s, z = bench_ctx
    H = ctx.schur()
    assert ctx.factor(shift) == 0
    b = np.random.default_rng(12).standard_normal((prob.n, 2))
    x = ctx.solve_many(b)
    xo = np.linalg.solve(H, b)  # refined against the unshifted Schur complement
    assert np.max(np.abs(x - xo)) <= 1e-9 * np.max(np.abs(xo))
