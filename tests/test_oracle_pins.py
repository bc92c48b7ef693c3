"""Pin the CPU oracle to the reference's own known answers (no GPU needed).

Known answers restated from the reference's tests:
  * crates/solver/tests/it/basic_sdp.rs:28-56: projection SDP, refsol / refobj 4.840076866013861,
    checked at 1e-6 with kkt_form condensed (basic_sdp.rs:97-113);
  * crates/solver/tests/it/sampled_solver.rs:8-105: x = 16/9 each, 2x after doubling b,
    bound 128 * tol with tol = 1e-9 in binary64;
  * crates/solver/src/solver/sampled/tests.rs:407-446: analytic Schur entries 16, 36, 0.
"""
import numpy as np
import pytest

from oracle import ipm
from sdpx_b200 import problems as P

REFSOL = np.array([-3.0729833267361095, 0.3696004167288786, -0.022226685581313674,
                   0.31441213129613066, -0.026739700851545107, -0.016084530571308823])
REFOBJ = 4.840076866013861


def test_basic_sdp_known_answer():
    r = ipm.solve(P.basic_projection_sdp())
    assert r.status == ipm.SOLVED
    assert np.linalg.norm(r.x - REFSOL) <= 1e-6
    assert abs(r.objective - REFOBJ) <= 1e-6


@pytest.mark.parametrize("scale", [1.0, 2.0])
def test_sampled_two_by_two_known_answer(scale):
    tol = 1e-9
    r = ipm.solve(P.sampled_two_by_two(scale), tol_feas=tol, tol_gap_abs=tol, tol_gap_rel=tol)
    assert r.status == ipm.SOLVED
    bound = 128 * tol * (4 if scale != 1.0 else 1)
    assert np.all(np.abs(r.x - scale * 16 / 9) <= bound)
    # residual b - A x - s = 0 in original coordinates
    prob = P.sampled_two_by_two(scale)
    assert np.max(np.abs(prob.b - prob.A @ r.x - r.s)) <= 128 * tol


def test_analytic_schur_entries():
    """Schur entry w_p w_q (v_p' G v_q)^2 of rank-one columns (sampled/tests.rs:407-446)."""
    # identity scaling, v_p = (1, 1), v_q = (1, 1): <A_p, A_q> = (v_p'v_q)^2 = 4^2 / ... cases
    cone = ipm.PsdCone(2)
    cases = [((1.0, 1.0), (1.0, 1.0), 4.0 ** 2 / 1.0),  # (|v|^2)^2 with |v|^2 = 2 -> 4; w = 2
             ]
    v = np.array([1.0, 1.0])
    col = P.svec(2.0 * np.outer(v, v))  # w = 2: entry w^2 (v'v)^2 = 4 * 4 = 16
    H = cone.schur_block(col[:, None])
    assert abs(H[0, 0] - 16.0) <= 1e-12
    v3 = np.array([1.0, 1.0]) * np.sqrt(1.5)
    col3 = P.svec(2.0 * np.outer(v3, v3))  # w^2 (v'v)^2 = 4 * 9 = 36
    assert abs(cone.schur_block(col3[:, None])[0, 0] - 36.0) <= 1e-12
    u = np.array([1.0, -1.0])
    colu = P.svec(np.outer(u, u))
    Hpq = cone.schur_block(np.stack([col, colu], axis=1))
    assert abs(Hpq[0, 1]) <= 1e-12  # orthogonal bases: exactly 0
    del cases


def test_dense_sdp_small_solves():
    r = ipm.solve(P.dense_sdp(n=12, m=30, seed=3))
    assert r.status == ipm.SOLVED
    assert r.gap_rel < 1e-8 and r.res_primal < 1e-8 and r.res_dual < 1e-8


def test_rank1_operator_matches_csc():
    """The Gram (rank-one) description and the CSC operator are the same linear map."""
    prob = P.rank1_sdp(blocks=4, m=40, seed=1, nmin=4, nmax=9)
    r1 = prob.rank1
    offs = np.concatenate([[0], np.cumsum([P.tri(d) for _, d in prob.cones])])
    x = np.random.default_rng(0).standard_normal(prob.n)
    Ax = np.zeros(prob.m)
    for (ci, j, col), w in zip(r1.terms, r1.weights):
        v = r1.bases[j][:, col]
        Ax[offs[j]:offs[j + 1]] += x[ci] * P.svec(w * np.outer(v, v))
    assert np.allclose(Ax, prob.A @ x, rtol=1e-13, atol=1e-13)


def test_generator_feasibility():
    """X0 = I is primal feasible and C - sum y0 A_i = I (strict dual feasibility)."""
    prob = P.dense_sdp(n=6, m=10, seed=5)
    y0 = prob.meta["y0"]
    slack = prob.b - prob.A @ y0
    assert np.allclose(slack, P.svec(np.eye(6)))
    assert np.allclose(prob.A.T @ P.svec(np.eye(6)), -prob.q)
