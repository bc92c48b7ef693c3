"""Factor-authoritative sampled input (sdpx_prepare_sampled) on the GPU Gram form.

* The reference's analytic Schur pins, exactly (crates/solver/src/solver/sampled/tests.rs:407-446):
  basis columns (1, 1) and (1, -1), weights 2 and -3, identity scaling: entries exactly 16, 36
  and 0; with R^-1 = diag(1, 1 + delta), delta = 2^-13 (binary64: precision 53 / 4), the
  cancellation-sensitive cell -6 (2 delta + delta^2)^2 within 4096 eps and negative.
* The reference's sampled solver test (crates/solver/tests/it/sampled_solver.rs:8-105): basis
  (1, 1/4), (1/4, 1), weights -1, q = (1, 1), b = (-1, 0, -1), tolerance 1e-9: Solved with both
  x = 16/9 within 128 tol; the same objective as the materialised (generic) problem; the factors
  reproduce b - A x = s; after b -> 2b, x = 32/9 within 4 * 128 tol.
* Matrix-valued blocks (dim > 1, columns w sym(e_r e_s') (x) q q'): whole solves agree with the
  materialised problem and the oracle; the Schur complement at an NT scaling agrees with the
  oracle's ordinary PSD Schur of the materialised columns (1e-11).
* Invalid blocks are refused with return code 1 before any device work (CPU).
"""
import numpy as np
import pytest
import scipy.sparse as sp

from sdpx_b200 import _lib
from sdpx_b200 import problems as P
from sdpx_b200.solver import DefaultSettings, DefaultSolver, KernelContext

EPS = float(np.finfo(np.float64).eps)


def _analytic_ctx():
    ctx = KernelContext()
    block = {"row_start": 0, "column_start": 0, "dim": 1,
             "basis": np.array([[1.0, 1.0], [1.0, -1.0]]), "weights": np.array([2.0, -3.0])}
    ctx.upload_sampled(sp.csc_matrix((3, 2)), [2], [block])
    return ctx


@pytest.mark.gpu
def test_analytic_schur_identity_scaling_exact():
    ctx = _analytic_ctx()
    ctx.set_scaling([np.eye(2)], [np.eye(2)])
    H = ctx.schur()
    assert H[0, 0] == 16.0
    assert H[1, 1] == 36.0
    assert H[0, 1] == 0.0 and H[1, 0] == 0.0


@pytest.mark.gpu
def test_analytic_schur_cancellation_cell():
    ctx = _analytic_ctx()
    delta = 2.0 ** -(53 // 4)
    rinv = np.diag([1.0, 1.0 + delta])
    ctx.set_scaling([np.diag([1.0, 1.0 / (1.0 + delta)])], [rinv])
    H = ctx.schur()
    cross = -(2.0 * delta + delta * delta)
    expected = -6.0 * cross * cross
    assert abs(H[0, 1] - expected) <= 4096 * EPS * abs(expected)
    assert H[0, 1] < 0.0


def _reference_sampled(scale=1.0):
    q = np.ones(2)
    b = np.array([-1.0, 0.0, -1.0]) * scale
    block = {"row_start": 0, "column_start": 0, "dim": 1,
             "basis": np.array([[1.0, 0.25], [0.25, 1.0]]), "weights": np.array([-1.0, -1.0])}
    return q, b, block


@pytest.mark.gpu
def test_sampled_solver_known_answer():
    tol = 1e-9
    st = DefaultSettings(tol_feas=tol, tol_gap_abs=tol, tol_gap_rel=tol, kkt_form="condensed")
    q, b, block = _reference_sampled()
    s = DefaultSolver.new_sampled(None, q, sp.csc_matrix((3, 2)), b, [("psd", 2)], [block], st)
    sol = s.solve()
    bound = 128 * tol
    assert sol.status == "Solved"
    assert np.all(np.abs(sol.x - 16.0 / 9.0) <= bound)
    generic = DefaultSolver(None, q, P.sampled_two_by_two().A, b, [("psd", 2)], st).solve()
    assert generic.status == "Solved"
    assert abs(sol.obj_val - generic.obj_val) <= bound
    # the original factors reproduce b - A x = s
    Q, w = block["basis"], block["weights"]
    Ax = sum(w[k] * sol.x[k] * P.svec(np.outer(Q[:, k], Q[:, k])) for k in range(2))
    assert np.max(np.abs(b - Ax - sol.s)) <= bound
    s.update(q, 2.0 * b)
    sol2 = s.solve()
    assert sol2.status == "Solved"
    assert np.all(np.abs(sol2.x - 32.0 / 9.0) <= 4 * bound)


def test_sampled_block_validation():
    """Invalid sampled blocks are refused before any device work (return code 1): wrong weight
    count for the dim, a block not aligned with its cone."""
    q, b, block = _reference_sampled()
    bad = dict(block, dim=2, basis=np.ones((1, 1)), weights=np.ones(2))  # tri(2) * 1 = 3 weights
    with pytest.raises(_lib.SdpxError) as e:
        DefaultSolver.new_sampled(None, np.ones(3), sp.csc_matrix((3, 3)), b, [("psd", 2)], [bad])
    assert e.value.code == 1
    bad = dict(block, row_start=1)
    with pytest.raises(_lib.SdpxError) as e:
        DefaultSolver.new_sampled(None, q, sp.csc_matrix((3, 2)), b, [("psd", 2)], [bad])
    assert e.value.code == 1


def _matrix_sampled(D=2, h=3, c=4, seed=0):
    """A matrix-valued sampled block (dim D, basis h x c) and its materialised columns:
    primitive (s, r, k) is w svec(sym(e_r e_s') (x) q_k q_k') (sampled/mod.rs:9-29)."""
    rng = np.random.default_rng(seed)
    Q = rng.standard_normal((h, c))
    w = rng.uniform(0.5, 2.0, size=D * (D + 1) // 2 * c)
    n = D * h
    cols, t = [], 0
    for s in range(D):
        for r in range(s + 1):
            for k in range(c):
                E = np.zeros((D, D))
                E[r, s] += 0.5
                E[s, r] += 0.5
                cols.append(P.svec(w[t] * np.kron(E, np.outer(Q[:, k], Q[:, k]))))
                t += 1
    A = np.stack(cols, axis=1)
    # strictly feasible: s = b - A x = I at x = 0; bounded: q = -A' z0 with z0 = svec(I + 0.1 G G')
    G = rng.standard_normal((n, n))
    z0 = P.svec(np.eye(n) + 0.1 * G @ G.T / n)
    q = -A.T @ z0
    b = P.svec(np.eye(n))
    block = {"row_start": 0, "column_start": 0, "dim": D, "basis": Q, "weights": w}
    return A, q, b, n, block


@pytest.mark.gpu
def test_matrix_valued_sampled_solve_matches_materialised_and_oracle():
    from oracle import ipm
    A, q, b, n, block = _matrix_sampled()
    cones = [("psd", n)]
    st = DefaultSettings(kkt_form="condensed")
    g = DefaultSolver.new_sampled(None, q, sp.csc_matrix((A.shape[0], A.shape[1])), b, cones, [block], st).solve()
    gen = DefaultSolver(None, q, sp.csc_matrix(A), b, cones, st).solve()
    prob = P.ConicProblem(P=None, q=q, A=sp.csc_matrix(A), b=b, cones=cones)
    o = ipm.solve(prob)
    assert g.status == gen.status == "Solved" and o.status == ipm.SOLVED
    assert abs(g.iterations - o.iterations) <= 1
    assert abs(g.obj_val - o.objective) <= 1e-8 * max(1.0, abs(o.objective))
    assert abs(g.obj_val - gen.obj_val) <= 1e-8 * max(1.0, abs(gen.obj_val))


@pytest.mark.gpu
def test_matrix_valued_sampled_schur_matches_oracle():
    from oracle import ipm
    A, q, b, n, block = _matrix_sampled(D=3, h=2, c=5, seed=4)
    ctx = KernelContext()
    ctx.upload_sampled(sp.csc_matrix((A.shape[0], A.shape[1])), [n], [block])
    rng = np.random.default_rng(2)
    S = rng.standard_normal((n, n))
    Z = rng.standard_normal((n, n))
    s, z = P.svec(S @ S.T / n + 0.2 * np.eye(n)), P.svec(Z @ Z.T / n + 0.2 * np.eye(n))
    assert ctx.nt_scale(s, z)[1] == 0
    H = ctx.schur()
    cone = ipm.PsdCone(n)
    assert cone.update_scaling(s, z)
    Ho = cone.schur_block(A)
    assert np.max(np.abs(H - Ho)) <= 1e-11 * np.max(np.abs(Ho))
