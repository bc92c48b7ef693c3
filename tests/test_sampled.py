"""Factor-authoritative sampled input (sdpx_prepare_sampled) on the GPU Gram form.

* The reference's analytic Schur pins, exactly (crates/solver/src/solver/sampled/tests.rs:407-446):
  basis columns (1, 1) and (1, -1), weights 2 and -3, identity scaling: entries exactly 16, 36
  and 0; with R^-1 = diag(1, 1 + delta), delta = 2^-13 (binary64: precision 53 / 4), the
  cancellation-sensitive cell -6 (2 delta + delta^2)^2 within 4096 eps and negative.
* The reference's sampled solver test (crates/solver/tests/it/sampled_solver.rs:8-105): basis
  (1, 1/4), (1/4, 1), weights -1, q = (1, 1), b = (-1, 0, -1), tolerance 1e-9: Solved with both
  x = 16/9 within 128 tol; the same objective as the materialised (generic) problem; the factors
  reproduce b - A x = s; after b -> 2b, x = 32/9 within 4 * 128 tol.
* Matrix-valued blocks (dim > 1) are refused with return code 2 before any device work (CPU).
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


def test_sampled_matrix_valued_block_unsupported():
    q, b, block = _reference_sampled()
    block = dict(block, dim=2, basis=np.ones((1, 1)), weights=np.ones(3))
    with pytest.raises(_lib.SdpxError) as e:
        DefaultSolver.new_sampled(None, np.ones(3), sp.csc_matrix((3, 3)), b, [("psd", 2)], [block])
    assert e.value.code == 2
