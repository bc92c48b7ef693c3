"""Adjoint of the conic QP solution map (sdpx_b200_adjoint) for the loss L = 1/2 |x* - t|^2.

Checks, on conic QPs of the differentiation workload (orthant rows + one PSD block + P):
  * against central finite differences of L along random directions in (q, b, A), solving to
    gap 1e-10 with h = 1e-5: relative error of the directional derivative <= 1e-3 (an SDP's x is
    accurate to roughly the square root of the gap tolerance, so the step stays well above that);
  * against the oracle's dense FP64 solve of the reference's KKT system [P A'; A -Hs]
    (oracle/adjoint.py), Hs the NT scaling at the solution re-centred as the library does
    (eigenbasis of S - Z per PSD block, the smaller partner of each orthant pair at 1e-9 x the
    larger, in the equilibrated coordinates): dq, db, dA within 1e-6 relative;
  * through a torch.autograd.Function wrapper (a thin harness that lives in this test only):
    loss.backward() delivers the library's adjoint unchanged;
  * through BatchSolver.solve_adjoint: bitwise the single-handle gradients.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle import adjoint as oracle_adjoint
from sdpx_b200 import problems as P
from sdpx_b200.solver import DefaultSettings, DefaultSolver

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _settings():
    return DefaultSettings(kkt_form="condensed", tol_gap_abs=TOL, tol_gap_rel=TOL, tol_feas=TOL)


def _solve(prob, q=None, b=None, A=None):
    s = DefaultSolver(prob.P, prob.q if q is None else q, prob.A if A is None else A,
                      prob.b if b is None else b, prob.cones, _settings())
    sol = s.solve()
    assert sol.status in ("Solved", "AlmostSolved"), sol.status
    return s, sol


def _loss(x, t):
    return 0.5 * float(np.sum((x - t) ** 2))


@pytest.mark.parametrize("seed", [0, 1])
def test_directional_derivatives_match_finite_differences(seed):
    prob = P.conic_qp(seed, n=20, n_nn=15, psd=4, rank=5)
    t = prob.meta["t"]
    s, sol = _solve(prob)
    dq, db, dA = s.adjoint(sol.x - t)
    A = sp.csc_matrix(prob.A)
    rng = np.random.default_rng(10 + seed)
    h = 1e-5
    for _ in range(3):
        vq = rng.standard_normal(prob.n)
        vb = rng.standard_normal(prob.m)
        vA = sp.csc_matrix((rng.standard_normal(A.nnz), A.indices, A.indptr), shape=A.shape)
        analytic = dq @ vq + db @ vb + float(dA.multiply(vA).sum())
        _, sp_ = _solve(prob, q=prob.q + h * vq, b=prob.b + h * vb, A=A + h * vA)
        _, sm_ = _solve(prob, q=prob.q - h * vq, b=prob.b - h * vb, A=A - h * vA)
        fd = (_loss(sp_.x, t) - _loss(sm_.x, t)) / (2 * h)
        assert abs(analytic - fd) <= 1e-3 * max(1.0, abs(fd)), (analytic, fd)


@pytest.mark.parametrize("kw", [dict(n=20, n_nn=15, psd=4, rank=5), dict()])
def test_adjoint_matches_dense_fp64_kkt_solve(kw):
    prob = P.conic_qp(2, **kw)
    t = prob.meta["t"]
    s, sol = _solve(prob)
    dq, db, dA = s.adjoint(sol.x - t)
    rq, rb, rA = oracle_adjoint.adjoint(prob, sol.x, sol.s, sol.z, sol.x - t)
    scale = max(np.max(np.abs(rq)), np.max(np.abs(rb)), 1.0)
    assert np.max(np.abs(dq - rq)) <= 1e-6 * scale
    assert np.max(np.abs(db - rb)) <= 1e-6 * scale
    assert np.max(np.abs(dA.toarray() - rA.toarray())) <= 1e-6 * scale * max(1.0, np.max(np.abs(sol.x)),
                                                                   np.max(np.abs(sol.z)))


def test_torch_autograd_wrapper():
    torch = pytest.importorskip("torch")

    prob = P.conic_qp(4, n=20, n_nn=15, psd=4, rank=5)
    pattern = sp.csc_matrix(prob.A)

    class ConicQP(torch.autograd.Function):
        """x*(q, b, A) on the GPU library, with the adjoint as its backward."""

        @staticmethod
        def forward(ctx, q, b, a_vals):
            A = sp.csc_matrix((a_vals.detach().cpu().numpy(), pattern.indices, pattern.indptr),
                              shape=pattern.shape)
            s, sol = _solve(prob, q=q.detach().cpu().numpy(), b=b.detach().cpu().numpy(), A=A)
            ctx.solver = s
            return torch.from_numpy(sol.x.copy())

        @staticmethod
        def backward(ctx, gx):
            dq, db, dA = ctx.solver.adjoint(gx.detach().cpu().numpy())
            return torch.from_numpy(dq), torch.from_numpy(db), torch.from_numpy(dA.data.copy())

    q = torch.tensor(prob.q, requires_grad=True)
    b = torch.tensor(prob.b, requires_grad=True)
    a = torch.tensor(pattern.data.copy(), requires_grad=True)
    t = torch.tensor(prob.meta["t"])
    loss = 0.5 * ((ConicQP.apply(q, b, a) - t) ** 2).sum()
    loss.backward()
    # the autograd path delivers exactly the library adjoint of the same solution
    s, sol = _solve(prob)
    dq, db, dA = s.adjoint(sol.x - prob.meta["t"])
    assert np.allclose(q.grad.numpy(), dq, rtol=1e-12, atol=1e-12)
    assert np.allclose(b.grad.numpy(), db, rtol=1e-12, atol=1e-12)
    assert np.allclose(a.grad.numpy(), dA.data, rtol=1e-12, atol=1e-12)


def test_batch_adjoint_equals_single_handle():
    """BatchSolver.solve_adjoint (re-prepared handles, eager launches, concurrent workers) gives
    bitwise the gradients of a fresh handle per instance."""
    from sdpx_b200.solver import BatchSolver

    probs = [P.conic_qp(20 + i, n=24, n_nn=16, psd=4, rank=6) for i in range(6)]
    bs = BatchSolver(workers=3, settings=_settings())
    sols, grads = bs.solve_adjoint(probs, lambda i, sol: sol.x - probs[i].meta["t"])
    for p, sol, g in zip(probs, sols, grads):
        s, ref = _solve(p)
        assert np.array_equal(sol.x, ref.x)
        dq, db, dA = s.adjoint(ref.x - p.meta["t"])
        assert np.array_equal(g[0], dq) and np.array_equal(g[1], db)
        assert np.array_equal(g[2].data, dA.data)
