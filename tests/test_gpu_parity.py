"""GPU parity: libsdpx_b200 (CUDA, through its C ABI) against the CPU oracle.

Bars (stated per test):
  * whole solves: same termination status, iteration count within 1, objective within 1e-8
    relative of the oracle; the reference's own known answers at the reference's tolerances;
  * kernel-level operations: float64 agreement within the stated relative tolerances (the
    GPU and the oracle round differently; no bitwise claim for float64 kernels).
"""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle import ipm
from sdpx_b200 import problems as P
from sdpx_b200.solver import DefaultSettings, DefaultSolver, KernelContext, solve_problem

pytestmark = pytest.mark.gpu

REFSOL = np.array([-3.0729833267361095, 0.3696004167288786, -0.022226685581313674,
                   0.31441213129613066, -0.026739700851545107, -0.016084530571308823])
REFOBJ = 4.840076866013861
OBJ_RTOL = 1e-8


def _rel(a, b):
    return abs(a - b) / max(1.0, abs(b))


# ------------------------------------------------------------------ known answers
def test_basic_sdp_known_answer():
    s = solve_problem(P.basic_projection_sdp(), DefaultSettings(kkt_form="condensed"))
    assert s.solution.status == "Solved"
    assert np.linalg.norm(s.solution.x - REFSOL) <= 1e-6
    assert abs(s.solution.obj_val - REFOBJ) <= 1e-6


@pytest.mark.parametrize("scale", [1.0, 2.0])
def test_sampled_two_by_two_known_answer(scale):
    tol = 1e-9
    st = DefaultSettings(tol_feas=tol, tol_gap_abs=tol, tol_gap_rel=tol, kkt_form="condensed")
    s = solve_problem(P.sampled_two_by_two(scale), st)
    assert s.solution.status == "Solved"
    bound = 128 * tol * (4 if scale != 1.0 else 1)
    assert np.all(np.abs(s.solution.x - scale * 16 / 9) <= bound)


# ------------------------------------------------------------------ whole-solve parity
def _parity(prob, **overrides):
    o = ipm.solve(prob, **overrides)
    st = DefaultSettings(kkt_form="condensed", **overrides)
    g = solve_problem(prob, st)
    assert g.solution.status_code == o.status, (g.solution.status, o.status)
    assert abs(g.solution.iterations - o.iterations) <= 1, (g.solution.iterations, o.iterations)
    assert _rel(g.solution.obj_val, o.objective) <= OBJ_RTOL
    assert _rel(g.solution.obj_val_dual, o.dual_objective) <= OBJ_RTOL
    return g, o


@pytest.mark.parametrize("n,m,seed", [(8, 20, 0), (20, 60, 1), (33, 100, 2), (50, 200, 0)])
def test_dense_sdp_parity(n, m, seed):
    g, o = _parity(P.dense_sdp(n, m, seed))
    # primal solution of the dual-form SDP (y) agrees with the oracle
    assert np.max(np.abs(g.solution.x - o.x)) <= 1e-6 * max(1.0, np.max(np.abs(o.x)))


@pytest.mark.parametrize("blocks,m,seed", [(4, 60, 0), (8, 200, 1)])
def test_rank1_sdp_parity(blocks, m, seed):
    _parity(P.rank1_sdp(blocks, m, seed, nmin=6, nmax=24))


def test_schur_tiles_cross_64_boundary():
    """m = 130 > 2 tiles of 64 exercises the panel/trailing kernels and a ragged last tile."""
    _parity(P.dense_sdp(12, 130, seed=7))


def test_repeat_solves_are_bitwise_identical():
    prob = P.dense_sdp(16, 40, seed=4)
    a = solve_problem(prob).solution
    b = solve_problem(prob).solution
    assert a.iterations == b.iterations
    assert np.array_equal(a.x, b.x) and np.array_equal(a.z, b.z)


def test_update_q_b_resolves():
    prob = P.sampled_two_by_two(1.0)
    s = DefaultSolver(prob.P, prob.q, prob.A, prob.b, prob.cones,
                      DefaultSettings(tol_feas=1e-9, tol_gap_abs=1e-9, tol_gap_rel=1e-9))
    s.solve()
    s.update(prob.q, 2.0 * prob.b)
    sol = s.solve()
    assert sol.status == "Solved"
    assert np.all(np.abs(sol.x - 32 / 9) <= 4 * 128 * 1e-9)
    dec = s.result_decimal()
    assert len(dec) == prob.n + 2 * prob.m + 6
    assert abs(float(dec[0]) - sol.x[0]) <= 1e-15 * abs(sol.x[0])


# ------------------------------------------------------------------ kernel-level parity
def _interior_point(prob, seed):
    """A strictly interior (s, z) pair on the cone rows of prob."""
    rng = np.random.default_rng(seed)
    s, z = [], []
    for _, d in prob.cones:
        for out in (s, z):
            B = rng.standard_normal((d, d))
            out.append(P.svec(B @ B.T / d + 0.1 * np.eye(d)))
    return np.concatenate(s), np.concatenate(z)


@pytest.fixture(scope="module")
def kctx_prob():
    prob = P.rank1_sdp(6, 90, seed=3, nmin=5, nmax=40)
    ctx = KernelContext()
    ctx.upload(prob.A, [d for _, d in prob.cones])
    cones = [ipm.PsdCone(d) for _, d in prob.cones]
    rng = []
    r = 0
    for c in cones:
        rng.append(slice(r, r + c.numel))
        r += c.numel
    return prob, ctx, cones, rng


def test_nt_scale_matches_oracle(kctx_prob):
    prob, ctx, cones, rng = kctx_prob
    s, z = _interior_point(prob, 1)
    lam, status = ctx.nt_scale(s, z)
    assert status == 0
    for c, r in zip(cones, rng):
        assert c.update_scaling(s[r], z[r])
    lam_o = np.concatenate([c.lam for c in cones])
    assert np.allclose(lam, lam_o, rtol=1e-12, atol=0)


def test_cone_operators_match_oracle(kctx_prob):
    prob, ctx, cones, rng = kctx_prob
    s, z = _interior_point(prob, 2)
    ctx.nt_scale(s, z)
    for c, r in zip(cones, rng):
        assert c.update_scaling(s[r], z[r])
    x = np.random.default_rng(5).standard_normal(prob.m)
    # R is unique up to the signs of its columns (singular-vector signs), so W itself is
    # compared through invariants: Hs = W'W and Hs^-1 entrywise, W^-1 W = W' W^-T = I, and
    # the Frobenius norm of W x per block.
    ops = {4: lambda c, v: c.mul_Hs(v), 5: lambda c, v: c.mul_Hinv(v)}
    for op, f in ops.items():
        y = ctx.cone_apply(op, x)
        yo = np.concatenate([f(c, x[r]) for c, r in zip(cones, rng)])
        assert np.max(np.abs(y - yo)) <= 1e-11 * max(1.0, np.max(np.abs(yo))), op
    assert np.max(np.abs(ctx.cone_apply(2, ctx.cone_apply(0, x)) - x)) <= 1e-10
    assert np.max(np.abs(ctx.cone_apply(1, ctx.cone_apply(3, x)) - x)) <= 1e-10
    wx = ctx.cone_apply(0, x)
    for c, r in zip(cones, rng):
        assert abs(np.linalg.norm(wx[r]) - np.linalg.norm(c.mul_W(x[r]))) <= 1e-11 * np.linalg.norm(wx[r])
    # W^-T s = lambda on the diagonal (NT scaling point)
    y = ctx.cone_apply(3, s)
    for c, r in zip(cones, rng):
        M = ipm.svec_to_mat(y[r], c.n)
        assert np.allclose(M, np.diag(c.lam), atol=1e-10 * c.lam.max())


def test_schur_matches_oracle(kctx_prob):
    prob, ctx, cones, rng = kctx_prob
    s, z = _interior_point(prob, 3)
    ctx.nt_scale(s, z)
    for c, r in zip(cones, rng):
        c.update_scaling(s[r], z[r])
    H = ctx.schur()
    A = sp.csc_matrix(prob.A)
    Ho = np.zeros((prob.n, prob.n))
    for c, r in zip(cones, rng):
        sub = A[r, :]
        cols = np.flatnonzero(sub.getnnz(axis=0))
        Ho[np.ix_(cols, cols)] += c.schur_block(sub[:, cols].toarray())
    assert np.allclose(H, H.T, rtol=0, atol=0)
    assert np.max(np.abs(H - Ho)) <= 1e-11 * np.max(np.abs(Ho))


@pytest.mark.parametrize("shift", [1e-8, 1e-3])
def test_factor_and_refined_solve(kctx_prob, shift):
    prob, ctx, cones, rng = kctx_prob
    s, z = _interior_point(prob, 4)
    ctx.nt_scale(s, z)
    H = ctx.schur()
    assert ctx.factor(shift) == 0
    b = np.random.default_rng(9).standard_normal((prob.n, 2))
    x = ctx.solve_many(b)
    xo = np.linalg.solve(H, b)  # refined against the unshifted Schur complement
    assert np.max(np.abs(x - xo)) <= 1e-9 * np.max(np.abs(xo))


def test_dynamic_pivot_rule_replaces_tiny_pivot():
    """A singular PSD Schur (repeated constraint) factors with the dynamic rule
    (kkt/ldl/dense_block.rs:334-365) and fails without it."""
    prob = P.dense_sdp(6, 10, seed=2)
    A = sp.hstack([prob.A, prob.A[:, :1]]).tocsc()  # duplicate column: singular Schur
    ctx = KernelContext()
    ctx.upload(A, [6])
    ctx.identity_scaling()
    H = ctx.schur()
    assert np.linalg.matrix_rank(H) < H.shape[0]
    assert ctx.factor(0.0, dynamic=True) == 0
    assert ctx.factor(0.0, dynamic=False) != 0


def test_step_length_matches_oracle(kctx_prob):
    prob, ctx, cones, rng = kctx_prob
    s, z = _interior_point(prob, 6)
    ctx.nt_scale(s, z)
    for c, r in zip(cones, rng):
        c.update_scaling(s[r], z[r])
    g = np.random.default_rng(8)
    for scale in (0.1, 1.0, 10.0):
        dz = scale * g.standard_normal(prob.m)
        ds = scale * g.standard_normal(prob.m)
        a, st = ctx.step_length(dz, ds, 1.0)
        assert st == 0
        ao = 1.0
        for c, r in zip(cones, rng):
            az, as_ = c.step_length(dz[r], ds[r], 1.0)
            ao = min(ao, az, as_)
        assert abs(a - ao) <= 1e-10 * max(ao, 1e-300)
        # admission: amax = 0.999 a admitted, 1.001 a rejected (unless capped at 1)
        adm, _ = ctx.step_length(dz, ds, 0.999 * a, mode=1)
        assert adm == pytest.approx(0.999 * a)
        if a < 1.0:
            rej, _ = ctx.step_length(dz, ds, min(1.0, 1.001 * a), mode=1)
            assert rej == 0.0


def test_kkt_solve_residual(kctx_prob):
    prob, ctx, cones, rng = kctx_prob
    s, z = _interior_point(prob, 7)
    ctx.nt_scale(s, z)
    ctx.schur()
    assert ctx.factor(1e-8) == 0
    g = np.random.default_rng(10)
    bx, bz = g.standard_normal(prob.n), g.standard_normal(prob.m)
    x, zz = ctx.kkt_solve(bx, bz)
    ex, ez, nrm = ctx.residual(bx, bz, x, zz)
    assert nrm <= 1e-9 * max(np.max(np.abs(bx)), np.max(np.abs(bz)))


@pytest.mark.parametrize("orders", [[1, 2, 3, 4, 5, 7, 8, 9], [16, 33, 63, 64]])
def test_nt_scale_edge_orders_match_oracle(orders):
    """The register-resident Jacobi at the orders that exercise its layout: one pair slot (1, 2),
    odd orders (a zero column that never rotates), and 63 / 64 (every lane and row in use);
    lambda to 1e-12 and the scaling through Hs, W^-1 W = I and W^-T s = diag(lambda)."""
    tri = [d * (d + 1) // 2 for d in orders]
    m = sum(tri)
    A = sp.random(m, 7, density=0.3, random_state=np.random.default_rng(11), format="csc")
    ctx = KernelContext()
    ctx.upload(A, orders)
    rng = np.random.default_rng(13)
    s, z, rows = [], [], []
    r0 = 0
    for d, t in zip(orders, tri):
        for out in (s, z):
            B = rng.standard_normal((d, d))
            out.append(P.svec(B @ B.T / d + 0.1 * np.eye(d)))
        rows.append(slice(r0, r0 + t))
        r0 += t
    s, z = np.concatenate(s), np.concatenate(z)
    lam, status = ctx.nt_scale(s, z)
    assert status == 0
    cones = [ipm.PsdCone(d) for d in orders]
    for c, r in zip(cones, rows):
        assert c.update_scaling(s[r], z[r])
    assert np.allclose(lam, np.concatenate([c.lam for c in cones]), rtol=1e-12, atol=0)
    x = np.random.default_rng(17).standard_normal(m)
    y = ctx.cone_apply(4, x)
    yo = np.concatenate([c.mul_Hs(x[r]) for c, r in zip(cones, rows)])
    assert np.max(np.abs(y - yo)) <= 1e-11 * max(1.0, np.max(np.abs(yo)))
    assert np.max(np.abs(ctx.cone_apply(2, ctx.cone_apply(0, x)) - x)) <= 1e-10
    y = ctx.cone_apply(3, s)
    for c, r in zip(cones, rows):
        M = ipm.svec_to_mat(y[r], c.n)
        assert np.allclose(M, np.diag(c.lam), atol=1e-10 * c.lam.max())
