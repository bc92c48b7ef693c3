"""Split-precision (Ozaki-II, INT8 tensor cores) FP64 products and the split factorisation form.

Bars:
  * sdpxg_split_dgemm_device against numpy's FP64 product: every entry within
    2^-50 * K * max|row of op(A)| * max|column of op(B)| (the quantisation bound is 2^-b with
    b >= 55 at these K, plus FP64's own rounding of the reference), all four transposes, ragged
    shapes, alpha/beta, zero rows;
  * integer operands small enough that every product is exact in FP64: bitwise equal (this pins
    the tensor-core GEMM itself: residues, swizzled TMA tiles, TMEM epilogue, Garner);
  * the split factorisation at m = 2000 (the bench's Schur dimension): refined solves within
    1e-9 of numpy's LU solve of the same Schur complement, like the plain form;
  * whole solves of the benchmarked workloads in the split form: status, iterations within 1,
    objectives within 1e-8 of the oracle fixtures (tests/golden).
"""
from pathlib import Path

import numpy as np
import pytest

from sdpx_b200 import problems as P
from sdpx_b200.solver import DefaultSettings, DefaultSolver, KernelContext, solve_problem

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


def _dev(a):
    import torch
    return torch.from_numpy(np.asfortranarray(a).ravel(order="F").copy()).cuda()


def _split_gemm(ctx, ta, tb, A, B, Cin, alpha, beta):
    import torch
    m = A.shape[0] if ta == "N" else A.shape[1]
    k = A.shape[1] if ta == "N" else A.shape[0]
    n = B.shape[1] if tb == "N" else B.shape[0]
    dA, dB, dC = _dev(A), _dev(B), _dev(Cin)
    torch.cuda.synchronize()
    st = ctx.split_dgemm_device(ta, tb, m, n, k, alpha, dA.data_ptr(), A.shape[0], dB.data_ptr(),
                                B.shape[0], beta, dC.data_ptr(), m)
    assert st == 0
    return dC.cpu().numpy().reshape((n, m)).T


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T"), ("T", "T")])
@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (130, 70, 257), (300, 520, 1000), (1024, 976, 1024)])
def test_split_gemm_matches_fp64(ta, tb, m, n, k):
    rng = np.random.default_rng(m * 7 + n * 3 + k)
    A = rng.standard_normal((m, k) if ta == "N" else (k, m))
    B = rng.standard_normal((k, n) if tb == "N" else (n, k))
    A *= np.exp2(rng.integers(-20, 20, size=A.shape))  # wide exponent ranges inside rows
    if m > 2:
        (A[2, :] if ta == "N" else A[:, 2])[:] = 0.0  # a zero row of op(A)
    Cin = rng.standard_normal((m, n))
    opA = A if ta == "N" else A.T
    opB = B if tb == "N" else B.T
    got = _split_gemm(KernelContext(), ta, tb, A, B, Cin, 0.75, -0.5)
    ref = 0.75 * (opA @ opB) - 0.5 * Cin
    bound = 2.0 ** -50 * k * np.outer(np.abs(opA).max(axis=1), np.abs(opB).max(axis=0)) + 1e-15 * np.abs(Cin)
    assert np.all(np.abs(got - ref) <= bound + 4 * np.finfo(float).eps * np.abs(ref))


def test_split_gemm_exact_on_integers():
    """Small integers: every product and sum is exact in FP64, so the split product is bitwise."""
    rng = np.random.default_rng(5)
    m, n, k = 257, 300, 1153
    A = rng.integers(-1000, 1000, size=(m, k)).astype(np.float64)
    B = rng.integers(-1000, 1000, size=(k, n)).astype(np.float64)
    got = _split_gemm(KernelContext(), "N", "N", A, B, np.zeros((m, n)), 1.0, 0.0)
    assert np.array_equal(got, A @ B)


def _interior_point(prob, seed):
    rng = np.random.default_rng(seed)
    s, z = [], []
    for _, d in prob.cones:
        for out in (s, z):
            Bm = rng.standard_normal((d, d))
            out.append(P.svec(Bm @ Bm.T / d + 0.1 * np.eye(d)))
    return np.concatenate(s), np.concatenate(z)


@pytest.mark.parametrize("shift", [1e-8, 1e-3])
def test_split_factor_refined_solve_m2000(shift):
    prob = P.rank1_sdp(32, 2000, seed=0)
    ctx = KernelContext()
    ctx.upload(prob.A, [d for _, d in prob.cones])
    ctx.set_factor_form(1)
    s, z = _interior_point(prob, 11)
    assert ctx.nt_scale(s, z)[1] == 0
    H = ctx.schur()
    assert ctx.factor(shift) == 0
    b = np.random.default_rng(12).standard_normal((prob.n, 2))
    x = ctx.solve_many(b)
    xo = np.linalg.solve(H, b)
    assert np.max(np.abs(x - xo)) <= 1e-9 * np.max(np.abs(xo))


def _rel(a, b):
    return abs(a - b) / max(1.0, abs(b))


@pytest.mark.parametrize("name,blocks,m", [("rank1_b32_m2000_s0", 32, 2000),
                                           ("rank1_b64_m4000_s0", 64, 4000)])
def test_split_form_whole_solve_matches_oracle(name, blocks, m):
    fx = np.load(GOLDEN / f"solve_{name}.npz")
    prob = P.rank1_sdp(blocks, m, seed=0)
    s = DefaultSolver(prob.P, prob.q, prob.A, prob.b, prob.cones, DefaultSettings(kkt_form="condensed"))
    s.set_form(DefaultSolver.FORM_SPLIT)
    g = s.solve()
    assert g.status_code == int(fx["status"])
    assert abs(g.iterations - int(fx["iterations"])) <= 1
    assert _rel(g.obj_val, float(fx["objective"])) <= 1e-8
    assert _rel(g.obj_val_dual, float(fx["dual_objective"])) <= 1e-8
