"""Float64 restatement of SDPX's homogeneous self-dual interior-point method -- TEST ORACLE.

Test infrastructure only (see ``oracle/__init__``).  Follows the reference solver
yongjunx23-del/SDPX.rs v0.9.5; each function cites the file:line it restates
(paths relative to the reference's ``crates/solver/src/solver/``).

Scope: binary64 settings defaults, symmetric cones (PSD triangle and nonnegative orthant),
``kkt_form = condensed`` (every cone row eliminated into the Schur complement on x).  The
heuristics that are off in binary64 (tau chase, fixed-tau phase, split steps, tau-kappa
proximity, GMRES-IR fallback) are not restated; Gondzio correctors only act on orthant or
second-order rows and are not restated either (pure-PSD workloads never reach them).
"""
from __future__ import annotations

import dataclasses
import math
from dataclasses import dataclass
from typing import Dict, List, Optional, Tuple

import numpy as np
import scipy.linalg as sla
import scipy.sparse as sp

EPS = float(np.finfo(np.float64).eps)
SQRT2 = math.sqrt(2.0)

# Solver status codes of include/sdpx.h:76-80.
UNSOLVED, SOLVED, PRIMAL_INFEASIBLE, DUAL_INFEASIBLE, ALMOST_SOLVED = 0, 1, 2, 3, 4
ALMOST_PRIMAL_INFEASIBLE, ALMOST_DUAL_INFEASIBLE, MAX_ITERATIONS = 5, 6, 7
MAX_TIME, NUMERICAL_ERROR, INSUFFICIENT_PROGRESS = 8, 9, 10


@dataclass
class Settings:
    """Binary64 defaults of default/settings.rs:17-314."""
    max_iter: int = 200
    max_step_fraction: float = 0.99
    tol_gap_abs: float = 1e-8
    tol_gap_rel: float = 1e-8
    tol_feas: float = 1e-8
    tol_infeas_abs: float = 1e-8
    tol_infeas_rel: float = 1e-8
    tol_ktratio: float = 1e-6
    reduced_tol_gap_abs: float = 5e-5
    reduced_tol_gap_rel: float = 5e-5
    reduced_tol_feas: float = 1e-4
    reduced_tol_infeas_abs: float = 5e-12
    reduced_tol_infeas_rel: float = 5e-5
    reduced_tol_ktratio: float = 1e-4
    tol_original: Optional[float] = 1e-6
    equilibrate_enable: bool = True
    equilibrate_max_iter: int = 10
    equilibrate_min_scaling: float = 1e-4
    equilibrate_max_scaling: float = 1e4
    static_regularization_enable: bool = True
    static_regularization_constant: float = 1e-8
    static_regularization_proportional: float = EPS * EPS
    dynamic_regularization_enable: bool = True
    dynamic_regularization_eps: float = 1e-13
    dynamic_regularization_delta: float = 2e-7
    iterative_refinement_enable: bool = True
    iterative_refinement_reltol: float = 1e-13
    iterative_refinement_abstol: float = 1e-12
    iterative_refinement_max_iter: int = 10
    iterative_refinement_stop_ratio: float = 5.0


# ---------------------------------------------------------------------------------------
# svec helpers (cones/psdtrianglecone.rs svec_to_mat / mat_to_svec; include/sdpx.h:32-33)
# ---------------------------------------------------------------------------------------
_IDX: Dict[int, Tuple[np.ndarray, np.ndarray]] = {}


def _svec_idx(n):
    if n not in _IDX:
        j, i = np.tril_indices(n)
        _IDX[n] = (i, j)
    return _IDX[n]


def svec_to_mat(v, n):
    """Batched: v[..., tri(n)] -> [..., n, n]."""
    i, j = _svec_idx(n)
    v = np.asarray(v)
    w = np.where(i == j, v, v / SQRT2)
    M = np.zeros(v.shape[:-1] + (n, n))
    M[..., i, j] = w
    M[..., j, i] = w
    return M


def mat_to_svec(M):
    n = M.shape[-1]
    i, j = _svec_idx(n)
    v = M[..., i, j].copy()
    v[..., i != j] *= SQRT2
    return v


def diag_index(n):
    """triangular_index(k) for k < n: svec slot of the diagonal entry (k, k)."""
    k = np.arange(n)
    return (k + 1) * (k + 2) // 2 - 1


# ---------------------------------------------------------------------------------------
# Cones
# ---------------------------------------------------------------------------------------
class PsdCone:
    """cones/psdtrianglecone.rs: NT scaling, Jordan ops, step length."""

    def __init__(self, n):
        self.n = n
        self.numel = n * (n + 1) // 2
        self.degree = n
        self.set_identity()

    def set_identity(self):
        n = self.n
        self.R = np.eye(n)
        self.Rinv = np.eye(n)
        self.lam = np.ones(n)
        self.lisqrt = np.ones(n)
        self.G = np.eye(n)
        self.Ginv = np.eye(n)

    # psdtrianglecone.rs:311-439
    def update_scaling(self, s, z):
        n = self.n
        S = svec_to_mat(s, n)
        Z = svec_to_mat(z, n)
        try:
            L1 = np.linalg.cholesky(S)
            L2 = np.linalg.cholesky(Z)
        except np.linalg.LinAlgError:
            return False
        M = L2.T @ L1
        try:
            _, sv, Vt = np.linalg.svd(M)
        except np.linalg.LinAlgError:
            return False
        if not (np.all(np.isfinite(sv)) and np.all(sv > 0)):
            return False
        self.lam = sv.copy()
        root = np.sqrt(sv)
        self.lisqrt = 1.0 / root
        self.R = (L1 @ Vt.T) * self.lisqrt[None, :]
        X = sla.solve_triangular(L1, Vt.T, lower=True, trans="T")  # L1' X = V
        self.Rinv = root[:, None] * X.T
        self.G = self.R @ self.R.T
        # condensed/kkt.rs:1077-1180 sync: Ginv = Rinv' Rinv
        self.Ginv = self.Rinv.T @ self.Rinv
        return True

    # W x = svec(R' X R), W' x = svec(R X R'); Winv uses Rinv  (psdtrianglecone.rs:860-917)
    def mul_W(self, x, trans=False):
        X = svec_to_mat(x, self.n)
        Y = self.R @ X @ self.R.T if trans else self.R.T @ X @ self.R
        return mat_to_svec(Y)

    def mul_Winv(self, x, trans=False):
        X = svec_to_mat(x, self.n)
        Y = self.Rinv @ X @ self.Rinv.T if trans else self.Rinv.T @ X @ self.Rinv
        return mat_to_svec(Y)

    # Binary64 applies Hs = W'W and its inverse through the factor in two congruences,
    # never through the squared G / Ginv (condensed/psd.rs:1968-2002).
    def mul_Hs(self, x):
        Y = self.R.T @ svec_to_mat(x, self.n) @ self.R
        Y = 0.5 * (Y + Y.T)
        return mat_to_svec(self.R @ Y @ self.R.T)

    def mul_Hinv(self, x):
        Y = self.Rinv @ svec_to_mat(x, self.n) @ self.Rinv.T
        Y = 0.5 * (Y + Y.T)
        return mat_to_svec(self.Rinv.T @ Y @ self.Rinv)

    def affine_ds(self):  # psdtrianglecone.rs:455-460
        ds = np.zeros(self.numel)
        ds[diag_index(self.n)] = self.lam * self.lam
        return ds

    def circ_op(self, y, z):  # psdtrianglecone.rs:927-938
        Y = svec_to_mat(y, self.n)
        Z = svec_to_mat(z, self.n)
        return mat_to_svec(0.5 * (Y @ Z + Z @ Y))

    def lam_inv_circ_op(self, z):  # psdtrianglecone.rs:757-780
        Z = svec_to_mat(z, self.n)
        lam = self.lam
        return mat_to_svec(2.0 * Z / (lam[:, None] + lam[None, :]))

    def shift_unit(self, v, a):
        v = v.copy()
        v[diag_index(self.n)] += a
        return v

    def margins(self, z):  # psdtrianglecone.rs:~610 (margins)
        e = np.linalg.eigvalsh(svec_to_mat(z, self.n))
        return e.min(), np.sum(np.maximum(e, 0.0))

    def unit(self):
        return self.shift_unit(np.zeros(self.numel), 1.0)

    def _scaled_delta(self, d, primal):
        if primal:
            D = self.Rinv @ svec_to_mat(d, self.n) @ self.Rinv.T  # W^-T ds
        else:
            D = self.R.T @ svec_to_mat(d, self.n) @ self.R  # W dz
        return self.lisqrt[:, None] * D * self.lisqrt[None, :]

    @staticmethod
    def _admits(D, a):  # psdtrianglecone.rs:1168-1178
        try:
            np.linalg.cholesky(np.eye(D.shape[0]) + a * D)
            return True
        except np.linalg.LinAlgError:
            return False

    def _component(self, d, primal, amax):  # psdtrianglecone.rs:1180-1231
        if d.size == 0:
            return amax
        D = self._scaled_delta(d, primal)
        if self.n > 3 and self._admits(D, amax):
            return amax
        g = np.linalg.eigvalsh(D)[0]
        return min(-1.0 / g, amax) if g < 0 else amax

    def step_length(self, dz, ds, amax):
        az = self._component(dz, False, amax)
        a_s = self._component(ds, True, az)
        return az, a_s

    def step_admits(self, dz, ds, a):
        return (self._admits(self._scaled_delta(dz, False), a)
                and self._admits(self._scaled_delta(ds, True), a))

    def schur_block(self, Acols):
        """A_j' Hs^-1 A_j for dense columns (tri(n) x k) -- condensed/psd.rs:1120-1570."""
        Mats = svec_to_mat(Acols.T, self.n)  # k x n x n
        T = self.Ginv[None] @ Mats @ self.Ginv[None]
        return Acols.T @ mat_to_svec(T).T

    def dist(self, v):
        return max(0.0, -np.linalg.eigvalsh(svec_to_mat(v, self.n))[0]) if self.n else 0.0


class NonnegCone:
    """cones/nonnegativecone.rs."""

    def __init__(self, d):
        self.n = d
        self.numel = d
        self.degree = d
        self.set_identity()

    def set_identity(self):
        self.w = np.ones(self.n)
        self.lam = np.ones(self.n)

    def update_scaling(self, s, z):
        if np.any(s <= 0) or np.any(z <= 0):
            return False
        self.w = np.sqrt(s / z)
        self.lam = np.sqrt(s * z)
        return True

    def mul_W(self, x, trans=False):
        return self.w * x

    def mul_Winv(self, x, trans=False):
        return x / self.w

    def mul_Hs(self, x):
        return self.w * self.w * x

    def mul_Hinv(self, x):
        return x / (self.w * self.w)

    def affine_ds(self):
        return self.lam * self.lam

    def circ_op(self, y, z):
        return y * z

    def lam_inv_circ_op(self, z):
        return z / self.lam

    def shift_unit(self, v, a):
        return v + a

    def margins(self, z):
        return z.min(), np.sum(np.maximum(z, 0.0))

    def unit(self):
        return np.ones(self.n)

    def step_length(self, dz, ds, amax):
        def one(x, d):
            neg = d < 0
            return min(amax, np.min(-x[neg] / d[neg])) if np.any(neg) else amax
        return one(self._z, dz), one(self._s, ds)

    def step_admits(self, dz, ds, a):
        return np.all(self._z + a * dz >= 0) and np.all(self._s + a * ds >= 0)

    def schur_block(self, Acols):
        h = 1.0 / (self.w * self.w)
        return Acols.T @ (h[:, None] * Acols)

    def dist(self, v):
        return max(0.0, -v.min()) if v.size else 0.0


def make_cones(cones):
    out = []
    for kind, d in cones:
        if kind == "psd":
            out.append(PsdCone(d))
        elif kind == "nonneg":
            out.append(NonnegCone(d))
        else:
            raise NotImplementedError(f"oracle cone kind {kind}")
    return out


# ---------------------------------------------------------------------------------------
# Problem data + Ruiz equilibration (default/problemdata.rs:639-735)
# ---------------------------------------------------------------------------------------
class Data:
    def __init__(self, prob, settings: Settings):
        n, m = prob.n, prob.m
        self.n, self.m = n, m
        P = prob.P if prob.P is not None else sp.csc_matrix((n, n))
        self.P = sp.triu(sp.csc_matrix(P, dtype=np.float64)).tocsc()
        self.A = sp.csc_matrix(prob.A, dtype=np.float64).copy()
        self.q = np.array(prob.q, dtype=np.float64)
        self.b = np.array(prob.b, dtype=np.float64)
        self.cone_kinds = list(prob.cones)
        self.cones = make_cones(prob.cones)
        self.rng = []
        r = 0
        for c in self.cones:
            self.rng.append(slice(r, r + c.numel))
            r += c.numel
        assert r == m
        self.orig = (self.P.copy(), self.q.copy(), self.A.copy(), self.b.copy())
        self.d = np.ones(n)
        self.e = np.ones(m)
        self.c = 1.0
        if settings.equilibrate_enable:
            self._equilibrate(settings)
        self.dinv = 1.0 / self.d
        self.einv = 1.0 / self.e
        self.normb = np.max(np.abs(self.b * self.einv)) if m else 0.0
        self.normq = (np.max(np.abs(self.q * self.dinv)) if n else 0.0) / self.c
        self.degree = sum(c.degree for c in self.cones)
        self.Pfull = (self.P + sp.triu(self.P, 1).T).tocsc()

    @staticmethod
    def _col_inf(M):
        M = sp.csc_matrix(M)
        out = np.zeros(M.shape[1])
        if M.nnz:
            absM = abs(M)
            out = np.asarray(absM.max(axis=0).todense()).ravel()
        return out

    def _equilibrate(self, st: Settings):
        smin, smax = st.equilibrate_min_scaling, st.equilibrate_max_scaling
        for _ in range(st.equilibrate_max_iter):
            Psym = self.P + sp.triu(self.P, 1).T
            dwork = np.maximum(self._col_inf(Psym), self._col_inf(self.A))
            ework = self._col_inf(self.A.T.tocsc())
            dwork[dwork == 0] = 1.0
            ework[ework == 0] = 1.0
            dwork = 1.0 / np.sqrt(dwork)
            ework = 1.0 / np.sqrt(ework)
            dwork = np.clip(dwork, smin / self.d, smax / self.d)
            ework = np.clip(ework, smin / self.e, smax / self.e)
            D = sp.diags(dwork)
            E = sp.diags(ework)
            self.P = (D @ self.P @ D).tocsc()
            self.A = (E @ self.A @ D).tocsc()
            self.q = self.q * dwork
            self.b = self.b * ework
            self.d *= dwork
            self.e *= ework
            mean_col_norm_P = self._col_inf(self.P).mean() if self.P.nnz else 0.0
            inf_norm_q = np.max(np.abs(self.q)) if self.q.size else 0.0
            if mean_col_norm_P != 0.0 and inf_norm_q != 0.0:
                ctmp = 1.0 / max(inf_norm_q, mean_col_norm_P)
                ctmp = min(max(ctmp, smin / self.c), smax / self.c)
                self.P = (self.P * ctmp).tocsc()
                self.q = self.q * ctmp
                self.c *= ctmp
        # rectify_equilibration: PSD cones take one scalar, mean(e) (psdtrianglecone.rs:252-255)
        delta = np.ones(self.m)
        rect = False
        for c, r in zip(self.cones, self.rng):
            if isinstance(c, PsdCone) and c.numel:
                er = self.e[r]
                delta[r] = er.mean() / er
                rect = True
        if rect:
            self.A = (sp.diags(delta) @ self.A).tocsc()
            self.b = self.b * delta
            self.e *= delta


# ---------------------------------------------------------------------------------------
# Condensed KKT: Schur assembly, dense Cholesky with dynamic pivots, refinement
# ---------------------------------------------------------------------------------------
def potrf_dynamic(H, eps, delta):
    """Upper Cholesky H = U'U with the dynamic pivot rule (kkt/ldl/dense_block.rs:334-365)."""
    a = np.array(H, dtype=np.float64)
    n = a.shape[0]
    diag = np.diag(a).copy()
    for k in range(n):
        d = a[k, k]
        if not np.isfinite(d):
            return None
        if d <= eps:
            if d < -64.0 * EPS * n * abs(diag[k]):
                return None
            d = delta
        r = math.sqrt(d)
        a[k, k] = r
        a[k, k + 1:] /= r
        row = a[k, k + 1:]
        a[k + 1:, k + 1:] -= np.triu(np.outer(row, row))
    return np.triu(a)


class CondensedKKT:
    """kkt/condensed + kkt/direct/solver.rs:758-877 + kkt/ldl/dense_block.rs + kkt/refinement.rs."""

    def __init__(self, data: Data, st: Settings):
        self.data = data
        self.st = st
        self.reg_boost = 0
        self.U = None
        self.M = None
        self.counts = {"factor": 0, "solves": 0, "refine_outer": 0, "refine_inner": 0}
        # per cone: dense column block of A restricted to the cone rows and its columns
        self.blocks = []
        A = data.A
        for c, r in zip(data.cones, data.rng):
            sub = A[r, :]
            cols = np.flatnonzero(sub.getnnz(axis=0)) if sub.nnz else np.zeros(0, np.int64)
            dense = sub[:, cols].toarray() if cols.size else np.zeros((c.numel, 0))
            self.blocks.append((cols, dense))

    # condensed/mod.rs:1962-2147 (assemble): M = P + sum_j A_j' Hs_j^-1 A_j
    def assemble(self):
        d = self.data
        M = d.Pfull.toarray() if d.P.nnz else np.zeros((d.n, d.n))
        for c, (cols, dense) in zip(d.cones, self.blocks):
            if cols.size:
                M[np.ix_(cols, cols)] += c.schur_block(dense)
        self.M = 0.5 * (M + M.T)
        return bool(np.all(np.isfinite(self.M)))

    def _shift(self):
        st = self.st
        diag = np.max(np.abs(np.diag(self.M))) if self.M.size else 0.0
        base = st.static_regularization_constant + st.static_regularization_proportional * diag
        if self.reg_boost == 0:
            return base
        return base * 100.0 ** self.reg_boost

    # direct/solver.rs:758-877 + dense_block.rs:95-316
    def factor(self):
        self.counts["factor"] += 1
        st = self.st
        eps = self._shift() if st.static_regularization_enable else 0.0
        self.eps = eps
        H = self.M + eps * np.eye(self.M.shape[0])
        U = None
        try:
            U = sla.cholesky(H, lower=False)
            if st.dynamic_regularization_enable and np.any(np.diag(U) ** 2 <= st.dynamic_regularization_eps):
                U = None
        except np.linalg.LinAlgError:
            U = None
        if U is None and st.dynamic_regularization_enable:
            U = potrf_dynamic(H, st.dynamic_regularization_eps, st.dynamic_regularization_delta)
        if U is None or not np.all(np.isfinite(U)) or np.any(np.diag(U) <= 0):
            self.U = None
            return False
        self.U = U
        return True

    def escalate(self):  # direct/solver.rs:511-520
        if self.reg_boost >= 3:
            return False
        self.reg_boost += 1
        return True

    def update(self):
        return self.assemble() and self.factor()

    def _chol_solve(self, r):
        y = sla.solve_triangular(self.U, r, trans="T", lower=False)
        return sla.solve_triangular(self.U, y, lower=False)

    def _stationary(self, x, b, residual, solve, key):
        """refinement.rs:118-191 (stationary IR, stop ratio, acceptance)."""
        st = self.st
        if not st.iterative_refinement_enable:
            return x, True
        normb = np.max(np.abs(b)) if b.size else 0.0
        tol = st.iterative_refinement_abstol + st.iterative_refinement_reltol * normb
        e = residual(x)
        norme = np.max(np.abs(e)) if e.size else 0.0
        if not np.isfinite(norme):
            return x, False
        converged = norme <= tol
        for _ in range(st.iterative_refinement_max_iter):
            if converged:
                break
            previous = norme
            self.counts[key] += 1
            cand = x + solve(e)
            e2 = residual(cand)
            norme = np.max(np.abs(e2)) if e2.size else 0.0
            if not np.isfinite(norme):
                return x, False
            ratio = previous / norme if norme > 0 else np.inf
            if ratio < st.iterative_refinement_stop_ratio:
                if ratio > 1.0:
                    x, e = cand, e2
                break
            x, e = cand, e2
            converged = norme <= tol
        return x, True

    def reduced_solve(self, r):
        """Reduced solve refined against the unshifted Schur complement (direct/solver.rs:1046-1125)."""
        x = self._chol_solve(r)
        x, ok = self._stationary(x, r, lambda v: r - self.M @ v, self._chol_solve, "refine_inner")
        return x, ok

    def hinv(self, v):
        d = self.data
        out = np.empty_like(v)
        for c, r in zip(d.cones, d.rng):
            out[r] = c.mul_Hinv(v[r])
        return out

    def hs(self, v):
        d = self.data
        out = np.empty_like(v)
        for c, r in zip(d.cones, d.rng):
            out[r] = c.mul_Hs(v[r])
        return out

    def solve_raw(self, bx, bz):
        """condensed/mod.rs:2606-2622: condense, reduced solve, recover."""
        d = self.data
        xhat = bx + d.A.T @ self.hinv(bz)  # prepare_rhs (mod.rs:2416-2507)
        x, ok = self.reduced_solve(xhat)
        z = self.hinv(d.A @ x - bz)  # recover_rhs (mod.rs:2511-2604)
        return x, z, ok

    def residual_full(self, bx, bz, x, z):
        """condensed/mod.rs:2631-2871: e = b - [P A'; A -Hs] [x; z] (unshifted)."""
        d = self.data
        ex = bx - d.Pfull @ x - d.A.T @ z
        ez = bz - d.A @ x + self.hs(z)
        return ex, ez

    def solve(self, bx, bz):
        """condensed/kkt.rs:275-318: solve_raw then outer refinement on the original operator."""
        self.counts["solves"] += 1
        n = self.data.n
        if self.U is None or not (np.all(np.isfinite(bx)) and np.all(np.isfinite(bz))):
            return None, None, False
        x, z, ok = self.solve_raw(bx, bz)
        if not ok:
            return None, None, False
        b = np.concatenate([bx, bz])

        def residual(v):
            ex, ez = self.residual_full(bx, bz, v[:n], v[n:])
            return np.concatenate([ex, ez])

        def corr(e):
            cx, cz, _ = self.solve_raw(e[:n], e[n:])
            return np.concatenate([cx, cz])

        v, ok = self._stationary(np.concatenate([x, z]), b, residual, corr, "refine_outer")
        if not ok:
            return None, None, False
        return v[:n], v[n:], True


# ---------------------------------------------------------------------------------------
# The HSD driver
# ---------------------------------------------------------------------------------------
@dataclass
class Vars:
    x: np.ndarray
    s: np.ndarray
    z: np.ndarray
    tau: float
    kappa: float

    def copy(self):
        return Vars(self.x.copy(), self.s.copy(), self.z.copy(), self.tau, self.kappa)


@dataclass
class Result:
    status: int
    iterations: int
    x: np.ndarray
    s: np.ndarray
    z: np.ndarray
    objective: float
    dual_objective: float
    res_primal: float
    res_dual: float
    gap_abs: float
    gap_rel: float
    trace: List[dict]
    counts: Dict[str, int]


class Solver:
    def __init__(self, prob, settings: Optional[Settings] = None):
        self.st = settings or Settings()
        self.data = Data(prob, self.st)
        self.kkt = CondensedKKT(self.data, self.st)
        self.status = UNSOLVED
        self.trace = []

    # ---- residuals (default/residuals.rs:340-490) and info (default/info.rs:89-192) ----
    def _residuals(self, v: Vars):
        d = self.data
        Px = d.Pfull @ v.x
        xPx = float(v.x @ Px)
        qx = float(d.q @ v.x)
        rx_inf = -(d.A.T @ v.z)
        rz_inf = d.A @ v.x + v.s
        bz = float(d.b @ v.z)
        sz = float(v.s @ v.z)
        rx = -Px - v.tau * d.q + rx_inf
        rz = rz_inf - v.tau * d.b
        rtau = qx + bz + v.kappa + xPx / v.tau
        return dict(Px=Px, xPx=xPx, qx=qx, rx_inf=rx_inf, rz_inf=rz_inf, bz=bz, sz=sz,
                    rx=rx, rz=rz, rtau=rtau)

    def _info(self, v: Vars, r):
        d = self.data
        nrm = np.linalg.norm
        tinv = 1.0 / v.tau
        cinv = 1.0 / d.c
        xpx = r["xPx"] * tinv * tinv / 2.0
        cp = (r["qx"] * tinv + xpx) * cinv
        cd = (-r["bz"] * tinv - xpx) * cinv
        normx = nrm(v.x * d.d)
        normz = nrm(v.z * d.e) * cinv
        norms = nrm(v.s * d.einv)
        rx_inf_ns = nrm(r["rx_inf"] * d.dinv)
        px_ns = nrm(r["Px"] * d.dinv)
        rz_inf_ns = nrm(r["rz_inf"] * d.einv)
        rz_ns = nrm(r["rz"] * d.einv)
        rx_ns = nrm(r["rx"] * d.dinv)
        info = {}
        info["res_primal_inf"] = (rx_inf_ns * cinv) / max(1.0, normz)
        info["res_dual_inf"] = max(px_ns / max(1.0, normx), rz_inf_ns / max(1.0, normx + norms))
        normx *= tinv
        normz *= tinv
        norms *= tinv
        info["residual_norms"] = (rz_ns, rx_ns)
        info["res_primal"] = rz_ns * tinv / max(1.0, d.normb + normx + norms)
        info["res_dual"] = rx_ns * tinv * cinv / max(1.0, d.normq + normx + normz)
        info["cost_primal"] = cp
        info["cost_dual"] = cd
        info["gap_abs"] = abs(cp - cd)
        info["gap_rel"] = info["gap_abs"] / max(1.0, min(abs(cp), abs(cd)))
        info["ktratio"] = v.kappa * tinv
        return info

    def _is_solved(self, info, ga, gr, feas):
        return ((info["gap_abs"] < ga or info["gap_rel"] < gr)
                and info["res_primal"] < feas and info["res_dual"] < feas)

    def _check_convergence(self, info, r, full=True):
        st = self.st
        if full:
            t = (st.tol_gap_abs, st.tol_gap_rel, st.tol_feas, st.tol_infeas_abs,
                 st.tol_infeas_rel, st.tol_ktratio)
            codes = (SOLVED, PRIMAL_INFEASIBLE, DUAL_INFEASIBLE)
        else:
            t = (st.reduced_tol_gap_abs, st.reduced_tol_gap_rel, st.reduced_tol_feas,
                 st.reduced_tol_infeas_abs, st.reduced_tol_infeas_rel, st.reduced_tol_ktratio)
            codes = (ALMOST_SOLVED, ALMOST_PRIMAL_INFEASIBLE, ALMOST_DUAL_INFEASIBLE)
        if info["ktratio"] <= 1.0 and self._is_solved(info, t[0], t[1], t[2]):
            self.status = codes[0]
        elif info["ktratio"] > (1.0 / t[5]) * 1000.0:
            if r["bz"] < -t[3] and info["res_primal_inf"] < -t[4] * r["bz"]:
                self.status = codes[1]
            elif r["qx"] < -t[3] and info["res_dual_inf"] < -t[4] * r["qx"]:
                self.status = codes[2]

    # default/info.rs:263-327
    def _check_termination(self, info, r, iters):
        st = self.st
        self._check_convergence(info, r, True)
        prev = self.prev_info
        if self.status == UNSOLVED and iters > 1 and prev is not None and (
                info["res_dual"] > prev["res_dual"] or info["res_primal"] > prev["res_primal"]):
            if info["ktratio"] < EPS * 100.0 and (prev["gap_abs"] < st.tol_gap_abs
                                                  or prev["gap_rel"] < st.tol_gap_rel):
                self.status = INSUFFICIENT_PROGRESS
            if info["ktratio"] < 1.0:
                if ((info["res_dual"] > st.tol_feas * 100.0 and info["res_dual"] > prev["res_dual"] * 100.0)
                        or (info["res_primal"] > st.tol_feas * 100.0
                            and info["res_primal"] > prev["res_primal"] * 100.0)):
                    self.status = INSUFFICIENT_PROGRESS
        if self.status == UNSOLVED and st.max_iter == iters:
            self.status = MAX_ITERATIONS
        return self.status != UNSOLVED

    # default/original_check.rs + default/solution.rs:169-193
    def _unscaled(self, v: Vars):
        d = self.data
        tinv = 1.0 / v.tau
        return (v.x * d.d * tinv, v.s * d.einv * tinv, v.z * d.e * (tinv / d.c))

    def _original_ratio(self, v: Vars, reduced=False):
        st = self.st
        if st.tol_original is None:
            return None
        x, s, z = self._unscaled(v)
        P, q, A, b = self.data.orig
        Pf = P + sp.triu(P, 1).T
        px = Pf @ x
        xpx = float(x @ px)
        r = b - A @ x
        rd = px + A.T @ z + q
        primal, dual = 0.0, 0.0
        for c, rg in zip(self.data.cones, self.data.rng):
            if isinstance(c, NonnegCone):
                primal = max(primal, np.max(np.abs(r[rg] - s[rg])), np.max(np.maximum(-r[rg], -s[rg])))
                dual = max(dual, np.max(-z[rg]))
            else:
                primal = max(primal, np.max(np.abs(r[rg] - s[rg])), c.dist(s[rg]), c.dist(r[rg]))
                dual = max(dual, c.dist(z[rg]))
        normb = np.max(np.abs(b)) if b.size else 0.0
        normq = np.max(np.abs(q)) if q.size else 0.0
        primal /= (1.0 + normb)
        dual = max(np.max(np.abs(rd)) if rd.size else 0.0, dual) / (1.0 + normq)
        obj = float(q @ x) + xpx / 2.0
        dobj = -float(b @ z) - xpx / 2.0
        gap_abs = abs(obj - dobj)
        gap_rel = gap_abs / (1.0 + abs(obj))
        if reduced:
            tf = max(st.tol_original, st.reduced_tol_feas)
            ta = max(st.tol_original, st.reduced_tol_gap_abs)
            tr = max(st.tol_original, st.reduced_tol_gap_rel)
        else:
            tf = ta = tr = st.tol_original
        gap = min(gap_abs / ta, gap_rel / tr)
        return max(primal / tf, dual / tf, gap)

    # ---- cone collection helpers ----
    def _cones(self):
        return zip(self.data.cones, self.data.rng)

    def _scale(self, v: Vars):
        return all(c.update_scaling(v.s[r], v.z[r]) for c, r in self._cones())

    def _shift_interior(self, z):
        """variables.rs:577-620 (_shift_to_cone_interior / interior_shifts)."""
        mins, poss = [], []
        for c, r in self._cones():
            a, b = c.margins(z[r])
            mins.append(a)
            poss.append(b)
        min_margin = min(mins) if mins else np.inf
        pos_margin = sum(poss)
        target = max(1.0, (pos_margin * 0.1) / self.data.degree)
        if min_margin <= 0:
            shifts = [-min_margin, target]
        elif min_margin < target:
            shifts = [target - min_margin]
        else:
            shifts = [0.0]
        z = z.copy()
        for a in shifts:
            for c, r in self._cones():
                z[r] = c.shift_unit(z[r], a)
        return z

    # core/solver.rs:1209-1322 default_start; kktsystem.rs:462-527 solve_initial_point
    def _default_start(self):
        d = self.data
        for c in d.cones:
            c.set_identity()
        ok = self._kkt_update()
        v = Vars(np.zeros(d.n), np.zeros(d.m), np.zeros(d.m), 1.0, 1.0)
        if ok:
            if d.P.nnz == 0:
                x, zz, ok1 = self.kkt.solve(np.zeros(d.n), d.b.copy())
                ok = ok1
                if ok:
                    v.x = x
                    v.s = -zz
                    _, z2, ok2 = self.kkt.solve(-d.q, np.zeros(d.m))
                    ok = ok2
                    if ok:
                        v.z = z2
            else:
                x, zz, ok = self.kkt.solve(-d.q, d.b.copy())
                if ok:
                    v.x = x
                    v.z = zz
                    v.s = -zz
        if ok:
            scale = max(np.max(np.abs(d.b)) if d.m else 0, np.max(np.abs(d.q)) if d.n else 0,
                        abs(d.A).max() if d.A.nnz else 0, 1.0)
            bound = 1e12 * scale
            if not (np.max(np.abs(v.x), initial=0) <= bound and np.max(np.abs(v.z), initial=0) <= bound):
                ok = False
        if ok:
            v.s = self._shift_interior(v.s)
            v.z = self._shift_interior(v.z)
            v.tau, v.kappa = 1.0, 1.0
        else:
            v.x = np.zeros(d.n)
            v.s = np.concatenate([c.unit() for c in d.cones]) if d.cones else np.zeros(0)
            v.z = v.s.copy()
            v.tau, v.kappa = 1.0, 1.0
            tau0 = min(1.0, 1.0 / max(1.0, d.d.max(initial=1.0)))
            if tau0 < 1.0:
                v.tau, v.kappa = tau0, 1.0 / tau0
        return v

    def _kkt_update(self):
        if not self.kkt.update():
            while self.st.static_regularization_enable and self.kkt.escalate():
                if self.kkt.factor():
                    return True
            return False
        return True

    # default/kktsystem.rs:190-274 update_affine + solve (276-460)
    def _hsd_solve(self, v: Vars, rhs_x, workz, rhs_tau, rhs_kappa, rhs_z, cached=None):
        d = self.data
        if cached is None:
            x1, z1, ok = self.kkt.solve(rhs_x, workz)
            if not ok:
                return None
        else:
            x1, z1 = cached
        x2, z2 = self.const
        xi = v.x / v.tau
        q1 = float(d.q @ x1)
        b1 = float(d.b @ z1)
        quad1 = float(xi @ (d.Pfull @ x1))
        xi = xi - x2
        q2 = float(d.q @ x2)
        b2 = float(d.b @ z2)
        delta = float(xi @ (d.Pfull @ xi))
        quad2 = float(x2 @ (d.Pfull @ x2))
        num = rhs_tau - rhs_kappa / v.tau + q1 + b1 + 2.0 * quad1
        den = v.kappa / v.tau - q2 - b2
        den += delta - quad2
        dtau = num / den
        dx = x1 + dtau * x2
        dz = z1 + dtau * z2
        # condensed binary64: Δs from the linear row A Δx + Δs - b Δτ = -r_z (kktsystem.rs:403-418)
        ds = -rhs_z + dtau * d.b - d.A @ dx
        dk = -(rhs_kappa + v.kappa * dtau) / v.tau
        return Vars(dx, ds, dz, dtau, dk)

    def _step_bounds(self, v: Vars, step: Vars):
        at = -v.tau / step.tau if step.tau < 0 else np.inf
        ak = -v.kappa / step.kappa if step.kappa < 0 else np.inf
        a = min(at, ak, 1.0)
        az_all, as_all = a, a
        for c, r in self._cones():
            if isinstance(c, NonnegCone):
                c._z, c._s = v.z[r], v.s[r]
            az, as_ = c.step_length(step.z[r], step.s[r], a)
            az_all = min(az_all, az)
            as_all = min(as_all, as_)
        return min(az_all, as_all)

    def _step_admits(self, v: Vars, step: Vars, t):
        a = t / self.st.max_step_fraction
        if not (a <= 1.0 and v.tau + a * step.tau >= 0 and v.kappa + a * step.kappa >= 0):
            return False
        for c, r in self._cones():
            if isinstance(c, NonnegCone):
                c._z, c._s = v.z[r], v.s[r]
            if not c.step_admits(step.z[r], step.s[r], a):
                return False
        return True

    def solve(self) -> Result:
        st = self.st
        d = self.data
        v = self._default_start()
        self.prev_info = None
        it, mu, sigma, alpha = 0, 0.0, 1.0, 0.0
        best = None
        prev_vars = v.copy()
        orig_progress = [None, 0]
        info = r = None
        while True:
            r = self._residuals(v)
            mu = (r["sz"] + v.tau * v.kappa) / (d.degree + 1)
            info = self._info(v, r)
            self.trace.append(dict(iter=it, mu=mu, alpha=alpha, sigma=sigma, pcost=info["cost_primal"],
                                   dcost=info["cost_dual"], gap_rel=info["gap_rel"],
                                   pres=info["res_primal"], dres=info["res_dual"], tau=v.tau, kappa=v.kappa))
            stop = self._check_termination(info, r, it)
            if stop and self.status == SOLVED:
                ratio = self._original_ratio(v)
                if ratio is not None and not ratio <= 1.0:
                    b0, stale = orig_progress
                    if b0 is None or ratio < b0 * 0.5:
                        orig_progress = [ratio, 0]
                    else:
                        orig_progress = [b0, stale + 1]
                    if orig_progress[1] >= 3:
                        self.status = INSUFFICIENT_PROGRESS
                    elif it >= st.max_iter:
                        self.status = MAX_ITERATIONS
                    else:
                        self.status = UNSOLVED
                        stop = False
            if stop:
                if self.status == INSUFFICIENT_PROGRESS:
                    # strategy_checkpoint_insufficient_progress: roll back one iterate
                    v = prev_vars.copy()
                    if self.prev_info is not None:
                        info = dict(info, **{k: self.prev_info[k] for k in
                                             ("cost_primal", "cost_dual", "res_primal", "res_dual",
                                              "gap_abs", "gap_rel")})
                break
            # scale (core/solver.rs:831-850)
            if not self._scale(v):
                self.status = NUMERICAL_ERROR
                break
            it += 1
            # ---------- direction (core/solver.rs:852-949) ----------
            ok = self._kkt_update()
            affine = None
            if ok:
                # constant column [-q; b] and affine column [rx; s - rz]
                x2, z2, okc = self.kkt.solve(-d.q, d.b.copy())
                while not okc:
                    if not (st.static_regularization_enable and self.kkt.escalate() and self.kkt.factor()):
                        break
                    x2, z2, okc = self.kkt.solve(-d.q, d.b.copy())
                ok = okc
                if ok:
                    self.const = (x2, z2)
                    xa, za, oka = self.kkt.solve(r["rx"], v.s - r["rz"])
                    ok = oka
                    if ok:
                        step = self._hsd_solve(v, r["rx"], None, r["rtau"], v.tau * v.kappa, r["rz"],
                                               cached=(xa, za))
                        ok = step is not None
            if not ok:
                self.status = NUMERICAL_ERROR
                alpha = 0.0
                break
            affine = step.copy()
            # affine step length: no step fraction (variables.rs:223-249, 673-690)
            alpha = self._step_bounds(v, step)
            sigma = max((1.0 - alpha) ** 3, 0.0)
            mfac = alpha if it == 1 else 1.0  # reduced Mehrotra correction in iteration 1
            # combined rhs (variables.rs:752-788, symmetric_common.rs:50-81)
            rhs_x = (1.0 - sigma) * r["rx"]
            rhs_tau = (1.0 - sigma) * r["rtau"]
            rhs_kappa = -sigma * mu + mfac * step.tau * step.kappa + v.tau * v.kappa
            dz_scaled = step.z * mfac
            rhs_s = np.empty(d.m)
            for c, rg in self._cones():
                wdz = c.mul_W(dz_scaled[rg], trans=False)
                wds = c.mul_Winv(step.s[rg], trans=True)
                shift = c.shift_unit(c.circ_op(wds, wdz), -sigma * mu)
                rhs_s[rg] = c.affine_ds() + shift
            rhs_z = (1.0 - sigma) * r["rz"]
            # Δs offset c = W'(λ \ ds)  (symmetric_common.rs:86-92)
            cvec = np.empty(d.m)
            for c, rg in self._cones():
                cvec[rg] = c.mul_W(c.lam_inv_circ_op(rhs_s[rg]), trans=True)
            step = self._hsd_solve(v, rhs_x, cvec - rhs_z, rhs_tau, rhs_kappa, rhs_z)
            if step is None:
                self.status = NUMERICAL_ERROR
                alpha = 0.0
                break
            # ---------- step length (core/solver.rs:951-1012) ----------
            alpha = self._step_bounds(v, step) * st.max_step_fraction
            if 0.0 < alpha < 0.9:
                for frac in (0.5, 0.25):
                    t = alpha + (1.0 - alpha) * frac
                    if t * (1.0 - sigma * t) <= 1.01 * alpha * (1.0 - sigma):
                        continue
                    trial = Vars((1 - t) * affine.x + t * step.x, (1 - t) * affine.s + t * step.s,
                                 (1 - t) * affine.z + t * step.z, (1 - t) * affine.tau + t * step.tau,
                                 (1 - t) * affine.kappa + t * step.kappa)
                    if self._step_admits(v, trial, t):
                        step = trial
                        alpha = t
                        break
            if alpha <= 0.0:
                self.status = INSUFFICIENT_PROGRESS
                break
            self.prev_info = info
            # best iterate (core/solver.rs:420-428)
            tm = max(max(info["res_primal"], info["res_dual"]) / st.tol_feas,
                     min(info["gap_abs"] / st.tol_gap_abs, info["gap_rel"] / st.tol_gap_rel))
            if best is None or tm < best[0]:
                best = (tm, v.copy())
            prev_vars = v.copy()
            v = Vars(v.x + alpha * step.x, v.s + alpha * step.s, v.z + alpha * step.z,
                     v.tau + alpha * step.tau, v.kappa + alpha * step.kappa)
        # finish (core/solver.rs:1128-1207)
        before = self.status
        if before in (NUMERICAL_ERROR, INSUFFICIENT_PROGRESS, MAX_ITERATIONS, MAX_TIME):
            r = self._residuals(v)
            info = self._info(v, r)
            now = max(max(info["res_primal"], info["res_dual"]) / st.tol_feas,
                      min(info["gap_abs"] / st.tol_gap_abs, info["gap_rel"] / st.tol_gap_rel))
            if best is not None and best[0] < now:
                v = best[1]
                r = self._residuals(v)
                info = self._info(v, r)
            self._check_convergence(info, r, False)
            if self.status == ALMOST_SOLVED and before != ALMOST_SOLVED:
                ratio = self._original_ratio(v, reduced=True)
                if ratio is not None and not ratio <= 1.0:
                    self.status = before
        x, s, z = self._unscaled(v)
        return Result(status=self.status, iterations=it, x=x, s=s, z=z,
                      objective=info["cost_primal"], dual_objective=info["cost_dual"],
                      res_primal=info["res_primal"], res_dual=info["res_dual"],
                      gap_abs=info["gap_abs"], gap_rel=info["gap_rel"], trace=self.trace,
                      counts=dict(self.kkt.counts))


def solve(prob, settings: Optional[Settings] = None, **overrides) -> Result:
    st = settings or Settings()
    if overrides:
        st = dataclasses.replace(st, **overrides)
    return Solver(prob, st).solve()
