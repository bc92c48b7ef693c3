"""Host-side mirror of the reference solver API over the CUDA library.

Mirrors ``DefaultSolver::new(&P, &q, &A, &b, &cones, settings)`` /
``solver.solve()`` / ``solver.solution`` / ``solver.info`` of the reference
(crates/solver/src/solver/default/solver.rs:260, solution.rs, info.rs) with the same
argument meaning, status names and error behaviour (invalid input raises, like the
reference's ``Result`` error), calling the reference-compatible C ABI ``sdpx_*`` of
libsdpx_b200.so.  ``KernelContext`` wraps the kernel-level ``sdpxg_*`` entry points.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np
import scipy.sparse as sp

from . import _lib
from ._lib import dptr

STATUS_NAMES = {
    0: "Unsolved", 1: "Solved", 2: "PrimalInfeasible", 3: "DualInfeasible", 4: "AlmostSolved",
    5: "AlmostPrimalInfeasible", 6: "AlmostDualInfeasible", 7: "MaxIterations", 8: "MaxTime",
    9: "NumericalError", 10: "InsufficientProgress", 11: "CallbackTerminated", 12: "DualFeasible",
}
CONE_KINDS = {"zero": 0, "nonneg": 1, "soc": 2, "psd": 3}


def PSDTriangleConeT(n: int) -> Tuple[str, int]:
    return ("psd", int(n))


@dataclass
class DefaultSettings:
    """Subset of DefaultSettings (default/settings.rs:17-314) carried by the C ABI."""
    max_iter: int = 200
    time_limit: float = float("inf")
    verbose: bool = False
    tol_gap_abs: Optional[float] = None
    tol_gap_rel: Optional[float] = None
    tol_feas: Optional[float] = None
    tol_infeas_abs: Optional[float] = None
    tol_infeas_rel: Optional[float] = None
    equilibrate_enable: bool = True
    presolve_enable: bool = True
    chordal_decomposition_enable: bool = True
    kkt_form: str = "auto"
    precision_bits: int = 53

    def to_c(self) -> Tuple[_lib.Settings, list]:
        s = _lib.Settings()
        _lib.call("sdpx_default_settings_v4", C.byref(s))
        s.max_iter = self.max_iter
        s.time_limit = self.time_limit
        s.verbose = int(bool(self.verbose))
        s.precision_bits = self.precision_bits
        s.kkt_form = {"auto": 0, "augmented": 1, "condensed": 2}[self.kkt_form]
        s.preprocessing_flags = (int(self.equilibrate_enable) | 2 * int(self.presolve_enable)
                                 | 4 * int(self.chordal_decomposition_enable))
        keep = []
        for name in ("tol_gap_abs", "tol_gap_rel", "tol_feas", "tol_infeas_abs", "tol_infeas_rel"):
            v = getattr(self, name)
            if v is not None:
                b = repr(float(v)).encode()
                keep.append(b)
                setattr(s, name, b)
        return s, keep


@dataclass
class Solution:
    x: np.ndarray
    z: np.ndarray
    s: np.ndarray
    status: str
    status_code: int
    obj_val: float
    obj_val_dual: float
    r_prim: float
    r_dual: float
    iterations: int
    solve_time: float


@dataclass
class SolveInfo:
    status: str
    iterations: int
    cost_primal: float
    cost_dual: float
    res_primal: float
    res_dual: float
    gap_abs: float
    gap_rel: float
    solve_time: float
    phase_times: dict = field(default_factory=dict)
    counts: dict = field(default_factory=dict)


def _scalars(a: np.ndarray) -> _lib.Scalars:
    s = _lib.Scalars()
    s.kind = 0
    s.reserved = 0
    s.count = a.size
    s.f64 = dptr(a)
    s.decimal = None
    return s


class _CscHold:
    """Keeps the numpy buffers of a C CSC view alive."""

    def __init__(self, M: sp.spmatrix):
        M = sp.csc_matrix(M, dtype=np.float64)
        M.sort_indices()
        self.colptr = np.ascontiguousarray(M.indptr, dtype=np.uint64)
        self.rowval = np.ascontiguousarray(M.indices, dtype=np.uint64)
        self.values = np.ascontiguousarray(M.data, dtype=np.float64)
        c = _lib.Csc()
        c.rows, c.cols, c.nnz = M.shape[0], M.shape[1], M.nnz
        c.colptr = self.colptr.ctypes.data_as(_lib.PU64)
        c.rowval = self.rowval.ctypes.data_as(_lib.PU64)
        c.values = _scalars(self.values)
        self.c = c


class CProblem:
    """A problem in the C ABI's host layout: sdpx_csc / sdpx_scalars / sdpx_cone / sdpx_settings
    views over numpy buffers this object keeps alive (what a C or Rust caller of sdpx_prepare
    holds).  Building it converts scipy/numpy inputs once; sdpx_prepare then reads it."""

    def __init__(self, P, q, A, b, cones: Sequence[Tuple[str, int]],
                 settings: Optional["DefaultSettings"] = None):
        settings = settings or DefaultSettings()
        A = sp.csc_matrix(A, dtype=np.float64)
        n = A.shape[1]
        P = sp.csc_matrix((n, n)) if P is None else sp.triu(sp.csc_matrix(P, dtype=np.float64)).tocsc()
        self.q = np.ascontiguousarray(q, dtype=np.float64)
        self.b = np.ascontiguousarray(b, dtype=np.float64)
        self.P, self.A = _CscHold(P), _CscHold(A)
        cone_arr = (_lib.Cone * max(len(cones), 1))()
        for i, (kind, d) in enumerate(cones):
            cone_arr[i].kind = CONE_KINDS[kind]
            cone_arr[i].reserved = 0
            cone_arr[i].dim = int(d)
            cone_arr[i].alpha = _scalars(np.zeros(0))
        cs, self._keep = settings.to_c()
        self.cones, self.cs = cone_arr, cs
        self.n, self.m = n, A.shape[0]
        self.args = (C.byref(self.P.c), C.byref(_scalars(self.q)), C.byref(self.A.c),
                     C.byref(_scalars(self.b)), cone_arr, len(cones), C.byref(cs))


class DefaultSolver:
    """GPU solve through the reference-compatible C ABI (sdpx_prepare / sdpx_solve)."""

    def __init__(self, P, q, A, b, cones: Sequence[Tuple[str, int]],
                 settings: Optional[DefaultSettings] = None):
        self._prepare(CProblem(P, q, A, b, cones, settings))

    @classmethod
    def new_sampled(cls, P, q, A_linear, b, cones: Sequence[Tuple[str, int]],
                    blocks: Sequence[dict], settings: Optional[DefaultSettings] = None) -> "DefaultSolver":
        """sdpx_prepare_sampled: factor-authoritative sampled PSD blocks (the reference's
        DefaultSolver::new_sampled).  Each block is a dict with row_start, column_start, dim,
        basis (basis_rows x basis_cols array) and weights (tri(dim) * basis_cols values)."""
        self = cls.__new__(cls)
        cp = CProblem(P, q, A_linear, b, cones, settings)
        self._hold(cp)
        arr = (_lib.SampledBlock * max(len(blocks), 1))()
        keep = []
        for i, blk in enumerate(blocks):
            Q = np.asfortranarray(blk["basis"], dtype=np.float64)
            w = np.ascontiguousarray(blk["weights"], dtype=np.float64)
            qv = Q.ravel(order="F").copy()
            keep += [qv, w]
            arr[i].row_start, arr[i].column_start = int(blk["row_start"]), int(blk["column_start"])
            arr[i].dim, arr[i].basis_rows, arr[i].basis_cols = int(blk.get("dim", 1)), Q.shape[0], Q.shape[1]
            arr[i].basis, arr[i].weights = _scalars(qv), _scalars(w)
        self._sampled_keep = (arr, keep)
        h = C.c_void_p()
        _lib.call("sdpx_prepare_sampled", *cp.args, arr, len(blocks), C.byref(h))
        self._h = h
        self.solution = None
        self.info = None
        return self

    @classmethod
    def from_c_problem(cls, cp: CProblem) -> "DefaultSolver":
        """sdpx_prepare on a problem already in the C ABI's host layout."""
        self = cls.__new__(cls)
        self._prepare(cp)
        return self

    def _prepare(self, cp: CProblem):
        self._hold(cp)
        h = C.c_void_p()
        _lib.call("sdpx_prepare", *cp.args, C.byref(h))
        self._h = h
        self.solution: Optional[Solution] = None
        self.info: Optional[SolveInfo] = None

    def _hold(self, cp: CProblem):
        self._cp, self._A = cp, cp.A
        self.n, self.m = cp.n, cp.m

    def close(self):
        """sdpx_destroy now (otherwise at garbage collection)."""
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _lib.load().sdpx_destroy(h)
            self._h = None

    def reprepare(self, P, q, A, b, cones: Sequence[Tuple[str, int]],
                  settings: Optional[DefaultSettings] = None):
        """Load another problem into this handle, reusing its device buffers and stream."""
        cp = CProblem(P, q, A, b, cones, settings)
        self._hold(cp)
        _lib.call("sdpx_b200_reprepare", self._h, *cp.args)
        self.solution = None
        self.info = None

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.load().sdpx_destroy(h)
            except Exception:
                pass
            self._h = None

    def solve(self) -> Solution:
        _lib.call("sdpx_solve", self._h)
        info = _lib.Info()
        _lib.call("sdpx_get_info", self._h, C.byref(info))
        need = C.c_uint64()
        _lib.call("sdpx_result_f64", self._h, None, 0, C.byref(need))
        out = np.empty(need.value)
        _lib.call("sdpx_result_f64", self._h, dptr(out), need.value, C.byref(need))
        n, m = self.n, self.m
        times = np.zeros(7)
        counts = np.zeros(4, dtype=np.uint64)
        _lib.call("sdpx_b200_phase_times", self._h, dptr(times), counts.ctypes.data_as(_lib.PU64))
        status = STATUS_NAMES.get(info.status, str(info.status))
        self.solution = Solution(x=out[:n].copy(), z=out[n:n + m].copy(), s=out[n + m:n + 2 * m].copy(),
                                 status=status, status_code=info.status, obj_val=out[-6],
                                 obj_val_dual=out[-5], r_prim=out[-4], r_dual=out[-3],
                                 iterations=info.iterations, solve_time=info.solve_time)
        names = ["scale", "assemble", "factor", "kkt_solve", "step", "residual", "other"]
        self.info = SolveInfo(status=status, iterations=info.iterations, cost_primal=info.objective,
                              cost_dual=info.dual_objective, res_primal=info.primal_residual,
                              res_dual=info.dual_residual, gap_abs=info.gap_abs,
                              gap_rel=info.gap_rel, solve_time=info.solve_time,
                              phase_times=dict(zip(names, times.tolist())),
                              counts=dict(zip(["factorizations", "kkt_solves", "outer_refinements",
                                               "inner_refinements"], counts.tolist())))
        return self.solution

    KERNEL_PHASES = ["scale", "assemble", "factor", "trisolve", "cone", "step", "symv", "trinv", "split"]

    def set_kernel_timing(self, on: bool):
        _lib.call("sdpx_b200_set_kernel_timing", self._h, int(bool(on)))

    def kernel_times(self) -> dict:
        ms = np.zeros(len(self.KERNEL_PHASES))
        cnt = np.zeros(len(self.KERNEL_PHASES), dtype=np.uint64)
        _lib.call("sdpx_b200_kernel_times", self._h, dptr(ms), cnt.ctypes.data_as(_lib.PU64))
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(self.KERNEL_PHASES)}

    def update(self, q, b):
        self._q = np.ascontiguousarray(q, dtype=np.float64)
        self._b = np.ascontiguousarray(b, dtype=np.float64)
        _lib.call("sdpx_update", self._h, C.byref(_scalars(self._q)), C.byref(_scalars(self._b)))

    def adjoint(self, dl_dx, dl_dz=None, dl_ds=None):
        """Gradients of a loss of the last solution: returns (dq, db, dA) with dA a CSC matrix on
        the sparsity pattern of A (sdpx_b200_adjoint)."""
        gx = np.ascontiguousarray(dl_dx, dtype=np.float64)
        gz = None if dl_dz is None else np.ascontiguousarray(dl_dz, dtype=np.float64)
        gs = None if dl_ds is None else np.ascontiguousarray(dl_ds, dtype=np.float64)
        dq, db = np.empty(self.n), np.empty(self.m)
        nnz = int(self._A.values.size)
        dA = np.empty(nnz)
        _lib.call("sdpx_b200_adjoint", self._h, dptr(gx), dptr(gz), dptr(gs), dptr(dq), dptr(db),
                  dptr(dA), nnz)
        A = sp.csc_matrix((dA, self._A.rowval.astype(np.int64), self._A.colptr.astype(np.int64)),
                          shape=(self.m, self.n))
        return dq, db, A

    def set_graphs(self, on: bool):
        """Replay the KKT solve's captured CUDA graphs (default) or launch eagerly."""
        _lib.call("sdpx_b200_set_graphs", self._h, int(bool(on)))

    FORM_PLAIN, FORM_SPLIT = 0, 1

    def set_form(self, form: int):
        """Factorisation form of later solves: FORM_PLAIN (FP64) or FORM_SPLIT (split-precision
        INT8 tensor-core products for the large blocks, FP64 diagonal blocks and refinement)."""
        _lib.call("sdpx_b200_set_form", self._h, int(form))

    def kkt_paths(self) -> dict:
        """KKT solves of the last solve refined on the device (one graph each) and from the host."""
        d, h = C.c_uint64(), C.c_uint64()
        _lib.call("sdpx_b200_kkt_paths", self._h, C.byref(d), C.byref(h))
        return {"device": int(d.value), "host": int(h.value)}

    def schur_forms(self) -> dict:
        """PSD blocks in the rank-one Gram form and in the ordinary dense-column form."""
        g, o = C.c_uint32(), C.c_uint32()
        _lib.call("sdpx_b200_schur_forms", self._h, C.byref(g), C.byref(o))
        return {"gram": int(g.value), "ordinary": int(o.value)}

    def solver_name(self) -> str:
        need = C.c_uint64()
        _lib.call("sdpx_get_solver_name", self._h, None, 0, C.byref(need))
        buf = C.create_string_buffer(need.value)
        _lib.call("sdpx_get_solver_name", self._h, buf, need.value, C.byref(need))
        return buf.value.decode()

    def result_decimal(self) -> List[str]:
        need = C.c_uint64()
        _lib.call("sdpx_result_decimal", self._h, None, 0, C.byref(need))
        buf = C.create_string_buffer(need.value)
        _lib.call("sdpx_result_decimal", self._h, buf, need.value, C.byref(need))
        return [s.decode() for s in buf.raw[:need.value].split(b"\0")[:-1]]


class BatchSolver:
    """Many independent problems on one GPU: ``workers`` host threads each own one handle (its
    own CUDA stream) and re-prepare it for every instance they take, so instances run
    concurrently on the device and no device memory is allocated or freed between them.
    The GIL is released inside every library call."""

    def __init__(self, workers: int = 16, settings: Optional[DefaultSettings] = None,
                 graphs: bool = False):
        self.workers = max(1, int(workers))
        self.settings = settings
        self.graphs = graphs  # graph capture costs more than it saves on one small instance
        self._solvers: List[Optional[DefaultSolver]] = [None] * self.workers

    def solve(self, problems) -> List[Solution]:
        return self._run(problems, None)[0]

    def solve_adjoint(self, problems, grad) -> Tuple[List[Solution], list]:
        """Solve every problem and, on the same handle right after its solve, the adjoint of a
        loss with dL/dx = grad(index, solution): per instance (dq, db, dA) as
        ``DefaultSolver.adjoint`` returns them (None where the solve did not succeed)."""
        return self._run(problems, grad)

    def _run(self, problems, grad):
        import threading
        from concurrent.futures import ThreadPoolExecutor
        problems = list(problems)
        out: List[Optional[Solution]] = [None] * len(problems)
        grads: list = [None] * len(problems)
        lock = threading.Lock()
        nxt = [0]

        def work(w: int):
            while True:
                with lock:
                    i = nxt[0]
                    nxt[0] += 1
                if i >= len(problems):
                    return
                p = problems[i]
                s = self._solvers[w]
                if s is None:
                    s = DefaultSolver(p.P, p.q, p.A, p.b, p.cones, self.settings)
                    s.set_graphs(self.graphs)
                    self._solvers[w] = s
                else:
                    s.reprepare(p.P, p.q, p.A, p.b, p.cones, self.settings)
                sol = s.solve()
                out[i] = sol
                if grad is not None and sol.status in ("Solved", "AlmostSolved"):
                    grads[i] = s.adjoint(grad(i, sol))

        with ThreadPoolExecutor(self.workers) as ex:
            for f in [ex.submit(work, w) for w in range(self.workers)]:
                f.result()
        return out, grads


def solve_problem(prob, settings: Optional[DefaultSettings] = None) -> DefaultSolver:
    """Prepare and solve a ``problems.ConicProblem``."""
    s = DefaultSolver(prob.P, prob.q, prob.A, prob.b, prob.cones, settings)
    s.solve()
    return s


class KernelContext:
    """The kernel-level ABI (sdpxg_*): one hot-path operation per call on host arrays."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        _lib.call("sdpxg_ctx_create", device, 0, C.byref(h))
        self._h = h
        self.n = self.m = 0

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.load().sdpxg_ctx_destroy(h)
            except Exception:
                pass
            self._h = None

    def upload(self, A, psd_orders: Sequence[int], P=None):
        A = sp.csc_matrix(A, dtype=np.float64)
        self._A = _CscHold(A)
        self._P = _CscHold(sp.triu(sp.csc_matrix(P)).tocsc()) if P is not None else None
        orders = np.ascontiguousarray(psd_orders, dtype=np.uint64)
        _lib.call("sdpxg_problem_upload", self._h, C.byref(self._P.c) if self._P else None,
                  C.byref(self._A.c), orders.ctypes.data_as(_lib.PU64), orders.size)
        self.m, self.n = A.shape
        self.nlam = int(orders.sum())

    def upload_sampled(self, A_linear, psd_orders: Sequence[int], blocks: Sequence[dict], P=None):
        """sdpxg_problem_upload_sampled: blocks as in DefaultSolver.new_sampled (dim 1)."""
        A_linear = sp.csc_matrix(A_linear, dtype=np.float64)
        self._A = _CscHold(A_linear)
        self._P = _CscHold(sp.triu(sp.csc_matrix(P)).tocsc()) if P is not None else None
        orders = np.ascontiguousarray(psd_orders, dtype=np.uint64)
        arr = (_lib.SampledBlock * max(len(blocks), 1))()
        keep = []
        for i, blk in enumerate(blocks):
            Q = np.asfortranarray(blk["basis"], dtype=np.float64)
            w = np.ascontiguousarray(blk["weights"], dtype=np.float64)
            qv = Q.ravel(order="F").copy()
            keep += [qv, w]
            arr[i].row_start, arr[i].column_start = int(blk["row_start"]), int(blk["column_start"])
            arr[i].dim, arr[i].basis_rows, arr[i].basis_cols = int(blk.get("dim", 1)), Q.shape[0], Q.shape[1]
            arr[i].basis, arr[i].weights = _scalars(qv), _scalars(w)
        _lib.call("sdpxg_problem_upload_sampled", self._h, C.byref(self._P.c) if self._P else None,
                  C.byref(self._A.c), orders.ctypes.data_as(_lib.PU64), orders.size, arr, len(blocks))
        self.m, self.n = A_linear.shape
        self.nlam = int(orders.sum())

    def set_scaling(self, R_blocks, Rinv_blocks):
        """sdpxg_set_scaling: per PSD block R and R^-1 (lists of square arrays, cone order)."""
        R = np.concatenate([np.asfortranarray(r, dtype=np.float64).ravel(order="F") for r in R_blocks])
        Ri = np.concatenate([np.asfortranarray(r, dtype=np.float64).ravel(order="F") for r in Rinv_blocks])
        _lib.call("sdpxg_set_scaling", self._h, dptr(R), dptr(Ri))

    def nt_scale(self, s, z):
        s = np.ascontiguousarray(s, dtype=np.float64)
        z = np.ascontiguousarray(z, dtype=np.float64)
        lam = np.empty(self.nlam)
        st = C.c_uint32()
        _lib.call("sdpxg_nt_scale", self._h, dptr(s), dptr(z), dptr(lam), C.byref(st))
        return lam, st.value

    def identity_scaling(self):
        _lib.call("sdpxg_identity_scaling", self._h)

    def schur(self):
        H = np.empty((self.n, self.n), order="F")
        _lib.call("sdpxg_schur_assemble", self._h, H.ctypes.data_as(_lib.PD))
        return H

    def factor(self, shift, dynamic=True, eps=1e-13, delta=2e-7):
        st = C.c_uint32()
        _lib.call("sdpxg_factor", self._h, float(shift), int(dynamic), eps, delta, C.byref(st))
        return st.value

    def solve_many(self, rhs):
        rhs = np.asfortranarray(np.atleast_2d(np.asarray(rhs, dtype=np.float64).T).T)
        out = np.empty_like(rhs, order="F")
        _lib.call("sdpxg_solve_many", self._h, rhs.ctypes.data_as(_lib.PD),
                  out.ctypes.data_as(_lib.PD), rhs.shape[1])
        return out

    def kkt_solve(self, bx, bz):
        bx = np.ascontiguousarray(bx, dtype=np.float64)
        bz = np.ascontiguousarray(bz, dtype=np.float64)
        x, z = np.empty(self.n), np.empty(self.m)
        _lib.call("sdpxg_kkt_solve", self._h, dptr(bx), dptr(bz), dptr(x), dptr(z))
        return x, z

    def residual(self, bx, bz, x, z):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (bx, bz, x, z)]
        ex, ez = np.empty(self.n), np.empty(self.m)
        nrm = C.c_double()
        _lib.call("sdpxg_residual", self._h, *[dptr(a) for a in arrs], dptr(ex), dptr(ez), C.byref(nrm))
        return ex, ez, nrm.value

    def step_length(self, dz, ds, amax, mode=0):
        dz = np.ascontiguousarray(dz, dtype=np.float64)
        ds = np.ascontiguousarray(ds, dtype=np.float64)
        a = C.c_double()
        st = C.c_uint32()
        _lib.call("sdpxg_step_length", self._h, dptr(dz), dptr(ds), float(amax), int(mode),
                  C.byref(a), C.byref(st))
        return a.value, st.value

    RNS_INT8, RNS_FP64 = 0, 1

    def set_factor_form(self, form: int):
        """sdpxg_factor form: 0 plain FP64, 1 split precision (see DefaultSolver.set_form)."""
        _lib.call("sdpxg_set_factor_form", self._h, int(form))

    def split_dgemm_device(self, ta: str, tb: str, m: int, n: int, k: int, alpha: float, d_A: int,
                           lda: int, d_B: int, ldb: int, beta: float, d_C: int, ldc: int) -> int:
        """Split-precision (INT8 tensor-core) C = alpha op(A) op(B) + beta C on device buffers."""
        st = C.c_uint32()
        _lib.call("sdpxg_split_dgemm_device", self._h, ta.encode(), tb.encode(), m, n, k,
                  float(alpha), C.c_void_p(d_A), lda, C.c_void_p(d_B), ldb, float(beta),
                  C.c_void_p(d_C), ldc, C.byref(st))
        return st.value

    @staticmethod
    def i8_tuning() -> str:
        """The INT8 GEMM autotuner's table (one line per shape class: chosen configuration and the
        time of each)."""
        lib = _lib.load()
        req = C.c_uint64()
        lib.sdpx_b200_i8_tuning(None, 0, C.byref(req))
        buf = C.create_string_buffer(max(req.value, 1))
        _lib.call("sdpx_b200_i8_tuning", buf, req.value, C.byref(req))
        return buf.value.decode()

    def set_rns_form(self, form: int):
        """Residue products on INT8 tensor cores (RNS_INT8, the default) or in FP64 (RNS_FP64)."""
        _lib.call("sdpxg_rns_set_form", self._h, int(form))

    def rns_gemm(self, limbs: int, ta: str, tb: str, m: int, n: int, k: int, A: bytes, lda: int,
                 B: bytes, ldb: int, upper_only: bool = False, form: Optional[int] = None):
        """Exact MpFloat<limbs> product (raw element bytes in, raw bytes out)."""
        if form is not None:
            self.set_rns_form(form)
        esz = 8 * limbs + 8
        out = C.create_string_buffer(max(m * n * esz, 1))
        st = C.c_uint32()
        _lib.call("sdpxg_rns_gemm", self._h, limbs, ta.encode(), tb.encode(), m, n, k,
                  C.c_char_p(A), lda, C.c_char_p(B), ldb, int(upper_only), out, C.byref(st))
        return out.raw[:m * n * esz], st.value

    def rns_congruence(self, limbs: int, ta: str, m: int, k: int, A: bytes, lda: int, X: bytes,
                       ldx: int, upper_only: bool = False):
        """Exact op(A) X op(A)' of MpFloat<limbs> matrices (raw bytes in, raw bytes out)."""
        esz = 8 * limbs + 8
        out = C.create_string_buffer(max(m * m * esz, 1))
        st = C.c_uint32()
        _lib.call("sdpxg_rns_congruence", self._h, limbs, ta.encode(), m, k, C.c_char_p(A), lda,
                  C.c_char_p(X), ldx, int(upper_only), out, C.byref(st))
        return out.raw[:m * m * esz], st.value

    def rns_diag_congruence(self, limbs: int, m: int, k: int, A: bytes, lda: int, d: bytes,
                            upper_only: bool = False):
        """Exact A' diag(d) A (A k x m) of MpFloat<limbs> arrays: (raw bytes m x m, status)."""
        esz = 8 * limbs + 8
        out = C.create_string_buffer(max(m * m * esz, 1))
        st = C.c_uint32()
        _lib.call("sdpxg_rns_diag_congruence", self._h, limbs, m, k, C.c_char_p(A), lda, C.c_char_p(d),
                  int(upper_only), out, C.byref(st))
        return out.raw[:m * m * esz], st.value

    def rns_svec_quadratic(self, limbs: int, h: int, kmax: int, Q: bytes, x: bytes, sqrt2: bytes,
                           abs_q: bool = False):
        """Exact svec quadratic forms (one MpFloat<limbs> per basis column): (raw bytes, status)."""
        esz = 8 * limbs + 8
        out = C.create_string_buffer(max(kmax * esz, 1))
        st = C.c_uint32()
        _lib.call("sdpxg_rns_svec_quadratic", self._h, limbs, h, kmax, C.c_char_p(Q), int(abs_q),
                  C.c_char_p(x), C.c_char_p(sqrt2), out, C.byref(st))
        return out.raw[:kmax * esz], st.value

    def rns_symmetric_bilinear(self, limbs: int, h: int, columns: int, Q: bytes, X: bytes, pairs):
        """Exact q_a' X q_b for the given (a, b) pairs: (raw bytes, status)."""
        esz = 8 * limbs + 8
        flat = [int(v) for ab in pairs for v in ab]
        arr = (C.c_uint64 * max(len(flat), 1))(*flat)
        out = C.create_string_buffer(max(len(pairs) * esz, 1))
        st = C.c_uint32()
        _lib.call("sdpxg_rns_symmetric_bilinear", self._h, limbs, h, columns, C.c_char_p(Q), C.c_char_p(X),
                  len(pairs), arr, out, C.byref(st))
        return out.raw[:len(pairs) * esz], st.value

    def rns_gemm_blocks_upper(self, limbs: int, m: int, blocks):
        """Upper triangle of sum_b (diag(d_b) Y_b)' Y_b over blocks (y bytes, d bytes, columns,
        width): (raw bytes m x m, status)."""
        esz = 8 * limbs + 8
        widths = (C.c_uint64 * max(len(blocks), 1))(*[b[3] for b in blocks])
        counts = (C.c_uint64 * max(len(blocks), 1))(*[len(b[2]) for b in blocks])
        cols = [int(c) for b in blocks for c in b[2]]
        carr = (C.c_uint64 * max(len(cols), 1))(*cols)
        y = b"".join(b[0] for b in blocks)
        d = b"".join(b[1] for b in blocks)
        out = C.create_string_buffer(max(m * m * esz, 1))
        st = C.c_uint32()
        _lib.call("sdpxg_rns_gemm_blocks_upper", self._h, limbs, m, len(blocks), widths, counts,
                  C.c_char_p(y) if y else None, C.c_char_p(d) if d else None, carr, out, C.byref(st))
        return out.raw[:m * m * esz], st.value

    def mp_nt_scale(self, limbs: int, orders, s: bytes, z: bytes):
        """MPFR NT scaling of PSD blocks (svec s, z as raw MpFloat bytes, concatenated): returns
        (lambda, lisqrt, R, Rinv, G raw bytes concatenated per block, block status list, status)."""
        esz = 8 * limbs + 8
        nb = len(orders)
        lin = sum(orders)
        sq = sum(n * n for n in orders)
        arr = (C.c_uint64 * max(nb, 1))(*orders)
        lam = C.create_string_buffer(max(lin * esz, 1))
        lis = C.create_string_buffer(max(lin * esz, 1))
        R = C.create_string_buffer(max(sq * esz, 1))
        Ri = C.create_string_buffer(max(sq * esz, 1))
        G = C.create_string_buffer(max(sq * esz, 1))
        bst = (C.c_int32 * max(nb, 1))()
        st = C.c_uint32()
        _lib.call("sdpxg_mp_nt_scale", self._h, limbs, nb, arr, C.c_char_p(s), C.c_char_p(z), lam, lis, R, Ri,
                  G, bst, C.byref(st))
        return (lam.raw[:lin * esz], lis.raw[:lin * esz], R.raw[:sq * esz], Ri.raw[:sq * esz],
                G.raw[:sq * esz], list(bst)[:nb], st.value)

    def mp_step_length(self, limbs: int, orders, primal: bool, d: bytes, Rx: bytes, lisqrt: bytes,
                       alpha_max: bytes):
        """MPFR step-length bounds per PSD block: returns (alpha raw bytes per block, path list,
        status)."""
        esz = 8 * limbs + 8
        nb = len(orders)
        arr = (C.c_uint64 * max(nb, 1))(*orders)
        al = C.create_string_buffer(max(nb * esz, 1))
        pth = (C.c_int32 * max(nb, 1))()
        st = C.c_uint32()
        _lib.call("sdpxg_mp_step_length", self._h, limbs, nb, arr, int(primal), C.c_char_p(d), C.c_char_p(Rx),
                  C.c_char_p(lisqrt), C.c_char_p(alpha_max), al, pth, C.byref(st))
        return al.raw[:nb * esz], list(pth)[:nb], st.value

    def mp_ldl(self, limbs: int, n: int, A: bytes, lda: int, reg: Optional[bytes] = None):
        """The reference's dense MPFR LDL' of an n x n MpFloat<limbs> matrix (raw bytes):
        returns (L bytes n x n, dinv bytes n, status)."""
        esz = 8 * limbs + 8
        L = C.create_string_buffer(max(n * n * esz, 1))
        D = C.create_string_buffer(max(n * esz, 1))
        st = C.c_uint32()
        _lib.call("sdpxg_mp_ldl", self._h, limbs, n, C.c_char_p(A), lda,
                  C.c_char_p(reg) if reg is not None else None, L, D, C.byref(st))
        return L.raw[:n * n * esz], D.raw[:n * esz], st.value

    def mp_potrf(self, limbs: int, uplo: str, n: int, A: bytes, lda: int):
        """The reference's exact MpFloat Cholesky (xpotrf): returns (factor bytes, info, status)."""
        buf = C.create_string_buffer(bytes(A), len(A))
        info, st = C.c_int32(), C.c_uint32()
        _lib.call("sdpxg_mp_potrf", self._h, limbs, uplo.encode(), n, buf, lda, C.byref(info), C.byref(st))
        return buf.raw[:len(A)], info.value, st.value

    def rns_gemm_device(self, limbs: int, ta: str, tb: str, m: int, n: int, k: int, d_A: int,
                        lda: int, d_B: int, ldb: int, d_C: int, upper_only: bool = False):
        """Exact product on device buffers (addresses of MpFloat arrays in device memory)."""
        st = C.c_uint32()
        _lib.call("sdpxg_rns_gemm_device", self._h, limbs, ta.encode(), tb.encode(), m, n, k,
                  C.c_void_p(d_A), lda, C.c_void_p(d_B), ldb, int(upper_only), C.c_void_p(d_C),
                  C.byref(st))
        return st.value

    def cone_apply(self, op, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(self.m)
        _lib.call("sdpxg_cone_apply", self._h, int(op), dptr(x), dptr(y))
        return y
