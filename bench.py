#!/usr/bin/env python
"""Time-to-gap benchmark of the SDPX interior-point hot path on B200.

Workload: the bootstrap-shaped Float64 SDP -- 32 PSD blocks of order U{10..60} with Chebyshev
bases, m = 2000 constraints of four rank-one terms each, seed 0 -- solved to the reference's
default gap 1e-8 with the condensed KKT form.  One "step" is one complete solve to the gap.
Both factorisation forms solve it in the same process: the plain FP64 form and the
split-precision form (INT8 tensor-core Ozaki-II products for the large blocks of the Schur
factorisation and its inverse, FP64 diagonal blocks, pivots and refinement).

  value     time-to-gap (s) of the split-precision form with the problem already resident in HBM
            (sdpx_solve), max over ranks; `forms` gives both forms and plain / split
  precision_f64  the same comparison on the 64-block m = 4000 workload at Float64
  rns_256   exact 256-bit products (2000^3) in both residue forms (INT8 tensor cores, FP64)
  e2e       the same metric through the C ABI with host buffers in the ABI's layout (built before
            the timed region, as a C caller holds them): sdpx_prepare (copy and validation, Ruiz
            equilibration, operator packing, H2D upload) + sdpx_solve + sdpx_result_f64 (D2H) +
            sdpx_destroy
  roofline  the dominant device phase of the split form, timed with CUDA events on the library's
            stream; int8_gemm: the INT8 tensor-core GEMM's achieved TOP/s against an INT8 GEMM peak
            measured in the same run
  cpu_baseline  the oracle (reference-algorithm CPU restatement, numpy/OpenBLAS, all host cores)
            solving the same instance to the gap once (measured, not projected)

``--impl reference`` times the reference's CPU path (the oracle port; the Rust reference cannot be
built on this image) on rank 0 and prints the same metric.  Multi-GPU runs are independent
replicas (the solve does not shard): each rank solves the same instance on its own GPU.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "sdpx.rs_b200"))

METRIC = ("time-to-gap 1e-8 (Float64): split-precision form (INT8 tensor-core Ozaki-II products, "
          "FP64 pivots and refinement) vs the plain FP64 GPU form")
WORKLOAD = {"workload": "rank1_sdp: 32 PSD blocks n_j~U{10..60}, Chebyshev bases s_j=2n_j, "
                        "m=2000 constraints x 4 rank-one terms, seed 0, gap 1e-8, kkt_form condensed",
            "blocks": 32, "m": 2000, "seed": 0, "precision_bits": 53,
            "l2": "inputs resident; the Schur complement (32 MB) and its factor are rewritten every "
                  "iteration, per-solve working set ~0.2 GB > 126 MB L2"}


def make_problem():
    from sdpx_b200 import problems
    return problems.rank1_sdp(32, 2000, seed=0)


def dist_backend():
    """NCCL between GPUs; gloo where there is no GPU (the multi-process tests on CPU).
    SDPX_B200_DIST_BACKEND overrides."""
    b = os.environ.get("SDPX_B200_DIST_BACKEND")
    if b:
        return b
    import torch
    return "nccl" if torch.cuda.is_available() else "gloo"


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = dist_backend()
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world, value):
    """The largest of the ranks' values (device timings: the slowest rank sets the job time)."""
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in Path(self.path).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons, "samples": len(rows)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def fp64_gemm_peak():
    """cuBLAS DGEMM throughput on this GPU (TFLOP/s): the FP64 roofline denominator."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(4):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


def schur_model(prob, gram=False):
    """Algorithmic work per launch of the timed phases (flop or bytes).

    factor: m^3/3 (Cholesky of the m x m Schur complement); trinv: m^3/3 (inverse of the
    triangular factor); assemble: sum_j 4 k_j n_j^3 + k_j^2 n_j (n_j + 1) in the ordinary form,
    sum_j 8 n_j^3 + 3 k_j^2 in the rank-one Gram form; scale: 20 n_j^3 per block; trisolve and
    symv: 8 m^2 bytes (two triangles, or the full matrix once).
    """
    import numpy as np
    n = prob.n
    orders = [d for _, d in prob.cones]
    A = prob.A.tocsc()
    k = []
    r0 = 0
    for d in orders:
        t = d * (d + 1) // 2
        sub = A[r0:r0 + t, :]
        k.append(int(np.count_nonzero(sub.getnnz(axis=0))))
        r0 += t
    if gram:
        assemble = sum(8.0 * d ** 3 + 3.0 * kj * kj for kj, d in zip(k, orders))
    else:
        assemble = sum(4.0 * kj * d ** 3 + 2.0 * kj * kj * d * (d + 1) / 2 for kj, d in zip(k, orders))
    return {"n": n, "factor_flops": n ** 3 / 3.0, "trisolve_bytes": 8.0 * n * n,
            "symv_bytes": 8.0 * n * n, "assemble_flops": assemble,
            "scale_flops": sum(20.0 * d ** 3 for d in orders)}


def traffic_from_profile(phase):
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        d = json.loads(p.read_text())
        v = d.get(phase)
        if isinstance(v, dict):
            return v.get("bytes_per_launch")
    return None


def cpu_baseline(prob):
    """The oracle solved to the gap once on the host cores: a measured time-to-gap, no projection."""
    from oracle import ipm
    t0 = time.perf_counter()
    r = ipm.Solver(prob, ipm.Settings()).solve()
    dt = time.perf_counter() - t0
    return {"value": dt, "unit": "s", "cores": os.cpu_count(), "kind": "port",
            "sample": f"one complete oracle solve (numpy + OpenBLAS, all host threads) of the "
                      f"same instance to the gap: status {r.status}, {r.iterations} iterations",
            "iterations": r.iterations, "status": r.status,
            "seconds_per_iteration": dt / max(r.iterations, 1)}


def _oracle_warmup():
    """Imports, BLAS thread pools and page faults: one small oracle solve (untimed)."""
    from oracle import ipm
    from sdpx_b200 import problems
    ipm.solve(problems.dense_sdp(16, 40, seed=0))


REFERENCE_BUDGET_S = 150.0  # wall-clock cap of the reference arm's timed solves


def run_reference(args, world, rank):
    """The reference's CPU path (the oracle port: the Rust reference cannot be built here) timed to
    the gap on rank 0.  Every timed step is one complete solve; steps beyond what fits in
    REFERENCE_BUDGET_S are not run (at least one always is), and the line says how many ran."""
    if rank != 0:
        return 0
    prob = make_problem()
    for _ in range(args.warmup):
        _oracle_warmup()
    vals = []
    t0 = time.perf_counter()
    for _ in range(max(args.steps, 1)):
        vals.append(cpu_baseline(prob))
        elapsed = time.perf_counter() - t0
        if elapsed + elapsed / len(vals) > REFERENCE_BUDGET_S:
            break
    wall = time.perf_counter() - t0
    v = statistics.mean(x["value"] for x in vals)
    cb = dict(vals[-1])
    cb["value"] = v
    cb["sample"] += f"; {len(vals)} complete solve(s) timed"
    line = {"metric": METRIC, "value": v, "unit": "s", "n_gpus": args.gpus, "steps": len(vals),
            "steps_requested": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * wall / len(vals), "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": WORKLOAD,
            "impl": "reference", "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def time_solves(solver, steps):
    """Device-clock seconds per solve (CUDA events around `steps` solves; every solve returns
    to the host with its result, so the events bracket complete solves), wall seconds per solve
    and kernel launches."""
    import torch
    from sdpx_b200 import _lib
    lib = _lib.load()
    launches0 = lib.sdpx_b200_launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record()
    t0 = time.perf_counter()
    for _ in range(steps):
        solver.solve()
    ev1.record()
    torch.cuda.synchronize()
    wall = (time.perf_counter() - t0) / steps
    return ev0.elapsed_time(ev1) / 1e3 / steps, wall, lib.sdpx_b200_launch_count() - launches0


def int8_peak():
    """cuBLASLt INT8 GEMM throughput (torch._int_mm, 8192^3): the INT8 roofline denominator
    (INT8 is not in MEASURED_PEAKS.json)."""
    import torch
    n = 8192
    a = torch.randint(-128, 127, (n, n), dtype=torch.int8, device="cuda")
    b = torch.randint(-128, 127, (n, n), dtype=torch.int8, device="cuda")
    for _ in range(2):
        torch._int_mm(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(4):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch._int_mm(a, b)
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


def i8_measure(fn):
    """Run fn with the INT8 GEMM launches timed: (ms, executed ops, algorithmic ops, launches)."""
    from sdpx_b200 import _lib
    lib = _lib.load()
    lib.sdpx_b200_set_i8_timing(1)
    fn()
    ms, ops, alg = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    cnt = ctypes.c_uint64()
    lib.sdpx_b200_i8_times(ctypes.byref(ms), ctypes.byref(ops), ctypes.byref(alg), ctypes.byref(cnt))
    lib.sdpx_b200_set_i8_timing(0)
    return ms.value, ops.value, alg.value, cnt.value


def precision_f64(args):
    """The precision workload at Float64 (64 blocks, m = 4000): both forms to the gap."""
    from sdpx_b200 import problems
    from sdpx_b200.solver import DefaultSettings, DefaultSolver
    prob = problems.rank1_sdp(64, 4000, seed=0)
    out = {"workload": "rank1_sdp: 64 PSD blocks n_j~U{10..60}, m=4000, seed 0, gap 1e-8, Float64"}
    for name, form in (("plain", 0), ("split", 1)):
        s = DefaultSolver(prob.P, prob.q, prob.A, prob.b, prob.cones, DefaultSettings(kkt_form="condensed"))
        s.set_form(form)
        s.solve()
        dev, wall, _ = time_solves(s, max(2, args.steps // 2))
        out[name] = {"s": dev, "status": s.solution.status, "iterations": s.solution.iterations,
                     "objective": s.solution.obj_val}
        s.close()
    out["plain_over_split"] = out["plain"]["s"] / out["split"]["s"]
    return out


def dense_c0(args):
    """The plain Float64 dense SDP (one PSD block n = 50, m = 200 dense constraints, ordinary Schur
    form on the FP64 tensor cores): time to the gap per solve, problem resident."""
    from sdpx_b200 import problems
    from sdpx_b200.solver import DefaultSettings, DefaultSolver
    prob = problems.dense_sdp(50, 200, seed=0)
    s = DefaultSolver(prob.P, prob.q, prob.A, prob.b, prob.cones, DefaultSettings(kkt_form="condensed"))
    s.solve()
    dev, wall, _ = time_solves(s, max(3, args.steps))
    out = {"workload": "dense_sdp: one PSD block n=50, m=200 dense constraints, seed 0, gap 1e-8, Float64",
           "s": dev, "status": s.solution.status, "iterations": s.solution.iterations,
           "objective": s.solution.obj_val, "iterations_per_s": s.solution.iterations / dev}
    s.close()
    return out


def _random_mp(count, limbs, rng, spread=4):
    """Random MpFloat<limbs> values in the reference's layout (top mantissa bit set, sign in the
    kind, exponents in [-spread, spread], 5 % zeros) as raw bytes."""
    import numpy as np
    dt = np.dtype([("l", "<u8", (limbs,)), ("kind", "<i4"), ("exp", "<i4")])
    a = np.zeros(count, dtype=dt)
    a["l"] = rng.integers(0, 2 ** 63, size=(count, limbs), dtype=np.uint64) * np.uint64(2) + np.uint64(1)
    a["l"][:, limbs - 1] |= np.uint64(1) << np.uint64(63)
    a["kind"] = np.where(rng.random(count) < 0.5, 3, -3)
    a["exp"] = rng.integers(-spread, spread + 1, size=count)
    zero = rng.random(count) < 0.05
    a["l"][zero] = 0
    a["kind"][zero] = 2
    a["exp"][zero] = 0
    return a.tobytes()


def rns_256(args, peak_i8):
    """Exact 256-bit products (MpFloat<4>) of 2000 x 2000 matrices, both residue forms, on device
    buffers: the trailing-update shape of the precision workload's factorisation."""
    import numpy as np
    import torch
    from sdpx_b200.solver import KernelContext
    n, limbs = 2000, 4
    rng = np.random.default_rng(7)
    esz = 8 * limbs + 8
    dA = torch.from_numpy(np.frombuffer(_random_mp(n * n, limbs, rng), dtype=np.uint8).copy()).cuda()
    dB = torch.from_numpy(np.frombuffer(_random_mp(n * n, limbs, rng), dtype=np.uint8).copy()).cuda()
    outs, res = {}, {"shape": f"{n} x {n} x {n}, 256-bit (MpFloat<4>), exponent spread 4, device buffers"}
    ctx = KernelContext()
    for name, form in (("int8", 0), ("fp64", 1)):
        ctx.set_rns_form(form)
        dC = torch.zeros(n * n * esz, dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()
        ctx.rns_gemm_device(limbs, "N", "N", n, n, n, dA.data_ptr(), n, dB.data_ptr(), n, dC.data_ptr())
        reps = 2
        t0 = time.perf_counter()
        for _ in range(reps):
            ctx.rns_gemm_device(limbs, "N", "N", n, n, n, dA.data_ptr(), n, dB.data_ptr(), n, dC.data_ptr())
        dt = (time.perf_counter() - t0) / reps
        res[name] = {"s": dt, "exact_macs_per_s": n ** 3 / dt}
        if form == 0:
            ms, ops, alg, cnt = i8_measure(lambda: ctx.rns_gemm_device(
                limbs, "N", "N", n, n, n, dA.data_ptr(), n, dB.data_ptr(), n, dC.data_ptr()))
            res[name]["i8_gemm"] = {"ms": ms, "launches": cnt, "tops_executed": ops / ms / 1e9,
                                    "tops_algorithmic": alg / ms / 1e9,
                                    "frac_of_int8_peak": (ops / ms / 1e9) / peak_i8}
        outs[name] = dC.cpu().numpy().tobytes()
        del dC
    res["bitwise_equal_forms"] = outs["int8"] == outs["fp64"]
    res["fp64_over_int8"] = res["fp64"]["s"] / res["int8"]["s"]
    return res


def _mp_from_f64(vals, limbs):
    """Binary64 values as MpFloat<limbs> bytes (exact: the 53-bit mantissa in the top limb)."""
    import numpy as np
    v = np.asarray(vals, dtype=np.float64)
    f, e = np.frexp(v)
    dt = np.dtype([("l", "<u8", (limbs,)), ("kind", "<i4"), ("exp", "<i4")])
    a = np.zeros(v.size, dtype=dt)
    a["l"][:, limbs - 1] = (np.abs(f) * 2.0 ** 64).astype(np.uint64)
    a["kind"] = np.where(v == 0, 2, np.where(f < 0, -3, 3))
    a["exp"] = np.where(v == 0, 0, e)
    return a.tobytes()


def mp_chain_256(args, m_ldl):
    """The per-iteration MPFR kernels of the 256-bit precision workload (64 PSD blocks of the
    bootstrap generator's orders, Schur dimension m_ldl): NT scaling of every block, the step
    bounds of both sides, and the dense LDL' of an m_ldl x m_ldl 256-bit matrix in both residue
    forms (the trailing products on the INT8 tensor cores or in FP64).  Host-built interior
    points, directions and a diagonally dominant Schur stand-in, all device work timed by
    wall clock around the synchronous entry points (each LDL' form after one warm-up call)."""
    import ctypes as C
    import numpy as np
    import torch
    from sdpx_b200 import _lib, problems
    from sdpx_b200.solver import KernelContext
    limbs, esz = 4, 40
    rng = np.random.default_rng(11)
    orders = [d for _, d in problems.rank1_sdp(64, 4000, seed=0).cones]

    def svec_spd(k):
        A = rng.standard_normal((k, k))
        S = A @ A.T / k + 0.3 * np.eye(k)
        return [S[i, j] if i == j else S[i, j] * np.sqrt(2.0) for j in range(k) for i in range(j + 1)]

    def svec_sym(k):
        A = rng.standard_normal((k, k))
        S = (A + A.T) / 2
        return [S[i, j] if i == j else S[i, j] * np.sqrt(2.0) for j in range(k) for i in range(j + 1)]
    s = _mp_from_f64(np.concatenate([svec_spd(k) for k in orders]), limbs)
    z = _mp_from_f64(np.concatenate([svec_spd(k) for k in orders]), limbs)
    ctx = KernelContext()
    res = {"workload": f"64 PSD blocks (orders of rank1_sdp(64, 4000, seed 0), n {min(orders)}..{max(orders)}), "
                       f"256-bit (MpFloat<4>); LDL' of a {m_ldl} x {m_ldl} diagonally dominant matrix"}
    t0 = time.perf_counter()
    lam, lis, R, Rinv, G, bst, st = ctx.mp_nt_scale(limbs, orders, s, z)
    res["nt_scale_s"] = time.perf_counter() - t0
    res["nt_scale_status"] = sorted(set(bst))
    d = _mp_from_f64(np.concatenate([svec_sym(k) for k in orders]), limbs)
    amax = _mp_from_f64([1.0], limbs)
    t0 = time.perf_counter()
    _, pz, _ = ctx.mp_step_length(limbs, orders, False, d, R, lis, amax)
    _, ps, _ = ctx.mp_step_length(limbs, orders, True, d, Rinv, lis, amax)
    res["step_bounds_s"] = time.perf_counter() - t0
    res["step_paths"] = {str(p): (pz + ps).count(p) for p in sorted(set(pz + ps))}
    m = m_ldl
    off = rng.standard_normal((m, m))
    H = (off + off.T) / 2
    H[np.diag_indices(m)] = 4.0 * m
    src = torch.from_numpy(np.frombuffer(_mp_from_f64(H.T.ravel(), limbs), dtype=np.uint8).copy()).cuda()
    A = torch.empty_like(src)
    dinv = torch.zeros(m * esz, dtype=torch.uint8, device="cuda")
    lib = _lib.load()
    outs = {}
    for name, form in (("int8", 0), ("fp64", 1)):
        ctx.set_rns_form(form)
        for rep in range(2):  # the first call warms up (the INT8 GEMM's autotuner times its shapes)
            A.copy_(src)
            torch.cuda.synchronize()
            stw = C.c_uint32()
            t0 = time.perf_counter()
            rc = lib.sdpxg_mp_ldl_device(ctx._h, limbs, m, C.c_void_p(A.data_ptr()), m, None,
                                         C.c_void_p(dinv.data_ptr()), C.byref(stw))
            torch.cuda.synchronize()
            dt = time.perf_counter() - t0
            if rc != 0:
                raise RuntimeError(_lib.last_error())
        res[f"ldl_{name}_s"] = dt
        outs[name] = dinv.cpu().numpy().tobytes()
    ctx.set_rns_form(0)
    res["ldl_bitwise_equal_forms"] = outs["int8"] == outs["fp64"]
    res["ldl_exact_macs"] = m ** 3 / 6
    res["per_iteration_int8_s"] = res["nt_scale_s"] + res["step_bounds_s"] + res["ldl_int8_s"]
    res["per_iteration_fp64_s"] = res["nt_scale_s"] + res["step_bounds_s"] + res["ldl_fp64_s"]
    res["fp64_over_int8"] = res["per_iteration_fp64_s"] / res["per_iteration_int8_s"]
    return res


def run_ours(args, world, rank, local):
    import numpy as np
    import torch
    os.environ["SDPX_B200_DEVICE"] = str(local)
    torch.cuda.set_device(local)
    from sdpx_b200 import _lib
    from sdpx_b200.solver import CProblem, DefaultSettings, DefaultSolver

    prob = make_problem()
    settings = DefaultSettings(kkt_form="condensed")
    arms = {}
    for name, form in (("plain", DefaultSolver.FORM_PLAIN), ("split", DefaultSolver.FORM_SPLIT)):
        s = DefaultSolver(prob.P, prob.q, prob.A, prob.b, prob.cones, settings)
        s.set_form(form)
        for _ in range(args.warmup):
            s.solve()
        arms[name] = s
    clocks = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    timed = {}
    for name in ("plain", "split"):  # the chosen (split) arm last: the headline value
        timed[name] = time_solves(arms[name], args.steps)
    barrier(world)
    clk = clocks.stop()
    solver = arms["split"]
    dev_s, wall, launches = timed["split"]
    value = max_over_ranks(world, dev_s)
    plain_s = max_over_ranks(world, timed["plain"][0])
    iters, status = solver.solution.iterations, solver.solution.status
    forms = {name: {"s": max_over_ranks(world, timed[name][0]), "status": arms[name].solution.status,
                    "iterations": arms[name].solution.iterations,
                    "objective": arms[name].solution.obj_val,
                    "gpu_launches_per_solve": timed[name][2] / args.steps} for name in arms}
    forms["plain_over_split"] = plain_s / value
    timed_host = {k: round(v, 5) for k, v in solver.info.phase_times.items()}
    # per-phase device times from one more solve per arm with phase events on (outside the
    # timed region: the events synchronize the host at every phase boundary)
    ktimes = {}
    for name, s in arms.items():
        s.set_kernel_timing(True)
        s.solve()
        ktimes[name] = s.kernel_times()
        s.set_kernel_timing(False)
    # INT8 tensor-core GEMM of the split form, timed inside one more solve
    i8 = i8_measure(lambda: solver.solve())

    # ---- end-to-end through the C ABI with host buffers (split form) ----
    e2e_times = []
    h2d = d2h = 0
    lib = _lib.load()
    cnt_h2d, cnt_d2h = ctypes.c_uint64(), ctypes.c_uint64()
    for i in range(args.warmup + args.steps):
        # the problem in the C ABI's host layout (what a caller of sdpx_prepare holds)
        cp = CProblem(prob.P, prob.q, prob.A, prob.b, prob.cones, settings)
        barrier(world)
        torch.cuda.synchronize()
        lib.sdpx_b200_transfer_bytes(ctypes.byref(cnt_h2d), ctypes.byref(cnt_d2h))
        b0 = (cnt_h2d.value, cnt_d2h.value)
        t0 = time.perf_counter()
        s2 = DefaultSolver.from_c_problem(cp)  # sdpx_prepare: validate, equilibrate, upload
        s2.set_form(DefaultSolver.FORM_SPLIT)
        s2.solve()                             # sdpx_solve, sdpx_get_info, sdpx_result_f64
        s2.close()                             # sdpx_destroy
        torch.cuda.synchronize()
        if i >= args.warmup:
            e2e_times.append(time.perf_counter() - t0)
            lib.sdpx_b200_transfer_bytes(ctypes.byref(cnt_h2d), ctypes.byref(cnt_d2h))
            h2d, d2h = cnt_h2d.value - b0[0], cnt_d2h.value - b0[1]  # bytes the library copied
    e2e = max_over_ranks(world, statistics.mean(e2e_times))
    model = schur_model(prob, gram=solver.schur_forms()["ordinary"] == 0)

    # ---- roofline of the dominant device phase of the chosen (split) arm ----
    hbm, hbm_kind = measured_peaks()
    kt = ktimes["split"]
    dom = max(kt, key=lambda k: kt[k][0])
    ms, cnt = kt[dom]
    per = ms / 1e3 / max(cnt, 1)
    peak_i8 = int8_peak()
    nh = model["n"] // 2
    half_flops = ((nh + 63) // 64 * 64) ** 3 / 3.0
    if dom == "split":
        achieved = i8[1] / (i8[0] / 1e3) / 1e12
        roof = {"bound": "tensor", "achieved": achieved, "peak": peak_i8, "unit": "TOP/s",
                "frac": achieved / peak_i8, "traffic": traffic_from_profile("i8_gemm"),
                "kernel": "k_i8_mod_gemm", "launch_ms": i8[0] / max(i8[3], 1),
                "note": "INT8 pipe; peak = cuBLASLt INT8 GEMM 8192^3 (torch._int_mm) measured in this run"}
    elif dom in ("factor", "trinv", "assemble", "scale", "cone", "step"):
        fp64 = fp64_gemm_peak()
        flops = {"factor": half_flops, "trinv": half_flops,
                 "assemble": model["assemble_flops"], "scale": model["scale_flops"]}.get(dom)
        if flops is None:
            flops = sum(4.0 * d ** 3 for _, d in prob.cones)
        achieved = flops / per / 1e12
        roof = {"bound": "tensor", "achieved": achieved, "peak": fp64, "unit": "TFLOP/s",
                "frac": achieved / fp64, "traffic": traffic_from_profile(dom),
                "kernel": "k_chol_dataflow" if dom == "factor" else dom, "launch_ms": per * 1e3,
                "note": "FP64 pipe; the split form factors two diagonal halves of order ~m/2 "
                        "(n^3/3 flop per launch); peak = cuBLAS DGEMM 8192^3 measured in this run "
                        "(FP64 is not in MEASURED_PEAKS.json)"}
    else:
        nbytes = model["trisolve_bytes"] if dom == "trisolve" else model["symv_bytes"]
        achieved = nbytes / per / 1e9
        roof = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "traffic": traffic_from_profile(dom), "kernel": dom,
                "launch_ms": per * 1e3, "note": f"peak {hbm_kind} (MEASURED_PEAKS.json hbm_gbs)"}
    i8_obj = {"ms_per_solve": i8[0], "launches_per_solve": i8[3],
              "tops_executed": i8[1] / (i8[0] / 1e3) / 1e12 if i8[0] else None,
              "tops_algorithmic": i8[2] / (i8[0] / 1e3) / 1e12 if i8[0] else None,
              "int8_peak_tops": peak_i8}
    phases = {arm: {k: {"ms_total": v[0], "launches": v[1]} for k, v in kt_.items()}
              for arm, kt_ in ktimes.items()}

    extra = {}
    if rank == 0 and not args.quick:
        extra["precision_f64"] = precision_f64(args)
        extra["dense_c0"] = dense_c0(args)
        extra["rns_256"] = rns_256(args, peak_i8)
        try:  # a supplementary measurement: its failure is reported, the headline line still prints
            extra["mp_256_iteration"] = mp_chain_256(args, 4000)
        except Exception as e:  # noqa: BLE001
            extra["mp_256_iteration"] = {"error": f"{type(e).__name__}: {e}"}
    cb = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cb = cpu_baseline(prob)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": value * 1e3,
                "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": dict(WORKLOAD, parallelism=f"replicas{world}"),
                "status": status, "iterations": iters, "wall_s_per_step": wall,
                "forms": forms,
                "e2e": {"value": e2e, "unit": "s", "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h},
                "roofline": roof, "int8_gemm": i8_obj, "phases": phases,
                "host_phase_s_timed_solve": timed_host,
                "gpu_launches": int(launches),
                "clocks": clk, "cpu_baseline": cb}
        line.update(extra)
        print(json.dumps(line))
    return 0


def run_i8(args, world, rank, local):
    """INT8 tensor-core GEMM microbenchmark: the cuBLASLt INT8 peak (torch._int_mm 8192^3), the
    split-precision DGEMM (Ozaki-II, 16 INT8 modular products) of --size^3 against cuBLAS DGEMM,
    and the exact 256-bit RNS product of --size^3 (INT8 form) -- each with the INT8 kernel's own
    event-timed TOP/s."""
    import numpy as np
    import torch
    torch.cuda.set_device(local)
    from sdpx_b200.solver import KernelContext
    n, reps = args.size, args.reps
    ctx = KernelContext(local)
    rng = np.random.default_rng(3)
    A = torch.from_numpy(rng.standard_normal((n, n))).cuda()
    B = torch.from_numpy(rng.standard_normal((n, n))).cuda()
    C = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    split = lambda: ctx.split_dgemm_device("N", "N", n, n, n, 1.0, A.data_ptr(), n, B.data_ptr(), n, 0.0,
                                           C.data_ptr(), n)
    split()
    t0 = time.perf_counter()
    for _ in range(reps):
        split()
    t_split = (time.perf_counter() - t0) / reps
    ms, ops, alg, cnt = i8_measure(split)
    # column-major device buffers: C = A B in BLAS terms is B^T A^T on torch's row-major views
    ref = (A.T @ B.T).T
    err = float((C - ref).abs().max() / ref.abs().max())
    torch.cuda.synchronize()
    s_, e_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s_.record()
    for _ in range(reps):
        torch.matmul(A, B)
    e_.record()
    torch.cuda.synchronize()
    t_dgemm = s_.elapsed_time(e_) / 1e3 / reps
    del A, B, C, ref
    torch.cuda.empty_cache()
    peak = int8_peak()
    limbs, esz = 4, 40
    dA = torch.from_numpy(np.frombuffer(_random_mp(n * n, limbs, rng), dtype=np.uint8).copy()).cuda()
    dB = torch.from_numpy(np.frombuffer(_random_mp(n * n, limbs, rng), dtype=np.uint8).copy()).cuda()
    dC = torch.zeros(n * n * esz, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    rns = lambda: ctx.rns_gemm_device(limbs, "N", "N", n, n, n, dA.data_ptr(), n, dB.data_ptr(), n, dC.data_ptr())
    rns()
    t0 = time.perf_counter()
    for _ in range(reps):
        rns()
    t_rns = (time.perf_counter() - t0) / reps
    rms, rops, ralg, rcnt = i8_measure(rns)
    if rank == 0:
        print(json.dumps({
            "metric": "INT8 tensor-core GEMM throughput (tcgen05 kind::i8 modular GEMM)", "value": ops / ms / 1e9,
            "unit": "TOP/s", "n_gpus": 1, "steps": reps, "warmup": 1, "higher_is_better": True,
            "data": "synthetic", "int8_peak_tops": peak,
            "split_dgemm": {"n": n, "s": t_split, "tflops_fp64_equivalent": 2.0 * n ** 3 / t_split / 1e12,
                            "cublas_dgemm_s": t_dgemm, "dgemm_over_split": t_dgemm / t_split,
                            "max_rel_err_vs_dgemm": err, "i8_gemm_ms": ms, "i8_launches": cnt,
                            "i8_tops_executed": ops / ms / 1e9, "i8_tops_algorithmic": alg / ms / 1e9,
                            "frac_of_int8_peak": ops / ms / 1e9 / peak},
            "rns_256": {"n": n, "s": t_rns, "i8_gemm_ms": rms, "i8_launches": rcnt,
                        "i8_tops_executed": rops / rms / 1e9, "i8_tops_algorithmic": ralg / rms / 1e9,
                        "frac_of_int8_peak": rops / rms / 1e9 / peak},
            "autotuner": ctx.i8_tuning().strip().splitlines()}))
    return 0


BATCH_METRIC = "instances/s to gap 1e-8 (Float64), batch of independent small SDPs"


def run_batch(args, world, rank, local):
    """Batching workload: independent dense SDPs, one PSD block each, n ~ U{8..64},
    m ~ U{20..300}, data as the dense generator from seed + index.  The instances are generated
    before the timed region; each timed step solves the whole batch from host buffers through
    BatchSolver (one re-prepared handle and stream per worker thread), so a step includes every
    instance's validation, equilibration, upload, solve and result read."""
    import numpy as np
    import torch
    os.environ["SDPX_B200_DEVICE"] = str(local)
    torch.cuda.set_device(local)
    from oracle import ipm
    from sdpx_b200 import problems as Pm
    from sdpx_b200.solver import BatchSolver, DefaultSettings

    count = args.instances or 4096
    probs = Pm.batch_sdps(count, seed=1000 * rank)  # replicas: each rank its own instances
    settings = DefaultSettings(kkt_form="condensed")
    bs = BatchSolver(workers=args.workers, settings=settings)
    for _ in range(args.warmup):
        bs.solve(probs[: min(count, 4 * args.workers)])
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        sols = bs.solve(probs)
    torch.cuda.synchronize()
    wall = (time.perf_counter() - t0) / args.steps
    wall = max_over_ranks(world, wall)
    statuses = {}
    for s_ in sols:
        statuses[s_.status] = statuses.get(s_.status, 0) + 1
    # accuracy against the oracle on a bounded, evenly spaced sample
    ns = args.oracle_sample or 32
    sample = list(range(0, count, max(1, count // ns)))[:ns]
    obj_err, x_err = [], []
    t1 = time.perf_counter()
    for i in sample:
        o = ipm.solve(probs[i])
        g = sols[i]
        obj_err.append(abs(g.obj_val - o.objective) / max(1.0, abs(o.objective)))
        x_err.append(float(np.max(np.abs(g.x - o.x)) / max(1.0, float(np.max(np.abs(o.x))))))
    cpu_per_instance = (time.perf_counter() - t1) / max(len(sample), 1)
    if rank == 0:
        line = {"metric": BATCH_METRIC, "value": world * count / wall, "unit": "instances/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": wall * 1e3, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": f"batch of {count} dense SDPs, n~U{{8..64}}, m~U{{20..300}}, "
                                       "seed+index, gap 1e-8", "workers": args.workers,
                           "parallelism": f"replicas{world}"},
                "statuses": statuses,
                "accuracy_vs_oracle": {"sample": len(sample),
                                       "obj_rel_p50": float(np.percentile(obj_err, 50)),
                                       "obj_rel_p99": float(np.percentile(obj_err, 99)),
                                       "x_rel_p50": float(np.percentile(x_err, 50)),
                                       "x_rel_p99": float(np.percentile(x_err, 99))},
                "cpu_baseline": {"value": 1.0 / cpu_per_instance, "unit": "instances/s",
                                 "cores": os.cpu_count(), "kind": "port",
                                 "sample": f"oracle on {len(sample)} instances of the batch"}}
        print(json.dumps(line))
    return 0


ADJOINT_METRIC = ("instances/s, solve to gap 1e-8 plus the adjoint of 1/2|x*-t|^2 w.r.t. q, b, A "
                  "(Float64), batch of conic QPs")


def run_adjoint(args, world, rank, local):
    """Differentiation workload: conic QPs x in R^200, P = LL' + 0.1 I (L 200 x 50), 150 orthant
    rows and one 20 x 20 PSD block, loss 1/2 |x* - t|^2.  Each timed step solves the whole batch
    from host buffers through BatchSolver and, on the same handle after each solve, computes
    dL/dq, dL/db, dL/dA (the KKT system re-factored at the re-centred solution).  Gradients are
    checked on an evenly spaced sample against the oracle's dense FP64 KKT solve at the same
    solution; the CPU baseline is the oracle's solve plus that adjoint."""
    import numpy as np
    import torch
    os.environ["SDPX_B200_DEVICE"] = str(local)
    torch.cuda.set_device(local)
    from oracle import adjoint as oracle_adjoint
    from oracle import ipm
    from sdpx_b200 import problems as Pm
    from sdpx_b200.solver import BatchSolver, DefaultSettings

    count = args.instances or 256
    probs = [Pm.conic_qp(1000 * rank + i) for i in range(count)]
    settings = DefaultSettings(kkt_form="condensed")
    bs = BatchSolver(workers=args.workers, settings=settings)

    def grad(i, sol):
        return sol.x - probs[i].meta["t"]

    for _ in range(args.warmup):
        bs.solve_adjoint(probs[: min(count, 2 * args.workers)], grad)
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        sols, grads = bs.solve_adjoint(probs, grad)
    torch.cuda.synchronize()
    wall = (time.perf_counter() - t0) / args.steps
    wall = max_over_ranks(world, wall)
    statuses = {}
    for s_ in sols:
        statuses[s_.status] = statuses.get(s_.status, 0) + 1
    ns = args.oracle_sample or 16
    sample = list(range(0, count, max(1, count // ns)))[:ns]
    errs, cpu_t = [], 0.0
    for i in sample:
        if grads[i] is None:
            continue
        g, (dq, db, dA) = sols[i], grads[i]
        rq, rb, rA = oracle_adjoint.adjoint(probs[i], g.x, g.s, g.z, g.x - probs[i].meta["t"])
        scale = max(float(np.max(np.abs(rq))), float(np.max(np.abs(rb))), 1.0)
        errs.append(max(float(np.max(np.abs(dq - rq))), float(np.max(np.abs(db - rb)))) / scale)
        t1 = time.perf_counter()
        o = ipm.solve(probs[i])
        oracle_adjoint.adjoint(probs[i], o.x, o.s, o.z, o.x - probs[i].meta["t"])
        cpu_t += time.perf_counter() - t1
    if rank == 0:
        line = {"metric": ADJOINT_METRIC, "value": world * count / wall, "unit": "instances/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": wall * 1e3, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": f"{count} conic QPs n=200, P=LL'+0.1I (L 200x50), 150 orthant "
                                       "rows + 20x20 PSD, seed+index, gap 1e-8, adjoint of "
                                       "1/2|x*-t|^2", "workers": args.workers,
                           "parallelism": f"replicas{world}"},
                "statuses": statuses,
                "gradient_vs_oracle": {"sample": len(errs),
                                       "rel_p50": float(np.percentile(errs, 50)) if errs else None,
                                       "rel_max": float(np.max(errs)) if errs else None},
                "cpu_baseline": {"value": len(errs) / cpu_t if cpu_t else None,
                                 "unit": "instances/s", "cores": os.cpu_count(), "kind": "port",
                                 "sample": f"oracle solve + dense FP64 KKT adjoint on {len(errs)} "
                                           "instances of the batch"}}
        print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--quick", action="store_true",
                    help="skip the nested precision-workload and 256-bit RNS measurements")
    ap.add_argument("--size", type=int, default=2048, help="i8 workload: matrix order")
    ap.add_argument("--reps", type=int, default=3, help="i8 workload: timed repetitions")
    ap.add_argument("--workload", default="rank1", choices=["rank1", "batch", "adjoint", "i8", "mp256"],
                    help="rank1: the 32-block bootstrap SDP (default line); batch: independent "
                         "small SDPs, instances/s; adjoint: conic QPs solved and differentiated; "
                         "i8: the INT8 GEMM; mp256: the 256-bit per-iteration kernels (--size: "
                         "the LDL' order)")
    ap.add_argument("--instances", type=int, default=None,
                    help="batch workloads: instances (default 4096 for batch, 256 for adjoint)")
    ap.add_argument("--workers", type=int, default=16, help="batch workload: worker handles")
    ap.add_argument("--oracle-sample", type=int, default=None,
                    help="batch workloads: instances checked against the oracle (default 32 for "
                         "batch, 16 for adjoint)")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            rc = run_reference(args, world, rank)
        elif args.workload == "i8":
            rc = run_i8(args, world, rank, local)
        elif args.workload == "mp256":
            import torch
            torch.cuda.set_device(local)
            if rank == 0:
                print(json.dumps({"metric": "256-bit per-iteration MPFR kernels (s)", "n_gpus": 1,
                                  "data": "synthetic", **mp_chain_256(args, args.size)}))
            rc = 0
        elif args.workload == "batch":
            rc = run_batch(args, world, rank, local)
        elif args.workload == "adjoint":
            rc = run_adjoint(args, world, rank, local)
        else:
            rc = run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    return rc


if __name__ == "__main__":
    sys.exit(main())
