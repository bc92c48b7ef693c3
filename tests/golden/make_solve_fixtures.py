"""Generate the whole-solve fixtures of the benchmarked workloads from the oracle.

Runs the oracle (oracle/ipm.py, the Float64 restatement of the reference's HSD solver) on the
bootstrap-shaped SDPs the benchmark times and writes, per workload, one compressed ``.npz`` with
the oracle's termination status, iteration count, primal and dual objectives, residuals, gaps and
the solution x.  The GPU parity tests (tests/test_bench_parity.py) solve the same seeded
instances through the C ABI and compare against these files, so the box that runs them needs
neither the oracle's minutes of CPU time nor anything outside the repository.

    python tests/golden/make_solve_fixtures.py [name ...]

Workloads (all gap 1e-8, kkt_form condensed, Float64):
  rank1_b32_m2000_s0   32 PSD blocks n_j ~ U{10..60}, m = 2000, seed 0 (the default bench line)
  rank1_b64_m4000_s0   64 PSD blocks n_j ~ U{10..60}, m = 4000, seed 0 (the precision workload
                       at Float64)
"""
from __future__ import annotations

import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
for p in (ROOT, ROOT / "sdpx.rs_b200"):
    sys.path.insert(0, str(p))

WORKLOADS = {
    "rank1_b32_m2000_s0": dict(blocks=32, m=2000, seed=0),
    "rank1_b64_m4000_s0": dict(blocks=64, m=4000, seed=0),
}


def make(name: str) -> Path:
    from oracle import ipm
    from sdpx_b200 import problems

    spec = WORKLOADS[name]
    prob = problems.rank1_sdp(spec["blocks"], spec["m"], seed=spec["seed"])
    t0 = time.perf_counter()
    r = ipm.Solver(prob, ipm.Settings()).solve()
    dt = time.perf_counter() - t0
    out = HERE / f"solve_{name}.npz"
    np.savez_compressed(out, status=r.status, iterations=r.iterations, objective=r.objective,
                        dual_objective=r.dual_objective, res_primal=r.res_primal,
                        res_dual=r.res_dual, gap_abs=r.gap_abs, gap_rel=r.gap_rel, x=r.x,
                        oracle_seconds=dt, blocks=spec["blocks"], m=spec["m"], seed=spec["seed"])
    print(f"{name}: status {r.status}, {r.iterations} iterations, objective {r.objective!r}, "
          f"{dt:.1f} s -> {out.name}", flush=True)
    return out


if __name__ == "__main__":
    for name in (sys.argv[1:] or list(WORKLOADS)):
        make(name)
