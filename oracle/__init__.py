"""CPU oracle for the SDPX interior-point hot path -- TEST INFRASTRUCTURE ONLY.

This package restates, on the CPU, the algorithm of the reference solver
(yongjunx23-del/SDPX.rs v0.9.5, pure Rust) for the path the CUDA library accelerates.  It is
the checker: only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import it.  The product (``sdpx.rs_b200``) never calls it and has no CPU
fallback.

Modules
-------
``ipm``    Float64 HSD predictor/corrector with the condensed PSD Schur complement, the
           dense Cholesky with the dynamic pivot rule, two-level iterative refinement,
           Ruiz equilibration and the reference's termination rules.
``exact``  exact-rounding restatement of the MPFR contract (dot rounded once, RNE at 64N
           bits) and of the RNS exact product used under the MPFR path.

Parity pinning: the reference cannot be built here (no Rust toolchain).  ``ipm`` is pinned to
the reference's own known answers (crates/solver/tests/it/basic_sdp.rs:28-56,
crates/solver/tests/it/sampled_solver.rs:8-105, crates/solver/src/solver/sampled/tests.rs:407-446);
iteration counts on the synthetic workloads are therefore pinned only through this restatement
("iteration parity unpinned" against the Rust binary).  ``exact`` is pinned by the
definition of correct rounding, cross-checked against mpmath.
"""
