"""sdpx_b200: the SDPX interior-point hot path on NVIDIA B200 (sm_100a).

The compute lives in ``libsdpx_b200.so`` (hand-written CUDA + a C++ host driver behind the
reference-compatible C ABI, see include/sdpx_b200.h).  This package holds the ctypes binding
(``_lib``), the host-side mirror of the reference solver API (``solver``) and the synthetic
workload generators (``problems``).
"""
from . import problems  # noqa: F401
from .solver import (DefaultSettings, DefaultSolver, KernelContext, PSDTriangleConeT,  # noqa: F401
                     STATUS_NAMES, solve_problem)

__all__ = ["problems", "DefaultSettings", "DefaultSolver", "KernelContext", "PSDTriangleConeT",
           "STATUS_NAMES", "solve_problem"]
