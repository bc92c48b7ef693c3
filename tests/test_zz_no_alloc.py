"""sdpxg_solve_noalloc: the reduced solve for callers that cannot allocate device memory.

Some hosts own all of their device memory through their own pool, or run a latency-bound loop in
which a cudaMalloc (which can synchronise the whole device) is not allowed.  The entry point takes
device pointers and keeps its per-call scratch in a static device array of the library, so such a
caller can solve without any allocation inside the call.  Its results must match the allocating
entry point sdpxg_solve_many on the same factorization, on two calls in a row (the static scratch
keeps the previous call's contents; nothing may depend on it being clean), and the library's
count of device blocks must not move across those calls.  This file is collected last so a
failure here does not hide any other test's result.
"""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

from sdpx_b200 import _lib
from sdpx_b200 import problems as P
from sdpx_b200.solver import KernelContext

pytestmark = pytest.mark.gpu


def _interior(prob, seed):
    rng = np.random.default_rng(seed)
    s, z = [], []
    for _, d in prob.cones:
        for out in (s, z):
            B = rng.standard_normal((d, d))
            out.append(P.svec(B @ B.T / d + 0.1 * np.eye(d)))
    return np.concatenate(s), np.concatenate(z)


def _factored_context(seed=5):
    prob = P.rank1_sdp(6, 150, seed=seed, nmin=5, nmax=30)
    ctx = KernelContext()
    ctx.upload(prob.A, [d for _, d in prob.cones])
    s, z = _interior(prob, 2)
    lam, st = ctx.nt_scale(s, z)
    assert st == 0
    ctx.schur()
    assert ctx.factor(1e-8) == 0
    return prob, ctx


def test_noalloc_solve_matches_solve_many():
    import torch

    prob, ctx = _factored_context()
    n = prob.n
    rhs = np.asfortranarray(np.random.default_rng(3).standard_normal((n, 2)))
    ref = ctx.solve_many(rhs)
    d_rhs = torch.from_numpy(rhs.ravel(order="F").copy()).to("cuda")
    d_out = torch.full((2 * n,), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()  # the entry point does not wait for the caller's stream
    lib = _lib.load()
    allocs = lib.sdpx_b200_device_allocations()
    for call in range(2):
        rc = lib.sdpxg_solve_noalloc(ctx._h, C.c_void_p(d_rhs.data_ptr()), C.c_void_p(d_out.data_ptr()), 2)
        assert rc == 0, _lib.last_error()
        assert lib.sdpx_b200_device_allocations() == allocs, call
        out = d_out.cpu().numpy().reshape((n, 2), order="F")
        err = np.max(np.abs(out - ref)) / np.max(np.abs(ref))
        assert err <= 1e-12, (call, err)


def test_noalloc_rejects_stale_factor_and_host_pointers():
    import torch

    prob, ctx = _factored_context(seed=7)
    n = prob.n
    lib = _lib.load()
    host = np.zeros(n)
    d = torch.zeros(n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = lib.sdpxg_solve_noalloc(ctx._h, C.c_void_p(host.ctypes.data), C.c_void_p(d.data_ptr()), 1)
    assert rc == 1 and "device pointers" in _lib.last_error()
    ctx.upload(prob.A, [d_ for _, d_ in prob.cones])  # a new upload invalidates the factor
    rc = lib.sdpxg_solve_noalloc(ctx._h, C.c_void_p(d.data_ptr()), C.c_void_p(d.data_ptr()), 1)
    assert rc == 1 and "sdpxg_factor" in _lib.last_error()


def test_noalloc_rejects_sizes_beyond_maximum():
    import torch

    n = 4097  # one above the compiled maximum
    A = sp.csc_matrix((np.ones(n), (np.zeros(n, dtype=int), np.arange(n))), shape=(3, n))
    ctx = KernelContext()
    ctx.upload(A, [2])
    d = torch.zeros(n, dtype=torch.float64, device="cuda")
    rc = _lib.load().sdpxg_solve_noalloc(ctx._h, C.c_void_p(d.data_ptr()), C.c_void_p(d.data_ptr()), 1)
    assert rc == 2
    assert "4096" in _lib.last_error()
