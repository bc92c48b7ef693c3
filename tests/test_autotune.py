"""The INT8 tensor-core GEMM's tile-configuration autotuner (sdpx_b200_i8_config / _i8_tuning).

Every configuration computes the same exact integers, so the split-precision product and the
exact RNS product must be bitwise equal whichever configuration runs (forced 0, 1 or 2,
autotuned), and the autotuner must have recorded the shape classes it timed.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import exact as X
from sdpx_b200 import _lib
from sdpx_b200.solver import KernelContext

pytestmark = pytest.mark.gpu


def _tuning_table():
    lib = _lib.load()
    req = C.c_uint64()
    lib.sdpx_b200_i8_tuning(None, 0, C.byref(req))
    buf = C.create_string_buffer(req.value)
    assert lib.sdpx_b200_i8_tuning(buf, req.value, C.byref(req)) == 0
    return buf.value.decode()


def test_configurations_agree_bitwise():
    import torch
    lib = _lib.load()
    ctx = KernelContext()
    rng = np.random.default_rng(9)
    m, n, k = 300, 500, 700
    A = torch.from_numpy(rng.standard_normal((k, m))).cuda()  # column-major m x k
    B = torch.from_numpy(rng.standard_normal((n, k))).cuda()  # column-major k x n
    outs = []
    n_mp, mm, nn, kk = 4, 40, 70, 300
    lcg = X.Lcg(5)
    Am = X.pack_array(X.random_values(n_mp, lcg, mm * kk, 20))
    Bm = X.pack_array(X.random_values(n_mp, lcg, kk * nn, 20))
    try:
        for cfg in (0, 1, 2, -1):
            assert lib.sdpx_b200_i8_config(cfg) == 0
            Cd = torch.zeros((n, m), dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            assert ctx.split_dgemm_device("N", "N", m, n, k, 1.0, A.data_ptr(), m, B.data_ptr(), k, 0.0,
                                          Cd.data_ptr(), m) == 0
            raw, st = ctx.rns_gemm(n_mp, "N", "N", mm, nn, kk, Am, mm, Bm, kk, form=0)
            assert st == 0
            outs.append((Cd.cpu().numpy().tobytes(), raw))
    finally:
        lib.sdpx_b200_i8_config(-1)
    assert outs[0] == outs[1] == outs[2] == outs[3]
    table = _tuning_table()
    assert "digits 1" in table and "digits 2" in table, table
