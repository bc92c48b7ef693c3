"""C-ABI surface of libsdpx_b200.so on the CPU: loads, exports every declared symbol, struct
layouts match the reference ABI 4, and validation errors are reported before any device work
(crates/ffi/src/lib.rs:292-325 validation, return codes of include/sdpx.h:15-17)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest
import scipy.sparse as sp

from sdpx_b200 import _lib
from sdpx_b200.solver import DefaultSettings, DefaultSolver

HEADER = Path(__file__).resolve().parent.parent / "include" / "sdpx_b200.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:int32_t|uint64_t)\s+(\w+)\s*\(", text, re.M)))


def test_header_symbols_exported(lib):
    names = declared_symbols()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, name


def test_struct_sizes_match_reference_abi():
    assert C.sizeof(_lib.Settings) == 88
    assert C.sizeof(_lib.Info) == 112


def test_default_settings(lib):
    s = _lib.Settings()
    assert lib.sdpx_default_settings_v4(C.byref(s)) == 0
    assert s.abi_version == 4 and s.struct_size == 88 and s.precision_bits == 53
    assert s.max_iter == 200 and s.preprocessing_flags == 7 and s.kkt_form == 0
    assert lib.sdpx_mpi_world_size() == 1


def _tiny():
    A = sp.identity(3, format="csc")
    return None, np.zeros(3), A, np.array([1.0, 0.0, 1.0]), [("psd", 2)]


def test_rejects_wrong_abi_version(lib):
    s = _lib.Settings()
    lib.sdpx_default_settings_v4(C.byref(s))
    s.abi_version = 3
    h = C.c_void_p()
    A = sp.identity(3, format="csc")
    from sdpx_b200.solver import _CscHold, _scalars
    a = _CscHold(A)
    q = np.zeros(3)
    b = np.ones(3)
    cone = (_lib.Cone * 1)()
    cone[0].kind, cone[0].dim = 3, 2
    rc = lib.sdpx_prepare(None, C.byref(_scalars(q)), C.byref(a.c), C.byref(_scalars(b)), cone, 1,
                          C.byref(s), C.byref(h))
    assert rc == 1
    assert "ABI" in _lib.last_error()


@pytest.mark.parametrize("field,value,code", [("precision_bits", 256, 2), ("kkt_form", 1, 2),
                                              ("kkt_form", 3, 1), ("verbose", 2, 1)])
def test_settings_validation(field, value, code):
    P, q, A, b, cones = _tiny()
    st = DefaultSettings()
    with pytest.raises(_lib.SdpxError) as e:
        if field == "precision_bits":
            DefaultSolver(P, q, A, b, cones, DefaultSettings(precision_bits=value))
        elif field == "kkt_form" and value == 1:
            DefaultSolver(P, q, A, b, cones, DefaultSettings(kkt_form="augmented"))
        else:
            s, keep = st.to_c()
            setattr(s, field, value)
            from sdpx_b200.solver import _CscHold, _scalars
            a = _CscHold(A)
            cone = (_lib.Cone * 1)()
            cone[0].kind, cone[0].dim = 3, 2
            h = C.c_void_p()
            _lib.call("sdpx_prepare", None, C.byref(_scalars(q)), C.byref(a.c), C.byref(_scalars(b)),
                      cone, 1, C.byref(s), C.byref(h))
    assert e.value.code == code


def test_rejects_nonfinite_and_bad_csc():
    P, q, A, b, cones = _tiny()
    with pytest.raises(_lib.SdpxError) as e:
        DefaultSolver(P, np.array([np.nan, 0, 0]), A, b, cones)
    assert e.value.code == 1
    with pytest.raises(_lib.SdpxError) as e:
        DefaultSolver(P, q, A, b, [("psd", 3)])  # 6 rows expected, 3 given
    assert e.value.code == 1
    with pytest.raises(_lib.SdpxError) as e:
        DefaultSolver(P, q, A, b, [("soc", 3)])  # second-order cones are not on the GPU path
    assert e.value.code == 2
    with pytest.raises(_lib.SdpxError) as e:
        DefaultSolver(P, q, A, np.ones(2), cones)
    assert e.value.code == 1


def test_last_error_truncates(lib):
    P, q, A, b, cones = _tiny()
    with pytest.raises(_lib.SdpxError):
        DefaultSolver(P, q, A, b, [("psd", 3)])
    need = lib.sdpx_last_error(None, 0)
    buf = C.create_string_buffer(4)
    assert lib.sdpx_last_error(buf, 4) == need
    assert len(buf.value) == 3


def test_null_handle_and_destroy(lib):
    assert lib.sdpx_destroy(None) == 0
    assert lib.sdpx_solve(None) == 1


def test_last_error_is_per_thread(lib):
    """Each host thread reads its own last error (batches call the library from many threads)."""
    import threading

    problems = []

    def worker(tid):
        from sdpx_b200.solver import _CscHold, _scalars
        s = _lib.Settings()
        lib.sdpx_default_settings_v4(C.byref(s))
        s.abi_version = 100 + tid  # rejected with a message naming this thread's version
        a = _CscHold(sp.identity(3, format="csc"))
        q, b = np.zeros(3), np.ones(3)
        cone = (_lib.Cone * 1)()
        cone[0].kind, cone[0].dim = 3, 2
        h = C.c_void_p()
        buf = C.create_string_buffer(256)
        for _ in range(200):
            rc = lib.sdpx_prepare(None, C.byref(_scalars(q)), C.byref(a.c), C.byref(_scalars(b)),
                                  cone, 1, C.byref(s), C.byref(h))
            lib.sdpx_last_error(buf, 256)
            msg = buf.value.decode()
            if rc != 1 or f"version {100 + tid};" not in msg:
                problems.append((tid, rc, msg))

    threads = [threading.Thread(target=worker, args=(t,)) for t in range(8)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not problems, problems[:3]
