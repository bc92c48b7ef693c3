"""ctypes binding of libsdpx_b200.so (declarations mirror include/sdpx_b200.h).

The library is the product: there is no Python or CPU fallback.  Loading fails loudly when the
shared object is missing (build it with ``python sdpx.rs_b200/build.py``).
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libsdpx_b200.so"

u32, u64, i32, f64 = C.c_uint32, C.c_uint64, C.c_int32, C.c_double
PD = C.POINTER(C.c_double)
PU64 = C.POINTER(C.c_uint64)
PU32 = C.POINTER(C.c_uint32)


class Scalars(C.Structure):
    _fields_ = [("kind", u32), ("reserved", u32), ("count", u64), ("f64", PD),
                ("decimal", C.POINTER(C.c_char_p))]


class Csc(C.Structure):
    _fields_ = [("rows", u64), ("cols", u64), ("nnz", u64), ("colptr", PU64), ("rowval", PU64),
                ("values", Scalars)]


class Cone(C.Structure):
    _fields_ = [("kind", u32), ("reserved", u32), ("dim", u64), ("alpha", Scalars)]


class SampledBlock(C.Structure):
    _fields_ = [("row_start", u64), ("column_start", u64), ("dim", u64), ("basis_rows", u64),
                ("basis_cols", u64), ("basis", Scalars), ("weights", Scalars)]


class Settings(C.Structure):
    _fields_ = [("abi_version", u32), ("struct_size", u32), ("precision_bits", u32),
                ("max_iter", u32), ("verbose", u32), ("preprocessing_flags", u32),
                ("max_threads", u32), ("kkt_form", u32), ("reserved_0", u32),
                ("time_limit", f64), ("tol_gap_abs", C.c_char_p), ("tol_gap_rel", C.c_char_p),
                ("tol_feas", C.c_char_p), ("tol_infeas_abs", C.c_char_p),
                ("tol_infeas_rel", C.c_char_p)]


class Info(C.Structure):
    _fields_ = [("abi_version", u32), ("struct_size", u32), ("status", u32), ("iterations", u32),
                ("working_bits", u32), ("backend_threads", u32), ("cone_threads", u32),
                ("kkt_form", u32), ("reserved_0", u32), ("n", u64), ("m", u64),
                ("solve_time", f64), ("objective", f64), ("dual_objective", f64),
                ("primal_residual", f64), ("dual_residual", f64), ("gap_abs", f64),
                ("gap_rel", f64)]


# name -> (restype, argtypes); every symbol declared in include/sdpx_b200.h
SIGNATURES = {
    "sdpx_default_settings_v4": (i32, [C.POINTER(Settings)]),
    "sdpx_mpi_world_size": (i32, []),
    "sdpx_prepare": (i32, [C.POINTER(Csc), C.POINTER(Scalars), C.POINTER(Csc), C.POINTER(Scalars),
                           C.POINTER(Cone), u64, C.POINTER(Settings), C.POINTER(C.c_void_p)]),
    "sdpx_prepare_sampled": (i32, [C.POINTER(Csc), C.POINTER(Scalars), C.POINTER(Csc),
                                   C.POINTER(Scalars), C.POINTER(Cone), u64, C.POINTER(Settings),
                                   C.POINTER(SampledBlock), u64, C.POINTER(C.c_void_p)]),
    "sdpx_solve": (i32, [C.c_void_p]),
    "sdpx_b200_reprepare": (i32, [C.c_void_p, C.POINTER(Csc), C.POINTER(Scalars), C.POINTER(Csc),
                                  C.POINTER(Scalars), C.POINTER(Cone), u64, C.POINTER(Settings)]),
    "sdpx_update": (i32, [C.c_void_p, C.POINTER(Scalars), C.POINTER(Scalars)]),
    "sdpx_get_info": (i32, [C.c_void_p, C.POINTER(Info)]),
    "sdpx_get_solver_name": (i32, [C.c_void_p, C.c_char_p, u64, PU64]),
    "sdpx_result_f64": (i32, [C.c_void_p, PD, u64, PU64]),
    "sdpx_result_decimal": (i32, [C.c_void_p, C.c_char_p, u64, PU64]),
    "sdpx_last_error": (u64, [C.c_char_p, u64]),
    "sdpx_destroy": (i32, [C.c_void_p]),
    "sdpx_b200_phase_times": (i32, [C.c_void_p, PD, PU64]),
    "sdpx_b200_set_kernel_timing": (i32, [C.c_void_p, i32]),
    "sdpx_b200_kernel_times": (i32, [C.c_void_p, PD, PU64]),
    "sdpx_b200_launch_count": (u64, []),
    "sdpx_b200_device_allocations": (u64, []),
    "sdpx_b200_set_i8_timing": (i32, [i32]),
    "sdpx_b200_i8_config": (i32, [i32]),
    "sdpx_b200_i8_tuning": (i32, [C.c_char_p, u64, PU64]),
    "sdpx_b200_i8_times": (i32, [PD, PD, PD, PU64]),
    "sdpx_b200_transfer_bytes": (i32, [PU64, PU64]),
    "sdpx_b200_schur_forms": (i32, [C.c_void_p, PU32, PU32]),
    "sdpx_b200_kkt_paths": (i32, [C.c_void_p, PU64, PU64]),
    "sdpx_b200_set_graphs": (i32, [C.c_void_p, i32]),
    "sdpx_b200_set_form": (i32, [C.c_void_p, u32]),
    "sdpx_b200_adjoint": (i32, [C.c_void_p, PD, PD, PD, PD, PD, PD, u64]),
    "sdpxg_ctx_create": (i32, [i32, u32, C.POINTER(C.c_void_p)]),
    "sdpxg_ctx_destroy": (i32, [C.c_void_p]),
    "sdpxg_problem_upload": (i32, [C.c_void_p, C.POINTER(Csc), C.POINTER(Csc), PU64, u64]),
    "sdpxg_nt_scale": (i32, [C.c_void_p, PD, PD, PD, PU32]),
    "sdpxg_identity_scaling": (i32, [C.c_void_p]),
    "sdpxg_problem_upload_sampled": (i32, [C.c_void_p, C.POINTER(Csc), C.POINTER(Csc), PU64, u64,
                                           C.POINTER(SampledBlock), u64]),
    "sdpxg_set_scaling": (i32, [C.c_void_p, PD, PD]),
    "sdpxg_schur_assemble": (i32, [C.c_void_p, PD]),
    "sdpxg_factor": (i32, [C.c_void_p, f64, u32, f64, f64, PU32]),
    "sdpxg_solve_many": (i32, [C.c_void_p, PD, PD, u32]),
    "sdpxg_set_factor_form": (i32, [C.c_void_p, u32]),
    "sdpxg_split_dgemm_device": (i32, [C.c_void_p, C.c_char, C.c_char, u64, u64, u64, f64, C.c_void_p,
                                       u64, C.c_void_p, u64, f64, C.c_void_p, u64, PU32]),
    "sdpxg_solve_noalloc": (i32, [C.c_void_p, C.c_void_p, C.c_void_p, u32]),
    "sdpxg_kkt_solve": (i32, [C.c_void_p, PD, PD, PD, PD]),
    "sdpxg_residual": (i32, [C.c_void_p, PD, PD, PD, PD, PD, PD, PD]),
    "sdpxg_step_length": (i32, [C.c_void_p, PD, PD, f64, u32, PD, PU32]),
    "sdpxg_cone_apply": (i32, [C.c_void_p, u32, PD, PD]),
    "sdpxg_rns_gemm": (i32, [C.c_void_p, u32, C.c_char, C.c_char, u64, u64, u64, C.c_void_p, u64,
                             C.c_void_p, u64, u32, C.c_void_p, PU32]),
    "sdpxg_rns_gemm_device": (i32, [C.c_void_p, u32, C.c_char, C.c_char, u64, u64, u64, C.c_void_p,
                                    u64, C.c_void_p, u64, u32, C.c_void_p, PU32]),
    "sdpxg_rns_set_form": (i32, [C.c_void_p, u32]),
    "sdpxg_mp_ldl": (i32, [C.c_void_p, u32, u64, C.c_void_p, u64, C.c_void_p, C.c_void_p, C.c_void_p,
                           PU32]),
    "sdpxg_mp_ldl_device": (i32, [C.c_void_p, u32, u64, C.c_void_p, u64, C.c_void_p, C.c_void_p, PU32]),
    "sdpxg_mp_potrf": (i32, [C.c_void_p, u32, C.c_char, u64, C.c_void_p, u64, C.POINTER(i32), PU32]),
    "sdpxg_rns_congruence": (i32, [C.c_void_p, u32, C.c_char, u64, u64, C.c_void_p, u64, C.c_void_p,
                                   u64, u32, C.c_void_p, PU32]),
    "sdpxg_rns_diag_congruence": (i32, [C.c_void_p, u32, u64, u64, C.c_void_p, u64, C.c_void_p, u32,
                                        C.c_void_p, PU32]),
    "sdpxg_rns_svec_quadratic": (i32, [C.c_void_p, u32, u64, u64, C.c_void_p, u32, C.c_void_p,
                                       C.c_void_p, C.c_void_p, PU32]),
    "sdpxg_rns_symmetric_bilinear": (i32, [C.c_void_p, u32, u64, u64, C.c_void_p, C.c_void_p, u64,
                                           C.POINTER(u64), C.c_void_p, PU32]),
    "sdpxg_mp_step_length": (i32, [C.c_void_p, u32, u64, C.POINTER(u64), u32, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(i32), PU32]),
    "sdpxg_mp_nt_scale": (i32, [C.c_void_p, u32, u64, C.POINTER(u64), C.c_void_p, C.c_void_p, C.c_void_p,
                                C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(i32), PU32]),
    "sdpxg_rns_gemm_blocks_upper": (i32, [C.c_void_p, u32, u64, u64, C.POINTER(u64), C.POINTER(u64),
                                          C.c_void_p, C.c_void_p, C.POINTER(u64), C.c_void_p, PU32]),
}

_lib = None


def load() -> C.CDLL:
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        path = os.environ.get("SDPX_B200_LIB", str(LIB_PATH))
        if not Path(path).exists():
            raise ImportError(f"libsdpx_b200.so not found at {path}: run python sdpx.rs_b200/build.py")
        lib = C.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


class SdpxError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"sdpx error {code}: {message}")
        self.code = code


def last_error() -> str:
    lib = load()
    buf = C.create_string_buffer(4096)
    lib.sdpx_last_error(buf, 4096)
    return buf.value.decode(errors="replace")


def call(name: str, *args) -> int:
    rc = getattr(load(), name)(*args)
    if rc != 0:
        raise SdpxError(rc, last_error())
    return rc


def dptr(a):
    """Pointer to a contiguous float64 numpy array (None -> NULL)."""
    if a is None:
        return None
    return a.ctypes.data_as(PD)
