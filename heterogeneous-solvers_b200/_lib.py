"""ctypes binding of libhs_b200.so (the C ABI declared in include/hs_b200.h).

The shared library is built in place (``make -C heterogeneous-solvers_b200``)
and must be present: there is no fallback path, a missing or stale library
raises immediately.
"""
import ctypes
import os
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libhs_b200.so"
ABI_VERSION = 1

HS_OK = 0
STATUS_NAMES = {
    0: "HS_OK", 1: "HS_ERR_INVALID_ARG", 2: "HS_ERR_OOM", 3: "HS_ERR_NOT_SPD", 4: "HS_ERR_NO_CONVERGENCE",
    5: "HS_ERR_REFINEMENT_STALLED", 6: "HS_ERR_CUDA", 7: "HS_ERR_TIMEOUT", 8: "HS_ERR_UNSUPPORTED",
}


class HSError(RuntimeError):
    """A non-OK hs_status; ``status`` holds the code, the message is hs_last_error()."""

    def __init__(self, status, message):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class NotSPDError(HSError):
    pass


class NoConvergenceError(HSError):
    pass


class SolveReport(ctypes.Structure):
    _fields_ = [("info", ctypes.c_int64), ("iterations", ctypes.c_int64), ("assemble_ms", ctypes.c_double),
                ("factor_ms", ctypes.c_double), ("solve_ms", ctypes.c_double), ("total_ms", ctypes.c_double)]


class MixedReport(ctypes.Structure):
    _fields_ = [("refinement_steps", ctypes.c_int64), ("pcg_iterations", ctypes.c_int64),
                ("fallback_pcg", ctypes.c_int), ("factor_attempts", ctypes.c_int),
                ("precision_used", ctypes.c_int), ("reserved", ctypes.c_int), ("shift", ctypes.c_double),
                ("backward_error", ctypes.c_double),
                ("initial_backward_error", ctypes.c_double), ("norm_k_fro", ctypes.c_double),
                ("logdet", ctypes.c_double), ("factor_ms", ctypes.c_double), ("refine_ms", ctypes.c_double),
                ("total_ms", ctypes.c_double)]


class GpReport(ctypes.Structure):
    _fields_ = [("factor_ms", ctypes.c_double), ("adjoint_ms", ctypes.c_double), ("grad_ms", ctypes.c_double),
                ("total_ms", ctypes.c_double), ("data_fit", ctypes.c_double), ("logdet", ctypes.c_double)]


class KernelProfile(ctypes.Structure):
    _fields_ = [("launches", ctypes.c_int64), ("ms", ctypes.c_double), ("flops", ctypes.c_double),
                ("bytes", ctypes.c_double)]


# hs_kernel_id
KERNEL_IDS = {"update": 0, "potrf": 1, "trsm": 2, "symv": 3, "trsv": 4, "colupd": 5, "assemble": 6, "vector": 7,
              "adjoint": 8, "grad": 9, "update_side": 10}

_P = ctypes.c_void_p
_I = ctypes.c_int
_I64 = ctypes.c_int64
_D = ctypes.c_double

# name -> argument types (all return hs_status unless listed in _RESTYPES)
SIGNATURES = {
    "hs_abi_version": [],
    "hs_last_error": [],
    "hs_status_string": [_I],
    "hs_ctx_create": [_I, _P, ctypes.POINTER(_P)],
    "hs_ctx_destroy": [_P],
    "hs_ctx_set_stream": [_P, _P],
    "hs_ctx_release_buffers": [_P],
    "hs_selftest_bounded_wait": [_P, _I64],
    "hs_ctx_set_problem": [_P, _I64, _I],
    "hs_sync": [_P],
    "hs_packed_matrix_size": [_I64, _I],
    "hs_padded_vector_size": [_I64, _I],
    "hs_ctx_set_profiling": [_P, _I],
    "hs_ctx_read_profile": [_P, _I, ctypes.POINTER(KernelProfile)],
    "hs_ctx_reset_profile": [_P],
    "hs_ctx_launch_count": [_P],
    "hs_ctx_set_reference_order": [_P, _I],
    "hs_ctx_set_mixed_accumulation": [_P, _I],
    "hs_ctx_set_mixed_lookahead": [_P, _I, _I],
    "hs_potrf_block": [_P, _P, _I, _I],
    "hs_ctx_take_info": [_P, ctypes.POINTER(_I64)],
    "hs_trsm_panel": [_P, _P, _I, _I, _I, _I],
    "hs_syrk_diag": [_P, _P, _I, _I, _I, _I, _I],
    "hs_gemm_trailing": [_P, _P, _I, _I, _I, _I, _I],
    "hs_symv_block": [_P, _P, _P, _P, _I, _I, _I, _I, _I, _I],
    "hs_symv_block_noalloc": [_P, _P, _P, _P, _I, _I, _I, _I, _I, _I],
    "hs_trsv_block": [_P, _P, _P, _I, _I, _I],
    "hs_column_update": [_P, _P, _P, _I, _I, _I, _I, _I, _I],
    "hs_scale_block": [_P, _P, _D, _P, _I, _I],
    "hs_add_block": [_P, _P, _P, _P, _I, _I],
    "hs_sub_block": [_P, _P, _P, _P, _I, _I],
    "hs_axpy_block": [_P, _P, _D, _P, _P, _I, _I],
    "hs_dot_block": [_P, _P, _P, _P, _I, _I],
    "hs_rbf_assemble": [_P, _P, _P, _I, _P, _I, _D, _D],
    "hs_cholesky_factor": [_P, _P, ctypes.POINTER(_I64)],
    "hs_cholesky_solve": [_P, _P, _P],
    "hs_cg_solve": [_P, _P, _P, _P, _D, _I64, ctypes.POINTER(_I64), ctypes.POINTER(_D), ctypes.POINTER(_D)],
    "hs_gp_solve_host": [_P, _P, _P, _I, _P, _I, _D, _D, _I, _D, _I64, _P, ctypes.POINTER(SolveReport)],
    "hs_mixed_solve": [_P, _P, _P, _P, _I, _D, _I, ctypes.POINTER(MixedReport)],
    "hs_cholesky_logdet": [_P, _P, ctypes.POINTER(_D)],
    "hs_cholesky_adjoint": [_P, _P, _P],
    "hs_gp_test_kernel_matrix": [_P, _P, _P, _I64, _I, _P, _I, _D, _P],
    "hs_matrix_vector_gp": [_P, _P, _P, _P, _I64, _I64],
    "hs_gp_predict": [_P, _P, _P, _I64, _I, _P, _I, _D, _P, _P],
    "hs_gp_nlml_grad": [_P, _P, _P, _I, _P, _I, ctypes.POINTER(_D), _P, ctypes.POINTER(GpReport)],
    "hs_gp_nlml_grad_mixed": [_P, _P, _P, _I, _P, _I, _I, _D, ctypes.POINTER(_D), _P, ctypes.POINTER(GpReport),
                              ctypes.POINTER(MixedReport)],
}
_RESTYPES = {"hs_abi_version": _I, "hs_last_error": ctypes.c_char_p, "hs_status_string": ctypes.c_char_p,
             "hs_packed_matrix_size": _I64, "hs_padded_vector_size": _I64, "hs_ctx_launch_count": _I64}

_lib = None


def load():
    """Load the library once; raises if it is missing or has another ABI version."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with `make -C {_HERE}` (no CPU fallback exists)")
    lib = ctypes.CDLL(os.fspath(LIB_PATH))
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = _RESTYPES.get(name, _I)
    if lib.hs_abi_version() != ABI_VERSION:
        raise ImportError(f"{LIB_PATH}: ABI version {lib.hs_abi_version()} != {ABI_VERSION}")
    _lib = lib
    return lib


def check(status):
    if status == HS_OK:
        return
    msg = load().hs_last_error().decode(errors="replace")
    if status == 3:
        raise NotSPDError(status, msg)
    if status == 4:
        raise NoConvergenceError(status, msg)
    raise HSError(status, msg)


def call(name, *args):
    check(getattr(load(), name)(*args))
