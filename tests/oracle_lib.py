"""ctypes access to the CPU oracle (oracle/_build/libhs_oracle.so).

Test infrastructure only: the oracle is the checker, never the thing tested.
Built by `make -C oracle` (also run by __graft_entry__.build()).
"""
import ctypes
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
ORACLE_DIR = ROOT / "oracle"
ORACLE_SO = ORACLE_DIR / "_build" / "libhs_oracle.so"

_P = ctypes.c_void_p
_I = ctypes.c_int
_I64 = ctypes.c_int64
_D = ctypes.c_double

_SIGS = {
    "or_block_id": ([_I64, _I64, _I64], _I64),
    "or_potrf_block": ([_P, _I64, _I, _I, _I], None),
    "or_trsm_panel": ([_P, _I, _I, _I, _I, _I], None),
    "or_syrk_diag": ([_P, _I, _I, _I, _I, _I, _I], None),
    "or_gemm_trailing": ([_P, _I, _I, _I, _I, _I, _I], None),
    "or_symv_block": ([_P, _P, _P, _I, _I, _I, _I, _I, _I, _I], None),
    "or_trsv_block": ([_P, _P, _I64, _I, _I, _I, _I], None),
    "or_column_update": ([_P, _P, _I, _I, _I, _I, _I, _I, _I], None),
    "or_scale_block": ([_P, _D, _P, _I, _I, _I], None),
    "or_add_block": ([_P, _P, _P, _I, _I, _I], None),
    "or_sub_block": ([_P, _P, _P, _I, _I, _I], None),
    "or_axpy_block": ([_P, _D, _P, _P, _I, _I, _I], None),
    "or_dot_block": ([_P, _P, _I, _I, _I, _I], _D),
    "or_cholesky": ([_P, _I64, _I], None),
    "or_triangular_solve": ([_P, _P, _I64, _I], None),
    "or_cg": ([_P, _P, _P, _I64, _I, _D, _I64, _I, ctypes.POINTER(_D), ctypes.POINTER(_D)], _I64),
    "or_rbf_assemble": ([_P, _P, _I64, _I, _I, _P, _I, _D, _D], None),
    "or_window_inputs": ([_P, _I64, _P], None),
    "or_test_kernel_matrix": ([_P, _I64, _P, _I64, _I, _P, _I, _D, _P], None),
    "or_matrix_vector_gp": ([_P, _P, _P, _I64, _I64], None),
}

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not ORACLE_SO.exists():
            subprocess.run(["make", "-C", str(ORACLE_DIR)], check=True, capture_output=True)
        _lib = ctypes.CDLL(str(ORACLE_SO))
        for name, (args, res) in _SIGS.items():
            fn = getattr(_lib, name)
            fn.argtypes = args
            fn.restype = res
    return _lib


def ptr(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.c_void_p)


def block_id(i, j, nb):
    return i + nb * (nb - 1) // 2 - (nb - j - 1) * (nb - j) // 2


def packed_size(N, bsz):
    nb = -(-N // bsz)
    return nb * (nb + 1) // 2 * bsz * bsz


def rbf_assemble(X, bsz, ell, sf2, sn2):
    X = np.ascontiguousarray(X, dtype=np.float64)
    N, d = X.shape
    A = np.zeros(packed_size(N, bsz))
    ell = np.atleast_1d(np.asarray(ell, dtype=np.float64))
    lib().or_rbf_assemble(ptr(A), ptr(X), N, d, bsz, ptr(ell), ell.size, sf2, sn2)
    return A


def cholesky(A, N, bsz):
    L = np.array(A, dtype=np.float64, copy=True)
    lib().or_cholesky(ptr(L), N, bsz)
    return L


def triangular_solve(L, b, N, bsz):
    x = np.array(b, dtype=np.float64, copy=True)
    lib().or_triangular_solve(ptr(np.ascontiguousarray(L)), ptr(x), N, bsz)
    return x


def cg(A, b, N, bsz, eps, imax, chunks=8):
    x = np.zeros_like(b)
    dn, d0 = ctypes.c_double(), ctypes.c_double()
    it = lib().or_cg(ptr(np.ascontiguousarray(A)), ptr(np.ascontiguousarray(b)), ptr(x), N, bsz, eps, imax, chunks,
                     ctypes.byref(dn), ctypes.byref(d0))
    return x, it, dn.value, d0.value


def packed_to_dense(data, N, bsz, lower_only=False):
    nb = -(-N // bsz)
    full = np.zeros((nb * bsz, nb * bsz))
    for j in range(nb):
        for i in range(j, nb):
            s = block_id(i, j, nb) * bsz * bsz
            blk = np.asarray(data[s:s + bsz * bsz]).reshape(bsz, bsz)
            full[i * bsz:(i + 1) * bsz, j * bsz:(j + 1) * bsz] = blk
            if i != j and not lower_only:
                full[j * bsz:(j + 1) * bsz, i * bsz:(i + 1) * bsz] = blk.T
    return full[:N, :N]


def test_kernel_matrix(X, Xt, ell, sf2):
    """K_star (N_test x N, row major) of MatrixGenerator::generateTestKernelMatrix."""
    X = np.ascontiguousarray(X, dtype=np.float64)
    Xt = np.ascontiguousarray(Xt, dtype=np.float64)
    ell = np.atleast_1d(np.asarray(ell, dtype=np.float64))
    K = np.zeros((Xt.shape[0], X.shape[0]))
    lib().or_test_kernel_matrix(ptr(X), X.shape[0], ptr(Xt), Xt.shape[0], X.shape[1], ptr(ell), ell.size, sf2, ptr(K))
    return K


def matrix_vector_gp(A, b, n, m):
    A = np.ascontiguousarray(A, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    out = np.zeros(m)
    lib().or_matrix_vector_gp(ptr(A), ptr(b), ptr(out), n, m)
    return out


def window_inputs(series, N):
    s = np.ascontiguousarray(series, dtype=np.float64)
    X = np.zeros((N, 8))
    lib().or_window_inputs(ptr(s), N, ptr(X))
    return X
