"""Host-side mirror of the reference's operator and solver interface.

Names, argument order and meaning follow TimThuering/Heterogeneous-Solvers
(paths relative to its root); a ``Context`` takes the place of the
``sycl::queue`` argument and of the ``conf::N`` / ``conf::matrixBlockSize``
globals (src/utility/Configuration.hpp:21-118).  Device memory is held in
torch CUDA tensors (float64); every operator launches the CUDA kernels of
libhs_b200.so through its C ABI.  There is no CPU implementation here.
"""
import ctypes
import math
import time
from pathlib import Path

import numpy as np
import torch

from . import _lib
from ._lib import GpReport, HSError, MixedReport, NoConvergenceError, NotSPDError, SolveReport, call

__all__ = [
    "Context", "SymmetricMatrix", "RightHandSide", "MatrixOperations", "MatrixMatrixOperations",
    "MatrixVectorOperations", "VectorOperations", "Cholesky", "TriangularSystemSolver", "CG",
    "MatrixGenerator", "MatrixParser", "HSError", "NotSPDError", "NoConvergenceError", "block_id",
    "packed_size", "padded_size", "gp_solve_host", "MixedPrecisionSolver", "cholesky_logdet", "PRECISIONS",
    "cholesky_adjoint", "gp_nlml_grad", "GaussianProcessNLML", "GaussianProcess", "gp_predict",
    "UtilityFunctions", "fit_hyperparameters",
]

# hs_precision
PRECISIONS = {"fp64": 0, "tf32x3": 1, "bf16x3": 2, "f16x3": 3}


def block_id(i, j, nb):
    """Id of block (i, j), i >= j, in column-by-column order (SymmetricMatrix.hpp:9-35)."""
    return i + nb * (nb - 1) // 2 - (nb - j - 1) * (nb - j) // 2


def packed_size(N, bsz):
    nb = -(-N // bsz)
    return nb * (nb + 1) // 2 * bsz * bsz


def padded_size(N, bsz):
    return -(-N // bsz) * bsz


def _dptr(t, ctx=None):
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"expected a torch CUDA float64 tensor, got {type(t).__name__}")
    if not t.is_cuda or t.dtype != torch.float64 or not t.is_contiguous():
        raise TypeError(f"expected a contiguous CUDA float64 tensor, got {t.dtype} on {t.device}")
    if ctx is not None and t.device.index != ctx.device:
        raise ValueError(f"tensor on cuda:{t.device.index}, context on cuda:{ctx.device}")
    return ctypes.c_void_p(t.data_ptr())


class Context:
    """Device, stream and problem size of a sequence of calls.

    Replaces the sycl::queue of every reference call plus conf::N and
    conf::matrixBlockSize.  By default the context runs on torch's current
    stream of ``device`` so that it orders with torch's own work.
    """

    def __init__(self, device=0, stream=None, N=None, matrixBlockSize=None):
        _lib.load()
        self.device = int(device)
        if stream is None:
            stream = torch.cuda.current_stream(self.device)
        self.stream = stream
        handle = ctypes.c_void_p()
        call("hs_ctx_create", self.device, ctypes.c_void_p(stream.cuda_stream), ctypes.byref(handle))
        self.handle = handle
        self.N = None
        self.matrixBlockSize = None
        if N is not None:
            self.set_problem(N, matrixBlockSize)

    def set_problem(self, N, matrixBlockSize):
        call("hs_ctx_set_problem", self.handle, int(N), int(matrixBlockSize))
        self.N = int(N)
        self.matrixBlockSize = int(matrixBlockSize)
        return self

    @property
    def blockCountXY(self):
        return -(-self.N // self.matrixBlockSize)

    def sync(self):
        call("hs_sync", self.handle)

    def set_profiling(self, enable=True):
        call("hs_ctx_set_profiling", self.handle, int(bool(enable)))

    def read_profile(self, kernel):
        """(launches, device ms, algorithmic flops, algorithmic bytes) of one kernel family."""
        out = _lib.KernelProfile()
        call("hs_ctx_read_profile", self.handle, _lib.KERNEL_IDS[kernel], ctypes.byref(out))
        return {"launches": out.launches, "ms": out.ms, "flops": out.flops, "bytes": out.bytes}

    def reset_profile(self):
        call("hs_ctx_reset_profile", self.handle)

    def set_reference_order(self, cpu_chunks):
        """cpu_chunks > 0: matvec, dots, vector updates and CG follow the
        reference CPU path's accumulation order exactly (its dot product sums
        `cpu_chunks` = core-count chunks); 0 restores the fast kernels."""
        call("hs_ctx_set_reference_order", self.handle, int(cpu_chunks))

    def set_mixed_accumulation(self, panels):
        """Mixed-precision factor: the trailing-update products of `panels` (1, 2 or 4)
        panels are summed in the tensor cores' accumulator, a tile's units then in
        registers before one add into the FP32 matrix; fewer is the more accurate factor
        and log|K| (default 1)."""
        call("hs_ctx_set_mixed_accumulation", self.handle, int(panels))

    def set_mixed_lookahead(self, side_sms=16, min_rows=24576):
        """Mixed-precision factor: while at least `min_rows` rows follow the next group
        of panels, factor that group on `side_sms` SMs beside the current group's
        trailing update (0: look-ahead by one diagonal block).  The factor is the same
        bit for bit either way."""
        call("hs_ctx_set_mixed_lookahead", self.handle, int(side_sms), int(min_rows))

    def launch_count(self):
        return _lib.load().hs_ctx_launch_count(self.handle)

    def take_info(self):
        v = ctypes.c_int64()
        call("hs_ctx_take_info", self.handle, ctypes.byref(v))
        return v.value

    def close(self):
        if getattr(self, "handle", None) is not None and _lib._lib is not None:
            _lib._lib.hs_ctx_destroy(self.handle)
        self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SymmetricMatrix:
    """Packed lower block triangle (src/dataStructures/SymmetricMatrix.hpp:36-54).

    ``matrixData`` is a float64 tensor of T*bsz*bsz entries (host by default,
    ``device=`` for a CUDA tensor), zero-initialised like the reference's
    std::vector.
    """

    def __init__(self, N, blockSize, device=None):
        self.N = int(N)
        self.blockSize = int(blockSize)
        self.blockCountXY = int(math.ceil(self.N / self.blockSize))
        self.matrixData = torch.zeros(packed_size(self.N, self.blockSize), dtype=torch.float64,
                                      device=device if device is not None else "cpu")

    def block(self, i, j):
        """View of stored block (i, j), i >= j, as bsz x bsz."""
        b = self.blockSize
        s = block_id(i, j, self.blockCountXY) * b * b
        return self.matrixData[s:s + b * b].view(b, b)

    def to_dense(self):
        """Full N x N matrix (lower blocks mirrored) as a float64 numpy array."""
        b, nb = self.blockSize, self.blockCountXY
        data = self.matrixData.detach().cpu().numpy()
        full = np.zeros((nb * b, nb * b))
        for j in range(nb):
            for i in range(j, nb):
                s = block_id(i, j, nb) * b * b
                blk = data[s:s + b * b].reshape(b, b)
                full[i * b:(i + 1) * b, j * b:(j + 1) * b] = blk
                if i != j:
                    full[j * b:(j + 1) * b, i * b:(i + 1) * b] = blk.T
        return full[:self.N, :self.N]


class RightHandSide:
    """Zero-padded vector of nb*bsz entries (src/dataStructures/RightHandSide.hpp:12-30)."""

    def __init__(self, N, blockSize, device=None):
        self.N = int(N)
        self.blockSize = int(blockSize)
        self.blockCountX = int(math.ceil(self.N / self.blockSize))
        self.rightHandSideData = torch.zeros(self.blockCountX * self.blockSize, dtype=torch.float64,
                                             device=device if device is not None else "cpu")


# ------------------------------------------------------------------ operators
class MatrixOperations:
    """src/kernel/MatrixOperations.hpp:9-56 — POTRF of one diagonal block."""

    @staticmethod
    def cholesky(ctx, A, blockID, blockRow):
        call("hs_potrf_block", ctx.handle, _dptr(A, ctx), int(blockID), int(blockRow))

    cholesky_GPU = cholesky
    cholesky_optimizedGPU = cholesky


class MatrixMatrixOperations:
    """src/kernel/MatrixMatrixOperations.hpp:8-295 — TRSM, SYRK and GEMM steps."""

    @staticmethod
    def triangularSolve(ctx, A, blockID, blockRow, blockStart, blockCount):
        call("hs_trsm_panel", ctx.handle, _dptr(A, ctx), int(blockID), int(blockRow), int(blockStart),
             int(blockCount))

    triangularSolve_optimizedGPU = triangularSolve
    triangularSolve_optimizedCPU = triangularSolve

    @staticmethod
    def symmetricMatrixMatrixDiagonal(ctx, A, blockID, blockRow, blockStart, blockCount, blockCountXY):
        call("hs_syrk_diag", ctx.handle, _dptr(A, ctx), int(blockID), int(blockRow), int(blockStart),
             int(blockCount), int(blockCountXY))

    symmetricMatrixMatrixDiagonal_optimizedGPU = symmetricMatrixMatrixDiagonal
    symmetricMatrixMatrixDiagonal_optimizedCPU = symmetricMatrixMatrixDiagonal

    @staticmethod
    def matrixMatrixStep(ctx, A, blockID, blockRow, blockStart, blockCount, blockCountXY):
        call("hs_gemm_trailing", ctx.handle, _dptr(A, ctx), int(blockID), int(blockRow), int(blockStart),
             int(blockCount), int(blockCountXY))

    matrixMatrixStep_optimizedGPU = matrixMatrixStep
    matrixMatrixStep_optimizedGPU2 = matrixMatrixStep
    matrixMatrixStep_optimizedGPU3 = matrixMatrixStep
    matrixMatrixStep_optimizedCPU = matrixMatrixStep
    matrixMatrixStep_optimizedCPU2 = matrixMatrixStep


class MatrixVectorOperations:
    """src/kernel/MatrixVectorOperations.hpp:8-114 — SYMV, TRSV, column update."""

    @staticmethod
    def matrixVectorBlock(ctx, A, b, result, blockStart_i, blockStart_j, blockCount_i, blockCount_j,
                          blockCountXY, reset=True):
        call("hs_symv_block", ctx.handle, _dptr(A, ctx), _dptr(b, ctx), _dptr(result, ctx), int(blockStart_i),
             int(blockStart_j), int(blockCount_i), int(blockCount_j), int(blockCountXY), int(bool(reset)))

    matrixVectorBlock_GPU = matrixVectorBlock
    matrixVectorBlock_CPU = matrixVectorBlock

    @staticmethod
    def matrixVectorGP(ctx, A, b, result, n, m):
        """MatrixVectorOperations.cpp:379-395: result[i] = sum_k A[i*n+k] b[k], i < m."""
        call("hs_matrix_vector_gp", ctx.handle, _dptr(A, ctx), _dptr(b, ctx), _dptr(result, ctx), int(n), int(m))

    @staticmethod
    def triangularSolveBlockVector(ctx, A, b, blockRow, blockID, transposed):
        call("hs_trsv_block", ctx.handle, _dptr(A, ctx), _dptr(b, ctx), int(blockRow), int(blockID),
             int(bool(transposed)))

    @staticmethod
    def matrixVectorColumnUpdate(ctx, A, b, blockStart, blockCount, blockRow, blockID, blockCountXY, transposed):
        call("hs_column_update", ctx.handle, _dptr(A, ctx), _dptr(b, ctx), int(blockStart), int(blockCount),
             int(blockRow), int(blockID), int(blockCountXY), int(bool(transposed)))


def _dev_f64(x, ctx):
    t = x if isinstance(x, torch.Tensor) else torch.as_tensor(np.ascontiguousarray(x, dtype=np.float64))
    return _to_device(t.to(torch.float64), ctx).contiguous()


class VectorOperations:
    """src/kernel/VectorOperations.hpp:8-126 — block-range vector kernels."""

    @staticmethod
    def scaleVectorBlock(ctx, x, alpha, result, blockStart_i, blockCount_i):
        call("hs_scale_block", ctx.handle, _dptr(x, ctx), float(alpha), _dptr(result, ctx), int(blockStart_i),
             int(blockCount_i))

    @staticmethod
    def addVectorBlock(ctx, x, y, result, blockStart_i, blockCount_i):
        call("hs_add_block", ctx.handle, _dptr(x, ctx), _dptr(y, ctx), _dptr(result, ctx), int(blockStart_i),
             int(blockCount_i))

    @staticmethod
    def subVectorBlock(ctx, x, y, result, blockStart_i, blockCount_i):
        call("hs_sub_block", ctx.handle, _dptr(x, ctx), _dptr(y, ctx), _dptr(result, ctx), int(blockStart_i),
             int(blockCount_i))

    @staticmethod
    def scaleAndAddVectorBlock(ctx, x, alpha, y, result, blockStart_i, blockCount_i):
        call("hs_axpy_block", ctx.handle, _dptr(x, ctx), float(alpha), _dptr(y, ctx), _dptr(result, ctx),
             int(blockStart_i), int(blockCount_i))

    @staticmethod
    def scalarProduct(ctx, x, y, result, blockStart_i, blockCount_i):
        """Writes the finished dot product to result[0] and returns 1 (one
        partial), so that a following sumFinalScalarProduct is the identity —
        the reference's two calls (VectorOperations.cpp:84-185) in one."""
        call("hs_dot_block", ctx.handle, _dptr(x, ctx), _dptr(y, ctx), _dptr(result, ctx), int(blockStart_i),
             int(blockCount_i))
        return 1

    scalarProduct_CPU = scalarProduct

    @staticmethod
    def sumFinalScalarProduct(ctx, result, workGroupCount):
        if workGroupCount != 1:
            raise ValueError("workGroupCount must come from scalarProduct")

    sumFinalScalarProduct_CPU = sumFinalScalarProduct


# ------------------------------------------------------------------ solvers
def _to_device(t, ctx):
    return t if t.is_cuda else t.to(f"cuda:{ctx.device}", non_blocking=False).contiguous()


class Cholesky:
    """src/solver/cholesky/Cholesky.hpp:22-168: blocked right-looking Cholesky.

    ``solve_heterogeneous()`` factors A in place on the GPU (every block row on
    the GPU, no split or load balancing) and copies L back into
    ``A.matrixData`` when that lives on the host (copyResultFromGPU,
    Cholesky.cpp:361-397).  ``A_gpu`` keeps the device copy for the
    TriangularSystemSolver, as main.cpp:232 lends it.
    """

    def __init__(self, A, ctx):
        self.A = A
        self.ctx = ctx
        self.A_gpu = None
        self.info = -1
        self.factor_ms = None

    def solve_heterogeneous(self):
        ctx = self.ctx
        ctx.set_problem(self.A.N, self.A.blockSize)
        self.A_gpu = _to_device(self.A.matrixData, ctx)
        info = ctypes.c_int64(-1)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(ctx.stream)
        status = _lib.load().hs_cholesky_factor(ctx.handle, _dptr(self.A_gpu, ctx), ctypes.byref(info))
        ev1.record(ctx.stream)
        self.info = info.value
        _lib.check(status)
        ctx.stream.synchronize()
        self.factor_ms = ev0.elapsed_time(ev1)
        if not self.A.matrixData.is_cuda:
            self.A.matrixData.copy_(self.A_gpu.cpu())
        else:
            self.A.matrixData = self.A_gpu
        return self


class TriangularSystemSolver:
    """src/solver/cholesky/TriangularSystemSolver.hpp:10-39: forward then
    backward block substitution with the factor, in place on b."""

    def __init__(self, A, A_gpu, b, ctx):
        self.A = A
        self.A_gpu = A_gpu if A_gpu is not None else _to_device(A.matrixData, ctx)
        self.b = b
        self.ctx = ctx

    def solve(self):
        """Overwrites b.rightHandSideData with the solution; returns the time in ms."""
        ctx = self.ctx
        ctx.set_problem(self.A.N, self.A.blockSize)
        t0 = time.perf_counter()
        b_gpu = _to_device(self.b.rightHandSideData, ctx)
        if b_gpu is self.b.rightHandSideData:
            b_gpu = b_gpu.clone()
        call("hs_cholesky_solve", ctx.handle, _dptr(self.A_gpu, ctx), _dptr(b_gpu, ctx))
        ctx.stream.synchronize()
        if self.b.rightHandSideData.is_cuda:
            self.b.rightHandSideData.copy_(b_gpu)
        else:
            self.b.rightHandSideData.copy_(b_gpu.cpu())
        return (time.perf_counter() - t0) * 1e3


class CG:
    """src/solver/cg/CG.hpp:14-142: conjugate gradients on the packed matrix.

    ``solveHeterogeneous(epsilon, iMax)`` runs on the GPU (every block row);
    the solution lands in ``self.x`` (host tensor), the iteration count in
    ``self.iterations``.  Defaults follow Configuration.hpp:26-27.
    """

    def __init__(self, A, b, ctx):
        if A.N != b.N:
            raise ValueError(f"Dimensions of A and b do not match: {A.N} != {b.N}")
        if A.blockCountXY != b.blockCountX:
            raise ValueError(f"Block count of A and b do not match: {A.blockCountXY} != {b.blockCountX}")
        self.A = A
        self.b = b
        self.ctx = ctx
        self.x = torch.zeros_like(b.rightHandSideData, device="cpu")
        self.iterations = 0
        self.delta_new = None
        self.delta_zero = None

    def solveHeterogeneous(self, epsilon=1.0e-6, iMax=100000):
        ctx = self.ctx
        ctx.set_problem(self.A.N, self.A.blockSize)
        A_gpu = _to_device(self.A.matrixData, ctx)
        b_gpu = _to_device(self.b.rightHandSideData, ctx)
        x_gpu = torch.empty_like(b_gpu)
        it, dn, d0 = ctypes.c_int64(), ctypes.c_double(), ctypes.c_double()
        status = _lib.load().hs_cg_solve(ctx.handle, _dptr(A_gpu, ctx), _dptr(b_gpu, ctx), _dptr(x_gpu, ctx),
                                         float(epsilon), int(iMax), ctypes.byref(it), ctypes.byref(dn),
                                         ctypes.byref(d0))
        self.iterations, self.delta_new, self.delta_zero = it.value, dn.value, d0.value
        self.x = x_gpu.cpu()
        if status != 4:  # reaching iMax is reported but, as in the reference, not an exception
            _lib.check(status)
        return self


def cholesky_logdet(ctx, L):
    """log|K| = 2 sum log diag(L) of a packed device factor from Cholesky."""
    out = ctypes.c_double()
    call("hs_cholesky_logdet", ctx.handle, _dptr(L, ctx), ctypes.byref(out))
    return out.value


class MixedPrecisionSolver:
    """Mixed-precision solve of K x = b (no reference counterpart).

    The factor runs in FP32 with the panel TRSM and SYRK/GEMM trailing updates
    on the tensor cores as split products ("tf32x3": three TF32 products per
    FP32 product; "bf16x3" / "f16x3": the trailing updates as three BF16, or
    three FP16 products of the panel scaled by a power of two — 16 or 22
    significant bits at twice the TF32 rate) and every diagonal-block POTRF in
    FP64; FP64 iterative
    refinement then drives the backward error ||b - K x|| / (||K||_F ||x||)
    below ``tol``, continuing as CG preconditioned by the low-precision factor
    when refinement stalls.  K (packed, device) is left unchanged.
    """

    def __init__(self, A, ctx, precision="tf32x3"):
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
        self.A = A
        self.ctx = ctx
        self.precision = precision
        self.report = None

    def solve(self, b, tol=1e-14, max_steps=30, out=None):
        """b: padded RHS (device tensor or RightHandSide); returns x (device)."""
        ctx = self.ctx
        ctx.set_problem(self.A.N, self.A.blockSize)
        K = _to_device(self.A.matrixData, ctx)
        bd = b.rightHandSideData if isinstance(b, RightHandSide) else b
        bd = _to_device(bd, ctx)
        x = out if out is not None else torch.empty_like(bd)
        rep = MixedReport()
        status = _lib.load().hs_mixed_solve(ctx.handle, _dptr(K, ctx), _dptr(bd, ctx), _dptr(x, ctx),
                                            PRECISIONS[self.precision], float(tol), int(max_steps),
                                            ctypes.byref(rep))
        self.report = {f: getattr(rep, f) for f, _ in MixedReport._fields_ if f != "reserved"}
        _lib.check(status)
        return x


def cholesky_adjoint(ctx, L, Abar):
    """Reverse-mode blocked Cholesky: on entry ``Abar`` (packed, device) holds
    the adjoint of a scalar with respect to the lower blocks of the factor
    ``L``; on exit it holds the adjoint with respect to the lower entries of
    A = L L^T.  FP64 tensor-core products; L is not modified."""
    call("hs_cholesky_adjoint", ctx.handle, _dptr(L, ctx), _dptr(Abar, ctx))
    return Abar


def gp_nlml_grad(ctx, X, y, theta, n_ell=None, precision=None, tol=1e-14):
    """GP negative log marginal likelihood and its gradient with respect to
    theta = [log l_1..log l_n_ell, log sf2, log sn2] (FP64 factor, reverse-mode
    Cholesky and an on-the-fly dK/dtheta contraction).  X (N x d) and y (N)
    may be host or device float64 arrays; returns (nlml, grad ndarray, report).
    With ``precision`` ("tf32x3", "bf16x3" or "f16x3") the factor is the
    mixed-precision one (hs_gp_nlml_grad_mixed): alpha refined in FP64 to the
    backward error ``tol``; the report then also holds the solve's report under
    "mixed"."""
    if precision is not None and precision not in PRECISIONS:
        raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
    Xd = X if isinstance(X, torch.Tensor) else torch.as_tensor(np.ascontiguousarray(X, dtype=np.float64))
    yd = y if isinstance(y, torch.Tensor) else torch.as_tensor(np.ascontiguousarray(y, dtype=np.float64))
    Xd = _to_device(Xd.to(torch.float64), ctx).contiguous()
    yd = _to_device(yd.to(torch.float64), ctx).contiguous()
    if Xd.dim() != 2 or Xd.shape[0] != ctx.N or yd.numel() != ctx.N:
        raise ValueError("X must be N x d and y of length N (N of the context)")
    th = np.ascontiguousarray(np.asarray(theta, dtype=np.float64).ravel())
    if n_ell is None:
        n_ell = th.size - 2
    if th.size != n_ell + 2:
        raise ValueError("theta must hold n_ell + 2 values")
    nlml = ctypes.c_double()
    grad = np.zeros(n_ell + 2)
    rep = GpReport()
    if precision is None or precision == "fp64":
        call("hs_gp_nlml_grad", ctx.handle, _dptr(Xd, ctx), _dptr(yd, ctx), int(Xd.shape[1]),
             th.ctypes.data_as(ctypes.c_void_p), int(n_ell), ctypes.byref(nlml),
             grad.ctypes.data_as(ctypes.c_void_p), ctypes.byref(rep))
        return nlml.value, grad, {f: getattr(rep, f) for f, _ in GpReport._fields_}
    mrep = MixedReport()
    call("hs_gp_nlml_grad_mixed", ctx.handle, _dptr(Xd, ctx), _dptr(yd, ctx), int(Xd.shape[1]),
         th.ctypes.data_as(ctypes.c_void_p), int(n_ell), int(PRECISIONS[precision]), float(tol), ctypes.byref(nlml),
         grad.ctypes.data_as(ctypes.c_void_p), ctypes.byref(rep), ctypes.byref(mrep))
    out = {f: getattr(rep, f) for f, _ in GpReport._fields_}
    out["mixed"] = {f: getattr(mrep, f) for f, _ in MixedReport._fields_ if f != "reserved"}
    return nlml.value, grad, out


def fit_hyperparameters(ctx, X, y, theta0, maxiter=30, n_ell=None, bounds=None, precision=None, tol=1e-14):
    """Fit theta = [log l_1..log l_n_ell, log sf2, log sn2] by L-BFGS (scipy's
    L-BFGS-B) on the NLML and its analytic gradient (hs_gp_nlml_grad, or the
    mixed-precision form with ``precision``).  X and y are copied to the device
    once.  Returns a dict with theta, nlml, the number of L-BFGS iterations and
    function evaluations, and the wall time of every NLML + gradient
    evaluation."""
    from scipy.optimize import minimize

    Xd = X if isinstance(X, torch.Tensor) else torch.as_tensor(np.ascontiguousarray(X, dtype=np.float64))
    yd = y if isinstance(y, torch.Tensor) else torch.as_tensor(np.ascontiguousarray(y, dtype=np.float64))
    Xd = _to_device(Xd.to(torch.float64), ctx).contiguous()
    yd = _to_device(yd.to(torch.float64), ctx).contiguous()
    th0 = np.asarray(theta0, dtype=np.float64).ravel()
    n_ell = th0.size - 2 if n_ell is None else n_ell
    evals = []

    def fun(th):
        t0 = time.perf_counter()
        v, g, _ = gp_nlml_grad(ctx, Xd, yd, th, n_ell, precision=precision, tol=tol)
        evals.append({"seconds": time.perf_counter() - t0, "nlml": v})
        return v, g

    res = minimize(fun, th0, jac=True, method="L-BFGS-B", bounds=bounds, options={"maxiter": int(maxiter)})
    return {"theta": res.x, "nlml": float(res.fun), "iterations": int(res.nit), "evaluations": len(evals),
            "eval_seconds": [e["seconds"] for e in evals], "nlml_trace": [e["nlml"] for e in evals],
            "message": str(res.message)}


class GaussianProcessNLML(torch.autograd.Function):
    """torch.autograd.Function over hs_gp_nlml_grad: forward returns the NLML
    of theta (a float64 tensor of n_ell + 2 log-parameters), backward returns
    the library's analytic gradient times the incoming gradient.

        nlml = GaussianProcessNLML.apply(theta, X, y, ctx)
    """

    @staticmethod
    def forward(fctx, theta, X, y, ctx):
        th = theta.detach().to("cpu", torch.float64).numpy()
        value, grad, _ = gp_nlml_grad(ctx, X, y, th)
        fctx.save_for_backward(torch.from_numpy(grad).to(theta.device, theta.dtype))
        return torch.tensor(value, dtype=theta.dtype, device=theta.device)

    @staticmethod
    def backward(fctx, g):
        (grad,) = fctx.saved_tensors
        return g * grad, None, None, None


class MatrixGenerator:
    """src/utility/MatrixGenerator.hpp:11-65 — kernel-matrix generation on the GPU."""

    @staticmethod
    def windowInputs(series):
        """The reference's sliding window of 8 regressors (MatrixGenerator.cpp:76-99):
        X[i, k] = series[i + k - 7], zeros before the series start."""
        s = np.asarray(series, dtype=np.float64)
        padded = np.concatenate([np.zeros(7), s])
        return np.lib.stride_tricks.sliding_window_view(padded, 8)[: len(s)].copy()

    @staticmethod
    def assemble(ctx, A, X, lengthscale=1.0, signal_variance=1.0, noise_variance=0.01):
        """K = sf2 * exp(-|x_i - x_j|^2 / (2 l^2)) + sn2 I into the packed device
        tensor A; ``lengthscale`` is a scalar or one value per feature (ARD)."""
        Xd = X if isinstance(X, torch.Tensor) else torch.as_tensor(np.ascontiguousarray(X, dtype=np.float64))
        Xd = _to_device(Xd.to(torch.float64), ctx).contiguous()
        if Xd.dim() != 2 or Xd.shape[0] != ctx.N:
            raise ValueError("X must be N x d")
        ell = np.atleast_1d(np.asarray(lengthscale, dtype=np.float64))
        call("hs_rbf_assemble", ctx.handle, _dptr(A, ctx), _dptr(Xd, ctx), int(Xd.shape[1]),
             ell.ctypes.data_as(ctypes.c_void_p), int(ell.size), float(signal_variance), float(noise_variance))

    @staticmethod
    def generateTestKernelMatrix(ctx, X, X_test, lengthscale=1.0, signal_variance=1.0, out=None):
        """MatrixGenerator.cpp:163-213: K_star (N_test x N, row major, device)
        with K_star[j, i] = sf2 exp(-|x_i - x*_j|^2 / (2 l^2)) (l scalar or ARD)."""
        Xd, Xt = _dev_f64(X, ctx), _dev_f64(X_test, ctx)
        if Xd.dim() != 2 or Xd.shape[0] != ctx.N or Xt.dim() != 2 or Xt.shape[1] != Xd.shape[1]:
            raise ValueError("X must be N x d and X_test N_test x d")
        ell = np.atleast_1d(np.asarray(lengthscale, dtype=np.float64))
        K = out if out is not None else torch.empty((Xt.shape[0], Xd.shape[0]), dtype=torch.float64,
                                                    device=f"cuda:{ctx.device}")
        call("hs_gp_test_kernel_matrix", ctx.handle, _dptr(Xd, ctx), _dptr(Xt, ctx), int(Xt.shape[0]),
             int(Xd.shape[1]), ell.ctypes.data_as(ctypes.c_void_p), int(ell.size), float(signal_variance),
             _dptr(K, ctx))
        return K

    @staticmethod
    def generateSPDMatrix(ctx, series, N, matrixBlockSize, lengthscale=1.0, signal_variance=1.0,
                          noise_variance=0.01):
        """generateSPDMatrix (MatrixGenerator.cpp:73-162): the first N values of
        a 1-D series (array or path of one value per line), 8-sample window,
        defaults l = 1, sf2 = 1, sn2 = 0.01; returns a device SymmetricMatrix."""
        if isinstance(series, (str, Path)):
            series = np.loadtxt(series, dtype=np.float64, ndmin=1)
        series = np.asarray(series, dtype=np.float64)
        if series.size < N:
            raise ValueError("Not enough data available!")
        ctx.set_problem(N, matrixBlockSize)
        A = SymmetricMatrix(N, matrixBlockSize, device=f"cuda:{ctx.device}")
        MatrixGenerator.assemble(ctx, A.matrixData, MatrixGenerator.windowInputs(series[:N]), lengthscale,
                                 signal_variance, noise_variance)
        return A


def gp_predict(ctx, X, X_test, alpha, lengthscale=1.0, signal_variance=1.0):
    """Predictive mean K_star alpha with K_star recomputed on the fly (never
    stored); alpha = K^-1 y of length N (padding beyond N is ignored)."""
    Xd, Xt = _dev_f64(X, ctx), _dev_f64(X_test, ctx)
    al = _dev_f64(alpha, ctx)
    ell = np.atleast_1d(np.asarray(lengthscale, dtype=np.float64))
    mean = torch.empty(Xt.shape[0], dtype=torch.float64, device=f"cuda:{ctx.device}")
    call("hs_gp_predict", ctx.handle, _dptr(Xd, ctx), _dptr(Xt, ctx), int(Xt.shape[0]), int(Xd.shape[1]),
         ell.ctypes.data_as(ctypes.c_void_p), int(ell.size), float(signal_variance), _dptr(al, ctx), _dptr(mean, ctx))
    return mean


class GaussianProcess:
    """src/gaussianProcess/GaussianProcess.hpp:10-36: the prediction pipeline.

    ``start()`` solves K alpha = y with the Cholesky factor + substitution or
    with CG (GaussianProcess.cpp:20-40), then forms K_star from the training and
    test inputs and returns K_star alpha (:42-54), as a host numpy array.
    Inputs are the reference's one-value-per-line series files (or arrays),
    windowed into 8 regressors (MatrixGenerator.cpp:76-99), or N x d arrays.
    """

    def __init__(self, A, train_y, path_train, path_test, ctx, algorithm="cholesky", lengthscale=1.0,
                 signal_variance=1.0, N_test=None, fused=True):
        self.A = A
        self.train_y = train_y
        self.path_train = path_train
        self.path_test = path_test
        self.ctx = ctx
        self.algorithm = algorithm
        self.lengthscale = lengthscale
        self.signal_variance = signal_variance
        self.N_test = N_test
        self.fused = fused
        self.result = None

    @staticmethod
    def _inputs(src, n=None):
        """Series file / 1-D series -> 8-regressor window rows; N x d arrays as they are."""
        a = np.loadtxt(src, dtype=np.float64, ndmin=1) if isinstance(src, (str, Path)) else np.asarray(
            src, dtype=np.float64)
        if n is not None and a.shape[0] < n:
            raise ValueError("Not enough data available!")
        a = a[:n] if n is not None else a
        return MatrixGenerator.windowInputs(a) if a.ndim == 1 else a

    def start(self):
        ctx = self.ctx
        N = self.A.N
        if self.algorithm == "cg":
            cg = CG(self.A, self.train_y, ctx).solveHeterogeneous()
            alpha = cg.x.to(f"cuda:{ctx.device}")
        elif self.algorithm == "cholesky":
            chol = Cholesky(self.A, ctx).solve_heterogeneous()
            TriangularSystemSolver(self.A, chol.A_gpu, self.train_y, ctx).solve()
            alpha = _to_device(self.train_y.rightHandSideData, ctx)
        else:
            raise RuntimeError(f"Invalid algorithm: {self.algorithm}")
        X = self._inputs(self.path_train, N)
        Xt = self._inputs(self.path_test, self.N_test)
        ctx.set_problem(N, self.A.blockSize)
        if self.fused:
            mean = gp_predict(ctx, X, Xt, alpha[:N].contiguous(), self.lengthscale, self.signal_variance)
        else:
            Ks = MatrixGenerator.generateTestKernelMatrix(ctx, X, Xt, self.lengthscale, self.signal_variance)
            mean = torch.empty(Xt.shape[0], dtype=torch.float64, device=f"cuda:{ctx.device}")
            MatrixVectorOperations.matrixVectorGP(ctx, Ks, alpha[:N].contiguous(), mean, N, Xt.shape[0])
        self.result = mean.cpu().numpy()
        return self.result


class UtilityFunctions:
    """src/utility/UtilityFunctions.hpp: output helpers."""

    @staticmethod
    def writeResult(path, x):
        """UtilityFunctions.cpp:19-33: `x_result.txt` in `path`, every value with
        20 fixed decimals followed by a space, then a newline."""
        vals = x.detach().cpu().numpy() if isinstance(x, torch.Tensor) else np.asarray(x, dtype=np.float64)
        out = Path(path) / "x_result.txt"
        out.write_text("".join(f"{v:.20f} " for v in vals) + "\n")
        return out


class MatrixParser:
    """src/utility/MatrixParser.hpp:10-73 — the reference's text formats."""

    @staticmethod
    def _rows(text):
        lines = [ln for ln in text.strip().splitlines()]
        if not lines or not lines[0].startswith("#"):
            raise ValueError("Invalid matrix format. First line has to be '# <N>!'")
        return int(lines[0][2:]), lines[1:]

    @staticmethod
    def parseSymmetricMatrix(path, matrixBlockSize):
        """`# N` then row i holding its lower-triangle values `v; v; ...`
        (MatrixParser.cpp:11-41, processRow :107-168); diagonal blocks mirrored."""
        N, lines = MatrixParser._rows(Path(path).read_text())
        A = SymmetricMatrix(N, matrixBlockSize)
        b, nb = matrixBlockSize, A.blockCountXY
        data = A.matrixData.numpy()
        for i, line in enumerate(lines[:N]):
            vals = [float(v) for v in line.split(";")]
            if len(vals) != i + 1:
                raise ValueError(f"row {i} has {len(vals)} values, expected {i + 1}")
            bi, ri = divmod(i, b)
            for j, v in enumerate(vals):
                bj, rj = divmod(j, b)
                base = block_id(bi, bj, nb) * b * b
                data[base + ri * b + rj] = v
                if bi == bj:
                    data[base + rj * b + ri] = v
        return A

    @staticmethod
    def writeFullMatrix(path, matrix):
        """MatrixParser.cpp:214-274: every row of the padded matrix, the stored
        blocks left of and on the diagonal read row-wise and the blocks right of
        it read transposed, each value with 20 fixed decimals followed by ';'
        (non-negative values preceded by a space), one line per row."""
        b, nb = matrix.blockSize, matrix.blockCountXY
        data = matrix.matrixData.detach().cpu().numpy()
        with open(path, "w") as out:
            for row in range(nb * b):
                rb, ri = divmod(row, b)
                parts = []
                for cb in range(nb):
                    if cb <= rb:
                        s0 = block_id(rb, cb, nb) * b * b
                        vals = data[s0 + ri * b:s0 + (ri + 1) * b]
                    else:
                        s0 = block_id(cb, rb, nb) * b * b
                        vals = data[s0 + ri:s0 + b * b:b]
                    parts.extend((" " if v >= 0 else "") + f"{v:.20f};" for v in vals)
                out.write("".join(parts) + "\n")

    @staticmethod
    def parseRightHandSide(path, matrixBlockSize):
        """`# N` then one line `v; v; ...` (MatrixParser.cpp:43-72)."""
        N, lines = MatrixParser._rows(Path(path).read_text())
        vals = [float(v) for v in lines[0].split(";")]
        b = RightHandSide(N, matrixBlockSize)
        b.rightHandSideData[:N] = torch.tensor(vals[:N], dtype=torch.float64)
        return b


# hs_gp_solve_host algorithms
_ALGORITHMS = {"cholesky": 0, "cg": 1, "mixed": 2, "mixed_tf32x3": 2, "mixed_bf16x3": 3, "mixed_f16x3": 4}


def gp_solve_host(ctx, X, y, lengthscale=1.0, signal_variance=1.0, noise_variance=0.01, algorithm="cholesky",
                  epsilon=1e-10, iMax=100000, out=None):
    """End-to-end GP solve through host buffers (hs_gp_solve_host): host X
    (N x d) and y (N) in, host x = K^-1 y out, plus the phase report.
    ``algorithm`` is "cholesky", "cg", "mixed" / "mixed_tf32x3", "mixed_bf16x3" or "mixed_f16x3"
    (for the mixed forms, ``epsilon`` is the backward-error target and ``iMax``
    the refinement step limit).  X, y
    and ``out`` may be CPU torch tensors (pinned memory gives asynchronous
    copies) or numpy arrays."""
    if algorithm not in _ALGORITHMS:
        raise ValueError(f"algorithm must be one of {sorted(_ALGORITHMS)}")

    def host(a, shape=None):
        if isinstance(a, torch.Tensor):
            if a.is_cuda or a.dtype != torch.float64 or not a.is_contiguous():
                raise TypeError("host tensors must be contiguous CPU float64")
            return a, ctypes.c_void_p(a.data_ptr())
        a = np.ascontiguousarray(a, dtype=np.float64)
        return a, a.ctypes.data_as(ctypes.c_void_p)

    X, Xp = host(X)
    y, yp = host(y)
    N, d = X.shape
    if ctx.N != N:
        raise ValueError("context N differs from X")
    ell = np.atleast_1d(np.asarray(lengthscale, dtype=np.float64))
    x, xp = host(out if out is not None else np.empty(N, dtype=np.float64))
    rep = SolveReport()
    call("hs_gp_solve_host", ctx.handle, Xp, yp, d, ell.ctypes.data_as(ctypes.c_void_p), int(ell.size),
         float(signal_variance), float(noise_variance), _ALGORITHMS[algorithm], float(epsilon),
         int(iMax), xp, ctypes.byref(rep))
    return x, rep
