"""GPU suite: every reference GoogleTest case replayed against the CUDA kernels
through the C ABI (libhs_b200.so), with the reference's own golden arrays and
its tolerance (EXPECT_NEAR 1e-12)."""
import numpy as np
import pytest
import torch

from reference_cases import load_cases, run_case

pytestmark = pytest.mark.gpu

DATA = load_cases()
CASES = [c for c in DATA["cases"] if any(s["op"] == "call" for s in c["steps"])]


class GpuBackend:
    """Runs each reference kernel call on the GPU: numpy arrays are copied to
    CUDA tensors (aliases preserved), the operator runs, results are copied
    back in place."""

    def __init__(self, hs, ctx):
        self.hs = hs
        self.ctx = ctx

    def run(self, op, args, N, bsz):
        hs, ctx = self.hs, self.ctx
        ctx.set_problem(N, bsz)
        dev = {}
        targs = []
        for a in args:
            if isinstance(a, np.ndarray):
                if id(a) not in dev:
                    dev[id(a)] = (a, torch.from_numpy(a).to(f"cuda:{ctx.device}"))
                targs.append(dev[id(a)][1])
            else:
                targs.append(a)
        ret = None
        MO, MMO, MVO, VO = hs.MatrixOperations, hs.MatrixMatrixOperations, hs.MatrixVectorOperations, \
            hs.VectorOperations
        if op == "potrf":
            MO.cholesky(ctx, *targs)
        elif op == "trsm":
            MMO.triangularSolve(ctx, *targs)
        elif op == "syrk":
            MMO.symmetricMatrixMatrixDiagonal(ctx, *targs)
        elif op == "gemm":
            MMO.matrixMatrixStep(ctx, *targs)
        elif op == "symv":
            MVO.matrixVectorBlock(ctx, *targs)
        elif op == "trsv":
            MVO.triangularSolveBlockVector(ctx, *targs)
        elif op == "colupd":
            MVO.matrixVectorColumnUpdate(ctx, *targs)
        elif op == "scale":
            VO.scaleVectorBlock(ctx, *targs)
        elif op == "add":
            VO.addVectorBlock(ctx, *targs)
        elif op == "sub":
            VO.subVectorBlock(ctx, *targs)
        elif op == "axpy":
            VO.scaleAndAddVectorBlock(ctx, *targs)
        elif op == "dot":
            ret = VO.scalarProduct(ctx, *targs)
        elif op == "dotfinal":
            VO.sumFinalScalarProduct(ctx, *targs)
        else:
            raise KeyError(op)
        ctx.sync()
        for a, t in dev.values():
            a[...] = t.cpu().numpy()
        return ret


@pytest.mark.parametrize("case", CASES, ids=[f"{c['suite']}.{c['name']}" for c in CASES])
def test_gpu_matches_reference_golden(case, hs, ctx):
    key = f"{case['file']}::{case['suite']}"
    failures = run_case(case, DATA["suite_arrays"].get(key, {}), DATA["fixtures"], GpuBackend(hs, ctx))
    assert not failures, "; ".join(failures[:3])
