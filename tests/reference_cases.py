"""Replays the reference's GoogleTest cases (tests/golden/reference_cases.json).

Each case is the ordered list of steps of one TEST_F of the reference
(TimThuering/Heterogeneous-Solvers tests/*.cpp): configuration assignments,
fixture parsing, vector set-up, kernel calls with their literal argument
expressions, and expectations against the literal golden arrays.  A backend
executes the kernel calls: ``OracleBackend`` (CPU restatement, pins the
oracle) or the GPU backend in test_gpu_reference_cases.py (the CUDA library
through its C ABI).  Every reference kernel variant (CPU, GPU, optimised)
maps to the one implementation under test, as the variants compute the same
function.
"""
import json
import math
import re
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden" / "reference_cases.json"


def load_cases():
    return json.loads(GOLDEN.read_text())


class Matrix:
    """Stand-in for SymmetricMatrix: packed numpy data + shape fields."""

    def __init__(self, N, bsz):
        self.N = N
        self.blockSize = bsz
        self.blockCountXY = -(-N // bsz)
        nb = self.blockCountXY
        self.matrixData = np.zeros(nb * (nb + 1) // 2 * bsz * bsz)


class Rhs:
    def __init__(self, N, bsz):
        self.N = N
        self.blockSize = bsz
        self.blockCountX = -(-N // bsz)
        self.rightHandSideData = np.zeros(self.blockCountX * bsz)


def parse_matrix(fixture, bsz):
    """MatrixParser::parseSymmetricMatrix (MatrixParser.cpp:11-41, :107-168)."""
    N = fixture["N"]
    A = Matrix(N, bsz)
    nb = A.blockCountXY
    for i, row in enumerate(fixture["rows"]):
        bi, ri = divmod(i, bsz)
        for j, v in enumerate(row):
            bj, rj = divmod(j, bsz)
            base = (bi + nb * (nb - 1) // 2 - (nb - bj - 1) * (nb - bj) // 2) * bsz * bsz
            A.matrixData[base + ri * bsz + rj] = v
            if bi == bj:
                A.matrixData[base + rj * bsz + ri] = v
    return A


def parse_rhs(fixture, bsz):
    b = Rhs(fixture["N"], bsz)
    b.rightHandSideData[: fixture["N"]] = fixture["values"]
    return b


def to_py(expr):
    e = expr.replace(".data()", "").replace(".size()", ".size")
    e = re.sub(r"\btrue\b", "True", e)
    e = re.sub(r"\bfalse\b", "False", e)
    e = e.replace("std::sqrt", "math.sqrt")
    return e


# reference kernel name -> (operation, argument roles after the queue)
KERNELS = {
    "cholesky": "potrf", "cholesky_GPU": "potrf", "cholesky_optimizedGPU": "potrf",
    "triangularSolve": "trsm", "triangularSolve_optimizedGPU": "trsm", "triangularSolve_optimizedCPU": "trsm",
    "symmetricMatrixMatrixDiagonal": "syrk", "symmetricMatrixMatrixDiagonal_optimizedGPU": "syrk",
    "symmetricMatrixMatrixDiagonal_optimizedCPU": "syrk",
    "matrixMatrixStep": "gemm", "matrixMatrixStep_optimizedGPU": "gemm", "matrixMatrixStep_optimizedGPU2": "gemm",
    "matrixMatrixStep_optimizedGPU3": "gemm", "matrixMatrixStep_optimizedCPU": "gemm",
    "matrixMatrixStep_optimizedCPU2": "gemm",
    "matrixVectorBlock": "symv", "matrixVectorBlock_GPU": "symv", "matrixVectorBlock_CPU": "symv",
    "triangularSolveBlockVector": "trsv", "matrixVectorColumnUpdate": "colupd",
    "scaleVectorBlock": "scale", "addVectorBlock": "add", "subVectorBlock": "sub",
    "scaleAndAddVectorBlock": "axpy", "scalarProduct": "dot", "scalarProduct_CPU": "dot",
    "sumFinalScalarProduct": "dotfinal", "sumFinalScalarProduct_CPU": "dotfinal",
}


class OracleBackend:
    """Runs the kernel calls on the CPU oracle (oracle/hs_oracle.c)."""

    name = "oracle"

    def __init__(self):
        import oracle_lib
        self.o = oracle_lib
        self.lib = oracle_lib.lib()

    def run(self, op, args, N, bsz):
        p, lib = self.o.ptr, self.lib
        if op == "potrf":
            A, blockID, blockRow = args
            lib.or_potrf_block(p(A), N, bsz, blockID, blockRow)
        elif op == "trsm":
            A, blockID, blockRow, start, count = args
            lib.or_trsm_panel(p(A), bsz, blockID, blockRow, start, count)
        elif op == "syrk":
            A, blockID, blockRow, start, count, nb = args
            lib.or_syrk_diag(p(A), bsz, blockID, blockRow, start, count, nb)
        elif op == "gemm":
            A, blockID, blockRow, start, count, nb = args
            lib.or_gemm_trailing(p(A), bsz, blockID, blockRow, start, count, nb)
        elif op == "symv":
            A, b, res, bi0, bj0, nbi, nbj, nb = args[:8]
            reset = args[8] if len(args) > 8 else True
            lib.or_symv_block(p(A), p(b), p(res), bsz, bi0, bj0, nbi, nbj, nb, int(reset))
        elif op == "trsv":
            A, b, blockRow, blockID, tr = args
            lib.or_trsv_block(p(A), p(b), N, bsz, blockRow, blockID, int(tr))
        elif op == "colupd":
            A, b, start, count, blockRow, blockID, nb, tr = args
            lib.or_column_update(p(A), p(b), bsz, start, count, blockRow, blockID, nb, int(tr))
        elif op == "scale":
            x, alpha, res, bi0, nbi = args
            lib.or_scale_block(p(x), alpha, p(res), bsz, bi0, nbi)
        elif op in ("add", "sub"):
            x, y, res, bi0, nbi = args
            getattr(lib, f"or_{op}_block")(p(x), p(y), p(res), bsz, bi0, nbi)
        elif op == "axpy":
            x, alpha, y, res, bi0, nbi = args
            lib.or_axpy_block(p(x), alpha, p(y), p(res), bsz, bi0, nbi)
        elif op == "dot":
            x, y, res, bi0, nbi = args
            res[0] = lib.or_dot_block(p(x), p(y), bsz, bi0, nbi, 8)
            return 1
        elif op == "dotfinal":
            return None
        else:
            raise KeyError(op)
        return None


def run_case(case, suite_arrays, fixtures, backend, parse_matrix_fn=None):
    """Executes one reference test; returns a list of failure strings.
    ``parse_matrix_fn(fixture, bsz)`` replaces the built-in fixture parser."""
    parse_matrix_fn = parse_matrix_fn or parse_matrix
    conf = {}
    ns = {"math": math}
    ns.update({k: np.asarray(v) for k, v in suite_arrays.items()})
    ns.update({k: np.asarray(v) for k, v in case["arrays"].items()})
    failures = []
    N = None
    for step in case["steps"]:
        op = step["op"]
        if op == "conf":
            conf[step["key"]] = eval(to_py(step["value"]), {}, {})
        elif op == "parse_matrix":
            ns[step["var"]] = parse_matrix_fn(fixtures["matrix"], conf["matrixBlockSize"])
            N = fixtures["matrix"]["N"]
        elif op == "parse_rhs":
            ns[step["var"]] = parse_rhs(fixtures["vector"], conf["matrixBlockSize"])
            if N is None:
                N = fixtures["vector"]["N"]
        elif op == "resize":
            size = int(eval(to_py(step["size"]), {}, ns))
            ns[step["var"]] = np.full(size, step.get("fill", 0.0))
        elif op == "fill":
            lo = int(eval(to_py(step["lo"]), {}, ns))
            hi = int(eval(to_py(step["hi"]), {}, ns))
            vec = ns[step["var"]]
            for i in range(lo, hi):
                vec[i] = eval(to_py(step["expr"]), {"math": math}, {"i": i})
        elif op == "call":
            kern = KERNELS[step["fn"]]
            args = [eval(to_py(a), {}, ns) for a in step["args"][1:]]
            bsz = conf["matrixBlockSize"]
            n_eff = N
            if n_eff is None:  # vector-only test: the vector's own length
                n_eff = next(len(a) for a in args if isinstance(a, np.ndarray))
            ret = backend.run(kern, args, n_eff, bsz)
            if step.get("ret"):
                ns[step["ret"]] = ret
        elif op == "expect_loop":
            count = int(eval(to_py(step["count"]), {}, ns))
            act = np.array([eval(to_py(step["actual"]), {}, dict(ns, i=i)) for i in range(count)])
            exp = np.array([eval(to_py(step["expected"]), {}, dict(ns, i=i)) for i in range(count)])
            bad = np.nonzero(~(np.abs(act - exp) <= step["tol"]))[0]
            if bad.size:
                k = bad[0]
                failures.append(f"{step['actual']} at i={k}: {act[k]!r} vs {exp[k]!r} "
                                f"({bad.size} of {count} beyond {step['tol']})")
        elif op == "expect_near":
            act = float(eval(to_py(step["actual"]), {}, ns))
            exp = step["expected"]
            exp = float(exp) if not isinstance(exp, str) else float(eval(to_py(exp), {}, ns))
            if not abs(act - exp) <= step["tol"]:
                failures.append(f"{step['actual']}: {act!r} vs {exp!r}")
        elif op in ("expect_double_eq", "expect_eq"):
            act = eval(to_py(step["actual"]), {}, ns)
            exp = eval(to_py(step["expected"]), {}, ns)
            ok = (abs(float(act) - float(exp)) <= 4 * np.spacing(abs(float(exp)))) if op == "expect_double_eq" \
                else act == exp
            if not ok:
                failures.append(f"{op} {step['actual']}: {act!r} vs {exp!r}")
    return failures
