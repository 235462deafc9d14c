"""CPU suite: the oracle and the host-side parser against the reference's own
golden vectors (every TEST_F of the reference's tests/*.cpp, replayed)."""
import numpy as np
import pytest

from reference_cases import OracleBackend, load_cases, run_case

DATA = load_cases()
CASES = DATA["cases"]


def _id(case):
    return f"{case['suite']}.{case['name']}"


@pytest.fixture(scope="module")
def backend():
    return OracleBackend()


def test_extracted_every_reference_test():
    # 2 parser + 16 POTRF + 55 TRSM/SYRK/GEMM + 36 matvec + 27 vector tests in the reference
    assert len(CASES) == 136
    assert all(any(s["op"].startswith("expect") for s in c["steps"]) for c in CASES)


@pytest.mark.parametrize("case", CASES, ids=[_id(c) for c in CASES])
def test_oracle_matches_reference_golden(case, backend):
    key = f"{case['file']}::{case['suite']}"
    failures = run_case(case, DATA["suite_arrays"].get(key, {}), DATA["fixtures"], backend)
    assert not failures, "; ".join(failures[:3])


def _product_parser(hs, tmp_path):
    def parse(fixture, bsz):
        path = tmp_path / "matrix.txt"
        rows = ["; ".join(repr(v) for v in row) for row in fixture["rows"]]
        path.write_text(f"# {fixture['N']}\n" + "\n".join(rows) + "\n")
        A = hs.MatrixParser.parseSymmetricMatrix(path, bsz)
        A.matrixData = A.matrixData.numpy()
        return A
    return parse


PARSER_CASES = [c for c in CASES if c["suite"] == "SymmetricMatrixTest"]


@pytest.mark.parametrize("case", PARSER_CASES, ids=[_id(c) for c in PARSER_CASES])
def test_host_parser_matches_reference(case, backend, hs, tmp_path):
    key = f"{case['file']}::{case['suite']}"
    failures = run_case(case, DATA["suite_arrays"].get(key, {}), DATA["fixtures"], backend,
                        parse_matrix_fn=_product_parser(hs, tmp_path))
    assert not failures, "; ".join(failures[:3])


def test_gemm_block_ids_match_reference_formula():
    """The reference's GEMM addresses A_rc through its own closed form
    (MatrixMatrixOperations.cpp:397-404); it equals the storage formula."""
    from oracle_lib import block_id
    for nb in range(3, 12):
        for blockRow in range(0, nb - 2):
            blockID = block_id(blockRow, blockRow, nb)
            V = nb - blockRow - 2
            total = V * (V + 1) // 2
            for rowID in range(V):
                for colID in range(rowID + 1):
                    ref = (blockID + nb - blockRow + colID + 1 +
                           (total - ((nb - blockRow - 2 - colID) * (nb - blockRow - 2 - colID + 1) // 2)) +
                           rowID - colID)
                    assert ref == block_id(blockRow + 2 + rowID, blockRow + 1 + colID, nb)


class _PerturbingBackend:
    """Oracle backend whose outputs are nudged by 1e-9: the replay must notice."""

    def __init__(self, inner):
        self.inner = inner

    def run(self, op, args, N, bsz):
        ret = self.inner.run(op, args, N, bsz)
        for a in args:
            if isinstance(a, np.ndarray):
                a += 1e-9
        return ret


@pytest.mark.parametrize("name", ["choleskyKernelFullMatrix", "gemmFullLowerBlockTriangle", "fullMatrixVector",
                                  "testTRSV", "scalarProuctFull"])
def test_replay_detects_planted_error(name, backend):
    case = next(c for c in CASES if c["name"] == name)
    key = f"{case['file']}::{case['suite']}"
    failures = run_case(case, DATA["suite_arrays"].get(key, {}), DATA["fixtures"], _PerturbingBackend(backend))
    assert failures
