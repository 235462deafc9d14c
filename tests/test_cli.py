"""CPU suite: the reference-compatible command line (flag parsing, defaults,
errors of src/main.cpp:37-186), the metrics.json layout and the factor writer
(MatrixParser::writeFullMatrix) on the reference's own 20x20 fixture."""
import json
import sys
from pathlib import Path

import numpy as np
import pytest
import torch

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "heterogeneous-solvers_b200"))
import cli  # noqa: E402


def test_defaults_follow_configuration_hpp():
    c = cli.parse_args(["--path_A", "A.txt", "--path_b", "b.txt"])
    assert c["algorithm"] == "cg" and c["matrixBlockSize"] == 128 and c["iMax"] == 100000
    assert c["epsilon"] == 1e-6 and c["mode"] == "static" and c["outputPath"] == "./output"
    assert not c["writeResult"] and not c["generateMatrix"]


def test_flags_and_booleans():
    c = cli.parse_args(["--gp_input", "x", "--gp_output", "y", "--size", "4096", "--test_size", "10",
                        "--algorithm", "cholesky", "--matrix_bsz", "256", "--write_result", "true", "--check_result",
                        "--eps", "1e-10", "--i_max", "500", "--init_gpu_perc", "1", "--mode", "power"])
    assert c["generateMatrix"] and c["N"] == 4096 and c["N_test"] == 10
    assert c["algorithm"] == "cholesky" and c["matrixBlockSize"] == 256 and c["workGroupSize"] == 256
    assert c["writeResult"] and c["checkResult"] and c["epsilon"] == 1e-10 and c["iMax"] == 500


@pytest.mark.parametrize("argv,msg", [
    (["--path_A", "a"], "No path to .txt file"),
    (["--gp_input", "x", "--gp_output", "y", "--mode", "fast"], "Invalid mode selected"),
    (["--gpr", "true", "--gp_input", "x", "--gp_output", "y"], "Not all required arguments for GPR"),
    (["--path_A", "a", "--path_b", "b", "--algorithm", "lu"], "Invalid algorithm"),
])
def test_errors_match_reference(argv, msg):
    with pytest.raises(RuntimeError, match=msg):
        cli.parse_args(argv)


def test_metrics_json_layout():
    c = cli.parse_args(["--path_A", "a", "--path_b", "b", "--algorithm", "cholesky"])
    c["N"] = 20
    m = cli.metrics_json(c, "B200", {"totalTime": 1.5, "choleskySolveStepTime": 0.5}, 3)
    cfg, rt = m["configuration"], m["runtime-metrics"]
    for k in ("algorithm", "N", "FP_type", "matrixBlockSize", "workGroupSize", "iMax", "epsilon", "mode"):
        assert k in cfg
    for k in ("iterationTimes", "memoryInitTime", "totalTime", "choleskySolveStepTime", "blockCounts_GPU",
              "matrixMatrixTimes_total", "triangularSolveTimes_GPU"):
        assert k in rt
    assert rt["totalTime"] == 1.5 and cfg["FP_type"] == "FP_64"
    json.dumps(m)


def test_write_full_matrix_round_trip(hs, tmp_path):
    """The reference's 20x20 fixture parsed with bsz 6 (padding 4), written in the
    reference's full-matrix format and read back: the symmetric matrix, padded."""
    fx = json.loads((ROOT / "tests" / "golden" / "reference_cases.json").read_text())["fixtures"]["matrix"]
    N = fx["N"]
    txt = tmp_path / "A.txt"
    txt.write_text(f"# {N}\n" + "\n".join(";".join(repr(v) for v in row) for row in fx["rows"]) + "\n")
    A = hs.MatrixParser.parseSymmetricMatrix(txt, 6)
    out = tmp_path / "A_chol_result"
    hs.MatrixParser.writeFullMatrix(out, A)
    lines = out.read_text().splitlines()
    assert len(lines) == 24
    got = np.array([[float(v) for v in ln.split(";")[:-1]] for ln in lines])
    dense = np.zeros((24, 24))
    dense[:N, :N] = A.to_dense()
    np.testing.assert_allclose(got, dense, rtol=0, atol=1e-15)
    assert lines[0].startswith(" ") or lines[0].startswith("-")
