"""GPU suite: the reference-compatible command line end to end on the
reference's 20x20 fixture and on generated GP systems; its outputs against the
oracle (the reference's CPU path)."""
import json
import sys
from pathlib import Path

import numpy as np
import pytest

import oracle_lib as ol

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "heterogeneous-solvers_b200"))
import cli  # noqa: E402

pytestmark = pytest.mark.gpu


def _fixture_files(tmp_path):
    g = json.loads((ROOT / "tests" / "golden" / "reference_cases.json").read_text())["fixtures"]
    m, v = g["matrix"], g["vector"]
    (tmp_path / "A.txt").write_text(f"# {m['N']}\n" + "\n".join(";".join(repr(x) for x in r) for r in m["rows"]) + "\n")
    (tmp_path / "b.txt").write_text(f"# {v['N']}\n" + ";".join(repr(x) for x in v["values"]) + "\n")
    return m, v


def test_cli_cholesky_on_reference_fixture(hs, tmp_path, monkeypatch):
    m, v = _fixture_files(tmp_path)
    monkeypatch.chdir(tmp_path)
    x = cli.main(["--path_A", "A.txt", "--path_b", "b.txt", "--algorithm", "cholesky", "--matrix_bsz", "6",
                  "--write_result", "true", "--write_matrix", "true", "--output", str(tmp_path / "out")])
    N = m["N"]
    dense = np.zeros((N, N))
    for i, row in enumerate(m["rows"]):
        dense[i, :i + 1] = row
        dense[:i, i] = row[:i]
    ref = np.linalg.solve(dense, np.asarray(v["values"]))
    got = np.array([float(t) for t in (tmp_path / "x_result.txt").read_text().split()])
    np.testing.assert_allclose(got[:N], ref, rtol=1e-12, atol=1e-12)
    lines = (tmp_path / "A_chol_result").read_text().splitlines()
    assert len(lines) == 24
    L = np.array([[float(t) for t in ln.split(";")[:-1]] for ln in lines])[:N, :N]
    np.testing.assert_allclose(np.tril(L) @ np.tril(L).T, dense, rtol=0, atol=1e-12)
    metrics = list((tmp_path / "out").glob("*/metrics.json"))
    assert len(metrics) == 1 and json.loads(metrics[0].read_text())["configuration"]["algorithm"] == "cholesky"


def test_cli_generated_cg_with_check(hs, tmp_path, monkeypatch, capsys):
    rng = np.random.default_rng(2)
    N = 300
    series = np.sin(np.linspace(0, 9, N)) + 0.05 * rng.standard_normal(N)
    (tmp_path / "x.txt").write_text("\n".join(f"{t:.17g}" for t in series) + "\n")
    (tmp_path / "y.txt").write_text("\n".join(f"{t:.17g}" for t in np.roll(series, -1)) + "\n")
    monkeypatch.chdir(tmp_path)
    x = cli.main(["--gp_input", "x.txt", "--gp_output", "y.txt", "--size", str(N), "--algorithm", "cg",
                  "--eps", "1e-12", "--matrix_bsz", "128", "--check_result", "true", "--output", "out"])
    out = capsys.readouterr().out
    err = float(out.split("Average error of Ax - b:")[1].split()[0])
    assert err < 1e-8
    X = ol.window_inputs(series, N)
    K = ol.packed_to_dense(ol.rbf_assemble(X, 128, 1.0, 1.0, 1e-2), N, 128)
    ref = np.linalg.solve(K, np.roll(series, -1))
    np.testing.assert_allclose(np.asarray(x)[:N], ref, rtol=1e-6, atol=1e-8)


def test_cli_gpr(hs, tmp_path, monkeypatch):
    rng = np.random.default_rng(3)
    N, Nt = 400, 50
    series = np.sin(np.linspace(0, 12, N + Nt)) + 0.02 * rng.standard_normal(N + Nt)
    (tmp_path / "x.txt").write_text("\n".join(f"{t:.17g}" for t in series[:N]) + "\n")
    (tmp_path / "y.txt").write_text("\n".join(f"{t:.17g}" for t in np.roll(series, -1)[:N]) + "\n")
    (tmp_path / "t.txt").write_text("\n".join(f"{t:.17g}" for t in series[N:]) + "\n")
    monkeypatch.chdir(tmp_path)
    mean = cli.main(["--gp_input", "x.txt", "--gp_output", "y.txt", "--gp_test", "t.txt", "--size", str(N),
                     "--test_size", str(Nt), "--gpr", "true", "--algorithm", "cholesky", "--write_result", "true"])
    X, Xt = ol.window_inputs(series[:N], N), ol.window_inputs(series[N:], Nt)
    K = ol.rbf_assemble(X, 128, 1.0, 1.0, 1e-2)
    yb = np.zeros(-(-N // 128) * 128)
    yb[:N] = np.roll(series, -1)[:N]
    alpha = ol.triangular_solve(ol.cholesky(K, N, 128), yb, N, 128)
    ref = ol.matrix_vector_gp(ol.test_kernel_matrix(X, Xt, 1.0, 1.0), alpha[:N], N, Nt)
    np.testing.assert_allclose(mean, ref, rtol=1e-10, atol=1e-12)
    written = np.array([float(t) for t in (tmp_path / "x_result.txt").read_text().split()])
    np.testing.assert_allclose(written, mean, rtol=1e-15)
