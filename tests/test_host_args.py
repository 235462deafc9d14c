"""CPU checks of the host mirror's argument validation (raised before any device
call): unknown split precisions and solve algorithms are rejected by name."""
import pytest


def test_mixed_solver_rejects_unknown_precision(hs):
    with pytest.raises(ValueError, match="precision must be one of"):
        hs.MixedPrecisionSolver(None, None, "fp8x3")
    for name in ("tf32x3", "bf16x3", "f16x3"):
        assert hs.MixedPrecisionSolver(None, None, name).precision == name


def test_gp_solve_host_rejects_unknown_algorithm(hs):
    with pytest.raises(ValueError, match="algorithm must be one of"):
        hs.gp_solve_host(None, [[0.0]], [0.0], algorithm="mixed_fp8")
