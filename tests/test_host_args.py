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


def test_context_setters_reject_bad_arguments_without_a_device(hs):
    """The context setters validate before touching a device: a null context or an
    accumulation width other than 1, 2 or 4 panels is HS_ERR_INVALID_ARG."""
    lib = hs._lib.load()
    assert lib.hs_ctx_set_mixed_accumulation(None, 2) == 1
    assert lib.hs_ctx_set_reference_order(None, 8) == 1
    assert lib.hs_ctx_set_mixed_accumulation(None, 3) == 1
    assert "panels must be 1, 2 or 4" in lib.hs_last_error().decode()


def test_gp_nlml_grad_rejects_unknown_precision(hs):
    with pytest.raises(ValueError, match="precision must be one of"):
        hs.gp_nlml_grad(None, [[0.0]], [0.0], [0.0, 0.0, 0.0], precision="fp8x3")


def test_lookahead_setter_rejects_bad_arguments_without_a_device(hs):
    lib = hs._lib.load()
    assert lib.hs_ctx_set_mixed_lookahead(None, 16, 0) == 1
    assert "side_sms must be in" in lib.hs_last_error().decode()
