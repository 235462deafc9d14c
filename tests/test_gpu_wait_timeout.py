"""GPU: the failure path of the library's bounded device-side waits.  A wait on a
flag that nothing sets runs out after its limit and comes back as HS_ERR_TIMEOUT
(no trap, no hang); the context then keeps working."""
import time

import pytest
import torch

pytestmark = pytest.mark.gpu


def test_expired_wait_returns_timeout_and_context_stays_usable(hs, ctx):
    lib = hs._lib.load()
    ctx.set_problem(256, 128)
    t0 = time.perf_counter()
    st = lib.hs_selftest_bounded_wait(ctx.handle, 50_000_000)  # 50 ms
    dt = time.perf_counter() - t0
    assert hs._lib.STATUS_NAMES[st] == "HS_ERR_TIMEOUT"
    assert "ran out" in lib.hs_last_error().decode()
    assert 0.045 <= dt < 5.0
    # the same context, right after: a dot product through the library
    x = torch.arange(256, dtype=torch.float64, device="cuda:0")
    out = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    hs.VectorOperations.scalarProduct(ctx, x, x, out, 0, 2)
    torch.cuda.synchronize()
    assert out.item() == float((x * x).sum().item())


def test_wait_limit_is_checked(hs, ctx):
    lib = hs._lib.load()
    ctx.set_problem(256, 128)
    for bad in (0, 999_999, 2_000_000_001):
        assert hs._lib.STATUS_NAMES[lib.hs_selftest_bounded_wait(ctx.handle, bad)] == "HS_ERR_INVALID_ARG"
