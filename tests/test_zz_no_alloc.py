"""GPU test of hs_symv_block_noalloc, the matvec entry point that allocates no
device memory (for callers whose allocator owns the device memory or who cannot
afford cudaMalloc's synchronisation).  It must give the same product as the
allocating hs_symv_block, including on a second call in a row, whose scratch
starts with the first call's leftovers.  The file name sorts last so that a run
stopping at the first failure has run every other test before it."""
import ctypes

import numpy as np
import pytest
import torch

import oracle_lib as ol

pytestmark = pytest.mark.gpu

MAX_DOUBLES = 2 * 1024 * 1024  # HS_SYMV_NOALLOC_MAX_DOUBLES in include/hs_b200.h


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _matvec_both(hs, ctx, A, b, rect, reset, start):
    """(allocating result, no-alloc result) for the same call; both outputs start from `start`."""
    lib = hs._lib.load()
    nb = ctx.blockCountXY
    out_ref = start.clone()
    out_new = start.clone()
    hs._lib.check(lib.hs_symv_block(ctx.handle, _p(A), _p(b), _p(out_ref), *rect, nb, reset))
    hs._lib.check(lib.hs_symv_block_noalloc(ctx.handle, _p(A), _p(b), _p(out_new), *rect, nb, reset))
    ctx.sync()
    return out_ref.cpu().numpy(), out_new.cpu().numpy()


@pytest.mark.parametrize("N,bsz", [(2000, 128), (1500, 256), (130, 20)])
def test_noalloc_matvec_matches_allocating_entry_point(hs, ctx, N, bsz):
    rng = np.random.default_rng(5)
    X = rng.random((N, 8))
    K = torch.from_numpy(ol.rbf_assemble(X, bsz, 0.5, 1.0, 1e-2)).cuda()
    ctx.set_problem(N, bsz)
    nb = ctx.blockCountXY
    n = nb * bsz
    # two calls in a row: a full product, then a sub-rectangle accumulating into
    # a non-zero vector with a different right-hand side
    b1 = torch.from_numpy(rng.standard_normal(n)).cuda()
    ref1, new1 = _matvec_both(hs, ctx, K, b1, (0, 0, nb, nb), 1, torch.zeros(n, dtype=torch.float64, device="cuda"))
    assert np.allclose(new1, ref1, rtol=1e-13, atol=1e-13)
    b2 = torch.from_numpy(rng.standard_normal(n)).cuda()
    start = torch.from_numpy(rng.standard_normal(n)).cuda()
    rect = (nb // 3, nb // 2, nb - nb // 3, nb - nb // 2)
    ref2, new2 = _matvec_both(hs, ctx, K, b2, rect, 0, start)
    assert np.allclose(new2, ref2, rtol=1e-13, atol=1e-13)
    # and against the dense product for the full call
    dense = ol.packed_to_dense(K.cpu().numpy(), N, bsz) @ b1.cpu().numpy()[:N]
    assert np.allclose(new1[:N], dense, rtol=1e-12, atol=1e-12)


def test_noalloc_matvec_rejects_rectangles_beyond_its_scratch(hs, ctx):
    # N = 131072, bsz = 256: a full matvec needs 512*512*256 doubles of partials
    ctx.set_problem(131072, 256)
    nb = ctx.blockCountXY
    assert nb * nb * 256 > MAX_DOUBLES
    dummy = torch.zeros(16, dtype=torch.float64, device="cuda")
    lib = hs._lib.load()
    st = lib.hs_symv_block_noalloc(ctx.handle, _p(dummy), _p(dummy), _p(dummy), 0, 0, nb, nb, nb, 1)
    assert st == 1  # HS_ERR_INVALID_ARG, nothing launched
    assert "static scratch holds" in lib.hs_last_error().decode()


def test_noalloc_matvec_allocates_nothing_on_a_fresh_context(hs, ctx):
    """On a context that has never run the allocating matvec, only the no-alloc
    entry point is called: the product matches the dense one and the device's free
    memory does not move.  The rectangle is the largest the static scratch takes
    (nb * nb * bsz == HS_SYMV_NOALLOC_MAX_DOUBLES: N = 16384, bsz = 128)."""
    N, bsz = 16384, 128
    rng = np.random.default_rng(8)
    X = rng.random((N, 4))
    lib = hs._lib.load()
    with hs.Context(device=0) as warm:  # kernels loaded once per process, outside the measurement
        warm.set_problem(256, 128)
        z = torch.zeros(hs.packed_size(256, 128), dtype=torch.float64, device="cuda")
        v = torch.zeros(256, dtype=torch.float64, device="cuda")
        w = torch.zeros(256, dtype=torch.float64, device="cuda")
        hs._lib.check(lib.hs_symv_block_noalloc(warm.handle, _p(z), _p(v), _p(w), 0, 0, 2, 2, 2, 1))
        warm.sync()
    K = torch.empty(hs.packed_size(N, bsz), dtype=torch.float64, device="cuda")
    b = torch.from_numpy(rng.standard_normal(N)).cuda()
    out = torch.full((N,), np.nan, dtype=torch.float64, device="cuda")
    with hs.Context(device=0) as fresh:
        fresh.set_problem(N, bsz)
        hs.MatrixGenerator.assemble(fresh, K, X, 0.5, 1.0, 1e-2)
        nb = fresh.blockCountXY
        assert nb * nb * bsz == MAX_DOUBLES
        fresh.sync()
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        for _ in range(2):
            hs._lib.check(lib.hs_symv_block_noalloc(fresh.handle, _p(K), _p(b), _p(out), 0, 0, nb, nb, nb, 1))
        fresh.sync()
        free1, _ = torch.cuda.mem_get_info()
        assert free1 == free0, (free0, free1)
        # one block row more than the scratch holds is rejected before any launch
        fresh.set_problem(N + bsz, bsz)
        nb1 = fresh.blockCountXY
        assert nb1 * nb * bsz > MAX_DOUBLES
        st = lib.hs_symv_block_noalloc(fresh.handle, _p(K), _p(b), _p(out), 0, 0, nb1, nb, nb1, 1)
        assert st == 1
    Kd = ol.packed_to_dense(K.cpu().numpy(), N, bsz)
    dense = Kd @ b.cpu().numpy()
    assert np.allclose(out.cpu().numpy(), dense, rtol=1e-12, atol=1e-12)


def test_noalloc_matvec_in_reference_order_mode_is_bitwise_equal(hs, ctx):
    """In reference-order mode both entry points run the reference-order kernel."""
    N, bsz = 700, 128
    rng = np.random.default_rng(9)
    X = rng.random((N, 8))
    K = torch.from_numpy(ol.rbf_assemble(X, bsz, 0.5, 1.0, 1e-2)).cuda()
    ctx.set_problem(N, bsz)
    nb = ctx.blockCountXY
    n = nb * bsz
    b = torch.from_numpy(rng.standard_normal(n)).cuda()
    ctx.set_reference_order(8)
    try:
        for _ in range(2):
            ref, new = _matvec_both(hs, ctx, K, b, (0, 0, nb, nb), 1, torch.zeros(n, dtype=torch.float64,
                                                                                  device="cuda"))
            assert np.array_equal(ref, new)
    finally:
        ctx.set_reference_order(0)
