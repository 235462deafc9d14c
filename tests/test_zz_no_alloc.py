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
