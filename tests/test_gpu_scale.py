"""GPU suite: size-independent properties at a size no oracle finishes quickly
(N=32768, d=16, l=1, sn2=1e-2, bsz=256: the headline generator at a quarter of its
N), and the smallest and ragged shapes (N=1, N=bsz+1).

At scale there is no reference result to compare with, so the checks are the ones
the domain gives: backward errors of each form, agreement of the FP64 and mixed
solutions and log-determinants within what their backward errors and the
conditioning allow, CG converging to its tolerance with a true residual that
matches its recurrence, and reproducibility of the fixed-order kernels."""
import ctypes

import numpy as np
import pytest
import torch

import oracle_lib as ol

pytestmark = pytest.mark.gpu


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _bwd(hs, ctx, A, x, b):
    """||b - K x|| / (||K||_F ||x||) with the library's matvec."""
    nb = ctx.blockCountXY
    r = torch.empty_like(b)
    hs.MatrixVectorOperations.matrixVectorBlock(ctx, A, x, r, 0, 0, nb, nb, nb)
    return r, torch.linalg.norm(r - b).item()


def test_full_scale_properties(hs, ctx):
    N, bsz, d = 32768, 256, 16
    rng = np.random.default_rng(2)
    X = rng.random((N, d))
    y = np.sin(X.sum(axis=1)) + 0.1 * rng.standard_normal(N)
    ctx.set_problem(N, bsz)
    nb = ctx.blockCountXY
    lib = hs._lib.load()
    Xd = torch.from_numpy(X).cuda()
    b = torch.zeros(hs.padded_size(N, bsz), dtype=torch.float64, device="cuda")
    b[:N] = torch.from_numpy(y).cuda()
    K = torch.empty(hs.packed_size(N, bsz), dtype=torch.float64, device="cuda")
    hs.MatrixGenerator.assemble(ctx, K, Xd, 1.0, 1.0, 1e-2)
    K2 = torch.empty_like(K)
    hs.MatrixGenerator.assemble(ctx, K2, Xd, 1.0, 1.0, 1e-2)
    assert torch.equal(K, K2), "assembly is deterministic"
    del K2
    blocks = K.view(-1, bsz * bsz)
    diag = torch.tensor([hs.block_id(k, k, nb) for k in range(nb)], device="cuda")
    sq = (blocks * blocks).sum(dim=1)
    kfro = float(torch.sqrt(2.0 * sq.sum() - sq[diag].sum()).item())
    # mixed form
    xm = torch.empty_like(b)
    rep = hs._lib.MixedReport()
    hs._lib.check(lib.hs_mixed_solve(ctx.handle, _p(K), _p(b), _p(xm), 3, 1e-14, 30, ctypes.byref(rep)))
    r, rn = _bwd(hs, ctx, K, xm, b)
    bwd_m = rn / (kfro * torch.linalg.norm(xm).item())
    # CG on the same system (the FP64 matvec, eps = 1e-10)
    xc = torch.empty_like(b)
    it, dn, d0 = ctypes.c_int64(), ctypes.c_double(), ctypes.c_double()
    hs._lib.check(lib.hs_cg_solve(ctx.handle, _p(K), _p(b), _p(xc), 1e-10, 20000, ctypes.byref(it), ctypes.byref(dn),
                                  ctypes.byref(d0)))
    _, rc = _bwd(hs, ctx, K, xc, b)
    true_rel = rc / torch.linalg.norm(b).item()
    # FP64 form (overwrites K with L)
    info = ctypes.c_int64()
    hs._lib.check(lib.hs_cholesky_factor(ctx.handle, _p(K), ctypes.byref(info)))
    ld64 = hs.cholesky_logdet(ctx, K)
    x64 = b.clone()
    hs._lib.check(lib.hs_cholesky_solve(ctx.handle, _p(K), _p(x64)))
    hs.MatrixGenerator.assemble(ctx, K, Xd, 1.0, 1.0, 1e-2)
    _, r64 = _bwd(hs, ctx, K, x64, b)
    bwd_64 = r64 / (kfro * torch.linalg.norm(x64).item())
    rel_x = (torch.linalg.norm(xm - x64) / torch.linalg.norm(x64)).item()
    rel_cg = (torch.linalg.norm(xc - x64) / torch.linalg.norm(x64)).item()
    print(f"N={N}: backward error FP64 {bwd_64:.2e}, mixed {bwd_m:.2e} ({rep.refinement_steps} steps); "
          f"x mixed vs FP64 {rel_x:.2e}; log|K| FP64 {ld64:.6f} mixed {rep.logdet:.6f}; CG {it.value} its, "
          f"recurrence {np.sqrt(dn.value / d0.value):.2e} true {true_rel:.2e}, x vs FP64 {rel_cg:.2e}")
    assert bwd_64 <= 1e-16
    assert bwd_m <= 1e-14
    assert rel_x <= 1e-8              # both backward stable; cond(K) ~1e6 at this N
    assert abs(rep.logdet - ld64) <= 1e-3 * abs(ld64)
    assert np.sqrt(dn.value / d0.value) <= 1e-10
    assert true_rel <= 2e-10          # the recurrence and the true residual agree
    assert rel_cg <= 1e-6


@pytest.mark.parametrize("N,bsz", [(1, 128), (1, 256), (129, 128), (257, 256), (5, 4)])
def test_smallest_and_ragged_shapes(hs, ctx, N, bsz):
    """One valid row in a whole padded block, and one row past a block boundary:
    factor, solve and CG against the oracle; the mixed solve (block sizes 128 / 256)
    to the FP64 backward-error target."""
    rng = np.random.default_rng(N + bsz)
    X = rng.random((N, 3))
    y = np.sin(X.sum(axis=1)) + 0.1 * rng.standard_normal(N)
    Kh = ol.rbf_assemble(X, bsz, 0.7, 1.0, 1e-2)
    bh = np.zeros(-(-N // bsz) * bsz)
    bh[:N] = y
    ctx.set_problem(N, bsz)
    lib = hs._lib.load()
    K = torch.from_numpy(Kh).cuda()
    Lref = ol.cholesky(Kh, N, bsz)
    xref = ol.triangular_solve(Lref, bh, N, bsz)
    L = K.clone()
    info = ctypes.c_int64()
    hs._lib.check(lib.hs_cholesky_factor(ctx.handle, _p(L), ctypes.byref(info)))
    assert info.value == -1
    Lg = L.cpu().numpy()
    assert np.linalg.norm(Lg - Lref) <= 1e-12 * np.linalg.norm(Lref)
    x = torch.from_numpy(bh).cuda()
    hs._lib.check(lib.hs_cholesky_solve(ctx.handle, _p(L), _p(x)))
    assert np.linalg.norm(x.cpu().numpy() - xref) <= 1e-12 * np.linalg.norm(xref)
    xc = torch.empty_like(x)
    it, dn, d0 = ctypes.c_int64(), ctypes.c_double(), ctypes.c_double()
    hs._lib.check(lib.hs_cg_solve(ctx.handle, _p(K), _p(torch.from_numpy(bh).cuda()), _p(xc), 1e-10, 1000,
                                  ctypes.byref(it), ctypes.byref(dn), ctypes.byref(d0)))
    assert np.linalg.norm(xc.cpu().numpy() - xref) <= 1e-8 * np.linalg.norm(xref)
    assert not xc.cpu().numpy()[N:].any()
    if bsz in (128, 256):
        bd = torch.from_numpy(bh).cuda()
        xm = torch.empty_like(bd)
        rep = hs._lib.MixedReport()
        hs._lib.check(lib.hs_mixed_solve(ctx.handle, _p(K), _p(bd), _p(xm), 3, 1e-14, 30, ctypes.byref(rep)))
        assert rep.backward_error <= 1e-14
        assert np.linalg.norm(xm.cpu().numpy() - xref) <= 1e-10 * np.linalg.norm(xref)
