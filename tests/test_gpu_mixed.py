"""GPU suite: the mixed-precision form (3xTF32 tensor-core factor, FP64
diagonal POTRF, FP64 iterative refinement, PCG fallback) against dense FP64
LAPACK and the plain FP64 path, on seeded RBF systems."""
import ctypes

import numpy as np
import pytest
import torch

import oracle_lib as ol

pytestmark = pytest.mark.gpu


def _system(hs, ctx, N, bsz, d, ell, sn2, seed=5, sf2=1.0):
    rng = np.random.default_rng(seed)
    X = rng.random((N, d))
    y = np.sin(X.sum(axis=1)) + 0.1 * rng.standard_normal(N)
    ctx.set_problem(N, bsz)
    A = hs.SymmetricMatrix(N, bsz, device="cuda:0")
    hs.MatrixGenerator.assemble(ctx, A.matrixData, X, ell, sf2, sn2)
    b = torch.zeros(hs.padded_size(N, bsz), dtype=torch.float64, device="cuda:0")
    b[:N] = torch.from_numpy(y)
    return A, b, X, y


@pytest.mark.parametrize("N,bsz,d,ell,sn2", [
    (1000, 128, 8, 0.5, 1e-2), (700, 256, 16, 1.0, 1e-2), (1024, 256, 8, 0.5, 1e-1), (300, 128, 8, 0.5, 1e-2),
    (2048, 256, 16, 1.0, 1e-2),
])
def test_mixed_solve_reaches_fp64_backward_error(hs, ctx, N, bsz, d, ell, sn2):
    A, b, X, y = _system(hs, ctx, N, bsz, d, ell, sn2)
    solver = hs.MixedPrecisionSolver(A, ctx, "tf32x3")
    x = solver.solve(b, tol=1e-14, max_steps=30)
    rep = solver.report
    Kd = A.to_dense()
    x_ref = np.linalg.solve(Kd, y)
    xg = x.cpu().numpy()
    assert np.all(xg[N:] == 0.0), "padding of x must stay zero"
    xg = xg[:N]
    bwd = np.linalg.norm(y - Kd @ xg) / (np.linalg.norm(Kd, "fro") * np.linalg.norm(xg))
    rel = np.linalg.norm(xg - x_ref) / np.linalg.norm(x_ref)
    print(f"N={N} bsz={bsz} sn2={sn2}: steps {rep['refinement_steps']} pcg {rep['pcg_iterations']} "
          f"bwd0 {rep['initial_backward_error']:.2e} bwd {rep['backward_error']:.2e} (host {bwd:.2e}) "
          f"x rel {rel:.2e}")
    assert rep["backward_error"] <= 1e-14
    assert bwd <= 2e-14
    # 3xTF32 products give an FP32-accurate factor: the unrefined solution's backward
    # error is ~1e-7; a plain TF32 product (10-bit mantissa) would leave ~1e-4
    assert rep["initial_backward_error"] <= 1e-5
    cond = np.linalg.cond(Kd)
    assert rel <= max(1e-12, 50 * cond * 1e-16)
    sign, logdet_ref = np.linalg.slogdet(Kd)
    assert sign > 0
    assert abs(rep["logdet"] - logdet_ref) <= 1e-4 * abs(logdet_ref) + 1e-3


def test_mixed_leaves_matrix_unchanged(hs, ctx):
    A, b, _, _ = _system(hs, ctx, 600, 128, 8, 0.5, 1e-2)
    before = A.matrixData.clone()
    hs.MixedPrecisionSolver(A, ctx).solve(b)
    torch.cuda.synchronize()
    assert torch.equal(before, A.matrixData)


def test_mixed_matches_fp64_path(hs, ctx):
    """The mixed solve and the FP64 factor + solve agree to the FP64 accuracy of the system."""
    A, b, _, y = _system(hs, ctx, 1536, 256, 8, 0.5, 1e-2, seed=9)
    x_mixed = hs.MixedPrecisionSolver(A, ctx).solve(b).cpu().numpy()
    L = A.matrixData.clone()
    info = ctypes.c_int64(-2)
    hs._lib.call("hs_cholesky_factor", ctx.handle, ctypes.c_void_p(L.data_ptr()), ctypes.byref(info))
    assert info.value == -1
    x64 = b.clone()
    hs._lib.call("hs_cholesky_solve", ctx.handle, ctypes.c_void_p(L.data_ptr()), ctypes.c_void_p(x64.data_ptr()))
    x64 = x64.cpu().numpy()
    rel = np.linalg.norm(x_mixed - x64) / np.linalg.norm(x64)
    assert rel <= 1e-10, rel


@pytest.mark.parametrize("N,bsz", [(1000, 128), (700, 256)])
def test_logdet_of_fp64_factor(hs, ctx, N, bsz):
    A, _, _, _ = _system(hs, ctx, N, bsz, 8, 0.5, 1e-2)
    Kd = A.to_dense()
    chol = hs.Cholesky(A, ctx).solve_heterogeneous()
    ld = hs.cholesky_logdet(ctx, chol.A_gpu)
    ref = np.linalg.slogdet(Kd)[1]
    assert abs(ld - ref) <= 1e-11 * abs(ref)


def test_mixed_ill_conditioned_falls_back_or_converges(hs, ctx):
    """sn2 = 1e-6: the FP32 factor is a poor approximation; the solve must still
    reach the backward-error target (refinement, then PCG with the factor)."""
    A, b, _, y = _system(hs, ctx, 1024, 128, 8, 0.5, 1e-6)
    solver = hs.MixedPrecisionSolver(A, ctx)
    x = solver.solve(b, tol=1e-14, max_steps=30)
    rep = solver.report
    print("ill-conditioned:", rep)
    Kd = A.to_dense()
    xg = x.cpu().numpy()[:1024]
    bwd = np.linalg.norm(y - Kd @ xg) / (np.linalg.norm(Kd, "fro") * np.linalg.norm(xg))
    assert bwd <= 2e-14


def test_gp_solve_host_mixed(hs):
    """hs_gp_solve_host, algorithm 2: host X, y in, host x out, through the mixed solve."""
    N, bsz, d = 900, 128, 8
    rng = np.random.default_rng(21)
    X = rng.random((N, d))
    y = np.sin(X.sum(axis=1)) + 0.1 * rng.standard_normal(N)
    with hs.Context(device=0) as c:
        c.set_problem(N, bsz)
        x, rep = hs.gp_solve_host(c, X, y, 0.5, 1.0, 1e-2, algorithm="mixed", epsilon=1e-14, iMax=30)
        A = hs.SymmetricMatrix(N, bsz, device="cuda:0")
        hs.MatrixGenerator.assemble(c, A.matrixData, X, 0.5, 1.0, 1e-2)
        Kd = A.to_dense()
        hs._lib.call("hs_ctx_release_buffers", c.handle)
        # a call after the release allocates again
        x2, _ = hs.gp_solve_host(c, X, y, 0.5, 1.0, 1e-2, algorithm="mixed", epsilon=1e-14, iMax=30)
    bwd = np.linalg.norm(y - Kd @ x) / (np.linalg.norm(Kd, "fro") * np.linalg.norm(x))
    assert bwd <= 2e-14
    assert rep.iterations >= 1
    np.testing.assert_array_equal(x, x2)


def test_mixed_factor_breakdown_falls_back_to_shifted_preconditioner(hs, ctx):
    """Duplicated inputs with sn2 = 1e-7 give pivots below the FP32 rounding noise,
    so the FP32 factor of K breaks down; the solve then factors K + shift*I and
    reaches the backward-error target with CG preconditioned by that factor."""
    N, bsz, d = 1024, 128, 4
    rng = np.random.default_rng(12)
    base = rng.random((N // 2, d))
    X = np.concatenate([base, base])[rng.permutation(N)]
    y = np.sin(X.sum(axis=1)) + 0.1 * rng.standard_normal(N)
    ctx.set_problem(N, bsz)
    A = hs.SymmetricMatrix(N, bsz, device="cuda:0")
    hs.MatrixGenerator.assemble(ctx, A.matrixData, X, 0.5, 1.0, 1e-7)
    b = torch.zeros(hs.padded_size(N, bsz), dtype=torch.float64, device="cuda:0")
    b[:N] = torch.from_numpy(y)
    solver = hs.MixedPrecisionSolver(A, ctx)
    x = solver.solve(b, tol=1e-14, max_steps=30)
    rep = solver.report
    print("breakdown case:", rep)
    Kd = A.to_dense()
    xg = x.cpu().numpy()[:N]
    bwd = np.linalg.norm(y - Kd @ xg) / (np.linalg.norm(Kd, "fro") * np.linalg.norm(xg))
    assert bwd <= 2e-14
    if rep["shift"] > 0:
        assert rep["factor_attempts"] > 1 and rep["fallback_pcg"] == 1
    else:
        assert rep["factor_attempts"] == 1


@pytest.mark.parametrize("prec", ["bf16x3", "f16x3"])
def test_mixed_split16_breakdown_falls_back_to_tf32(hs, ctx, prec):
    """A BF16-split factor that breaks down is redone with 3xTF32 products before
    any diagonal shift is tried.  A FP16-split factor (22 significant bits, finer
    than 3xTF32) that meets a negative pivot goes straight to a diagonal shift
    set from that pivot (3xTF32 only after an overflow of the scaled panel).  The
    solve reaches the target either way."""
    N, bsz, d = 1024, 128, 4
    rng = np.random.default_rng(12)
    base = rng.random((N // 2, d))
    X = np.concatenate([base, base])[rng.permutation(N)]
    y = np.sin(X.sum(axis=1)) + 0.1 * rng.standard_normal(N)
    ctx.set_problem(N, bsz)
    A = hs.SymmetricMatrix(N, bsz, device="cuda:0")
    hs.MatrixGenerator.assemble(ctx, A.matrixData, X, 0.5, 1.0, 1e-7)
    b = torch.zeros(hs.padded_size(N, bsz), dtype=torch.float64, device="cuda:0")
    b[:N] = torch.from_numpy(y)
    solver = hs.MixedPrecisionSolver(A, ctx, prec)
    x = solver.solve(b, tol=1e-14, max_steps=30)
    rep = solver.report
    print(f"{prec} breakdown case:", rep)
    if rep["factor_attempts"] > 1:
        if prec == "bf16x3":
            assert rep["precision_used"] == hs.PRECISIONS["tf32x3"]
        else:
            assert rep["precision_used"] == hs.PRECISIONS["tf32x3"] or rep["shift"] > 0
        assert rep["factor_attempts"] <= 6
    Kd = A.to_dense()
    xg = x.cpu().numpy()[:N]
    bwd = np.linalg.norm(y - Kd @ xg) / (np.linalg.norm(Kd, "fro") * np.linalg.norm(xg))
    assert bwd <= 2e-14


@pytest.mark.parametrize("N,bsz,sn2", [(1000, 128, 1e-2), (2048, 256, 1e-2), (700, 256, 1e-1)])
def test_mixed_bf16_split_reaches_fp64_backward_error(hs, ctx, N, bsz, sn2):
    """The BF16 split variant of the trailing update: a less accurate factor
    (~2^-16 per product instead of ~2^-21), still refined (or PCG-preconditioned)
    to the FP64 backward-error target."""
    A, b, X, y = _system(hs, ctx, N, bsz, 8, 0.5, sn2, seed=31)
    solver = hs.MixedPrecisionSolver(A, ctx, "bf16x3")
    x = solver.solve(b, tol=1e-14, max_steps=30)
    rep = solver.report
    Kd = A.to_dense()
    xg = x.cpu().numpy()[:N]
    bwd = np.linalg.norm(y - Kd @ xg) / (np.linalg.norm(Kd, "fro") * np.linalg.norm(xg))
    print(f"bf16x3 N={N} bsz={bsz} sn2={sn2}: steps {rep['refinement_steps']} pcg {rep['pcg_iterations']} "
          f"bwd0 {rep['initial_backward_error']:.2e} bwd {bwd:.2e}")
    assert bwd <= 2e-14
    # a BF16-split factor: unrefined backward error well below plain BF16's ~1e-3
    assert rep["initial_backward_error"] <= 1e-4


@pytest.mark.parametrize("N,bsz,sn2,sf2", [
    (1000, 128, 1e-2, 1.0), (2048, 256, 1e-2, 1.0), (700, 256, 1e-1, 1.0), (1536, 256, 1e-3, 1.0),
    (1000, 128, 1e4, 1e6), (1000, 128, 1e-8, 1e-6),
])
def test_mixed_f16_split_reaches_fp64_backward_error(hs, ctx, N, bsz, sn2, sf2):
    """The FP16 split of the trailing update (the panel scaled by a power of two set
    from the largest diagonal entry, 22 significant bits): refined to the FP64
    backward-error target, with no more refinement work than the BF16 split on the
    same system.  sf2 = 1e6 and 1e-6 move the scale far from 1 (2^5 and 2^25)."""
    A, b, X, y = _system(hs, ctx, N, bsz, 8, 0.5, sn2, seed=31, sf2=sf2)
    Kd = A.to_dense()
    reps = {}
    for prec in ("f16x3", "bf16x3"):
        solver = hs.MixedPrecisionSolver(A, ctx, prec)
        x = solver.solve(b, tol=1e-14, max_steps=30)
        rep = solver.report
        reps[prec] = rep
        xg = x.cpu().numpy()[:N]
        bwd = np.linalg.norm(y - Kd @ xg) / (np.linalg.norm(Kd, "fro") * np.linalg.norm(xg))
        print(f"{prec} N={N} bsz={bsz} sn2={sn2} sf2={sf2}: attempts {rep['factor_attempts']} "
              f"steps {rep['refinement_steps']} pcg {rep['pcg_iterations']} "
              f"bwd0 {rep['initial_backward_error']:.2e} bwd {bwd:.2e}")
        assert bwd <= 2e-14
    f, g = reps["f16x3"], reps["bf16x3"]
    assert f["factor_attempts"] == 1 and f["precision_used"] == hs.PRECISIONS["f16x3"] and f["shift"] == 0.0
    assert f["initial_backward_error"] <= 1e-5
    if g["factor_attempts"] == 1:
        assert f["refinement_steps"] + f["pcg_iterations"] <= g["refinement_steps"] + g["pcg_iterations"]
    sign, logdet_ref = np.linalg.slogdet(Kd)
    assert sign > 0
    assert abs(f["logdet"] - logdet_ref) <= 1e-4 * abs(logdet_ref) + 1e-3


def test_gp_solve_host_mixed_f16(hs):
    """hs_gp_solve_host, algorithm 4 (mixed, FP16 split): host X, y in, host x out."""
    N, bsz, d = 900, 128, 8
    rng = np.random.default_rng(22)
    X = rng.random((N, d))
    y = np.sin(X.sum(axis=1)) + 0.1 * rng.standard_normal(N)
    with hs.Context(device=0) as c:
        c.set_problem(N, bsz)
        x, rep = hs.gp_solve_host(c, X, y, 0.5, 1.0, 1e-2, algorithm="mixed_f16x3", epsilon=1e-14, iMax=30)
        A = hs.SymmetricMatrix(N, bsz, device="cuda:0")
        hs.MatrixGenerator.assemble(c, A.matrixData, X, 0.5, 1.0, 1e-2)
        Kd = A.to_dense()
    bwd = np.linalg.norm(y - Kd @ x) / (np.linalg.norm(Kd, "fro") * np.linalg.norm(x))
    assert bwd <= 2e-14
    assert rep.iterations >= 1


def test_per_panel_accumulation_is_more_accurate_and_deterministic(hs, ctx):
    """hs_ctx_set_mixed_accumulation(1): each panel's trailing-update product is added
    into the FP32 matrix on its own.  On an ARD system with sn2 = 1e-3 its log|K| is
    closer to the FP64 factor's than four panels an add (measured 0.48 against 2.81
    nats at N = 2048), every setting reaches the FP64 backward-error target, and two
    one-panel factors are identical bit for bit (the adds into an entry keep panel
    order)."""
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
    import gp_dense as g
    N, bsz, d = 2048, 256, 8
    rng = np.random.default_rng(40 + N)
    X = rng.random((N, d))
    ell = np.exp(rng.uniform(np.log(0.2), np.log(2.0), d))
    ctx.set_problem(N, bsz)
    A = hs.SymmetricMatrix(N, bsz, device="cuda:0")
    hs.MatrixGenerator.assemble(ctx, A.matrixData, X, list(ell), 1.0, 1e-3)
    K, _, _ = g.rbf_dense(X, ell, 1.0, 1e-3)
    ld_ref = np.linalg.slogdet(K)[1]
    b = torch.zeros(hs.padded_size(N, bsz), dtype=torch.float64, device="cuda:0")
    b[:N] = 1.0
    out = {}
    try:
        for mode in (4, 2, 1, 1):
            ctx.set_mixed_accumulation(mode)
            solver = hs.MixedPrecisionSolver(A, ctx, "f16x3")
            x = solver.solve(b, tol=1e-14, max_steps=30).clone()
            assert solver.report["backward_error"] <= 1e-14
            out.setdefault(mode, []).append((solver.report, x))
    finally:
        ctx.set_mixed_accumulation(1)
    err = {m: abs(v[0][0]["logdet"] - ld_ref) for m, v in out.items()}
    print("log|K| error by panels an add:", err, "steps", {m: v[0][0]["refinement_steps"] for m, v in out.items()})
    assert err[1] < 0.5 * err[4]
    assert out[1][0][0]["logdet"] == out[1][1][0]["logdet"]
    assert torch.equal(out[1][0][1], out[1][1][1])


@pytest.mark.parametrize("N,bsz,prec", [
    (3000, 128, "f16x3"), (2900, 256, "f16x3"), (1300, 128, "tf32x3"), (5000, 256, "bf16x3"),
    (700, 128, "f16x3"), (257, 128, "f16x3"), (128, 128, "f16x3"),
])
def test_group_lookahead_gives_the_same_factor(hs, ctx, N, bsz, prec):
    """hs_ctx_set_mixed_lookahead: factoring the next panel group on a few SMs beside
    the current group's trailing update (the update's tiles shared between two
    launches through a counter) adds the same products into every block in the same
    order as the look-ahead by one diagonal block, so log|K| and the refined x are
    identical bit for bit.  Run with the group look-ahead forced on for every group
    (min_rows 0), on 16 and on a single side SM, on ragged sizes and group counts that
    end on a partial group."""
    A, b, _, _ = _system(hs, ctx, N, bsz, 8, 0.5, 1e-2, seed=N)
    runs = {}
    try:
        for cfg in ((0, 0), (16, 0), (1, 0), (16, 24576)):
            ctx.set_mixed_lookahead(*cfg)
            solver = hs.MixedPrecisionSolver(A, ctx, prec)
            x = solver.solve(b, tol=1e-14, max_steps=30).clone()
            assert solver.report["backward_error"] <= 1e-14, (cfg, solver.report)
            runs[cfg] = (solver.report, x)
    finally:
        ctx.set_mixed_lookahead()
    rep0, x0 = runs[(0, 0)]
    for cfg, (rep, x) in runs.items():
        assert rep["logdet"] == rep0["logdet"], cfg
        assert rep["initial_backward_error"] == rep0["initial_backward_error"], cfg
        assert rep["refinement_steps"] == rep0["refinement_steps"], cfg
        assert torch.equal(x, x0), cfg
