"""GPU suite: the differentiation form (no reference counterpart).  The
tensor-core reverse-mode Cholesky against the dense adjoint formula, and the GP
NLML and its gradient against dense FP64 LAPACK and central finite differences
(the dense checkers are themselves pinned by FD in test_gp_oracle.py)."""
import ctypes
import sys
from pathlib import Path

import numpy as np
import pytest
import torch

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
import gp_dense as g  # noqa: E402

pytestmark = pytest.mark.gpu


def _lower_dense(hs, packed, N, bsz):
    """Packed lower blocks -> dense N x N lower-triangular array."""
    nb = -(-N // bsz)
    full = np.zeros((nb * bsz, nb * bsz))
    for j in range(nb):
        for i in range(j, nb):
            s = hs.block_id(i, j, nb) * bsz * bsz
            full[i * bsz:(i + 1) * bsz, j * bsz:(j + 1) * bsz] = packed[s:s + bsz * bsz].reshape(bsz, bsz)
    return np.tril(full)


def _pack_lower(hs, dense, N, bsz):
    nb = -(-N // bsz)
    full = np.zeros((nb * bsz, nb * bsz))
    full[:N, :N] = np.tril(dense)
    out = np.zeros(hs.packed_size(N, bsz))
    for j in range(nb):
        for i in range(j, nb):
            s = hs.block_id(i, j, nb) * bsz * bsz
            out[s:s + bsz * bsz] = full[i * bsz:(i + 1) * bsz, j * bsz:(j + 1) * bsz].ravel()
    return out


@pytest.mark.parametrize("N,bsz", [(1000, 128), (768, 256), (700, 256), (1536, 256), (128, 128)])
def test_cholesky_adjoint_matches_dense_formula(hs, ctx, N, bsz):
    rng = np.random.default_rng(N + bsz)
    X = rng.random((N, 8))
    ctx.set_problem(N, bsz)
    A = hs.SymmetricMatrix(N, bsz, device="cuda:0")
    hs.MatrixGenerator.assemble(ctx, A.matrixData, X, 0.6, 1.0, 1e-2)
    chol = hs.Cholesky(A, ctx).solve_heterogeneous()
    L = chol.A_gpu
    L_before = L.clone()
    Ld = _lower_dense(hs, L.cpu().numpy(), N, bsz)[:N, :N]
    Lbar = np.tril(rng.standard_normal((N, N)))
    Abar = torch.from_numpy(_pack_lower(hs, Lbar, N, bsz)).to("cuda:0")
    hs.cholesky_adjoint(ctx, L, Abar)
    torch.cuda.synchronize()
    assert torch.equal(L, L_before), "the factor must not be modified"
    got_full = _lower_dense(hs, Abar.cpu().numpy(), N, bsz)
    assert np.all(got_full[N:, :] == 0.0), "padding rows of the adjoint must be zero"
    got = got_full[:N, :N]
    ref = g.chol_adjoint_dense(Ld, Lbar)
    err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
    print(f"N={N} bsz={bsz}: adjoint max rel err {err:.2e}")
    assert err <= 1e-10


def _c4_problem(N, d, seed):
    """ARD RBF with l_k ~ LogUniform[0.2, 2], sf2 = 1, sn2 = 1e-3, X ~ U[0,1],
    y drawn from the GP prior plus noise (y ~ N(0, K))."""
    rng = np.random.default_rng(seed)
    X = rng.random((N, d))
    ell = np.exp(rng.uniform(np.log(0.2), np.log(2.0), d))
    theta = np.concatenate([np.log(ell), [0.0, np.log(1e-3)]])
    K, _, _ = g.rbf_dense(X, ell, 1.0, 1e-3)
    y = np.linalg.cholesky(K) @ rng.standard_normal(N)
    return X, y, theta


@pytest.mark.parametrize("N,bsz", [(2048, 256), (1000, 128)])
def test_nlml_grad_matches_dense_and_finite_differences(hs, ctx, N, bsz):
    d = 8
    X, y, theta = _c4_problem(N, d, seed=40 + N)
    ctx.set_problem(N, bsz)
    nlml, grad, rep = hs.gp_nlml_grad(ctx, X, y, theta)
    nlml_ref, grad_ref = g.nlml_dense(X, y, theta, d)
    fd = g.nlml_fd(X, y, theta, d, h=1e-6)
    fd4 = g.nlml_fd4(X, y, theta, d, h=3e-3)
    rel_dense = np.max(np.abs(grad - grad_ref) / np.abs(grad_ref))
    rel_fd4 = np.max(np.abs(grad - fd4) / np.abs(fd4))
    norm_fd = np.max(np.abs(grad - fd)) / np.max(np.abs(fd))
    print(f"N={N}: nlml {nlml:.12e} (dense {nlml_ref:.12e}) grad rel vs dense {rel_dense:.2e}, "
          f"vs 4th-order FD {rel_fd4:.2e}, vs central FD (h=1e-6, normwise) {norm_fd:.2e}; {rep}")
    assert abs(nlml - nlml_ref) <= 1e-10 * abs(nlml_ref)
    assert rel_dense <= 1e-8
    # every component within 1e-6 relative of a finite-difference gradient accurate
    # to ~1e-7 (fourth-order stencil, h = 3e-3 in log-parameter space)
    assert rel_fd4 <= 1e-6
    # the two-point stencil at h = 1e-6 is limited by rounding (eps |NLML| / h with
    # |NLML| ~ 2.5e3 and an ill-conditioned factor): ~5e-6 normwise even for the
    # exact dense gradient
    assert norm_fd <= 2e-5


def test_nlml_grad_isotropic(hs, ctx):
    N, bsz = 900, 128
    rng = np.random.default_rng(5)
    X = rng.random((N, 4))
    y = np.sin(X.sum(1)) + 0.1 * rng.standard_normal(N)
    theta = np.log([0.7, 1.3, 2e-2])
    ctx.set_problem(N, bsz)
    nlml, grad, _ = hs.gp_nlml_grad(ctx, X, y, theta, n_ell=1)
    nlml_ref, grad_ref = g.nlml_dense(X, y, theta, 1)
    assert abs(nlml - nlml_ref) <= 1e-10 * abs(nlml_ref)
    assert np.max(np.abs(grad - grad_ref) / np.abs(grad_ref)) <= 1e-8


def test_autograd_function(hs, ctx):
    N, bsz, d = 512, 128, 3
    X, y, _ = _c4_problem(N, d, seed=9)
    theta = torch.tensor(np.log([0.5, 0.9, 1.4, 1.0, 1e-2]), dtype=torch.float64, requires_grad=True)
    ctx.set_problem(N, bsz)
    Xd = torch.from_numpy(X).to("cuda:0")
    yd = torch.from_numpy(y).to("cuda:0")
    out = hs.GaussianProcessNLML.apply(theta, Xd, yd, ctx)
    (2.0 * out).backward()
    _, grad_ref = g.nlml_dense(X, y, theta.detach().numpy(), d)
    np.testing.assert_allclose(theta.grad.numpy(), 2.0 * grad_ref, rtol=1e-8)


def test_nlml_rejects_bad_arguments(hs, ctx):
    ctx.set_problem(256, 128)
    X = np.random.default_rng(0).random((256, 3))
    y = np.zeros(256)
    with pytest.raises(hs.HSError):
        hs.gp_nlml_grad(ctx, X, y, np.zeros(4), n_ell=2)  # n_ell must be 1 or d
    ctx.set_problem(256, 64)
    with pytest.raises(hs.HSError):
        hs.gp_nlml_grad(ctx, X, y, np.zeros(3), n_ell=1)  # block size 64 unsupported


def test_fit_hyperparameters_decreases_nlml(hs, ctx):
    """A few L-BFGS steps on the analytic gradient lower the NLML; the result
    agrees with the dense NLML at the returned theta."""
    N, bsz, d = 1024, 128, 3
    X, y, theta_true = _c4_problem(N, d, seed=17)
    theta0 = np.concatenate([np.zeros(d), [0.5, np.log(1e-2)]])
    ctx.set_problem(N, bsz)
    out = hs.fit_hyperparameters(ctx, X, y, theta0, maxiter=8)
    nlml0 = g.nlml_value(X, y, theta0, d)
    assert out["nlml"] < nlml0 - 1.0
    assert abs(out["nlml"] - g.nlml_value(X, y, out["theta"], d)) <= 1e-9 * abs(out["nlml"])


@pytest.mark.parametrize("prec", ["f16x3", "tf32x3"])
@pytest.mark.parametrize("N,bsz", [(2048, 256), (1000, 128)])
def test_mixed_nlml_grad_against_dense(hs, ctx, N, bsz, prec):
    """The NLML and gradient through the mixed-precision factor: the data-fit term
    1/2 y^T K^-1 y has FP64 accuracy (alpha is refined against the FP64 K); log|K|
    and the gradient carry the low-precision factor's error, bounded here at the
    sizes tested and reported by bench.py at N = 65536."""
    d = 8
    X, y, theta = _c4_problem(N, d, seed=40 + N)
    ctx.set_problem(N, bsz)
    nlml, grad, rep = hs.gp_nlml_grad(ctx, X, y, theta, precision=prec)
    nlml_ref, grad_ref = g.nlml_dense(X, y, theta, d)
    nlml64, grad64, rep64 = hs.gp_nlml_grad(ctx, X, y, theta)
    ell = np.exp(theta[:d])
    K, _, _ = g.rbf_dense(X, ell, 1.0, np.exp(theta[-1]))
    fit_ref = 0.5 * y @ np.linalg.solve(K, y)
    logdet_ref = np.linalg.slogdet(K)[1]
    rel_fit = abs(rep["data_fit"] - fit_ref) / abs(fit_ref)
    abs_logdet = abs(rep["logdet"] - logdet_ref)
    rel_grad = np.max(np.abs(grad - grad_ref) / np.abs(grad_ref))
    rel_grad_norm = np.linalg.norm(grad - grad_ref) / np.linalg.norm(grad_ref)
    print(f"{prec} N={N}: data fit rel {rel_fit:.2e}, log|K| abs {abs_logdet:.2e} (FP64 form "
          f"{abs(rep64['logdet'] - logdet_ref):.2e}), nlml abs {abs(nlml - nlml_ref):.2e}, grad rel max "
          f"{rel_grad:.2e} normwise {rel_grad_norm:.2e} (FP64 form "
          f"{np.max(np.abs(grad64 - grad_ref) / np.abs(grad_ref)):.2e}); {rep['mixed']}")
    assert rep["mixed"]["backward_error"] <= 1e-14
    # alpha to ~cond(K) x 1e-14 (cond ~6e5 here; measured 8e-12 / 2.3e-10)
    assert rel_fit <= 1e-8
    # the low-precision factor's share (measured: log|K| 2.8 nats and gradient 1.5e-2
    # normwise for the FP16 split at N = 2048, against 9e-12 and 1e-10 for the FP64 form)
    assert abs_logdet <= 2e-3 * N
    assert rel_grad_norm <= 5e-2
