"""CPU suite: the dense checkers of the two new forms (no reference
counterpart) are pinned by central finite differences, and the blocked reverse
sweep that the CUDA kernels run is checked against the dense adjoint formula."""
import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
import gp_dense as g  # noqa: E402


def _spd(n, seed):
    rng = np.random.default_rng(seed)
    M = rng.standard_normal((n, n))
    return M @ M.T + n * np.eye(n), rng


def test_dense_cholesky_adjoint_matches_finite_differences():
    A, rng = _spd(12, 0)
    L = np.linalg.cholesky(A)
    Lbar = np.tril(rng.standard_normal((12, 12)))
    ad = g.chol_adjoint_dense(L, Lbar)
    fd = g.chol_adjoint_fd(A, Lbar)
    assert np.max(np.abs(ad - fd)) <= 1e-7 * np.max(np.abs(fd))


@pytest.mark.parametrize("bsz", [4, 8, 16, 48])
def test_blocked_reverse_sweep_matches_dense(bsz):
    A, rng = _spd(96, 1)
    L = np.linalg.cholesky(A)
    Lbar = np.tril(rng.standard_normal((96, 96)))
    bl = g.chol_adjoint_blocked(L, Lbar, bsz)
    ad = g.chol_adjoint_dense(L, Lbar)
    assert np.max(np.abs(bl - ad)) <= 1e-13 * np.max(np.abs(ad))


def test_logdet_adjoint_is_inverse():
    """Lbar = diag(1/L_ii) (the adjoint of sum log L_ii = 1/2 log|A|) gives the
    lower representation of A^-1: off-diagonal entries, halved diagonal."""
    A, _ = _spd(40, 2)
    L = np.linalg.cholesky(A)
    ad = g.chol_adjoint_blocked(L, np.diag(1.0 / np.diag(L)), 8)
    Ai = np.linalg.inv(A)
    ref = np.tril(Ai, -1) + 0.5 * np.diag(np.diag(Ai))
    assert np.max(np.abs(ad - ref)) <= 1e-13 * np.max(np.abs(Ai))


@pytest.mark.parametrize("n_ell", [1, 3])
def test_dense_nlml_gradient_matches_finite_differences(n_ell):
    rng = np.random.default_rng(3)
    X = rng.random((150, 3))
    y = np.sin(X.sum(1)) + 0.1 * rng.standard_normal(150)
    theta = np.log([0.5, 0.8, 1.2][:n_ell] + [1.0, 1e-2])
    _, grad = g.nlml_dense(X, y, theta, n_ell)
    fd = g.nlml_fd(X, y, theta, n_ell, h=1e-6)
    assert np.all(np.abs(grad - fd) <= 1e-6 * np.abs(fd) + 1e-6)


def test_fourth_order_fd_agrees_with_central_fd():
    rng = np.random.default_rng(6)
    X = rng.random((120, 2))
    y = np.sin(X.sum(1)) + 0.1 * rng.standard_normal(120)
    theta = np.log([0.6, 1.1, 1.0, 5e-2])
    _, grad = g.nlml_dense(X, y, theta, 2)
    fd4 = g.nlml_fd4(X, y, theta, 2)
    assert np.all(np.abs(grad - fd4) <= 1e-7 * np.abs(fd4) + 1e-8)


def test_planted_error_is_detected():
    """A wrong factor of 2 on the data-fit term must fail the FD comparison."""
    rng = np.random.default_rng(4)
    X = rng.random((60, 2))
    y = rng.standard_normal(60)
    theta = np.log([0.7, 1.0, 1e-1])
    _, grad = g.nlml_dense(X, y, theta, 1)
    fd = g.nlml_fd(X, y, theta, 1)
    wrong = grad.copy()
    wrong[0] *= 1.01
    assert not np.all(np.abs(wrong - fd) <= 1e-6 * np.abs(fd) + 1e-6)
