"""CPU suite: the oracle's drivers (not covered by the reference's unit tests)
against dense LAPACK / numpy on the same seeded inputs."""
import numpy as np
import pytest

import oracle_lib as ol


def _problem(N, d, seed=3):
    rng = np.random.default_rng(seed)
    X = rng.random((N, d))
    y = np.sin(X.sum(axis=1)) + 0.1 * rng.standard_normal(N)
    return X, y


def _dense_rbf(X, ell, sf2, sn2):
    ell = np.atleast_1d(ell)
    Z = X / ell if ell.size > 1 else X
    D = ((Z[:, None, :] - Z[None, :, :]) ** 2).sum(-1)
    scale = 0.5 if ell.size > 1 else 0.5 / ell[0] ** 2
    return sf2 * np.exp(-scale * D) + sn2 * np.eye(len(X))


@pytest.mark.parametrize("N,bsz,d,ell", [(50, 8, 3, 0.7), (130, 32, 8, 0.5), (97, 20, 4, np.array([0.3, 1.0, 2.0, 0.5]))])
def test_rbf_assembly_matches_dense(N, bsz, d, ell):
    X, _ = _problem(N, d)
    A = ol.rbf_assemble(X, bsz, ell, 1.3, 1e-2)
    K = ol.packed_to_dense(A, N, bsz)
    assert np.allclose(K, _dense_rbf(X, ell, 1.3, 1e-2), rtol=1e-13, atol=1e-15)
    # padding stays zero
    nb = -(-N // bsz)
    last = A[ol.block_id(nb - 1, nb - 1, nb) * bsz * bsz:].reshape(bsz, bsz)
    r = N - (nb - 1) * bsz
    assert not last[r:, :].any() and not last[:, r:].any()


def test_window_inputs_match_reference_generator():
    s = np.arange(1.0, 11.0)
    X = np.zeros((10, 8))
    ol.lib().or_window_inputs(ol.ptr(s), 10, ol.ptr(X))
    assert X[0].tolist() == [0] * 7 + [1.0]
    assert X[9].tolist() == list(range(3, 11))


@pytest.mark.parametrize("N,bsz", [(64, 16), (100, 32), (130, 20)])
def test_cholesky_and_solve_match_lapack(N, bsz):
    X, y = _problem(N, 5)
    A = ol.rbf_assemble(X, bsz, 0.8, 1.0, 1e-2)
    K = ol.packed_to_dense(A, N, bsz)
    L = ol.cholesky(A, N, bsz)
    Ld = ol.packed_to_dense(L, N, bsz, lower_only=True)
    assert np.allclose(Ld, np.linalg.cholesky(K), rtol=1e-11, atol=1e-13)
    b = np.zeros(-(-N // bsz) * bsz)
    b[:N] = y
    x = ol.triangular_solve(L, b, N, bsz)
    assert np.allclose(x[:N], np.linalg.solve(K, y), rtol=1e-9, atol=1e-11)
    assert not x[N:].any()


def test_cg_matches_lapack():
    N, bsz = 120, 16
    X, y = _problem(N, 4)
    A = ol.rbf_assemble(X, bsz, 0.8, 1.0, 1e-1)
    K = ol.packed_to_dense(A, N, bsz)
    b = np.zeros(-(-N // bsz) * bsz)
    b[:N] = y
    x, it, dn, d0 = ol.cg(A, b, N, bsz, 1e-10, 10000)
    assert dn <= 1e-20 * d0 and it > 0
    assert np.allclose(x[:N], np.linalg.solve(K, y), rtol=1e-7, atol=1e-8)


def test_oracle_test_kernel_matrix_is_the_rbf_formula():
    """The restatement of generateTestKernelMatrix against the closed form."""
    rng = np.random.default_rng(0)
    X, Xt = rng.random((40, 8)), rng.random((13, 8))
    for ell in (1.0, np.linspace(0.3, 2.0, 8)):
        K = ol.test_kernel_matrix(X, Xt, ell, 1.7)
        e = np.broadcast_to(np.atleast_1d(ell), (8,))
        D = ((Xt[:, None, :] - X[None, :, :]) / e) ** 2
        np.testing.assert_allclose(K, 1.7 * np.exp(-0.5 * D.sum(-1)), rtol=1e-14)
    A, b = rng.standard_normal((5, 40)), rng.standard_normal(40)
    np.testing.assert_allclose(ol.matrix_vector_gp(A, b, 40, 5), A @ b, rtol=1e-13)
