"""Dense FP64 checkers for the two forms that have no counterpart in the
reference (test infrastructure only: imported by tests/ and nothing else).

* GP negative log marginal likelihood and its gradient, computed densely with
  LAPACK (scipy.linalg.cho_factor) from the kernel matrix of
  src/utility/MatrixGenerator.cpp:134-155 generalised to ARD lengthscales:
      K = sf2 exp(-1/2 sum_k (x_ik - x_jk)^2 / l_k^2) + sn2 I
      NLML = 1/2 y^T K^-1 y + 1/2 log|K| + N/2 log 2pi
      dNLML/dtheta = 1/2 tr((K^-1 - alpha alpha^T) dK/dtheta),  theta = log params
  and its central finite differences.
* The adjoint of the Cholesky factorisation: the dense level-3 formula
      Abar = tril_h(L^-T (H + H^T) L^-1),  H = tril_h(L^T Lbar)
  (tril_h = lower triangle, diagonal halved), its finite-difference check, and
  a blocked restatement of the reverse sweep the CUDA kernels run, so the
  blocked algorithm can be checked without a GPU.
"""
import numpy as np
import scipy.linalg as sla

LOG2PI = np.log(2.0 * np.pi)


def theta_split(theta, n_ell):
    theta = np.asarray(theta, dtype=np.float64)
    return np.exp(theta[:n_ell]), np.exp(theta[n_ell]), np.exp(theta[n_ell + 1])


def rbf_dense(X, ell, sf2, sn2):
    X = np.asarray(X, dtype=np.float64)
    ell = np.broadcast_to(np.atleast_1d(np.asarray(ell, dtype=np.float64)), (X.shape[1],))
    Xs = X / ell
    # exact pairwise differences (no |a|^2 + |b|^2 - 2ab cancellation)
    D2 = np.zeros((X.shape[0], X.shape[0]))
    for k in range(X.shape[1]):
        diff = Xs[:, k][:, None] - Xs[:, k][None, :]
        D2 += diff * diff
    Kr = sf2 * np.exp(-0.5 * D2)
    return Kr + sn2 * np.eye(X.shape[0]), Kr, Xs


def nlml_dense(X, y, theta, n_ell):
    """(nlml, grad) in FP64 with dense LAPACK."""
    ell, sf2, sn2 = theta_split(theta, n_ell)
    K, Kr, Xs = rbf_dense(X, ell, sf2, sn2)
    c, low = sla.cho_factor(K, lower=True)
    alpha = sla.cho_solve((c, low), y)
    N = len(y)
    nlml = 0.5 * y @ alpha + np.sum(np.log(np.diag(c))) + 0.5 * N * LOG2PI
    Kinv = sla.cho_solve((c, low), np.eye(N))
    W = Kinv - np.outer(alpha, alpha)
    grad = np.zeros(n_ell + 2)
    if n_ell == 1:
        D2 = np.zeros_like(K)
        for k in range(X.shape[1]):
            diff = Xs[:, k][:, None] - Xs[:, k][None, :]
            D2 += diff * diff
        grad[0] = 0.5 * np.sum(W * Kr * D2)
    else:
        for k in range(n_ell):
            diff = Xs[:, k][:, None] - Xs[:, k][None, :]
            grad[k] = 0.5 * np.sum(W * Kr * diff * diff)
    grad[n_ell] = 0.5 * np.sum(W * Kr)
    grad[n_ell + 1] = 0.5 * sn2 * np.trace(W)
    return nlml, grad


def nlml_value(X, y, theta, n_ell):
    ell, sf2, sn2 = theta_split(theta, n_ell)
    K, _, _ = rbf_dense(X, ell, sf2, sn2)
    c, low = sla.cho_factor(K, lower=True)
    alpha = sla.cho_solve((c, low), y)
    return 0.5 * y @ alpha + np.sum(np.log(np.diag(c))) + 0.5 * len(y) * LOG2PI


def nlml_fd(X, y, theta, n_ell, h=1e-6):
    """Central finite differences of the dense NLML in log-parameter space."""
    theta = np.asarray(theta, dtype=np.float64)
    g = np.zeros_like(theta)
    for q in range(len(theta)):
        tp, tm = theta.copy(), theta.copy()
        tp[q] += h
        tm[q] -= h
        g[q] = (nlml_value(X, y, tp, n_ell) - nlml_value(X, y, tm, n_ell)) / (2 * h)
    return g


def nlml_fd4(X, y, theta, n_ell, h=3e-3):
    """Fourth-order central differences (5-point stencil) of the dense NLML:
    truncation O(h^4), rounding ~eps |NLML| / h, so a larger step keeps both
    small where the 2-point stencil at h = 1e-6 is limited by rounding."""
    theta = np.asarray(theta, dtype=np.float64)
    g = np.zeros_like(theta)
    for q in range(len(theta)):
        f = []
        for s in (-2, -1, 1, 2):
            t = theta.copy()
            t[q] += s * h
            f.append(nlml_value(X, y, t, n_ell))
        g[q] = (f[0] - 8.0 * f[1] + 8.0 * f[2] - f[3]) / (12.0 * h)
    return g


def tril_h(M):
    T = np.tril(M)
    T[np.diag_indices_from(T)] *= 0.5
    return T


def chol_adjoint_dense(L, Lbar):
    """Adjoint of the lower entries of A = L L^T given Lbar (lower)."""
    Lbar = np.tril(Lbar)
    H = tril_h(L.T @ Lbar)
    Li = sla.solve_triangular(L, np.eye(L.shape[0]), lower=True)
    return tril_h(Li.T @ (H + H.T) @ Li)


def chol_adjoint_fd(A, Lbar, h=1e-6):
    """d/dA_ij (i >= j, symmetric perturbation) of f(A) = sum(Lbar * chol(A))."""
    n = A.shape[0]
    out = np.zeros_like(A)
    for i in range(n):
        for j in range(i + 1):
            E = np.zeros_like(A)
            E[i, j] = E[j, i] = h
            fp = np.sum(Lbar * np.linalg.cholesky(A + E))
            fm = np.sum(Lbar * np.linalg.cholesky(A - E))
            out[i, j] = (fp - fm) / (2 * h)
    return out


def chol_adjoint_blocked(L, Lbar, bsz):
    """The reverse sweep of the CUDA kernels on a dense array (n a multiple of
    bsz): for k = nb-1 .. 0, with P the panel rows below block k and D = L_kk,
      (i)   Lbar_P -= (Abar + Abar^T)_trailing L_P
      (ii)  Abar_P  = Lbar_P D^-1
      (iii) Dbar   -= tril(Abar_P^T L_P)
      (iv)  Abar_kk = tril_h(D^-T (H + H^T) D^-1),  H = tril_h(D^T Dbar)."""
    n = L.shape[0]
    nb = n // bsz
    Ab = np.tril(Lbar).copy()
    for k in range(nb - 1, -1, -1):
        s, e = k * bsz, (k + 1) * bsz
        D = L[s:e, s:e]
        Di = sla.solve_triangular(D, np.eye(bsz), lower=True)
        if e < n:
            Tr = Ab[e:, e:]
            S = Tr + Tr.T  # diagonal doubled, as (Abar_rr + Abar_rr^T)
            Ab[e:, s:e] -= S @ L[e:, s:e]
            Ab[e:, s:e] = Ab[e:, s:e] @ Di
            Ab[s:e, s:e] -= np.tril(Ab[e:, s:e].T @ L[e:, s:e])
        H = tril_h(D.T @ np.tril(Ab[s:e, s:e]))
        Ab[s:e, s:e] = tril_h(Di.T @ (H + H.T) @ Di)
    return Ab
