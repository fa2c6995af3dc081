"""The oracle's restatements of the smoothers checked against independent
NumPy mathematics on small matrices: ILU(0) of a tridiagonal matrix (no
fill) is its exact LU factorisation; each SPAI(1) row solves the
least-squares problem min ||e_i - A^T m|| over row i's pattern; the
Chebyshev power iteration approaches the largest eigenvalue of D^-1 A; one
serial Gauss-Seidel sweep equals a plain row loop; SPAI(0) is
a_ii / ||A_i,:||^2."""

import numpy as np
import scipy.sparse as sp

import oracle
from draugr import problems


def parts(A):
    A = A.tocsr()
    A.sort_indices()
    return A.shape[0], A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data.astype(np.float64)


def test_ilu0_of_tridiagonal_is_exact_lu():
    rng = np.random.default_rng(1)
    n = 12
    A = sp.diags([rng.uniform(-1, -0.5, n - 1), rng.uniform(3, 4, n), rng.uniform(-1, -0.5, n - 1)],
                 [-1, 0, 1], format="csr")
    n, rp, ci, v = parts(A)
    diag = oracle.ilu0_diag(n, rp, ci)
    Lf, Uf = oracle.ilu0_factor(n, rp, ci, v, diag)
    L = sp.csr_matrix((Lf, ci, rp), shape=(n, n)).toarray() + np.eye(n)
    U = sp.csr_matrix((Uf, ci, rp), shape=(n, n)).toarray()
    assert np.allclose(np.tril(L, -1) + np.eye(n), L) and np.allclose(np.triu(U), U)
    assert np.abs(L @ U - A.toarray()).max() < 1e-13


def test_spai1_rows_solve_their_least_squares_problems():
    A = problems.poisson2d(5)
    n, rp, ci, v = parts(A)
    M = oracle.spai1(n, rp, ci, v)
    Ad = A.toarray()
    for i in range(n):
        J = ci[rp[i]:rp[i + 1]]
        e = np.zeros(n)
        e[i] = 1.0
        m, *_ = np.linalg.lstsq(Ad[:, J], e, rcond=None)  # min ||e_i - A[:, J] m|| (A symmetric: A^T = A)
        assert np.allclose(M[rp[i]:rp[i + 1]], m, rtol=1e-10, atol=1e-12), i


def test_power_iteration_approaches_the_spectral_radius_of_dinv_a():
    A = problems.poisson1d(30)
    n, rp, ci, v = parts(A)
    inv = oracle.invdiag(n, rp, ci, v)
    lam_max = np.max(np.abs(np.linalg.eigvals(np.diag(inv) @ A.toarray())))
    v0 = np.random.default_rng(2).standard_normal(n)
    rho = oracle.spectral_radius(n, rp, ci, v, inv, v0 / np.linalg.norm(v0), niter=2000)
    assert abs(rho - lam_max) < 1e-3 * lam_max
    rho10 = oracle.spectral_radius(n, rp, ci, v, inv, v0 / np.linalg.norm(v0), niter=10)
    assert 0 < rho10 <= lam_max * (1 + 1e-12)  # an estimate from below, as the reference's


def test_serial_gs_and_spai0_match_plain_numpy():
    A = problems.poisson2d(6)
    n, rp, ci, v = parts(A)
    rng = np.random.default_rng(3)
    x0, b = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    inv = oracle.serial_gs_invdiag(n, rp, ci, v)
    x = x0.copy()
    Ad = A.toarray()
    for i in range(n):
        x[i] += inv[i] * (b[i] - Ad[i] @ x)
    assert np.allclose(oracle.serial_gs(n, rp, ci, v, inv, x0, b, 1), x, rtol=1e-14, atol=1e-15)
    m = oracle.spai0(n, rp, ci, v)
    assert np.allclose(m, np.diag(Ad) / (Ad ** 2).sum(axis=1), rtol=1e-15)
