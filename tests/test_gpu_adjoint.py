"""Differentiation through the solve (the C5 configurations, reduced in
size): loss L = ||C x - d||^2 with x = A(kappa)^-1 b and C sampling 1% of
the cells, gradients with respect to the cell coefficients kappa and to b.

The library's backward pass solves the adjoint system A^T lambda = dL/dx
on the GPU (BiCGStab with cycles on the transposed hierarchy for the
nonsymmetric convection-diffusion operator, PCG for the symmetric diffusion
operator) and forms dL/da_ij = -lambda_i x_j per nonzero; the problem's
Jacobian J = d(values)/d(kappa) maps that onto cells.  Checked against an
FP64 CPU adjoint with direct solves (scipy; 1e-10 normwise relative, the
iterative solves stopping at 1e-13) and against central finite differences
of the GPU forward solve on 20 seeded directions (h = 1e-6, relative step).
"""

import numpy as np
import pytest
import scipy.sparse.linalg as spla

import draugr
from draugr import problems

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

CFG = draugr.hypre_default_config(agg_trunc_factor=0.2, smoother=draugr.L1JacobiSmootherType(), seed=3)


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / (nb if nb > 0 else 1.0)


def cpu_adjoint(A, J, b, S, d):
    x = spla.spsolve(A.tocsc(), b)
    gx = np.zeros_like(x)
    gx[S] = 2 * (x[S] - d)
    lam = spla.spsolve(A.T.tocsc(), gx)
    rows = np.repeat(np.arange(A.shape[0]), np.diff(A.indptr))
    gvals = -lam[rows] * x[A.indices]
    return J.T @ gvals, lam


def gpu_grad(make, kappa, b, S, d, symmetric, h=None):
    A, J = make(kappa)
    if h is None:
        h = draugr.amg_setup(A, CFG)
    vals = torch.tensor(A.data, device="cuda", requires_grad=True)
    bt = torch.tensor(b, device="cuda", requires_grad=True)
    x = draugr.amg_solve_diff(vals, bt, h, CFG, tol=1e-13, maxiter=2000, symmetric=symmetric)
    St = torch.tensor(S, device="cuda")
    L = ((x[St] - torch.tensor(d, device="cuda")) ** 2).sum()
    L.backward()
    return h, float(L.detach()), J.T @ vals.grad.cpu().numpy(), bt.grad.cpu().numpy()


def gpu_loss(h, make, kappa, b, S, d, symmetric):
    A, _ = make(kappa)
    with torch.no_grad():
        x = draugr.amg_solve_diff(torch.tensor(A.data, device="cuda"), torch.tensor(b, device="cuda"), h,
                                  CFG, tol=1e-13, maxiter=2000, symmetric=symmetric)
    return float(((x.cpu().numpy()[S] - d) ** 2).sum())


CASES = {
    "convection_diffusion_2d": (lambda k: problems.convection_diffusion_2d(k, 50.0, seed=5), (64, 64), False),
    "diffusion_3d": (lambda k: problems.fv_diffusion_3d(k), (16, 16, 16), True),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_gradient_matches_cpu_adjoint_and_finite_differences(name):
    make, shape, symmetric = CASES[name]
    rng = np.random.default_rng(17)
    kappa = np.exp(rng.normal(0.0, 1.0, shape))
    n = kappa.size
    b = rng.uniform(-1, 1, n)
    S = np.sort(rng.choice(n, size=max(1, n // 100), replace=False))
    d = rng.uniform(-0.1, 0.1, len(S))
    A, J = make(kappa)
    if not symmetric:
        assert abs(A - A.T).max() > 1.0
    h, L, gk, gb = gpu_grad(make, kappa, b, S, d, symmetric)
    ref_k, ref_b = cpu_adjoint(A, J, b, S, d)
    assert rel(gk, ref_k) < 1e-10, rel(gk, ref_k)
    assert rel(gb, ref_b) < 1e-10, rel(gb, ref_b)
    eps = 1e-6
    for t in range(20):
        delta = rng.normal(size=shape) * kappa
        lp = gpu_loss(h, make, kappa + eps * delta, b, S, d, symmetric)
        lm = gpu_loss(h, make, kappa - eps * delta, b, S, d, symmetric)
        fd = (lp - lm) / (2 * eps)
        ad = float(gk @ delta.ravel())
        assert abs(fd - ad) <= 1e-5 * max(abs(ad), 1e-3 * abs(L)), (t, fd, ad)


def test_transposed_bicgstab_solves_the_adjoint_system():
    kappa = np.exp(np.random.default_rng(2).normal(0.0, 1.0, (48, 48)))
    A, _ = problems.convection_diffusion_2d(kappa, 50.0, seed=1)
    h = draugr.amg_setup(A, CFG)
    b = np.random.default_rng(3).uniform(-1, 1, A.shape[0])
    for transpose, M in ((False, A), (True, A.T.tocsr())):
        x, it, rr = draugr.bicgstab(np.zeros(A.shape[0]), b, h, CFG, tol=1e-10, maxiter=500,
                                    transpose=transpose)
        assert it < 500 and rr < 1e-10
        assert np.linalg.norm(b - M @ x) / np.linalg.norm(b) < 1e-10
