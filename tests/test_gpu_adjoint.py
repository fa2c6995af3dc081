"""Differentiation through the solve (the C5 configurations, at 64^2 / 16^3
and at the full 512^2 / 96^3): loss L = ||C x - d||^2 with x = A(kappa)^-1 b
and C sampling 1% of the cells, gradients with respect to the cell
coefficients kappa and to b.

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
import oracle
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


def gpu_grad(make, kappa, b, S, d, symmetric, h=None, tol=1e-13, precision="fp64"):
    A, J = make(kappa)
    if h is None:
        h = draugr.amg_setup(A, CFG)
    vals = torch.tensor(A.data, device="cuda", requires_grad=True)
    bt = torch.tensor(b, device="cuda", requires_grad=True)
    x = draugr.amg_solve_diff(vals, bt, h, CFG, tol=tol, maxiter=2000, symmetric=symmetric,
                              precision=precision)
    St = torch.tensor(S, device="cuda")
    L = ((x[St] - torch.tensor(d, device="cuda")) ** 2).sum()
    L.backward()
    return h, float(L.detach()), J.T @ vals.grad.cpu().numpy(), bt.grad.cpu().numpy()


def gpu_loss(h, make, kappa, b, S, d, symmetric, tol=1e-13, precision="fp64"):
    v = make(kappa, values_only=True)
    with torch.no_grad():
        x = draugr.amg_solve_diff(torch.tensor(v, device="cuda"), torch.tensor(b, device="cuda"), h,
                                  CFG, tol=tol, maxiter=3000, symmetric=symmetric, precision=precision)
    return float(((x.cpu().numpy()[S] - d) ** 2).sum())


def check_finite_differences(h, make, kappa, b, S, d, symmetric, L, gk, rng, ndir=20, tol=1e-13,
                             rtol=1e-5, precision="fp64"):
    """Central differences of the GPU forward solve's loss (h = 1e-6,
    relative step) along `ndir` seeded directions, against gk . delta
    (relative error `rtol`); the forward solves stop at relative residual
    `tol`."""
    eps = 1e-6
    shape = kappa.shape
    for t in range(ndir):
        delta = rng.normal(size=shape) * kappa
        lp = gpu_loss(h, make, kappa + eps * delta, b, S, d, symmetric, tol, precision)
        lm = gpu_loss(h, make, kappa - eps * delta, b, S, d, symmetric, tol, precision)
        fd = (lp - lm) / (2 * eps)
        ad = float(gk @ delta.ravel())
        assert abs(fd - ad) <= rtol * max(abs(ad), 1e-3 * abs(L)), (t, fd, ad)


CASES = {
    "convection_diffusion_2d": (lambda k, **kw: problems.convection_diffusion_2d(k, 50.0, seed=5, **kw),
                                (64, 64), False),
    "diffusion_3d": (lambda k, **kw: problems.fv_diffusion_3d(k, **kw), (16, 16, 16), True),
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
    check_finite_differences(h, make, kappa, b, S, d, symmetric, L, gk, rng)


FULL = {
    "convection_diffusion_2d_512": (CASES["convection_diffusion_2d"][0], (512, 512), False),
    "diffusion_3d_96": (CASES["diffusion_3d"][0], (96, 96, 96), True),
}


@pytest.mark.parametrize("name", sorted(FULL))
def test_full_size_gradient(name):
    """The C5 sizes: 512^2 upwind convection-diffusion (Peclet 50) and 96^3
    diffusion, kappa log-normal (sigma 1).  CPU FP64 adjoint: direct solves
    (scipy) for the 2D operator; for the 3D operator, whose direct
    factorisation does not fit a test, the oracle's FP64 AMG-PCG on the same
    hierarchy to 1e-15.  GPU solves to 1e-14 for the gradient (1e-12 against
    the CPU adjoint).  The finite differences need forward solves as exact
    as FP64 allows: at h = 1e-6 the loss changes by ~1e-9 of itself along a
    random direction, so they solve to 1e-15 (or until the iteration
    stalls), and the rounding left in the loss (~1e-13 of it, divided by h)
    sets a floor near 1e-5 relative on the 512^2 convection-diffusion
    operator: the bound is 1e-4 (a wrong gradient is off by O(1))."""
    make, shape, symmetric = FULL[name]
    rng = np.random.default_rng(23)
    kappa = np.exp(rng.normal(0.0, 1.0, shape))
    n = kappa.size
    b = rng.uniform(-1, 1, n)
    S = np.sort(rng.choice(n, size=n // 100, replace=False))
    d = rng.uniform(-0.1, 0.1, len(S))
    A, J = make(kappa)
    h, L, gk, gb = gpu_grad(make, kappa, b, S, d, symmetric, tol=1e-14)
    if symmetric:
        O = oracle.OracleHierarchy(h)
        x, itx, _ = O.pcg(np.zeros(n), b, tol=1e-15, maxiter=3000)
        gx = np.zeros(n)
        gx[S] = 2 * (x[S] - d)
        lam, itl, _ = O.pcg(np.zeros(n), gx, tol=1e-15, maxiter=3000)
        rows = np.repeat(np.arange(n), np.diff(A.indptr))
        ref_k, ref_b = J.T @ (-lam[rows] * x[A.indices]), lam
    else:
        ref_k, ref_b = cpu_adjoint(A, J, b, S, d)
    ek, eb = rel(gk, ref_k), rel(gb, ref_b)
    print(f"{name}: gradient vs CPU adjoint: kappa {ek:.2e}, b {eb:.2e}")
    assert ek < 1e-12 and eb < 1e-12, (ek, eb)
    check_finite_differences(h, make, kappa, b, S, d, symmetric, L, gk, rng, tol=1e-15, rtol=1e-4)


@pytest.mark.parametrize("smoother", ["l1_jacobi", "spai0"])
def test_transposed_bicgstab_solves_the_adjoint_system(smoother):
    kappa = np.exp(np.random.default_rng(2).normal(0.0, 1.0, (48, 48)))
    A, _ = problems.convection_diffusion_2d(kappa, 50.0, seed=1)
    cfg = CFG if smoother == "l1_jacobi" else draugr.hypre_default_config(
        agg_trunc_factor=0.2, smoother=draugr.SPAI0SmootherType(), seed=3)
    h = draugr.amg_setup(A, cfg)
    b = np.random.default_rng(3).uniform(-1, 1, A.shape[0])
    for transpose, M in ((False, A), (True, A.T.tocsr())):
        x, it, rr = draugr.bicgstab(np.zeros(A.shape[0]), b, h, cfg, tol=1e-10, maxiter=500,
                                    transpose=transpose)
        assert it < 500 and rr < 1e-10
        assert np.linalg.norm(b - M @ x) / np.linalg.norm(b) < 1e-10


@pytest.mark.parametrize("name", sorted(CASES) + sorted(FULL))
def test_fp32_cycle_gradient(name):
    """The precision the C5 configuration names: both solves of the
    gradient (forward, and the adjoint on the transposed hierarchy) with the
    FP32 cycle (FP32 copies of the hierarchy and of its transpose) inside
    the FP64 Krylov iteration, to 1e-13.  Checked against the FP64 CPU
    adjoint (direct solves; for the 96^3 diffusion operator the oracle's
    FP64 AMG-PCG to 1e-15) at 1e-10 normwise relative, and against central
    differences on 20 seeded directions (h = 1e-6): of the FP32-cycle
    forward solve at the small sizes (1e-5 relative), of the FP64 forward
    solve at the full sizes (1e-4 relative), where the differences need the
    forward solves to stop near 1e-15 and BiCGStab with the FP32 cycle
    stalls a little above that."""
    full = name in FULL
    make, shape, symmetric = FULL[name] if full else CASES[name]
    rng = np.random.default_rng(29)
    kappa = np.exp(rng.normal(0.0, 1.0, shape))
    n = kappa.size
    b = rng.uniform(-1, 1, n)
    S = np.sort(rng.choice(n, size=max(1, n // 100), replace=False))
    d = rng.uniform(-0.1, 0.1, len(S))
    A, J = make(kappa)
    h, L, gk, gb = gpu_grad(make, kappa, b, S, d, symmetric, tol=1e-13, precision="mixed")
    if full and symmetric:
        O = oracle.OracleHierarchy(h)
        x, _, _ = O.pcg(np.zeros(n), b, tol=1e-15, maxiter=3000)
        gx = np.zeros(n)
        gx[S] = 2 * (x[S] - d)
        lam, _, _ = O.pcg(np.zeros(n), gx, tol=1e-15, maxiter=3000)
        rows = np.repeat(np.arange(n), np.diff(A.indptr))
        ref_k, ref_b = J.T @ (-lam[rows] * x[A.indices]), lam
    else:
        ref_k, ref_b = cpu_adjoint(A, J, b, S, d)
    ek, eb = rel(gk, ref_k), rel(gb, ref_b)
    print(f"{name}, FP32 cycle: gradient vs FP64 CPU adjoint: kappa {ek:.2e}, b {eb:.2e}")
    assert ek < 1e-10 and eb < 1e-10, (ek, eb)
    if full:
        check_finite_differences(h, make, kappa, b, S, d, symmetric, L, gk, rng, tol=1e-15, rtol=1e-4)
    else:
        check_finite_differences(h, make, kappa, b, S, d, symmetric, L, gk, rng, precision="mixed")
