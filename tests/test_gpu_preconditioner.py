"""The preconditioner object (Draugr.jl's DraugrPreconditioner,
src/preconditioner.jl:12-102): update builds then resets up the hierarchy,
apply / ldiv zero x and run one cycle, and the SciPy LinearOperator view
preconditions scipy.sparse.linalg.cg and gmres (the Python counterpart of
the LinearSolve.jl / Krylov.jl hooks)."""

import numpy as np
import pytest
import scipy.sparse.linalg as spla

import draugr
import oracle
from draugr import problems

pytestmark = pytest.mark.gpu


def test_apply_is_one_cycle_from_zero_and_update_resets_up():
    A = problems.heterogeneous_diffusion_3d(12, seed=4)
    n = A.shape[0]
    P = draugr.DraugrPreconditioner(draugr.hypre_default_config(
        agg_trunc_factor=0.2, smoother=draugr.L1JacobiSmootherType()))
    assert P.nrows == 0
    P.update(A)
    assert P.nrows == n
    y = np.random.default_rng(1).uniform(-1, 1, n)
    x = P.ldiv(np.full(n, 7.0), y)  # x is zeroed first
    O = oracle.OracleHierarchy(P.hierarchy)
    ref = O.cycle(np.zeros(n), y, 1, 1, False)
    assert np.linalg.norm(x - ref) / np.linalg.norm(ref) < 1e-12
    h = P.hierarchy
    A2 = (2.0 * A).tocsr()
    P.update(A2)  # same pattern: partial resetup of the same hierarchy
    assert P.hierarchy is h
    x2 = P.apply(np.zeros(n), y)
    assert np.linalg.norm(x2 - 0.5 * x) / np.linalg.norm(x) < 1e-12


def test_scipy_krylov_with_the_preconditioner():
    A = problems.heterogeneous_diffusion_3d(16, seed=2)
    n = A.shape[0]
    b = np.random.default_rng(3).uniform(-1, 1, n)
    P = draugr.DraugrPreconditioner(coarsening=draugr.HMISCoarsening(0.5, draugr.ExtendedIInterpolation()),
                                    smoother=draugr.L1JacobiSmootherType()).update(A)
    M = P.as_linear_operator()
    its = {"amg": 0, "none": 0}

    def counter(key):
        def cb(_):
            its[key] += 1
        return cb

    x, info = spla.cg(A, b, rtol=1e-8, maxiter=500, M=M, callback=counter("amg"))
    assert info == 0 and np.linalg.norm(b - A @ x) / np.linalg.norm(b) < 1e-8
    x0, info0 = spla.cg(A, b, rtol=1e-8, maxiter=500, callback=counter("none"))
    assert its["amg"] * 5 < its["none"]
    xg, infog = spla.gmres(A, b, rtol=1e-8, restart=30, maxiter=50, M=M)
    assert infog == 0 and np.linalg.norm(b - A @ xg) / np.linalg.norm(b) < 1e-7


def test_apply_on_cuda_tensors():
    torch = pytest.importorskip("torch")
    A = problems.poisson3d(14)
    n = A.shape[0]
    P = draugr.DraugrPreconditioner(smoother=draugr.JacobiSmootherType()).update(A)
    y = np.random.default_rng(5).uniform(-1, 1, n)
    xh = P.apply(np.zeros(n), y)
    xd = P.apply(torch.ones(n, dtype=torch.float64, device="cuda"), torch.tensor(y, device="cuda"))
    assert np.array_equal(xd.cpu().numpy(), xh)
