"""Small and degenerate inputs through the C ABI on the GPU: the reference's
"Small/Trivial Systems" testset (test/runtests.jl:1798-1815: 1 x 1 and 2 x 2
systems with no AMG level), zero right-hand sides (solve, PCG, a zero column
of block PCG: no iterations, x = 0), and every smoother type on a small
multilevel problem against the oracle."""

import numpy as np
import pytest
import scipy.sparse as sp

import draugr
import oracle
from draugr import problems

pytestmark = pytest.mark.gpu

SMOOTHERS = ["JacobiSmootherType", "L1JacobiSmootherType", "ColoredGaussSeidelType",
             "L1ColoredGaussSeidelType", "SerialGaussSeidelType", "L1SerialGaussSeidelType",
             "SPAI0SmootherType", "SPAI1SmootherType", "ChebyshevSmootherType", "ILU0SmootherType",
             "SerialILU0SmootherType"]


def test_one_by_one_and_two_by_two():
    A1 = sp.csr_matrix(np.array([[5.0]]))
    cfg = draugr.AMGConfig(max_coarse_size=10)
    h = draugr.amg_setup(A1, cfg)
    assert h.nlevels == 0
    x, _ = draugr.amg_solve(np.zeros(1), np.array([3.0]), h, cfg, tol=1e-10)
    assert abs(x[0] - 0.6) < 1e-8
    A2 = sp.csr_matrix(np.array([[4.0, -1.0], [-1.0, 4.0]]))
    h2 = draugr.amg_setup(A2, cfg)
    b = np.ones(2)
    x, _ = draugr.amg_solve(np.zeros(2), b, h2, cfg, tol=1e-10)
    assert np.linalg.norm(b - A2 @ x) / np.linalg.norm(b) < 1e-10


def test_zero_right_hand_sides():
    torch = pytest.importorskip("torch")
    A = problems.poisson2d(20)
    n = A.shape[0]
    cfg = draugr.hypre_default_config(agg_trunc_factor=0.2, smoother=draugr.L1JacobiSmootherType())
    h = draugr.amg_setup(A, cfg)
    x, it = draugr.amg_solve(np.ones(n), np.zeros(n), h, cfg, tol=1e-8)
    assert it == 0 and not np.any(x)
    for precision in ("fp64", "mixed"):
        x, it, rel = draugr.pcg(np.ones(n), np.zeros(n), h, cfg, tol=1e-8, precision=precision)
        assert it == 0 and not np.any(x)
    B = torch.tensor(np.random.default_rng(1).uniform(-1, 1, (n, 4)), device="cuda")
    B[:, 2] = 0.0
    X = torch.zeros_like(B)
    X, its, rels = draugr.pcg_multi(X, B, h, cfg, tol=1e-8)
    assert its[2] == 0 and not torch.any(X[:, 2])
    assert all(its[c] > 0 and rels[c] < 1e-8 for c in (0, 1, 3))


@pytest.mark.parametrize("smoother", SMOOTHERS)
def test_every_smoother_on_a_small_hierarchy(smoother):
    """Each smoother type with the reference's per-smoother solve setting
    (default HMIS coarsening, V(2,2), the 10 x 10 Poisson matrix; levels of
    a few dozen rows): the GPU solve reaches 1e-8 in the oracle's number of
    cycles (+-1)."""
    A = problems.poisson2d(10)
    n = A.shape[0]
    cfg = draugr.AMGConfig(smoother=getattr(draugr, smoother)(), max_coarse_size=10,
                           pre_smoothing_steps=2, post_smoothing_steps=2)
    h = draugr.amg_setup(A, cfg)
    assert h.nlevels >= 1
    b = np.random.default_rng(3).uniform(-1, 1, n)
    x, it = draugr.amg_solve(np.zeros(n), b, h, cfg, tol=1e-8, maxiter=300)
    assert it < 300 and np.linalg.norm(b - A @ x) / np.linalg.norm(b) < 1e-8
    O = oracle.OracleHierarchy(h)
    _, ito, _ = O.solve(np.zeros(n), b, 2, 2, False, 1e-8, 300)
    assert abs(it - ito) <= 1, (it, ito)
