"""FGMRES and iterative refinement around the AMG cycle, through the C ABI.

The reference has no Krylov solver of its own: it hands amg_cycle! to
LinearSolve.jl as a preconditioner (ext/DraugrLinearSolveExt.jl:35-37,
src/preconditioner.jl:76-102).  These tests therefore check the mathematics:
every solution's residual is recomputed in FP64 on the host, FGMRES is
compared with a sparse direct solve on a small nonsymmetric system, and
iteration counts are compared with the library's own AMG-PCG where both
apply.

* Nonsymmetric: 2D upwind convection-diffusion (cell Peclet number up to
  50, seeded divergence-free velocity), hypre_default_config with
  l1-Jacobi: FGMRES with the FP64 cycle and with the FP32 cycle.
* Symmetric: the 3D heterogeneous-diffusion system (sigma = 3): FGMRES
  needs about as many iterations as PCG; iterative refinement with a mixed
  PCG inner solve (inner tolerance 1e-4) reaches 1e-8 in FP64 with at most
  1.5 times the iterations of one mixed PCG solve.
"""

import numpy as np
import pytest
import scipy.sparse.linalg as spla

import draugr
from draugr import problems

pytestmark = pytest.mark.gpu


def relres(A, x, b):
    return np.linalg.norm(b - A @ x) / np.linalg.norm(b)


def _cd(m, seed=5):
    kappa = np.exp(np.random.default_rng(seed).normal(0.0, 1.0, (m, m)))
    A, _ = problems.convection_diffusion_2d(kappa, 50.0, seed=seed)
    return A.tocsr()


@pytest.fixture(scope="module")
def cfg():
    return draugr.hypre_default_config(agg_trunc_factor=0.2, smoother=draugr.L1JacobiSmootherType())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_fgmres_nonsymmetric_matches_a_direct_solve(cfg, precision):
    A = _cd(64)
    n = A.shape[0]
    b = problems.rhs(n, 1)
    h = draugr.amg_setup(A, cfg)
    x, it, rel = draugr.fgmres(np.zeros(n), b, h, cfg, tol=1e-10, maxiter=300, precision=precision)
    assert 0 < it < 300 and rel < 1e-10
    assert relres(A, x, b) < 1e-10
    xd = spla.spsolve(A.tocsc(), b)
    assert np.linalg.norm(x - xd) / np.linalg.norm(xd) < 1e-7
    h.free()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_fgmres_nonsymmetric_512(cfg, precision):
    torch = pytest.importorskip("torch")
    A = _cd(512)
    n = A.shape[0]
    b = problems.rhs(n, 2)
    h = draugr.amg_setup(A, cfg)
    xd = torch.zeros(n, dtype=torch.float64, device="cuda")
    bd = torch.tensor(b, device="cuda")
    _, it, rel = draugr.fgmres(xd, bd, h, cfg, tol=1e-8, maxiter=400, precision=precision)
    assert it < 400 and rel < 1e-8
    assert relres(A, xd.cpu().numpy(), b) < 1e-8
    # a short restart length still converges
    xd.zero_()
    _, it5, rel5 = draugr.fgmres(xd, bd, h, cfg, tol=1e-8, maxiter=2000, restart=5, precision=precision)
    assert rel5 < 1e-8 and relres(A, xd.cpu().numpy(), b) < 1e-8
    assert it5 >= it
    h.free()


def test_fgmres_and_refinement_on_the_spd_system(cfg):
    A = problems.heterogeneous_diffusion_3d(32, sigma=3.0, corr_len=8.0, seed=7)
    n = A.shape[0]
    b = problems.rhs(n, 3)
    h = draugr.amg_setup(A, cfg)
    _, itp, _ = draugr.pcg(np.zeros(n), b, h, cfg, tol=1e-8, precision="mixed")
    for precision in ("fp64", "mixed"):
        x, it, rel = draugr.fgmres(np.zeros(n), b, h, cfg, tol=1e-8, maxiter=300, precision=precision)
        assert relres(A, x, b) < 1e-8
        assert it <= itp + 5, (precision, it, itp)
    for inner in ("pcg", "fgmres"):
        x, steps, inner_its, rel = draugr.refine(np.zeros(n), b, h, cfg, tol=1e-8, inner_tol=1e-4, inner=inner,
                                                 precision="mixed")
        assert relres(A, x, b) < 1e-8 and rel < 1e-8
        assert 1 <= steps <= 5
        assert inner_its <= int(1.5 * itp) + 5, (inner, inner_its, itp)
    # a zero right-hand side: x = 0, no iterations
    x, it, rel = draugr.fgmres(np.ones(n), np.zeros(n), h, cfg)
    assert it == 0 and not np.any(x)
    x, steps, inner_its, rel = draugr.refine(np.ones(n), np.zeros(n), h, cfg)
    assert steps == 0 and not np.any(x)
    h.free()


def test_argument_errors(cfg):
    A = problems.poisson2d(16)
    n = A.shape[0]
    h = draugr.amg_setup(A, cfg)
    with pytest.raises(draugr.DraugrError, match="restart"):
        draugr.fgmres(np.zeros(n), np.ones(n), h, cfg, restart=64)
    with pytest.raises(draugr.DraugrError, match="inner_tol"):
        draugr.refine(np.zeros(n), np.ones(n), h, cfg, inner_tol=1.5)
    h.free()
