"""The reference's coarsening testsets (test/runtests.jl), restated against
the library's CPU setup: PMIS, HMIS and aggressive C/F splittings, their
coarsening ratios and hierarchy depths, and solves through hierarchies with
isolated or disconnected rows.  The splitting is read back from the
host-only hierarchy (export "cf" of level 0); solves run the oracle's
amg_solve! on the CPU."""

import numpy as np
import pytest
import scipy.sparse as sp

import draugr
import oracle
from draugr import problems


def first_level(A, coarsening, **kw):
    cfg = draugr.AMGConfig(coarsening=coarsening, max_coarse_size=2, **kw)
    h = draugr.amg_setup(A, cfg, on_device=False)
    assert h.nlevels >= 1
    return h, h.export(0, "cf"), int(h.level_info(0)[2])


def oracle_solve(A, cfg, b, tol=1e-8, maxiter=200):
    h = draugr.amg_setup(A, cfg, on_device=False)
    O = oracle.OracleHierarchy(h)
    x, it, _ = O.solve(np.zeros(A.shape[0]), b, cfg.pre_smoothing_steps, cfg.post_smoothing_steps,
                       False, tol, maxiter)
    return x, it


def rel_res(A, x, b):
    return np.linalg.norm(b - A @ x) / np.linalg.norm(b)


def test_pmis_coarsening_1d():
    """testset "PMIS Coarsening" (test/runtests.jl:118-126): every point of
    the 1D Laplacian (20) decided, 0 < nc < 20."""
    _, cf, nc = first_level(problems.poisson1d(20), draugr.PMISCoarsening(0.25))
    assert len(cf) == 20 and np.all(np.abs(cf) == 1)
    assert 0 < nc < 20 and int(np.sum(cf == 1)) == nc


def test_hmis_coarsening_1d_fine_points_have_coarse_neighbours():
    """testset "HMIS Coarsening" (test/runtests.jl:933-956): 1D Laplacian
    (20), all points decided, 0 < nc < 20, every F-point has a C-point among
    its off-diagonal neighbours."""
    A = problems.poisson1d(20)
    _, cf, nc = first_level(A, draugr.HMISCoarsening(0.25))
    assert len(cf) == 20 and np.all(np.abs(cf) == 1) and 0 < nc < 20
    A = A.tocsr()
    for i in range(20):
        if cf[i] == -1:
            cols = A.indices[A.indptr[i]:A.indptr[i + 1]]
            assert any(j != i and cf[j] == 1 for j in cols), i


def test_hmis_coarsening_2d_count_and_ratio():
    """testsets "HMIS Coarsening - 2D" and "HMIS Coarsening ratio - 2D"
    (test/runtests.jl:958-977): on 8 x 8, 0 < nc < 64 and nc counts the
    C-points; on 20 x 20 with theta = 0.5, fewer than 60% of the points are
    coarse and all are decided."""
    _, cf, nc = first_level(problems.poisson2d(8), draugr.HMISCoarsening(0.25))
    assert 0 < nc < 64 and int(np.sum(cf == 1)) == nc
    _, cf, nc = first_level(problems.poisson2d(20), draugr.HMISCoarsening(0.5))
    assert nc / 400 < 0.6 and np.all(np.abs(cf) == 1)


def test_hmis_hierarchy_depth_2d():
    """testset "HMIS Hierarchy depth - 2D" (test/runtests.jl:979-987): HMIS
    (0.5) with extended+i interpolation on 50 x 50 gives at most 10 levels,
    counting the coarsest."""
    cfg = draugr.AMGConfig(coarsening=draugr.HMISCoarsening(0.5, draugr.ExtendedIInterpolation()))
    h = draugr.amg_setup(problems.poisson2d(50), cfg, on_device=False)
    assert h.nlevels + 1 <= 10


@pytest.mark.parametrize("coarsening", [draugr.PMISCoarsening(), draugr.HMISCoarsening(),
                                        draugr.AggressiveCoarsening()],
                         ids=["pmis", "hmis", "aggressive"])
def test_setup_and_solve_2d(coarsening):
    """testsets "AMG Setup - PMIS / Aggressive / HMIS" and "AMG Solve - PMIS
    / Aggressive" (test/runtests.jl:298-310, :346-372, :989-994): the 10 x
    10 Laplacian gets at least one level, and amg_solve! reaches 1e-8 in
    fewer than 200 cycles."""
    A = problems.poisson2d(10)
    cfg = draugr.AMGConfig(coarsening=coarsening)
    assert draugr.amg_setup(A, cfg, on_device=False).nlevels > 0
    b = np.random.default_rng(11).uniform(0, 1, 100)
    x, it = oracle_solve(A, cfg, b)
    assert it < 200 and rel_res(A, x, b) < 1e-8


def test_pmis_good_coarsening_ratios():
    """testset "PMIS - Good coarsening ratios" (test/runtests.jl:1335-1348):
    PMIS with direct interpolation on 20 x 20 builds at least one level and
    solves to 1e-8."""
    A = problems.poisson2d(20)
    cfg = draugr.AMGConfig(coarsening=draugr.PMISCoarsening(0.25, draugr.DirectInterpolation()))
    assert draugr.amg_setup(A, cfg, on_device=False).nlevels >= 1
    b = np.random.default_rng(12).uniform(0, 1, 400)
    x, _ = oracle_solve(A, cfg, b)
    assert rel_res(A, x, b) < 1e-8


def test_isolated_and_disconnected_rows():
    """testsets "Isolated diagonal-only rows" and "Block diagonal matrix"
    (test/runtests.jl:1353-1382): the default configuration solves a 5 x 5
    matrix with two diagonal-only rows, and two 2 x 2 blocks plus an
    isolated node, to 1e-8."""
    I = [0, 0, 1, 2, 2, 3, 4]
    J = [0, 1, 1, 2, 3, 3, 4]
    V = [4.0, -1.0, 5.0, -1.0, 4.0, -1.0, 3.0]
    A = sp.csr_matrix((V, (I, J)), shape=(5, 5))
    b = np.array([1.0, 2.0, 3.0, 4.0, 5.0])
    x, _ = oracle_solve(A, draugr.AMGConfig(), b, tol=1e-10, maxiter=100)
    assert rel_res(A, x, b) < 1e-8
    I = [0, 0, 1, 1, 2, 2, 3, 3, 4]
    J = [0, 1, 0, 1, 2, 3, 2, 3, 4]
    V = [4.0, -1.0, -1.0, 4.0, 4.0, -1.0, -1.0, 4.0, 3.0]
    A = sp.csr_matrix((V, (I, J)), shape=(5, 5))
    x, _ = oracle_solve(A, draugr.AMGConfig(), np.ones(5), tol=1e-10, maxiter=100)
    assert rel_res(A, x, np.ones(5)) < 1e-8


@pytest.mark.parametrize("coarsening", [draugr.PMISCoarsening(), draugr.HMISCoarsening(),
                                        draugr.RSCoarsening()], ids=["pmis", "hmis", "rs"])
def test_isolated_nodes(coarsening):
    """testset "Isolated nodes in PMIS/HMIS" (test/runtests.jl:1384-1413): a
    tridiagonal matrix with diagonal 100 and off-diagonals -1e-10 has no
    strong coupling worth the name; every splitting still gives a hierarchy
    that solves to 1e-8."""
    n = 10
    A = sp.diags([np.full(n - 1, -1e-10), np.full(n, 100.0), np.full(n - 1, -1e-10)],
                 [-1, 0, 1], format="csr")
    b = np.random.default_rng(13).uniform(0, 1, n)
    x, _ = oracle_solve(A, draugr.AMGConfig(coarsening=coarsening), b)
    assert rel_res(A, x, b) < 1e-8
