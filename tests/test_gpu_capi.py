"""The reference's C API lifecycle tests (test/runtests.jl:3513-3703),
restated against libdraugr_b200.so through ctypes: setup + solve + cycle +
free, partial / full resetup with and without restriction maps, zero-based
indexing and invalid handles."""

import ctypes as C

import numpy as np
import pytest

import draugr
from draugr import problems

pytestmark = pytest.mark.gpu


def p(a):
    return a.ctypes.data_as(C.c_void_p)


def laplacian_1d(n):
    rowptr, colval, nzval = [1], [], []
    for i in range(1, n + 1):
        if i > 1:
            colval.append(i - 1); nzval.append(-1.0)
        colval.append(i); nzval.append(2.0)
        if i < n:
            colval.append(i + 1); nzval.append(-1.0)
        rowptr.append(len(colval) + 1)
    return (np.array(rowptr, np.int32), np.array(colval, np.int32), np.array(nzval))


@pytest.fixture(scope="module")
def capi(lib):
    n = 20
    rowptr, colval, nzval = laplacian_1d(n)
    cfg = lib.draugr_amg_config_from_json(b"{}")
    assert cfg > 0
    yield lib, n, rowptr, colval, nzval, cfg
    lib.draugr_amg_config_free(cfg)


def test_setup_solve_cycle_free(capi):
    lib, n, rowptr, colval, nzval, cfg = capi
    nnz = len(nzval)
    h = lib.draugr_amg_setup(n, nnz, p(rowptr), p(colval), p(nzval), cfg, 1, 1)
    assert h > 0
    b = np.ones(n)
    x = np.zeros(n)
    niter = lib.draugr_amg_solve(h, n, p(x), p(b), cfg, 1e-10, 200)
    assert 0 < niter < 200
    x[:] = 0.0
    assert lib.draugr_amg_cycle(h, n, p(x), p(b), cfg) == 0
    assert np.linalg.norm(x) > 0
    assert lib.draugr_amg_free(h) == 0
    assert lib.draugr_amg_free(h) == -1


def test_partial_resetup(capi):
    lib, n, rowptr, colval, nzval, cfg = capi
    nnz = len(nzval)
    h = lib.draugr_amg_setup(n, nnz, p(rowptr), p(colval), p(nzval), cfg, 1, 1)
    nz2 = nzval * 1.5
    assert lib.draugr_amg_resetup(h, n, nnz, p(rowptr), p(colval), p(nz2), cfg, 1, 1, 1) == 0
    b, x = np.ones(n), np.zeros(n)
    niter = lib.draugr_amg_solve(h, n, p(x), p(b), cfg, 1e-10, 200)
    assert 0 < niter < 200
    lib.draugr_amg_free(h)


def test_full_resetup_variants(capi):
    lib, n, rowptr, colval, nzval, cfg = capi
    nnz = len(nzval)
    h = lib.draugr_amg_setup(n, nnz, p(rowptr), p(colval), p(nzval), cfg, 1, 0)
    assert h > 0
    nz2 = nzval * 2.0
    assert lib.draugr_amg_resetup(h, n, nnz, p(rowptr), p(colval), p(nz2), cfg, 1, 0, 1) == 0
    nz3 = nzval * 1.1
    assert lib.draugr_amg_resetup(h, n, nnz, p(rowptr), p(colval), p(nz3), cfg, 1, 1, 1) == 0
    b, x = np.ones(n), np.zeros(n)
    assert 0 < lib.draugr_amg_solve(h, n, p(x), p(b), cfg, 1e-10, 200) < 200
    lib.draugr_amg_free(h)


def test_zero_based(capi):
    lib, n, rowptr, colval, nzval, cfg = capi
    rp0, cv0 = rowptr - 1, colval - 1
    h = lib.draugr_amg_setup(n, len(nzval), p(rp0), p(cv0), p(nzval), cfg, 0, 1)
    assert h > 0
    b, x = np.ones(n), np.zeros(n)
    assert 0 < lib.draugr_amg_solve(h, n, p(x), p(b), cfg, 1e-10, 200) < 200
    lib.draugr_amg_free(h)


def test_invalid_handles_gpu(capi):
    lib, n, rowptr, colval, nzval, cfg = capi
    b, x = np.ones(n), np.zeros(n)
    assert lib.draugr_amg_resetup(9999, n, len(nzval), p(rowptr), p(colval), p(nzval), cfg,
                                  1, 1, 1) == -1
    assert len(draugr.last_error()) > 0
    assert lib.draugr_amg_solve(9999, n, p(x), p(b), cfg, 1e-10, 50) == -1
    assert lib.draugr_amg_cycle(9999, n, p(x), p(b), cfg) == -1
    assert lib.draugr_amg_free(9999) == -1


def test_partial_resetup_rejects_other_pattern(lib):
    A = problems.poisson2d(16)
    cfg = draugr.AMGConfig(coarsening=draugr.AggregationCoarsening())
    h = draugr.amg_setup(A, cfg)
    B = problems.poisson2d(17)
    with pytest.raises(draugr.DraugrError, match="sparsity pattern|pattern"):
        draugr.amg_resetup(h, B, cfg)
    h2 = draugr.amg_setup(A, cfg, allow_partial_resetup=False)
    with pytest.raises(draugr.DraugrError, match="allow_partial_resetup"):
        draugr.amg_resetup(h2, A, cfg)


def test_solve_reference_thresholds(lib):
    """amg_solve! reaches 1e-8 in fewer than 200 cycles for each coarsening,
    and W-cycles need no more cycles than V-cycles (test/runtests.jl:332-415,
    :1828-1855)."""
    A = problems.poisson2d(10)
    b = np.random.default_rng(0).uniform(0, 1, 100)
    for coars in (draugr.AggregationCoarsening(), draugr.PMISCoarsening(),
                  draugr.AggressiveCoarsening(), draugr.HMISCoarsening(0.5, draugr.ExtendedIInterpolation())):
        cfg = draugr.AMGConfig(coarsening=coars, max_coarse_size=10)
        h = draugr.amg_setup(A, cfg)
        x, it = draugr.amg_solve(np.zeros(100), b, h, cfg, tol=1e-8, maxiter=200)
        assert it < 200
        assert np.linalg.norm(b - A @ x) / np.linalg.norm(b) < 1e-8
    A = problems.poisson2d(32)
    b = np.random.default_rng(1).uniform(0, 1, A.shape[0])
    cv = draugr.AMGConfig(coarsening=draugr.AggregationCoarsening(), cycle_type="V")
    cw = draugr.AMGConfig(coarsening=draugr.AggregationCoarsening(), cycle_type="W")
    h = draugr.amg_setup(A, cv)
    _, itv = draugr.amg_solve(np.zeros(A.shape[0]), b, h, cv, tol=1e-8, maxiter=300)
    _, itw = draugr.amg_solve(np.zeros(A.shape[0]), b, h, cw, tol=1e-8, maxiter=300)
    assert itw <= itv
