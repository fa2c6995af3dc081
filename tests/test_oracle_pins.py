"""Pins of the oracle (the CPU restatement of Draugr.jl's arithmetic) to the
reference's own test assertions (test/runtests.jl), since the reference is
Julia and cannot run here and ships no golden vectors.  Each test names the
testset it restates.  Hierarchy structures come from the library's CPU setup
(host-only, no GPU), as they do for the parity tests."""

import numpy as np
import pytest
import scipy.sparse as sp

import draugr
import oracle
from draugr import problems


def parts(A):
    return oracle.csr_parts(A)


def explicit_P(h, l):
    info = h.level_info(l)
    return sp.csr_matrix((h.export(l, "P_nzval"), h.export(l, "P_colval"), h.export(l, "P_rowptr")),
                         shape=(int(info[0]), int(info[2])))


def agg_hierarchy(A, **kw):
    cfg = draugr.AMGConfig(coarsening=draugr.AggregationCoarsening(0.25), max_coarse_size=2, **kw)
    return draugr.amg_setup(A, cfg, on_device=False)


def test_strength_and_aggregation_coarsening():
    """testsets "Strength of Connection" and "Aggregation Coarsening"
    (:96-116): every off-diagonal entry of the 1D Laplacian (10) is strong
    at theta 0.25 (18 of them); aggregation of the 1D Laplacian (20) gives
    0 < nc < 20 aggregates covering every point, none of them empty."""
    n, rp, ci, v = parts(problems.poisson1d(10))
    assert int(np.sum(oracle.strength_abs(n, rp, ci, v, 0.25))) == 18
    h = agg_hierarchy(problems.poisson1d(20))
    P = explicit_P(h, 0)
    nc = P.shape[1]
    assert P.shape[0] == 20 and 0 < nc < 20
    assert np.all(np.diff(P.indptr) == 1)
    assert set(P.indices.tolist()) == set(range(nc))


def test_prolongation_and_restriction():
    """testset "Prolongation" (:138-179): aggregation P has one unit entry per
    row, P*ones = ones, restriction preserves the sum, the transpose map has
    nc+1 offsets ending at nnz(P)+1, and restrict! equals the explicit Pᵀr
    (atol 1e-12)."""
    A = problems.poisson1d(10)
    h = agg_hierarchy(A)
    P = explicit_P(h, 0)
    n, nc = P.shape
    assert np.all(np.diff(P.indptr) == 1) and np.all(P.data == 1.0)
    xf = oracle.prolongate(n, P.indptr.astype(np.int32), P.indices.astype(np.int32), P.data,
                           np.ones(nc), np.zeros(n))
    assert np.allclose(xf, 1.0)
    off, rows, pnz = oracle.transpose_map(n, nc, P.indptr.astype(np.int32), P.indices.astype(np.int32))
    assert len(off) == nc + 1 and off[0] == 0 and off[-1] == n
    bc = oracle.restrict(nc, off, rows, pnz, P.data, np.ones(n))
    assert np.isclose(bc.sum(), n)
    r = np.random.default_rng(0).standard_normal(n)
    bc = oracle.restrict(nc, off, rows, pnz, P.data, r)
    assert np.allclose(bc, P.T @ r, atol=1e-12)


def _galerkin_check(A, scale):
    h = agg_hierarchy(A)
    P = explicit_P(h, 0)
    n, nc = P.shape
    _, arp, aci, av = parts(A)
    prp, pci = P.indptr.astype(np.int32), P.indices.astype(np.int32)
    c_rp, c_ci, c_v, nz_off, tpi, tai, tpj = oracle.coarse_sparsity(n, nc, arp, aci, av, prp, pci, P.data)
    Ac = sp.csr_matrix((c_v, c_ci, c_rp), shape=(nc, nc)).toarray()
    assert np.allclose(Ac, (P.T @ A @ P).toarray(), atol=1e-12)
    assert len(nz_off) == len(c_ci) + 1 and nz_off[0] == 0
    assert np.all(np.diff(nz_off) >= 0)
    # in-place resetup with scaled values
    av2 = av * scale
    cv2 = np.zeros(len(c_ci))
    oracle.load().orc_galerkin(len(c_ci), oracle.ptr(nz_off), oracle.ptr(tpi), oracle.ptr(tai),
                               oracle.ptr(tpj), oracle.ptr(P.data), oracle.ptr(av2), oracle.ptr(cv2))
    Ac2 = sp.csr_matrix((cv2, c_ci, c_rp), shape=(nc, nc)).toarray()
    A2 = sp.csr_matrix((av2, aci, arp), shape=(n, n))
    assert np.allclose(Ac2, (P.T @ A2 @ P).toarray(), atol=1e-12)


def test_galerkin_product():
    """testsets "Galerkin Product" (:215-241), "contention-free kernel"
    (:181-212) and "In-place Galerkin Resetup" (:243-270)."""
    _galerkin_check(problems.poisson1d(10), 2.0)
    _galerkin_check(problems.poisson1d(20), 3.0)


def test_galerkin_multi_entry_p():
    """testset with PMIS + standard interpolation (:1219-1252): several
    entries per P row; the explicit PᵀAP agrees to 1e-10."""
    A = problems.poisson2d(10)
    cfg = draugr.AMGConfig(coarsening=draugr.PMISCoarsening(0.25, draugr.StandardInterpolation()),
                           max_coarse_size=4)
    h = draugr.amg_setup(A, cfg, on_device=False)
    P = explicit_P(h, 0)
    n, nc = P.shape
    _, arp, aci, av = parts(A)
    c_rp, c_ci, c_v, *_ = oracle.coarse_sparsity(n, nc, arp, aci, av, P.indptr.astype(np.int32),
                                                 P.indices.astype(np.int32), P.data)
    Ac = sp.csr_matrix((c_v, c_ci, c_rp), shape=(nc, nc)).toarray()
    assert np.allclose(Ac, (P.T @ A @ P).toarray(), atol=1e-10)


def test_jacobi_invdiag_and_smoothing():
    """testset "Jacobi Smoother" (:272-284): invdiag ≡ 0.5 on the 1D
    Laplacian; 10 steps reduce the residual."""
    A = problems.poisson1d(10)
    n, rp, ci, v = parts(A)
    inv = oracle.invdiag(n, rp, ci, v)
    assert np.allclose(inv, 0.5)
    b = np.ones(n)
    x = oracle.jacobi(n, rp, ci, v, inv, 2.0 / 3.0, np.zeros(n), b, 10)
    assert np.linalg.norm(b - A @ x) < np.linalg.norm(b)


def test_safe_inverse_diagonal():
    """testset "Safe Diagonal - Zero diagonal row" (test/runtests.jl:1784-1796):
    a row whose diagonal is 1e-20 gets a finite (zero) inverse.  (The
    library's diagonals equal the oracle's bit for bit in
    test_cpu_library.py::test_structure_matches_oracle.)"""
    A = sp.csr_matrix(np.array([[2.0, -1.0, 0.0], [-1.0, 1e-20, -1.0], [0.0, -1.0, 2.0]]))
    A.sort_indices()
    n, rp, ci, v = parts(A)
    inv = oracle.invdiag(n, rp, ci, v)
    assert np.all(np.isfinite(inv)) and inv[1] == 0.0


def test_l1_invdiag():
    """testset "L1 Colored GS Smoother - Build" (:607-617): interior row l1
    norm 4 -> invdiag 0.25."""
    A = problems.poisson1d(10)
    n, rp, ci, v = parts(A)
    inv = oracle.invdiag(n, rp, ci, v, l1=True)
    assert np.isclose(inv[4], 0.25)


def test_spai0_diagonal_smoothing_and_solve():
    """testsets "SPAI0 Smoother - Build / Smoothing" and "AMG Solve - SPAI0"
    (test/runtests.jl:754-788): interior row [-1 2 -1] gives m = 2/6; 10
    sweeps reduce the residual; amg_solve! with SPAI(0) on the 10 x 10
    Poisson matrix reaches 1e-8 in fewer than 200 cycles."""
    A = problems.poisson1d(10)
    n, rp, ci, v = parts(A)
    m = oracle.spai0(n, rp, ci, v)
    assert len(m) == 10 and np.isclose(m[4], 2.0 / 6.0)
    b = np.ones(n)
    x = oracle.spai0_smooth(n, rp, ci, v, m, np.zeros(n), b, 10)
    assert np.linalg.norm(b - A @ x) < np.linalg.norm(b)
    A = problems.poisson2d(10)
    b = np.random.default_rng(2).uniform(0, 1, 100)
    cfg = draugr.AMGConfig(smoother=draugr.SPAI0SmootherType())
    h = draugr.amg_setup(A, cfg, on_device=False)
    O = oracle.OracleHierarchy(h)
    x, it, rel = O.solve(np.zeros(100), b, tol=1e-8, maxiter=200)
    assert it < 200 and rel < 1e-8
    assert np.linalg.norm(b - A @ x) / np.linalg.norm(b) < 1e-8


def test_chebyshev_build_smoothing_solve_and_resetup():
    """testsets "Chebyshev Smoother - Build / Smoothing / AMG Solve" and
    "Chebyshev - Resetup" (test/runtests.jl:1913-1966): 0 < lambda_min <
    lambda_max and degree 3; 5 applications reduce the residual; amg_solve!
    with V(2,2) Chebyshev reaches 1e-8 in fewer than 200 cycles, also after
    a resetup with the values doubled."""
    A = problems.poisson1d(10)
    n, rp, ci, v = parts(A)
    inv = oracle.invdiag(n, rp, ci, v)
    v0 = np.random.default_rng(3).standard_normal(n)
    rho = oracle.spectral_radius(n, rp, ci, v, inv, v0 / np.linalg.norm(v0))
    lmax, lmin = 1.1 * rho, 1.1 * rho / 30.0
    assert lmax > lmin > 0
    coef = oracle.cheb_coef(rho, 3)
    assert len(coef) == 2 * 3 and np.isclose(coef[0], 2.0 / (lmax + lmin))
    b = np.ones(n)
    x = oracle.chebyshev(n, rp, ci, v, inv, coef, np.zeros(n), b, 5)
    assert np.linalg.norm(b - A @ x) < np.linalg.norm(b)
    for m in (10, 8):
        A = problems.poisson2d(m)
        N = m * m
        b = np.random.default_rng(m).uniform(0, 1, N)
        cfg = draugr.AMGConfig(smoother=draugr.ChebyshevSmootherType(), pre_smoothing_steps=2,
                               post_smoothing_steps=2, max_coarse_size=10)
        h = draugr.amg_setup(A, cfg, on_device=False)
        O = oracle.OracleHierarchy(h, with_rmaps=True)
        x, it, rel = O.solve(np.zeros(N), b, 2, 2, False, 1e-8, 200)
        assert it < 200 and np.linalg.norm(b - A @ x) / np.linalg.norm(b) < 1e-8
        if m == 8:
            O.resetup(2.0 * A.data)
            x, it, rel = O.solve(np.zeros(N), b, 2, 2, False, 1e-8, 200)
            assert it < 200 and np.linalg.norm(b - 2.0 * (A @ x)) / np.linalg.norm(b) < 1e-8


def _check_rs_splitting(A, cf, nc):
    """Every point C or F, nc = number of C-points, 0 < nc < n, and every
    F-point with a strong C-neighbour (the checks of the reference's RS
    testsets)."""
    n, rp, ci, v = parts(A)
    assert len(cf) == n and np.all(np.abs(cf) == 1)
    assert 0 < nc < n and int(np.sum(cf == 1)) == nc
    st = oracle.strength_abs(n, rp, ci, v, 0.25)
    for i in range(n):
        if cf[i] == -1:
            row = range(rp[i], rp[i + 1])
            assert any(ci[k] != i and st[k] and cf[ci[k]] == 1 for k in row), i


def test_rs_coarsening():
    """testsets "RS Coarsening - Basic / 2D / larger system / Solve /
    Standard Interpolation / Good coarsening ratios" (test/runtests.jl:
    1254-1334, :2567-2590): valid splittings of the 1D (20) and 2D (10 x 10,
    30 x 30) Laplacians; amg_solve! with V(2,2) reaches 1e-8 in fewer than
    200 cycles with direct and standard interpolation; every level of the
    30 x 30 hierarchy is smaller than the one above."""
    for A in (problems.poisson1d(20), problems.poisson2d(10), problems.poisson2d(30)):
        cfg = draugr.AMGConfig(coarsening=draugr.RSCoarsening(0.25), max_coarse_size=2)
        h = draugr.amg_setup(A, cfg, on_device=False)
        _check_rs_splitting(A, h.export(0, "cf"), int(h.level_info(0)[2]))
    A = problems.poisson2d(10)
    b = np.random.default_rng(7).uniform(0, 1, 100)
    for interp in (draugr.DirectInterpolation(), draugr.StandardInterpolation()):
        cfg = draugr.AMGConfig(coarsening=draugr.RSCoarsening(0.25, interp), pre_smoothing_steps=2,
                               post_smoothing_steps=2)
        h = draugr.amg_setup(A, cfg, on_device=False)
        assert h.nlevels >= 1
        O = oracle.OracleHierarchy(h)
        x, it, rel = O.solve(np.zeros(100), b, 2, 2, False, 1e-8, 200)
        assert it < 200 and np.linalg.norm(b - A @ x) / np.linalg.norm(b) < 1e-8
    h = draugr.amg_setup(problems.poisson2d(30), draugr.AMGConfig(coarsening=draugr.RSCoarsening(0.25)),
                         on_device=False)
    sizes = [int(h.level_info(l)[0]) for l in range(h.nlevels)] + [int(h.level_info(-1)[0])]
    assert all(b < a for a, b in zip(sizes, sizes[1:]))


def test_spai1_build_smoothing_and_solve():
    """testsets "SPAI1 Smoother - Build / Smoothing" and "AMG Solve - SPAI1"
    (test/runtests.jl:793-823): M has nnz(A) entries; 10 steps reduce the
    residual; amg_solve! with V(2,2) SPAI(1) reaches 1e-8 in fewer than 300
    cycles on the 10 x 10 Poisson matrix."""
    A = problems.poisson1d(5)
    n, rp, ci, v = parts(A)
    assert len(oracle.spai1(n, rp, ci, v)) == A.nnz
    A = problems.poisson1d(10)
    n, rp, ci, v = parts(A)
    M = oracle.spai1(n, rp, ci, v)
    b = np.ones(n)
    x = oracle.spai1_smooth(n, rp, ci, v, M, np.zeros(n), b, 10)
    assert np.linalg.norm(b - A @ x) < np.linalg.norm(b)
    A = problems.poisson2d(10)
    b = np.random.default_rng(6).uniform(0, 1, 100)
    cfg = draugr.AMGConfig(smoother=draugr.SPAI1SmootherType(), pre_smoothing_steps=2, post_smoothing_steps=2)
    h = draugr.amg_setup(A, cfg, on_device=False)
    O = oracle.OracleHierarchy(h)
    x, it, rel = O.solve(np.zeros(100), b, 2, 2, False, 1e-8, 300)
    assert it < 300 and np.linalg.norm(b - A @ x) / np.linalg.norm(b) < 1e-8


@pytest.mark.parametrize("l1", [False, True])
def test_serial_gs_build_smoothing_and_solve(l1):
    """testsets "Serial GS Smoother" and "L1 Serial GS Smoother" (test/
    runtests.jl:648-740): invdiag 0.5 (l1: 1/4 inside, 1/3 at the ends) on
    the 1D Laplacian; 10 sweeps reduce the residual; amg_solve! reaches 1e-8
    in fewer than 200 cycles on the 10 x 10 Poisson matrix."""
    A = problems.poisson1d(10)
    n, rp, ci, v = parts(A)
    inv = oracle.invdiag(n, rp, ci, v, l1=True) if l1 else oracle.serial_gs_invdiag(n, rp, ci, v)
    if l1:
        assert np.isclose(inv[4], 0.25) and np.isclose(inv[0], 1.0 / 3.0)
    else:
        assert np.allclose(inv, 0.5)
    b = np.ones(n)
    x = oracle.serial_gs(n, rp, ci, v, inv, np.zeros(n), b, 10)
    assert np.linalg.norm(b - A @ x) < np.linalg.norm(b)
    A = problems.poisson2d(10)
    b = np.random.default_rng(4).uniform(0, 1, 100)
    cfg = draugr.AMGConfig(smoother=draugr.L1SerialGaussSeidelType() if l1 else draugr.SerialGaussSeidelType())
    h = draugr.amg_setup(A, cfg, on_device=False)
    O = oracle.OracleHierarchy(h)
    x, it, rel = O.solve(np.zeros(100), b, tol=1e-8, maxiter=200)
    assert it < 200 and np.linalg.norm(b - A @ x) / np.linalg.norm(b) < 1e-8


def _anisotropic(nx, ny, kx=1e4, ky=1e-2):
    """anisotropic_csr of the reference's tests (test/runtests.jl:1681-1694)."""
    rows, cols, vals = [], [], []
    for j in range(ny):
        for i in range(nx):
            idx = j * nx + i
            nb = [(idx, 2 * kx + 2 * ky)]
            if i > 0:
                nb.append((idx - 1, -kx))
            if i < nx - 1:
                nb.append((idx + 1, -kx))
            if j > 0:
                nb.append((idx - nx, -ky))
            if j < ny - 1:
                nb.append((idx + nx, -ky))
            for c, v in nb:
                rows.append(idx); cols.append(c); vals.append(v)
    A = sp.csr_matrix((vals, (rows, cols)), shape=(nx * ny, nx * ny))
    A.sort_indices()
    return A


@pytest.mark.parametrize("smoother", ["ILU0SmootherType", "SerialILU0SmootherType"])
def test_ilu0_build_smoothing_solve_and_resetup(smoother):
    """testsets "ILU(0) Smoother - Build / Smoothing / AMG Solve / Resetup /
    Anisotropic" and their serial counterparts (test/runtests.jl:1972-2127):
    factors of nnz entries and at least 2 forward levels on the 1D
    Laplacian; 3 steps reduce the residual; amg_solve! reaches 1e-8 in fewer
    than 200 cycles on the 10 x 10 Poisson matrix, after a resetup with
    doubled values (8 x 8), and on the 8 x 8 anisotropic matrix."""
    A = problems.poisson1d(10)
    n, rp, ci, v = parts(A)
    diag = oracle.ilu0_diag(n, rp, ci)
    Lf, Uf = oracle.ilu0_factor(n, rp, ci, v, diag)
    assert len(Lf) == A.nnz and len(Uf) == A.nnz and len(diag) == 10
    cfg = draugr.AMGConfig(smoother=getattr(draugr, smoother)())
    h = draugr.amg_setup(problems.poisson2d(10), cfg, on_device=False)
    assert len(h.export(0, "ilu_fwd_offsets")) - 1 >= 2
    b = np.ones(n)
    x = oracle.ilu0_smooth(n, rp, ci, v, diag, Lf, Uf, np.zeros(n), b, 3)
    assert np.linalg.norm(b - A @ x) < np.linalg.norm(b)
    for A, m in ((problems.poisson2d(10), 10), (problems.poisson2d(8), 8), (_anisotropic(8, 8), 8)):
        N = A.shape[0]
        b = np.random.default_rng(m).uniform(0, 1, N)
        h = draugr.amg_setup(A, cfg, on_device=False)
        O = oracle.OracleHierarchy(h, with_rmaps=True)
        x, it, rel = O.solve(np.zeros(N), b, 1, 1, False, 1e-8, 200)
        assert it < 200 and np.linalg.norm(b - A @ x) / np.linalg.norm(b) < 1e-8
        if m == 8 and A.nnz == problems.poisson2d(8).nnz:
            O.resetup(2.0 * A.data)
            x, it, rel = O.solve(np.zeros(N), b, 1, 1, False, 1e-8, 200)
            assert it < 200 and np.linalg.norm(b - 2.0 * (A @ x)) / np.linalg.norm(b) < 1e-8


def test_coloring():
    """testsets "Graph Coloring" (:549-566) and "Colored GS Smoother" (:568-588)."""
    A = problems.poisson1d(10)
    n, rp, ci, v = parts(A)
    colors, ncol, off, order = oracle.greedy_coloring(n, rp, ci)
    assert len(colors) == 10 and np.all(colors > 0) and ncol >= 2
    for i in range(n):
        for k in range(rp[i], rp[i + 1]):
            if ci[k] != i:
                assert colors[i] != colors[ci[k]]
    inv = oracle.invdiag(n, rp, ci, v)
    b = np.ones(n)
    x = oracle.gs(n, rp, ci, v, inv, ncol, off, order, np.zeros(n), b, 10)
    assert np.linalg.norm(b - A @ x) < np.linalg.norm(b)


def test_solve_thresholds_and_w_cycle():
    """amg_solve! reaches 1e-8 in < 200 cycles (:332-415, :589-605) and the
    W-cycle needs no more cycles than the V-cycle (:1828-1855)."""
    A = problems.poisson2d(10)
    b = np.random.default_rng(0).uniform(0, 1, 100)
    for coars, smo in ((draugr.AggregationCoarsening(), draugr.L1ColoredGaussSeidelType()),
                       (draugr.PMISCoarsening(), draugr.L1ColoredGaussSeidelType()),
                       (draugr.AggressiveCoarsening(), draugr.L1ColoredGaussSeidelType()),
                       (draugr.HMISCoarsening(0.5, draugr.ExtendedIInterpolation()),
                        draugr.ColoredGaussSeidelType())):
        cfg = draugr.AMGConfig(coarsening=coars, smoother=smo, max_coarse_size=10)
        h = draugr.amg_setup(A, cfg, on_device=False)
        O = oracle.OracleHierarchy(h)
        x, it, rel = O.solve(np.zeros(100), b, tol=1e-8, maxiter=200)
        assert it < 200 and rel < 1e-8
        assert np.linalg.norm(b - A @ x) / np.linalg.norm(b) < 1e-8
    A = problems.poisson2d(32)
    b = np.random.default_rng(1).uniform(0, 1, A.shape[0])
    h = draugr.amg_setup(A, draugr.AMGConfig(coarsening=draugr.AggregationCoarsening()),
                         on_device=False)
    O = oracle.OracleHierarchy(h)
    _, itv, _ = O.solve(np.zeros(A.shape[0]), b, w=False, tol=1e-8, maxiter=300)
    _, itw, _ = O.solve(np.zeros(A.shape[0]), b, w=True, tol=1e-8, maxiter=300)
    assert itw <= itv


def test_resetup_keeps_pattern_and_solves():
    """testsets "AMG Resetup" (:392-415) and "Resetup Preserves Pattern"
    (:417-434), on the oracle's partial resetup."""
    A = problems.poisson2d(10)
    cfg = draugr.AMGConfig(coarsening=draugr.AggregationCoarsening(), max_coarse_size=10)
    h = draugr.amg_setup(A, cfg, on_device=False)
    O = oracle.OracleHierarchy(h, with_rmaps=True)
    pats = [(O.levels_np[l]["A_rp"].copy(), O.levels_np[l]["A_ci"].copy()) for l in range(O.nlevels)]
    b = np.random.default_rng(2).uniform(0, 1, 100)
    x1, _, r1 = O.solve(np.zeros(100), b, tol=1e-8, maxiter=200)
    assert r1 < 1e-8
    A2 = A * 2.0
    O.resetup(A2.data)
    for l, (rp, ci) in enumerate(pats):
        assert np.array_equal(O.levels_np[l]["A_rp"], rp) and np.array_equal(O.levels_np[l]["A_ci"], ci)
    x2, _, r2 = O.solve(np.zeros(100), b, tol=1e-8, maxiter=200)
    assert np.linalg.norm(b - A2 @ x2) / np.linalg.norm(b) < 1e-8
    assert not np.allclose(x1, x2, atol=1e-6)


def test_lu_matches_numpy():
    """The coarsest LU (getrf/getrs order) solves like a reference LU."""
    rng = np.random.default_rng(3)
    M = rng.standard_normal((17, 17)) + 17 * np.eye(17)
    lu, piv, info = oracle.lu_factor(M)
    assert info == 0
    b = rng.standard_normal(17)
    y = b.copy()
    a = np.ascontiguousarray(lu.T).ravel()
    oracle.load().orc_lu_solve(17, oracle.ptr(a), oracle.ptr(piv), oracle.ptr(y))
    assert np.allclose(y, np.linalg.solve(M, b), atol=1e-12)
    S = M.copy()
    S[:, 3] = 0.0
    assert oracle.lu_factor(S)[2] == 4  # SingularException(4)


def test_l1_jacobi_lu_refactorization_and_cpu_coarse_solve():
    """testsets "l1-Jacobi Smoother - Build / Smoothing / AMG Solve /
    Resetup" (:1857-1908), "In-place LU Refactorization" (:1103-1129), "AMG
    Solve - coarse_solve_on_cpu" (:374-390), "AMG Setup - Aggregation" and
    "AMG Cycle Convergence - Aggregation" (:286-330): the l1 inverse
    diagonal of an interior row of the 1D Laplacian is 1/4 and ten sweeps
    reduce the residual; l1-Jacobi and coarse_solve_on_cpu hierarchies solve
    10 x 10 to 1e-8 in fewer than 200 cycles; after a resetup with doubled
    values (which refactorises the coarsest LU) the solve again meets 1e-8;
    five V(2,2) cycles of an aggregation hierarchy on 20 x 20 reduce the
    residual of b = 1."""
    n, rp, ci, v = parts(problems.poisson1d(10))
    invd = oracle.invdiag(n, rp, ci, v, l1=True)
    assert len(invd) == 10 and invd[4] == pytest.approx(0.25)
    b = np.ones(10)
    x = oracle.jacobi(n, rp, ci, v, invd, 2.0 / 3.0, np.zeros(10), b, 10)
    A1 = problems.poisson1d(10)
    assert np.linalg.norm(b - A1 @ x) < np.linalg.norm(b)
    A = problems.poisson2d(10)
    b = np.random.default_rng(31).uniform(0, 1, 100)
    for cfg in (draugr.AMGConfig(smoother=draugr.L1JacobiSmootherType()),
                draugr.AMGConfig(coarse_solve_on_cpu=True)):
        h = draugr.amg_setup(A, cfg, on_device=False)
        x, it, _ = oracle.OracleHierarchy(h).solve(np.zeros(100), b, tol=1e-8, maxiter=200)
        assert it < 200 and np.linalg.norm(b - A @ x) / np.linalg.norm(b) < 1e-8
    A8 = problems.poisson2d(8)
    b8 = np.random.default_rng(32).uniform(0, 1, 64)
    for cfg in (draugr.AMGConfig(smoother=draugr.L1JacobiSmootherType()),
                draugr.AMGConfig(coarsening=draugr.AggregationCoarsening())):
        h = draugr.amg_setup(A8, cfg, on_device=False)
        O = oracle.OracleHierarchy(h, with_rmaps=True)
        x1, _, _ = O.solve(np.zeros(64), b8, tol=1e-8, maxiter=200)
        assert np.linalg.norm(b8 - A8 @ x1) / np.linalg.norm(b8) < 1e-8
        O.resetup(A8.data * 2.0)
        x2, _, _ = O.solve(np.zeros(64), b8, tol=1e-8, maxiter=200)
        assert np.linalg.norm(b8 - 2.0 * (A8 @ x2)) / np.linalg.norm(b8) < 1e-8
    h = draugr.amg_setup(A, draugr.AMGConfig(coarsening=draugr.AggregationCoarsening()), on_device=False)
    assert h.nlevels > 0
    assert all(h.level_info(l)[2] < h.level_info(l)[0] for l in range(h.nlevels))
    A20 = problems.poisson2d(20)
    cfg = draugr.AMGConfig(coarsening=draugr.AggregationCoarsening(), pre_smoothing_steps=2,
                           post_smoothing_steps=2)
    h = draugr.amg_setup(A20, cfg, on_device=False)
    assert h.nlevels > 0
    O = oracle.OracleHierarchy(h)
    b = np.ones(400)
    x = np.zeros(400)
    for _ in range(5):
        x = O.cycle(x, b, 2, 2)
    assert np.linalg.norm(b - A20 @ x) < np.linalg.norm(b)


@pytest.mark.parametrize("smoother", ["jacobi", "spai0", "l1_jacobi", "colored_gs", "l1_colored_gs", "ilu0",
                                      "chebyshev", "spai1", "serial_gs", "serial_ilu0", "l1_serial_gs"])
def test_every_smoother_type_smooths(smoother):
    """testsets "Standalone Smoother API - build_smoother / smooth! /
    update_smoother! / all types smooth correctly" (:2490-2562): on the 1D
    Laplacian (10), the smoother the library builds for each type (Jacobi's
    inverse diagonal is 0.5 throughout) takes ten sweeps of the oracle's
    smoother from zero to a smaller residual than b = 1."""
    A = problems.poisson1d(10)
    cls = {k.name: k for k in (draugr.JacobiSmootherType, draugr.SPAI0SmootherType, draugr.L1JacobiSmootherType,
                               draugr.ColoredGaussSeidelType, draugr.L1ColoredGaussSeidelType,
                               draugr.ILU0SmootherType, draugr.ChebyshevSmootherType, draugr.SPAI1SmootherType,
                               draugr.SerialGaussSeidelType, draugr.SerialILU0SmootherType,
                               draugr.L1SerialGaussSeidelType)}[smoother]
    h = draugr.amg_setup(A, draugr.AMGConfig(coarsening=draugr.AggregationCoarsening(), smoother=cls(),
                                             max_coarse_size=2), on_device=False)
    n, rp, ci, v = parts(A)
    b = np.ones(n)
    x0 = np.zeros(n)
    invd = h.export(0, "invdiag")
    omega = float(h.export(0, "omega")[0])
    if smoother in ("jacobi", "l1_jacobi"):
        if smoother == "jacobi":
            assert np.all(invd == 0.5)
        x = oracle.jacobi(n, rp, ci, v, invd, omega, x0, b, 10)
    elif smoother == "spai0":
        x = oracle.spai0_smooth(n, rp, ci, v, oracle.spai0(n, rp, ci, v), x0, b, 10)
    elif smoother in ("colored_gs", "l1_colored_gs"):
        off, order = h.export(0, "color_offsets"), h.export(0, "color_order")
        x = oracle.gs(n, rp, ci, v, invd, len(off) - 1, off, order, x0, b, 10)
    elif smoother in ("ilu0", "serial_ilu0"):
        x = oracle.ilu0_smooth(n, rp, ci, v, h.export(0, "ilu_diag"), h.export(0, "ilu_L"), h.export(0, "ilu_U"),
                               x0, b, 10)
    elif smoother == "chebyshev":
        x = oracle.chebyshev(n, rp, ci, v, invd, h.export(0, "cheb_coef"), x0, b, 10)
    elif smoother == "spai1":
        x = oracle.spai1_smooth(n, rp, ci, v, h.export(0, "spai1_M"), x0, b, 10)
    else:
        x = oracle.serial_gs(n, rp, ci, v, invd, x0, b, 10)
    assert np.linalg.norm(b - A @ x) < np.linalg.norm(b)
