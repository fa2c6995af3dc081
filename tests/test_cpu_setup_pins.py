"""The reference's setup testsets (test/runtests.jl) for interpolation,
initial coarsening, aggregation variants, strength, truncation options and
hypre_default_config, restated against the library's CPU setup.  Each test
names the testset it restates.  Solves run the oracle's amg_solve! (V or W
cycles, test/runtests.jl's tolerances) on the host-only hierarchy.  Where
the reference draws a random matrix from Julia's RNG, a seeded NumPy matrix
of the same construction stands in for it."""

import numpy as np
import pytest
import scipy.sparse as sp

import draugr
import oracle
from draugr import problems


def solve(A, cfg, b, tol=1e-8, maxiter=200):
    """amg_setup + amg_solve! from x = 0; returns (x, cycles, hierarchy)."""
    h = draugr.amg_setup(A, cfg, on_device=False)
    O = oracle.OracleHierarchy(h)
    x, it, _ = O.solve(np.zeros(A.shape[0]), b, cfg.pre_smoothing_steps, cfg.post_smoothing_steps,
                       cfg.cycle_type == "W", tol, maxiter)
    return x, it, h


def rel_res(A, x, b):
    return np.linalg.norm(b - A @ x) / np.linalg.norm(b)


def rhs(n, seed):
    return np.random.default_rng(seed).uniform(0, 1, n)


def reservoir_like(n):
    """reservoir_like_csr (test/runtests.jl:1664-1678): diagonal 10,
    off-diagonals -1 / -2 with positive entries on every third and fifth
    row."""
    rows, cols, vals = [], [], []
    for i in range(1, n + 1):
        rows.append(i); cols.append(i); vals.append(10.0)
        if i > 1:
            rows.append(i); cols.append(i - 1); vals.append(0.5 if i % 3 == 0 else -1.0)
        if i < n:
            rows.append(i); cols.append(i + 1); vals.append(0.3 if (i + 1) % 5 == 0 else -2.0)
    return sp.csr_matrix((vals, (np.array(rows) - 1, np.array(cols) - 1)), shape=(n, n))


def anisotropic(nx, ny, kx=1e4, ky=1e-2):
    """anisotropic_csr (test/runtests.jl:1681-1694)."""
    rows, cols, vals = [], [], []
    for j in range(ny):
        for i in range(nx):
            idx = j * nx + i
            rows.append(idx); cols.append(idx); vals.append(2 * kx + 2 * ky)
            for cond, off, v in ((i > 0, -1, -kx), (i < nx - 1, 1, -kx), (j > 0, -nx, -ky),
                                 (j < ny - 1, nx, -ky)):
                if cond:
                    rows.append(idx); cols.append(idx + off); vals.append(v)
    return sp.csr_matrix((vals, (rows, cols)), shape=(nx * ny, nx * ny))


V22 = dict(pre_smoothing_steps=2, post_smoothing_steps=2)


@pytest.mark.parametrize("coarsening", [
    draugr.PMISCoarsening(0.25, draugr.DirectInterpolation()),
    draugr.PMISCoarsening(0.25, draugr.StandardInterpolation()),
    draugr.PMISCoarsening(0.25, draugr.ExtendedIInterpolation()),
    draugr.HMISCoarsening(0.25, draugr.DirectInterpolation()),
    draugr.HMISCoarsening(0.25, draugr.StandardInterpolation()),
    draugr.HMISCoarsening(0.25, draugr.ExtendedIInterpolation()),
], ids=["pmis-direct", "pmis-standard", "pmis-exti", "hmis-direct", "hmis-standard", "hmis-exti"])
def test_interpolation_types_solve(coarsening):
    """testsets "PMIS - Direct / Standard / Extended+i Interpolation", "HMIS -
    Standard / Extended+i Interpolation" and "AMG Solve - HMIS Direct"
    (test/runtests.jl:996-1100): on 10 x 10, V(2,2), at least one level,
    1e-8 in fewer than 200 cycles; and "ExtendedI Convergence" (:1415-1447)
    on 15 x 15 for the extended+i pair."""
    cfg = draugr.AMGConfig(coarsening=coarsening, **V22)
    A = problems.poisson2d(10)
    b = rhs(100, 1)
    x, it, h = solve(A, cfg, b)
    assert h.nlevels > 0 and it < 200 and rel_res(A, x, b) < 1e-8
    if isinstance(coarsening.interpolation, draugr.ExtendedIInterpolation):
        A = problems.poisson2d(15)
        b = rhs(225, 2)
        x, it, _ = solve(A, cfg, b)
        assert it < 200 and rel_res(A, x, b) < 1e-8


def test_initial_coarsening_levels_and_solve():
    """testsets "Initial Coarsening - Default / Custom / Solve"
    (test/runtests.jl:1133-1180): the first initial_coarsening_levels levels
    use the initial coarsening (a C/F splitting here, read back as the
    level's "cf"), later levels the main one (aggregation, no splitting);
    PMIS for one level, then aggregation, solves 10 x 10 with V(2,2) to 1e-8
    in fewer than 200 cycles."""
    A = problems.poisson2d(30)
    cfg = draugr.AMGConfig(coarsening=draugr.AggregationCoarsening(),
                           initial_coarsening=draugr.PMISCoarsening(0.25, draugr.DirectInterpolation()),
                           initial_coarsening_levels=2, max_coarse_size=10)
    h = draugr.amg_setup(A, cfg, on_device=False)
    assert h.nlevels >= 3
    for l in range(h.nlevels):
        n_l = int(h.level_info(l)[0])
        assert len(h.export(l, "cf")) == (n_l if l < 2 else 0), l
    plain = draugr.amg_setup(A, draugr.AMGConfig(coarsening=draugr.AggregationCoarsening(),
                                                 max_coarse_size=10), on_device=False)
    assert len(plain.export(0, "cf")) == 0
    cfg = draugr.AMGConfig(coarsening=draugr.AggregationCoarsening(),
                           initial_coarsening=draugr.PMISCoarsening(0.25, draugr.DirectInterpolation()),
                           initial_coarsening_levels=1, **V22)
    A = problems.poisson2d(10)
    b = rhs(100, 3)
    x, it, h = solve(A, cfg, b)
    assert h.nlevels > 0 and it < 200 and rel_res(A, x, b) < 1e-8


@pytest.mark.parametrize("interp", [draugr.DirectInterpolation(), draugr.StandardInterpolation(),
                                    draugr.ExtendedIInterpolation()], ids=["direct", "standard", "exti"])
def test_cf_prolongation_rows(interp):
    """testsets "CF Prolongation - Coarse Points Identity / Fine Points Have
    Entries" (test/runtests.jl:1183-1218): PMIS on the 1D Laplacian (20); P
    is 20 x nc; a C-point's row is the single entry 1 in its own coarse
    column; every F-point's row has at least one entry."""
    A = problems.poisson1d(20)
    cfg = draugr.AMGConfig(coarsening=draugr.PMISCoarsening(0.25, interp), max_coarse_size=2)
    h = draugr.amg_setup(A, cfg, on_device=False)
    info = h.level_info(0)
    nc = int(info[2])
    cf = h.export(0, "cf")
    rp, ci, v = h.export(0, "P_rowptr"), h.export(0, "P_colval"), h.export(0, "P_nzval")
    assert int(info[0]) == 20 and len(rp) == 21 and 0 < nc < 20
    cmap = np.cumsum(cf == 1) - 1
    for i in range(20):
        if cf[i] == 1:
            assert rp[i + 1] - rp[i] == 1 and ci[rp[i]] == cmap[i] and v[rp[i]] == pytest.approx(1.0)
        else:
            assert rp[i + 1] - rp[i] >= 1
    assert ci.max() < nc


def test_aggregation_filtering_and_max_row_sum_solve():
    """testsets "Aggregation Filtering - Config / Solve" and "Max Row Sum -
    Config / Solve" (test/runtests.jl:1449-1469, :1492-1550): defaults
    (filtering off, max_row_sum 1.0), and 10 x 10 solves to 1e-8 in fewer
    than 200 cycles with filtering (0.1) and with max_row_sum 0.9."""
    assert draugr.AggregationCoarsening().filtering is False
    alg = draugr.AggregationCoarsening(0.25, True, 0.2)
    assert alg.filtering and alg.filter_tol == pytest.approx(0.2)
    assert draugr.AMGConfig().max_row_sum == pytest.approx(1.0)
    A = problems.poisson2d(10)
    b = rhs(100, 4)
    for cfg in (draugr.AMGConfig(coarsening=draugr.AggregationCoarsening(0.25, True, 0.1)),
                draugr.AMGConfig(max_row_sum=0.9)):
        x, it, _ = solve(A, cfg, b)
        assert it < 200 and rel_res(A, x, b) < 1e-8


def test_smoothed_aggregation():
    """testsets "Smoothed Aggregation - Config / Setup / Solve / Better than
    Plain Aggregation / With Filtering / Resetup" and "Smoothed Prolongation
    Construction" (test/runtests.jl:1552-1660)."""
    alg = draugr.SmoothedAggregationCoarsening()
    assert alg.theta == pytest.approx(0.25) and alg.omega == pytest.approx(2 / 3) and not alg.filtering
    A = problems.poisson2d(10)
    h = draugr.amg_setup(A, draugr.AMGConfig(coarsening=alg), on_device=False)
    assert h.nlevels >= 1 and int(h.level_info(0)[1]) > 0
    b = rhs(100, 5)
    for cfg in (draugr.AMGConfig(coarsening=alg, **V22),
                draugr.AMGConfig(coarsening=draugr.SmoothedAggregationCoarsening(0.25, 2 / 3, True, 0.1),
                                 **V22)):
        x, it, _ = solve(A, cfg, b)
        assert it < 200 and rel_res(A, x, b) < 1e-8
    # no more cycles than plain aggregation on 15 x 15
    A15 = problems.poisson2d(15)
    b15 = rhs(225, 6)
    _, it_plain, _ = solve(A15, draugr.AMGConfig(coarsening=draugr.AggregationCoarsening(), **V22), b15)
    _, it_sa, _ = solve(A15, draugr.AMGConfig(coarsening=alg, **V22), b15)
    assert it_sa <= it_plain
    # resetup with doubled values (P frozen) still solves to 1e-8
    cfg = draugr.AMGConfig(coarsening=alg, **V22)
    h = draugr.amg_setup(A, cfg, on_device=False)
    O = oracle.OracleHierarchy(h, with_rmaps=True)
    _, it1, _ = O.solve(np.zeros(100), b, 2, 2, False, 1e-8, 200)
    assert it1 < 200
    A2 = A.copy()
    A2.data = A2.data * 2.0
    O.resetup(A2.data)
    x2, _, _ = O.solve(np.zeros(100), b, 2, 2, False, 1e-8, 200)
    assert rel_res(A2, x2, b) < 1e-8
    # the smoothed P of the 1D Laplacian (10) keeps the tentative P's size
    # and has at least its nonzeros
    A1 = problems.poisson1d(10)
    ht = draugr.amg_setup(A1, draugr.AMGConfig(coarsening=draugr.AggregationCoarsening(),
                                               max_coarse_size=2), on_device=False)
    hs = draugr.amg_setup(A1, draugr.AMGConfig(coarsening=alg, max_coarse_size=2), on_device=False)
    it_, is_ = ht.level_info(0), hs.level_info(0)
    assert int(is_[0]) == 10 and int(is_[2]) == int(it_[2])
    assert int(is_[3]) >= int(it_[3])


def test_signed_strength_and_positive_off_diagonals():
    """testsets "SignedStrength - Solve" and "Positive Off-Diags - All
    smoothers converge" (test/runtests.jl:1724-1765): the reservoir-like
    matrix (50) solves to 1e-8 with signed strength, and with each of
    Jacobi, l1-Jacobi, colored GS, l1 colored GS, l1 serial GS, SPAI(0) and
    ILU(0)."""
    A = reservoir_like(50)
    b = rhs(50, 7)
    x, it, _ = solve(A, draugr.AMGConfig(strength_type=draugr.SignedStrength()), b)
    assert it < 200 and rel_res(A, x, b) < 1e-8
    for smoother in (draugr.JacobiSmootherType(), draugr.L1JacobiSmootherType(),
                     draugr.ColoredGaussSeidelType(), draugr.L1ColoredGaussSeidelType(),
                     draugr.L1SerialGaussSeidelType(), draugr.SPAI0SmootherType(),
                     draugr.ILU0SmootherType()):
        x, _, _ = solve(A, draugr.AMGConfig(smoother=smoother), b)
        assert rel_res(A, x, b) < 1e-8, smoother


def test_anisotropic_convergence():
    """testset "Anisotropic Matrix - Convergence" (test/runtests.jl:
    1767-1782): kx = 1e4, ky = 1e-2 on 8 x 8 solves to 1e-8 within 300
    cycles with the default smoother and l1-Jacobi (V(2,2)) and with
    ILU(0)."""
    A = anisotropic(8, 8)
    b = rhs(64, 8)
    for cfg in (draugr.AMGConfig(**V22), draugr.AMGConfig(smoother=draugr.L1JacobiSmootherType(), **V22),
                draugr.AMGConfig(smoother=draugr.ILU0SmootherType())):
        x, _, _ = solve(A, cfg, b, maxiter=300)
        assert rel_res(A, x, b) < 1e-8


def _random_matrix(n, seed, diag, nneigh, offv):
    rng = np.random.default_rng(seed)
    rows, cols, vals = [], [], []
    for i in range(n):
        rows.append(i); cols.append(i); vals.append(diag(rng))
        for _ in range(nneigh(rng)):
            j = int(rng.integers(0, n))
            if j == i:
                continue
            rows.append(i); cols.append(j); vals.append(offv(rng))
    return sp.csr_matrix((vals, (rows, cols)), shape=(n, n))


def test_aggregation_on_irregular_matrices():
    """testsets "Aggregation - no stalling on sparse irregular matrix",
    "Aggregation - theta auto-reduction fallback" and "MIS-based aggregation
    produces larger aggregates" (test/runtests.jl:2148-2212): fewer than 8
    levels with strictly shrinking sizes on a random 500 x 500 matrix; 1 to
    14 levels on a weakly coupled random 200 x 200; on 20 x 20, fewer than
    half the points are aggregates."""
    A = _random_matrix(500, 42, lambda r: 10 + 90 * r.uniform(), lambda r: int(r.integers(2, 6)),
                       lambda r: -(1 + 9 * r.uniform()))
    h = draugr.amg_setup(A, draugr.AMGConfig(coarsening=draugr.AggregationCoarsening(0.25), max_levels=20),
                         on_device=False)
    sizes = [int(h.level_info(l)[0]) for l in range(h.nlevels)]
    assert h.nlevels < 8 and all(b < a for a, b in zip(sizes, sizes[1:]))
    A = _random_matrix(200, 123, lambda r: 100.0, lambda r: int(r.integers(1, 3)),
                       lambda r: -(0.1 + r.uniform()))
    h = draugr.amg_setup(A, draugr.AMGConfig(coarsening=draugr.AggregationCoarsening(0.25)),
                         on_device=False)
    assert 1 <= h.nlevels < 15
    h = draugr.amg_setup(problems.poisson2d(20),
                         draugr.AMGConfig(coarsening=draugr.AggregationCoarsening(0.25), max_coarse_size=2),
                         on_device=False)
    nc = int(h.level_info(0)[2])
    assert nc < 0.5 * 400 and 400 / nc > 2.0


def test_hypre_default_config():
    """testsets "hypre_default_config construction / with custom params /
    solve - 2D Poisson" and "Interpolation trunc_factor"
    (test/runtests.jl:2214-2269)."""
    c = draugr.hypre_default_config()
    assert isinstance(c.coarsening, draugr.HMISCoarsening) and c.coarsening.theta == 0.5
    assert isinstance(c.coarsening.interpolation, draugr.ExtendedIInterpolation)
    assert c.coarsening.interpolation.trunc_factor == 0.3
    ic = c.initial_coarsening
    assert isinstance(ic, draugr.AggressiveCoarsening) and ic.theta == 0.5 and ic.base == "hmis"
    assert ic.interpolation.trunc_factor == 0.3 and c.initial_coarsening_levels == 1
    c = draugr.hypre_default_config(theta=0.3, agg_num_levels=2, agg_trunc_factor=0.5,
                                    smoother=draugr.ColoredGaussSeidelType())
    assert c.coarsening.theta == 0.3 and c.initial_coarsening.theta == 0.3
    assert c.initial_coarsening_levels == 2 and c.coarsening.interpolation.trunc_factor == 0.5
    assert isinstance(c.smoother, draugr.ColoredGaussSeidelType)
    for cls in (draugr.DirectInterpolation, draugr.StandardInterpolation, draugr.ExtendedIInterpolation):
        assert cls().trunc_factor == 0.0 and cls(0.3).trunc_factor == 0.3
    A = problems.poisson2d(12)
    b = rhs(144, 9)
    x, it, h = solve(A, draugr.hypre_default_config(), b)
    assert h.nlevels >= 1 and it < 200 and rel_res(A, x, b) < 1e-6


@pytest.mark.parametrize("base,main", [("hmis", draugr.HMISCoarsening), ("pmis", draugr.PMISCoarsening)])
def test_aggressive_coarsening_bases(base, main):
    """testsets "AggressiveCoarsening with HMIS / PMIS base" and
    "coarsen_aggressive_cf with HMIS / PMIS" (test/runtests.jl:2271-2312,
    :2329-2365): one aggressive level then HMIS or PMIS solves 10 x 10 to
    1e-6 in fewer than 200 cycles; the aggressive splitting of 10 x 10
    (theta 0.25) decides every point and keeps 0 < nc < N (below 0.6 N for
    the HMIS base), with coarse indices 0..nc-1."""
    cfg = draugr.AMGConfig(coarsening=main(0.5, draugr.ExtendedIInterpolation()),
                           initial_coarsening=draugr.AggressiveCoarsening(0.5, base,
                                                                          draugr.ExtendedIInterpolation(0.3)),
                           initial_coarsening_levels=1, **V22)
    A = problems.poisson2d(10)
    b = rhs(100, 10)
    x, it, h = solve(A, cfg, b)
    assert h.nlevels >= 1 and it < 200 and rel_res(A, x, b) < 1e-6
    cfg = draugr.AMGConfig(coarsening=draugr.AggressiveCoarsening(0.25, base), max_coarse_size=2)
    h = draugr.amg_setup(A, cfg, on_device=False)
    cf = h.export(0, "cf")
    nc = int(h.level_info(0)[2])
    assert np.all(np.abs(cf) == 1) and 0 < nc < 100 and int(np.sum(cf == 1)) == nc
    if base == "hmis":
        assert nc < 0.6 * 100
    assert h.export(0, "P_colval").max() == nc - 1


def test_consistent_theta_and_hmis_truncation():
    """testsets "Consistent theta in interpolation" and "HMIS with ExtendedI
    and trunc_factor" (test/runtests.jl:2313-2327, :2367-2384): HMIS (0.5)
    with direct interpolation on 8 x 8 and with extended+i (0.3) on 10 x 10
    solve to 1e-6."""
    for n, ip in ((8, draugr.DirectInterpolation()), (10, draugr.ExtendedIInterpolation(0.3))):
        A = problems.poisson2d(n)
        b = rhs(n * n, 11)
        x, it, h = solve(A, draugr.AMGConfig(coarsening=draugr.HMISCoarsening(0.5, ip), **V22), b)
        assert h.nlevels >= 1 and it < 200 and rel_res(A, x, b) < 1e-6


def test_extended_i_options():
    """testsets "ExtendedI max_elements", "ExtendedI norm_p and rescale
    fields", "ExtendedI norm_p truncation" and "ExtendedI rescale"
    (test/runtests.jl:2386-2489): field defaults; HMIS (0.5) on 10 x 10 with
    max_elements 2, 4, 8, 0, with norm_p 1 and 2, and with and without
    rescaling solves to 1e-6 within 300 cycles.  max_elements caps every F
    row of P."""
    E = draugr.ExtendedIInterpolation
    assert E().max_elements == 0 and E(0.3).max_elements == 0 and E(0.0, 8).max_elements == 8
    assert E().norm_p == 1 and E().rescale is False
    e3 = E(0.3, 4, 2, True)
    assert (e3.trunc_factor, e3.max_elements, e3.norm_p, e3.rescale) == (0.3, 4, 2, True)
    A = problems.poisson2d(10)
    b = rhs(100, 12)
    for ip in (E(0.0, 2), E(0.0, 4), E(0.0, 8), E(0.0, 0), E(0.3, 0, 1, False), E(0.3, 0, 2, False),
               E(0.3, 0, 1, True)):
        x, it, h = solve(A, draugr.AMGConfig(coarsening=draugr.HMISCoarsening(0.5, ip), **V22), b,
                         tol=1e-6, maxiter=300)
        assert h.nlevels >= 1 and rel_res(A, x, b) < 1e-6, ip
        if ip.max_elements:
            rp = h.export(0, "P_rowptr")
            assert np.diff(rp).max() <= ip.max_elements, ip
