"""Parity of the CUDA solve / resetup path with the oracle (the CPU
restatement of Draugr.jl's arithmetic), on the same hierarchy structure,
through the library's C ABI.

Tolerances (normwise relative): FP64 kernels and cycles 1e-12; the coarsest
LU solve is bit-exact (same operation order, no contraction); FP32 kernels
1e-5; Galerkin resetup values 1e-12 per level against the reference's
triple-map product.
"""

import numpy as np
import pytest

import draugr
import oracle
from cases import CASES

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 1e-5


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / (nb if nb > 0 else 1.0)


@pytest.fixture(scope="module", params=sorted(CASES))
def case(request):
    make, cfg = CASES[request.param]
    A = make()
    h = draugr.amg_setup(A, cfg)
    O = oracle.OracleHierarchy(h, with_rmaps=True)
    return request.param, A, cfg, h, O


def _level_arrays(O, l):
    d = O.levels_np[l]
    L = O._levels[l]
    return d, L


def test_level_kernels(case):
    name, A, cfg, h, O = case
    rng = np.random.default_rng(11)
    for l in range(h.nlevels):
        d, L = _level_arrays(O, l)
        n, nc = L.n, L.nc
        x = rng.uniform(-1, 1, n)
        b = rng.uniform(-1, 1, n)
        xc = rng.uniform(-1, 1, nc)
        ref = oracle.spmv(n, d["A_rp"], d["A_ci"], d["A_v"], x)
        assert rel(h.level_op(l, 0, x), ref) < TOL64
        assert rel(h.level_op(l, 0, x, precision=1), ref) < TOL32
        ref = oracle.residual(n, d["A_rp"], d["A_ci"], d["A_v"], x, b)
        assert rel(h.level_op(l, 1, x, b), ref) < TOL64
        ref = oracle.restrict(nc, d["T_off"], d["T_rows"], d["T_pnz"], d["P_v"], x)
        assert rel(h.level_op(l, 3, x), ref) < TOL64
        assert rel(h.level_op(l, 3, x, precision=1), ref) < TOL32
        ref = oracle.prolongate(n, d["P_rp"], d["P_ci"], d["P_v"], xc, x)
        assert rel(h.level_op(l, 4, x, xc), ref) < TOL64
        for steps in (1, 2, 3):
            if L.smoother in (0, 5):
                ref = oracle.jacobi(n, d["A_rp"], d["A_ci"], d["A_v"], d["invd"], L.omega, x, b, steps)
            elif L.smoother == 3:
                ref = oracle.spai0_smooth(n, d["A_rp"], d["A_ci"], d["A_v"], d["invd"], x, b, steps)
            elif L.smoother == 8:
                ref = oracle.chebyshev(n, d["A_rp"], d["A_ci"], d["A_v"], d["invd"], d["cheb_coef"], x, b, steps)
            elif L.smoother == 4:
                ref = oracle.spai1_smooth(n, d["A_rp"], d["A_ci"], d["A_v"], d["spai1_M"], x, b, steps)
            elif L.smoother in (2, 7):
                ref = oracle.serial_gs(n, d["A_rp"], d["A_ci"], d["A_v"], d["invd"], x, b, steps)
            elif L.smoother in (9, 10):
                ref = oracle.ilu0_smooth(n, d["A_rp"], d["A_ci"], d["A_v"], d["ilu_diag"], d["ilu_L"],
                                         d["ilu_U"], x, b, steps)
            else:
                ref = oracle.gs(n, d["A_rp"], d["A_ci"], d["A_v"], d["invd"], L.ncolors,
                                d["color_off"], d["color_order"], x, b, steps)
            assert rel(h.level_op(l, 2, x, b, steps=steps), ref) < TOL64, (l, steps)
            assert rel(h.level_op(l, 2, x, b, steps=steps, precision=1), ref) < TOL32
        if L.smoother in (0, 3, 5):
            x1 = (oracle.spai0_smooth(n, d["A_rp"], d["A_ci"], d["A_v"], d["invd"], np.zeros(n), b, 1)
                  if L.smoother == 3 else
                  oracle.jacobi(n, d["A_rp"], d["A_ci"], d["A_v"], d["invd"], L.omega, np.zeros(n), b, 1))
            r1 = oracle.residual(n, d["A_rp"], d["A_ci"], d["A_v"], x1, b)
            out = h.level_op(l, 6, b)
            assert rel(out[:n], x1) < TOL64
            assert rel(out[n:], r1) < TOL64


def test_coarse_solve_bit_exact(case):
    name, A, cfg, h, O = case
    rng = np.random.default_rng(5)
    bc = rng.uniform(-1, 1, O.nc)
    y = bc.copy()
    oracle.load().orc_lu_solve(O.nc, oracle.ptr(O.lu), oracle.ptr(O.piv), oracle.ptr(y))
    assert np.array_equal(h.level_op(0, 5, bc), y)


@pytest.mark.parametrize("wcycle", [False, True])
def test_cycle(case, wcycle):
    name, A, cfg, h, O = case
    n = A.shape[0]
    rng = np.random.default_rng(3)
    b = rng.uniform(-1, 1, n)
    x0 = rng.uniform(-1, 1, n)
    c2 = draugr.AMGConfig(**{**cfg.__dict__, "cycle_type": "W" if wcycle else "V"})
    ref = O.cycle(x0, b, cfg.pre_smoothing_steps, cfg.post_smoothing_steps, wcycle)
    x = x0.copy()
    draugr.amg_cycle(x, b, h, c2)
    assert rel(x, ref) < TOL64
    # zero initial guess (the path that fuses the first Jacobi step)
    ref0 = O.cycle(np.zeros(n), b, cfg.pre_smoothing_steps, cfg.post_smoothing_steps, wcycle)
    x = np.zeros(n)
    draugr.amg_cycle(x, b, h, c2)
    assert rel(x, ref0) < TOL64


def test_cycle_more_smoothing(case):
    name, A, cfg, h, O = case
    n = A.shape[0]
    b = np.random.default_rng(8).uniform(-1, 1, n)
    c2 = draugr.AMGConfig(**{**cfg.__dict__, "pre_smoothing_steps": 2, "post_smoothing_steps": 3})
    ref = O.cycle(np.zeros(n), b, 2, 3, False)
    x = np.zeros(n)
    draugr.amg_cycle(x, b, h, c2)
    assert rel(x, ref) < TOL64


def test_stationary_solve(case):
    name, A, cfg, h, O = case
    n = A.shape[0]
    b = np.random.default_rng(1).uniform(-1, 1, n)
    xr, itr, relr = O.solve(np.zeros(n), b, cfg.pre_smoothing_steps, cfg.post_smoothing_steps,
                            False, 1e-8, 300)
    x = np.zeros(n)
    x, it = draugr.amg_solve(x, b, h, cfg, tol=1e-8, maxiter=300)
    assert it == itr
    assert rel(x, xr) < 1e-9
    if it < 300:
        assert np.linalg.norm(b - A @ x) / np.linalg.norm(b) < 1e-8


def test_pcg_fp64_and_mixed(case):
    name, A, cfg, h, O = case
    n = A.shape[0]
    b = np.random.default_rng(2).uniform(-1, 1, n)
    xr, itr, relr = O.pcg(np.zeros(n), b, cfg.pre_smoothing_steps, cfg.post_smoothing_steps,
                          False, 1e-8, 500)
    x, it, rr = draugr.pcg(np.zeros(n), b, h, cfg, tol=1e-8, maxiter=500, precision="fp64")
    if "gs" not in name:   # colored GS cycles are not symmetric: CG is not guaranteed
        assert abs(it - itr) <= 1
        assert rel(x, xr) < 1e-7
        assert np.linalg.norm(b - A @ x) / np.linalg.norm(b) < 1e-8
        xm, itm, rm = draugr.pcg(np.zeros(n), b, h, cfg, tol=1e-8, maxiter=500, precision="mixed")
        assert np.linalg.norm(b - A @ xm) / np.linalg.norm(b) < 1e-8  # FP64-verified
        assert itm <= int(1.25 * it) + 2


def test_resetup_matches_reference_galerkin(case):
    name, A, cfg, h, O = case
    n = A.shape[0]
    rng = np.random.default_rng(4)
    dscale = rng.uniform(0.5, 2.0, n)
    A2 = A.multiply(dscale[:, None]).multiply(dscale[None, :]).tocsr()  # D A D, same pattern
    A2.sort_indices()
    assert np.array_equal(A2.indices, A.indices)
    draugr.amg_resetup(h, A2, cfg, partial=True)
    O.resetup(A2.data)
    for l in range(h.nlevels):
        dev = h.export(l, "A_nzval")
        ref = O.level_values(l)
        assert rel(dev, ref) < TOL64, f"level {l}"
        assert rel(h.export(l, "invdiag"), O.levels_np[l]["invd"]) < TOL64
        if "cheb_coef" in O.levels_np[l]:  # spectral radius and coefficients redone on the device
            assert rel(h.export(l, "cheb_coef"), O.levels_np[l]["cheb_coef"]) < TOL64
        if "spai1_M" in O.levels_np[l]:  # M recomputed from the level's new values
            assert rel(h.export(l, "spai1_M"), O.levels_np[l]["spai1_M"]) < TOL64
        if "ilu_L" in O.levels_np[l]:  # refactorised from the level's new values
            assert rel(h.export(l, "ilu_L"), O.levels_np[l]["ilu_L"]) < TOL64
            assert rel(h.export(l, "ilu_U"), O.levels_np[l]["ilu_U"]) < TOL64
    nc = O.nc
    assert rel(h.export(-1, "C_dense"), O.dense) < TOL64
    # the resetup hierarchy solves the new system
    b = rng.uniform(-1, 1, n)
    x, it = draugr.amg_solve(np.zeros(n), b, h, cfg, tol=1e-8, maxiter=400)
    if it < 400:
        assert np.linalg.norm(b - A2 @ x) / np.linalg.norm(b) < 1e-8
    # and the cycle after resetup still matches the oracle's
    xr = O.cycle(np.zeros(n), b, cfg.pre_smoothing_steps, cfg.post_smoothing_steps, False)
    x = np.zeros(n)
    draugr.amg_cycle(x, b, h, cfg)
    assert rel(x, xr) < 1e-11
    assert nc > 0


def test_device_pointer_entry_points(case):
    torch = pytest.importorskip("torch")
    name, A, cfg, h, O = case
    n = A.shape[0]
    b = np.random.default_rng(6).uniform(-1, 1, n)
    xh, ith = draugr.amg_solve(np.zeros(n), b, h, cfg, tol=1e-8, maxiter=200)
    xd = torch.zeros(n, dtype=torch.float64, device="cuda")
    bd = torch.tensor(b, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    xd, itd = draugr.amg_solve(xd, bd, h, cfg, tol=1e-8, maxiter=200)
    torch.cuda.synchronize()
    assert itd == ith
    assert np.array_equal(xd.cpu().numpy(), xh)


@pytest.fixture(scope="module", params=sorted(CASES))
def fresh_case(request):
    """A hierarchy straight from setup (the resetup test above changes the
    values of `case`; a GPU resetup's coarse values differ from the
    reference's triple-map values in the last bits)."""
    make, cfg = CASES[request.param]
    A = make()
    h = draugr.amg_setup(A, cfg)
    return request.param, A, cfg, h, oracle.OracleHierarchy(h)


def _single_lane(h, l):
    """(A, P, Pᵀ) rows all reduced in column order by the row kernel."""
    info = h.level_info(l)
    return int(info[7]) == 1, int(info[8]) == 1, int(info[9]) == 1


def test_single_lane_rows_are_bit_exact(fresh_case):
    """Rows reduced by one lane sum their products in column order, as the
    reference does, so those kernels reproduce the oracle bit for bit."""
    name, A, cfg, h, O = fresh_case
    rng = np.random.default_rng(21)
    checked = 0
    for l in range(h.nlevels):
        d, L = _level_arrays(O, l)
        n, nc = L.n, L.nc
        a1, p1, r1 = _single_lane(h, l)
        x = rng.uniform(-1, 1, n)
        b = rng.uniform(-1, 1, n)
        xc = rng.uniform(-1, 1, nc)
        if a1:
            assert np.array_equal(h.level_op(l, 0, x), oracle.spmv(n, d["A_rp"], d["A_ci"], d["A_v"], x))
            assert np.array_equal(h.level_op(l, 1, x, b),
                                  oracle.residual(n, d["A_rp"], d["A_ci"], d["A_v"], x, b))
            if L.smoother in (0, 5):
                for steps in (1, 2):
                    ref = oracle.jacobi(n, d["A_rp"], d["A_ci"], d["A_v"], d["invd"], L.omega, x, b, steps)
                    assert np.array_equal(h.level_op(l, 2, x, b, steps=steps), ref)
                x1 = oracle.jacobi(n, d["A_rp"], d["A_ci"], d["A_v"], d["invd"], L.omega,
                                   np.zeros(n), b, 1)
                r1v = oracle.residual(n, d["A_rp"], d["A_ci"], d["A_v"], x1, b)
                out = h.level_op(l, 6, b)
                assert np.array_equal(out[:n], x1) and np.array_equal(out[n:], r1v)
            checked += 1
        if r1:
            ref = oracle.restrict(nc, d["T_off"], d["T_rows"], d["T_pnz"], d["P_v"], x)
            assert np.array_equal(h.level_op(l, 3, x), ref)
        if p1:
            ref = oracle.prolongate(n, d["P_rp"], d["P_ci"], d["P_v"], xc, x)
            assert np.array_equal(h.level_op(l, 4, x, xc), ref)
    assert checked >= 1


def test_cycle_bit_exact_when_all_rows_single_lane(fresh_case):
    name, A, cfg, h, O = fresh_case
    jac = all(int(h.level_info(l)[4]) in (0, 5) for l in range(h.nlevels))
    single = all(all(_single_lane(h, l)) for l in range(h.nlevels))
    if not (jac and single):
        pytest.skip("hierarchy has multi-lane rows or Gauss-Seidel levels")
    n = A.shape[0]
    b = np.random.default_rng(9).uniform(-1, 1, n)
    x0 = np.random.default_rng(10).uniform(-1, 1, n)
    for w in (False, True):
        c2 = draugr.AMGConfig(**{**cfg.__dict__, "cycle_type": "W" if w else "V"})
        for start in (x0, np.zeros(n)):
            x = start.copy()
            draugr.amg_cycle(x, b, h, c2)
            assert np.array_equal(x, O.cycle(start, b, 1, 1, w))


def test_tail_flat_products_bit_exact(monkeypatch):
    """The coarse tail forms the products of levels with long rows flat over
    the block and then sums each row in column order: the same rounded
    products and sums, so the cycle still equals the oracle's bit for bit.
    DRAUGR_B200_TAIL_FLAT_ROW=0 makes every tail level take that path."""
    monkeypatch.setenv("DRAUGR_B200_TAIL_FLAT_ROW", "0")
    checked = 0
    for name in sorted(CASES):
        make, cfg = CASES[name]
        A = make()
        h = draugr.amg_setup(A, cfg)
        jac = all(int(h.level_info(l)[4]) in (0, 5) for l in range(h.nlevels))
        single = all(all(_single_lane(h, l)) for l in range(h.nlevels))
        if jac and single and h.nlevels >= 2:
            O = oracle.OracleHierarchy(h)
            n = A.shape[0]
            b = np.random.default_rng(12).uniform(-1, 1, n)
            for start in (np.zeros(n), np.random.default_rng(13).uniform(-1, 1, n)):
                x = start.copy()
                draugr.amg_cycle(x, b, h, cfg)
                assert np.array_equal(x, O.cycle(start, b, 1, 1, False)), name
            checked += 1
        h.free()
    assert checked >= 1


def test_cycle_from_level_timing(case):
    """draugr_b200_time_level_op op 8 times the V(1,1) cycle from a level
    >= 1 down (the coarse tail included) and rejects the finest level."""
    name, A, cfg, h, O = case
    if h.nlevels < 2 or any(int(h.level_info(l)[4]) not in (0, 3, 5) for l in range(h.nlevels)):
        pytest.skip("needs two levels with Jacobi-type smoothers")
    for l in range(1, h.nlevels):
        assert h.time_level_op(l, 8, 0, reps=2) > 0.0
        assert h.time_level_op(l, 8, 1, reps=2) > 0.0
    with pytest.raises(draugr.DraugrError, match="op 8"):
        h.time_level_op(0, 8, 0, reps=2)


def test_residual_entry_point(fresh_case):
    """draugr_b200_residual_device: r = b - A x and ||r|| on device vectors."""
    torch = pytest.importorskip("torch")
    import ctypes as C
    name, A, cfg, h, O = fresh_case
    n = A.shape[0]
    rng = np.random.default_rng(31)
    x = rng.uniform(-1, 1, n)
    b = rng.uniform(-1, 1, n)
    xd = torch.tensor(x, dtype=torch.float64, device="cuda")
    bd = torch.tensor(b, dtype=torch.float64, device="cuda")
    rd = torch.zeros(n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rn = C.c_double(0)
    rc = draugr.load().draugr_b200_residual_device(h.handle, n, xd.data_ptr(), bd.data_ptr(),
                                                   rd.data_ptr(), C.byref(rn))
    assert rc == 0, draugr.last_error()
    d, L = _level_arrays(O, 0)
    ref = oracle.residual(n, d["A_rp"], d["A_ci"], d["A_v"], x, b)
    r = rd.cpu().numpy()
    assert rel(r, ref) < TOL64
    if _single_lane(h, 0)[0]:
        assert np.array_equal(r, ref)
    assert abs(rn.value - np.linalg.norm(ref)) <= 1e-12 * np.linalg.norm(ref)


def test_resetup_reproduces_setup_values_bit_exact(fresh_case):
    """The GPU Galerkin products accumulate every entry in the order of the
    CPU setup's numeric product: a partial resetup with the setup's own
    values reproduces every level (and the coarsest dense matrix) exactly."""
    name, A, cfg, h, O = fresh_case
    before = [h.export(l, "A_nzval").copy() for l in range(h.nlevels)]
    dense = h.export(-1, "C_dense").copy()
    draugr.amg_resetup(h, A, cfg, partial=True)
    for l in range(h.nlevels):
        assert np.array_equal(h.export(l, "A_nzval"), before[l]), (name, l)
    assert np.array_equal(h.export(-1, "C_dense"), dense)
