"""CPU tests of the library: it loads, exports every symbol its headers
declare, parses configurations like the reference, reports errors like the
reference, and its CPU-built hierarchy structure equals the oracle's
restatement of the reference's structure routines (bit for bit)."""

import re

import numpy as np
import pytest
import scipy.sparse as sp

import draugr
import oracle
from conftest import ROOT
from draugr import problems
from draugr._lib import SIGNATURES, check

HEADERS = [ROOT / "include" / "draugr_amg.h", ROOT / "include" / "draugr_b200.h"]


def declared_functions():
    names = set()
    for h in HEADERS:
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", text):
            name = m.group(1)
            if name.startswith(("draugr_", "init_julia", "shutdown_julia")):
                names.add(name)
    return names


def test_library_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert "draugr_amg_setup" in names and "draugr_b200_pcg" in names
    for name in names:
        assert hasattr(lib, name), name
    # the ctypes signature table covers the same set
    assert names == set(SIGNATURES)


def test_config_defaults_and_errors(lib):
    h = lib.draugr_amg_config_from_json(None)
    assert h > 0
    assert lib.draugr_amg_config_from_json(b"{}") > h
    # string values are case-insensitive, numbers may be strings, unknown keys ignored
    ok = lib.draugr_amg_config_from_json(
        b'{"coarsening": "AGGREGATION", "theta": "0.25", "smoother": {"type": "Jacobi", '
        b'"omega": "0.5"}, "cycle": "W", "max_levels": 10.0, "whatever": [1, 2]}')
    assert ok > 0
    bad = lib.draugr_amg_config_from_json(b'{"coarsening": "nope"}')
    assert bad == -1
    msg = draugr.last_error()
    assert 'Unknown coarsening: "nope"' in msg and "aggregation" in msg
    assert lib.draugr_amg_config_from_json(b'{"smoother": 3}') == -1
    assert lib.draugr_amg_config_from_json(b'{"cycle": "x"}') == -1
    assert lib.draugr_amg_config_from_json(b"{not json") == -1
    assert lib.draugr_amg_config_free(ok) == 0
    assert lib.draugr_amg_config_free(ok) == -1
    assert "Invalid config handle" in draugr.last_error()


def test_invalid_handles(lib):
    x = np.zeros(4)
    b = np.ones(4)
    p = lambda a: a.ctypes.data_as(draugr._lib.C.c_void_p)
    cfg = draugr.config_handle(None)
    assert lib.draugr_amg_solve(9999, 4, p(x), p(b), cfg, 1e-8, 10) == -1
    assert len(draugr.last_error()) > 0
    assert lib.draugr_amg_cycle(9999, 4, p(x), p(b), cfg) == -1
    assert lib.draugr_amg_free(9999) == -1
    rp = np.array([0, 1], np.int32)
    ci = np.array([0], np.int32)
    v = np.array([1.0])
    assert lib.draugr_amg_resetup(9999, 1, 1, p(rp), p(ci), p(v), cfg, 0, 1, 1) == -1


def test_index_base_and_validation(lib):
    A = problems.poisson1d(200)
    n, rp, ci, v = oracle.csr_parts(A)
    p = lambda a: a.ctypes.data_as(draugr._lib.C.c_void_p)
    cfg = draugr.config_handle(draugr.AMGConfig(coarsening=draugr.AggregationCoarsening()))
    h0 = lib.draugr_b200_setup_host(n, len(ci), p(rp), p(ci), p(v), cfg, 0, 1)
    rp1, ci1 = rp + 1, ci + 1
    h1 = lib.draugr_b200_setup_host(n, len(ci), p(rp1), p(ci1), p(v), cfg, 1, 1)
    assert h0 > 0 and h1 > 0
    H0, H1 = draugr.Hierarchy(h0, n, None), draugr.Hierarchy(h1, n, None)
    for what in ("A_rowptr", "A_colval", "P_colval", "T_rows"):
        assert np.array_equal(H0.export(0, what), H1.export(0, what))
    assert lib.draugr_b200_setup_host(n, len(ci), p(rp), p(ci), p(v), cfg, 2, 1) == -1
    assert "index_base must be 0 or 1" in draugr.last_error()
    bad = ci.copy()
    bad[3] = n + 5
    assert lib.draugr_b200_setup_host(n, len(ci), p(rp), p(bad), p(v), cfg, 0, 1) == -1
    assert "column index out of range" in draugr.last_error()
    # every smoother and coarsening of the configuration is supported: an
    # unknown name fails at parsing, with the valid names in the message
    assert lib.draugr_amg_config_from_json(b'{"smoother": "no_such_smoother"}') == -1
    assert "Unknown smoother" in draugr.last_error() and "spai1" in draugr.last_error()
    cfg2 = draugr.config_handle(draugr.AMGConfig(coarsening=draugr.RSCoarsening()))
    assert lib.draugr_b200_setup_host(n, len(ci), p(rp), p(ci), p(v), cfg2, 0, 1) > 0


from cases import CASES as CONFIGS  # noqa: E402


@pytest.fixture(scope="module", params=sorted(CONFIGS))
def host_case(request):
    make, cfg = CONFIGS[request.param]
    A = make()
    h = draugr.amg_setup(A, cfg, on_device=False)
    return request.param, A, cfg, h


def test_structure_matches_oracle(host_case):
    """Transpose maps, Galerkin sparsity (compute_coarse_sparsity), colours
    and smoother diagonals equal the oracle's restatement exactly; setup
    values of the coarse operators agree to 1e-12 (different summation
    order than the reference's triple map)."""
    name, A, cfg, h = host_case
    nl = h.nlevels
    assert nl >= 1
    for l in range(nl):
        info = h.level_info(l)
        n, nc = int(info[0]), int(info[2])
        arp, aci, av = h.export(l, "A_rowptr"), h.export(l, "A_colval"), h.export(l, "A_nzval")
        prp, pci, pv = h.export(l, "P_rowptr"), h.export(l, "P_colval"), h.export(l, "P_nzval")
        off, rows, pnz = oracle.transpose_map(n, nc, prp, pci)
        assert np.array_equal(off, h.export(l, "T_offsets"))
        assert np.array_equal(rows, h.export(l, "T_rows"))
        assert np.array_equal(pnz, h.export(l, "T_pnz"))
        c_rp, c_ci, c_v, *_ = oracle.coarse_sparsity(n, nc, arp, aci, av, prp, pci, pv)
        if l + 1 < nl:
            nrp, nci, nv = (h.export(l + 1, "A_rowptr"), h.export(l + 1, "A_colval"),
                            h.export(l + 1, "A_nzval"))
        else:
            nrp, nci, nv = h.export(-1, "C_rowptr"), h.export(-1, "C_colval"), h.export(-1, "C_nzval")
        assert np.array_equal(c_rp, nrp), f"level {l}: coarse rowptr differs"
        assert np.array_equal(c_ci, nci), f"level {l}: coarse colval differs"
        scale = np.abs(c_v).max()
        assert np.abs(c_v - nv).max() <= 1e-12 * scale
        kind = int(info[4])
        if kind == 3:  # SPAI(0): m_i = a_ii / sum a_ij^2, swept with omega = 1
            inv = oracle.spai0(n, arp, aci, av)
            assert h.export(l, "omega")[0] == 1.0
        elif kind == 4:  # SPAI(1): M on A's pattern, against the reference's loop
            inv = oracle.invdiag(n, arp, aci, av)
            assert np.array_equal(oracle.spai1(n, arp, aci, av), h.export(l, "spai1_M"))
        elif kind in (2, 7):  # serial (l1) Gauss-Seidel: diagonal and sweep schedule
            inv = oracle.serial_gs_invdiag(n, arp, aci, av) if kind == 2 else oracle.invdiag(n, arp, aci, av, l1=True)
            order, off = h.export(l, "sgs_order"), h.export(l, "sgs_offsets")
            assert np.array_equal(np.sort(order), np.arange(n)) and off[0] == 0 and off[-1] == n
            level = np.empty(n, np.int64)
            for v in range(len(off) - 1):
                level[order[off[v]:off[v + 1]]] = v
            rr = np.repeat(np.arange(n), np.diff(arp))
            off_diag = rr != aci
            lo, hi = np.minimum(rr, aci)[off_diag], np.maximum(rr, aci)[off_diag]
            assert np.all(level[lo] < level[hi])  # every coupling ordered as the row sweep
        elif kind in (9, 10):  # ILU(0): factors and level schedules
            inv = oracle.invdiag(n, arp, aci, av)
            diag = oracle.ilu0_diag(n, arp, aci)
            assert np.array_equal(diag, h.export(l, "ilu_diag"))
            Lf, Uf = oracle.ilu0_factor(n, arp, aci, av, diag)
            assert np.array_equal(Lf, h.export(l, "ilu_L")) and np.array_equal(Uf, h.export(l, "ilu_U"))
            for which, lower in (("fwd", True), ("bwd", False)):
                order, off = h.export(l, f"ilu_{which}_order"), h.export(l, f"ilu_{which}_offsets")
                assert np.array_equal(np.sort(order), np.arange(n)) and off[0] == 0 and off[-1] == n
                level = np.empty(n, np.int64)
                for v in range(len(off) - 1):
                    level[order[off[v]:off[v + 1]]] = v
                for i in range(n):  # every dependency sits in an earlier level
                    deps = aci[arp[i]:diag[i]] if lower else aci[diag[i] + 1:arp[i + 1]]
                    assert np.all(level[deps] < level[i])
        elif kind == 8:  # Chebyshev: Jacobi diagonal, power iteration, coefficients
            inv = oracle.invdiag(n, arp, aci, av)
            rho = oracle.spectral_radius(n, arp, aci, av, inv, h.export(l, "cheb_v0"))
            assert np.array_equal(oracle.cheb_coef(rho, 3), h.export(l, "cheb_coef"))
        else:
            inv = oracle.invdiag(n, arp, aci, av, l1=kind in (5, 6))
        assert np.array_equal(inv, h.export(l, "invdiag"))
        if kind in (1, 6):
            colors, ncol, coff, order = oracle.greedy_coloring(n, arp, aci)
            assert ncol == int(info[5])
            assert np.array_equal(colors, h.export(l, "colors"))
            assert np.array_equal(coff, h.export(l, "color_offsets"))
            assert np.array_equal(order, h.export(l, "color_order"))
            # no two neighbours share a colour (test/runtests.jl:549-566)
            rr = np.repeat(np.arange(n), np.diff(arp))
            off_diag = rr != aci
            assert not np.any(colors[rr[off_diag]] == colors[aci[off_diag]])
    # coarsest LU equals the oracle's getf2
    nc = int(h.level_info(-1)[0])
    lu, piv, info = oracle.lu_factor(h.export(-1, "C_dense").reshape(nc, nc).T)
    assert info == 0
    assert np.array_equal(piv, h.export(-1, "C_piv"))
    assert np.array_equal(lu.T.reshape(-1), h.export(-1, "C_lu"))


def test_prolongation_properties(host_case):
    """Every fine row interpolates from at least one coarse point; C-point
    rows are unit rows; P columns are in range and sorted per row."""
    name, A, cfg, h = host_case
    for l in range(h.nlevels):
        info = h.level_info(l)
        prp, pci = h.export(l, "P_rowptr"), h.export(l, "P_colval")
        assert np.all(np.diff(prp) >= 1)
        assert pci.min() >= 0 and pci.max() < info[2]
        for i in range(0, int(info[0]), max(1, int(info[0]) // 200)):
            row = pci[prp[i]:prp[i + 1]]
            assert np.all(np.diff(row) > 0)


def test_hierarchy_summary(host_case):
    """testset "Verbose Output" (test/runtests.jl:830-856), the setup part:
    the summary carries the hierarchy header, the backend and block size,
    and the operator complexity; the level table names the smoothers as the
    reference's setup print does (src/setup.jl:478-488)."""
    name, A, cfg, h = host_case
    s = h.summary()
    for key in ("AMG Hierarchy Summary", "Operator complexity", "Backend", "Block size", "Direct (LU)"):
        assert key in s, key
    assert type(cfg.smoother).__name__ in s


def test_host_galerkin_reproduces_the_setup_product(host_case):
    """draugr_b200_galerkin_host with a level's own values gives the next
    level's values bit for bit (the same numeric product as the setup), and
    is linear in the values (2A gives twice the product exactly)."""
    name, A, cfg, h = host_case
    for l in range(h.nlevels):
        v = h.export(l, "A_nzval")
        nxt = h.export(l + 1, "A_nzval") if l + 1 < h.nlevels else h.export(-1, "C_nzval")
        assert np.array_equal(h.galerkin_host(l, v), nxt), (name, l)
        assert np.array_equal(h.galerkin_host(l, 2.0 * v), 2.0 * nxt), (name, l)
    with pytest.raises(draugr.DraugrError):
        h.galerkin_host(h.nlevels, np.zeros(1))


def test_allow_partial_resetup_false_has_no_maps():
    A = problems.poisson2d(16)
    h = draugr.amg_setup(A, draugr.AMGConfig(coarsening=draugr.AggregationCoarsening()),
                         allow_partial_resetup=False, on_device=False)
    for l in range(h.nlevels):
        assert h.level_info(l)[6] == -1


def test_setup_seed_determinism():
    A = problems.heterogeneous_diffusion_3d(10, seed=5)
    cfg = draugr.hypre_default_config(agg_trunc_factor=0.2, seed=7)
    h1 = draugr.amg_setup(A, cfg, on_device=False)
    h2 = draugr.amg_setup(A, cfg, on_device=False)
    for l in range(h1.nlevels):
        assert np.array_equal(h1.export(l, "P_colval"), h2.export(l, "P_colval"))
        assert np.array_equal(h1.export(l, "P_nzval"), h2.export(l, "P_nzval"))


def test_check_raises():
    with pytest.raises(draugr.DraugrError):
        check(-1, "x")


def test_preconditioner_before_update():
    """DraugrPreconditioner keeps the reference's lifecycle: no hierarchy
    (nrows 0) until update(A), and applying it before then is an error."""
    P = draugr.DraugrPreconditioner(smoother=draugr.L1JacobiSmootherType())
    assert P.nrows == 0 and P.hierarchy is None
    with pytest.raises(draugr.DraugrError):
        P.apply(np.zeros(4), np.ones(4))


def test_csr_from_raw_testsets(lib):
    """testset "csr_from_raw" (test/runtests.jl:3157-3224), through the C
    ABI: the same 3 x 3 matrix given one-based and zero-based arrives as
    the same CSR (read back as the coarsest matrix, 0-based) with A * 1 =
    (1, 0, 1); a zero-based 50 x 50 tridiagonal solves to 1e-6 with the
    default configuration; index_base 2 is rejected."""
    p = lambda a: a.ctypes.data_as(draugr._lib.C.c_void_p)
    cfg = draugr.config_handle(draugr.AMGConfig())
    v = np.array([2.0, -1.0, -1.0, 2.0, -1.0, -1.0, 2.0])
    got = []
    for base, rp, ci in ((1, [1, 3, 6, 8], [1, 2, 1, 2, 3, 2, 3]), (0, [0, 2, 5, 7], [0, 1, 0, 1, 2, 1, 2])):
        rp, ci = np.array(rp, np.int32), np.array(ci, np.int32)
        h = lib.draugr_b200_setup_host(3, 7, p(rp), p(ci), p(v), cfg, base, 1)
        assert h > 0, draugr.last_error()
        H = draugr.Hierarchy(h, 3, None)
        assert H.nlevels == 0
        A = sp.csr_matrix((H.export(-1, "C_nzval"), H.export(-1, "C_colval"), H.export(-1, "C_rowptr")),
                          shape=(3, 3))
        assert (A[0, 0], A[0, 1], A[1, 0], A[1, 1], A[2, 2]) == (2.0, -1.0, -1.0, 2.0, 2.0)
        assert np.array_equal(A @ np.ones(3), [1.0, 0.0, 1.0])
        got.append(A)
        H.free()
    assert (got[0] != got[1]).nnz == 0
    n = 50
    T = sp.diags([np.full(n - 1, -1.0), np.full(n, 2.0), np.full(n - 1, -1.0)], [-1, 0, 1], format="csr")
    h = draugr.amg_setup(T, draugr.AMGConfig(), on_device=False)
    O = oracle.OracleHierarchy(h)
    x, _, _ = O.solve(np.zeros(n), np.ones(n), tol=1e-6, maxiter=100)
    assert np.linalg.norm(np.ones(n) - T @ x) / np.sqrt(n) < 1e-6
    rp, ci = np.array([1, 3, 5], np.int32), np.array([1, 2, 1, 2], np.int32)
    assert lib.draugr_b200_setup_host(2, 4, p(rp), p(ci), p(np.array([1.0, 2.0, 3.0, 4.0])), cfg, 2, 1) == -1
    assert "index_base" in draugr.last_error()


def test_full_resetup_and_direct_solve_testsets():
    """testsets "AMG Resetup - partial=false", "... with
    allow_partial_resetup", "... partial=false, allow_partial_resetup=false"
    and "Small System Direct Solve" (test/runtests.jl:467-547), on host-only
    hierarchies: a full resetup rebuilds the hierarchy from the new values
    (the solve then meets 1e-8 on 2A and differs from the first), keeps or
    drops the Galerkin maps as allow_partial_resetup says, and a system no
    larger than max_coarse_size has no levels and is solved directly to
    1e-10.  (The partial resetup that follows in the second testset runs on
    the GPU and is covered there.)"""
    A = problems.poisson2d(10)
    cfg = draugr.AMGConfig(coarsening=draugr.AggregationCoarsening())
    b = np.random.default_rng(21).uniform(0, 1, 100)

    def solve(h, M):
        x, _, _ = oracle.OracleHierarchy(h).solve(np.zeros(100), b, tol=1e-8, maxiter=200)
        assert np.linalg.norm(b - M @ x) / np.linalg.norm(b) < 1e-8
        return x

    h = draugr.amg_setup(A, cfg, on_device=False)
    x1 = solve(h, A)
    A2 = A.copy()
    A2.data = A2.data * 2.0
    draugr.amg_resetup(h, A2, cfg, partial=False)
    x2 = solve(h, A2)
    assert not np.allclose(x1, x2, atol=1e-6)
    h = draugr.amg_setup(A, cfg, allow_partial_resetup=False, on_device=False)
    assert all(h.level_info(l)[6] == -1 for l in range(h.nlevels))
    draugr.amg_resetup(h, A, cfg, partial=False, allow_partial_resetup=True)
    assert h.nlevels > 0 and all(h.level_info(l)[6] >= 0 for l in range(h.nlevels))
    h = draugr.amg_setup(A, cfg, on_device=False)
    draugr.amg_resetup(h, A, cfg, partial=False, allow_partial_resetup=False)
    assert all(h.level_info(l)[6] == -1 for l in range(h.nlevels))
    solve(h, A)
    A5 = problems.poisson1d(5)
    h = draugr.amg_setup(A5, draugr.AMGConfig(max_coarse_size=10), on_device=False)
    assert h.nlevels == 0
    x, _, _ = oracle.OracleHierarchy(h).solve(np.zeros(5), np.ones(5), tol=1e-10)
    assert np.linalg.norm(np.ones(5) - A5 @ x) < 1e-10


def test_sparse_csc_input():
    """testset "SparseMatrixCSC convenience" (test/runtests.jl:3076-3106),
    in the Python mirror: a CSC matrix sets up the same hierarchy as its
    CSR form, solves the 50 x 50 tridiagonal system to 1e-6, and after new
    values (4, -2) the solve takes fewer than 100 cycles."""
    n = 50
    T = sp.diags([np.full(n - 1, -1.0), np.full(n, 2.0), np.full(n - 1, -1.0)], [-1, 0, 1], format="csc")
    cfg = draugr.AMGConfig(max_coarse_size=10)
    h = draugr.amg_setup(T, cfg, on_device=False)
    h2 = draugr.amg_setup(T.tocsr(), cfg, on_device=False)
    assert h.nlevels == h2.nlevels > 0
    for l in range(h.nlevels):
        for what in ("A_colval", "A_nzval", "P_colval", "P_nzval"):
            assert np.array_equal(h.export(l, what), h2.export(l, what))
    O = oracle.OracleHierarchy(h, with_rmaps=True)
    b = np.ones(n)
    x, _, _ = O.solve(np.zeros(n), b, tol=1e-6, maxiter=100)
    assert np.linalg.norm(b - T @ x) / np.linalg.norm(b) < 1e-6
    O.resetup((2.0 * T).tocsr().data)
    x, it, _ = O.solve(np.zeros(n), b, tol=1e-6, maxiter=100)
    assert it < 100 and np.linalg.norm(b - 2.0 * (T @ x)) / np.linalg.norm(b) < 1e-6


def _split_top(s):
    """Split s at commas outside (), {} and []."""
    out, depth, cur = [], 0, ""
    for ch in s:
        if ch in "({[":
            depth += 1
        elif ch in ")}]":
            depth -= 1
        if ch == "," and depth == 0:
            out.append(cur.strip())
            cur = ""
        else:
            cur += ch
    if cur.strip():
        out.append(cur.strip())
    return out


def _c_params():
    """name -> (return type, [parameter types]) of every declared function."""
    decls = {}
    for h in HEADERS:
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"([A-Za-z_][A-Za-z0-9_ \*]*?)\b(draugr_[A-Za-z0-9_]+|init_julia|shutdown_julia)"
                             r"\s*\(([^)]*)\)\s*;", text):
            params = [p.strip() for p in m.group(3).split(",") if p.strip() and p.strip() != "void"]
            decls[m.group(2)] = (m.group(1).strip(), params)
    return decls


def test_julia_bindings_match_the_c_header():
    """The Julia module cannot run here (no Julia in the image), so its
    ccall signatures are checked against include/*.h: every symbol is
    declared, with the same number of arguments, each of a matching kind
    (Int32 / Int64 / Float64 / pointer / string), and a matching return."""
    jl = "\n".join(f.read_text() for f in sorted((ROOT / "draugr.jl_b200" / "julia").rglob("*.jl")))
    decls = _c_params()

    def kind_c(t):
        t = t.replace("const", "").strip()
        if "char" in t and "*" in t:
            return "str"
        if "*" in t:
            return "ptr"
        base = t.split()[0]
        return {"int32_t": "i32", "int64_t": "i64", "double": "f64", "float": "f32", "void": "void"}[base]

    def kind_jl(t):
        if t.startswith(("Ptr", "CuPtr", "Ref")):
            return "ptr"
        if t == "Cstring":
            return "str"
        return {"Int32": "i32", "Int64": "i64", "Float64": "f64", "Float32": "f32", "Cvoid": "void",
                "Nothing": "void"}[t]

    seen = 0
    for m in re.finditer(r"ccall\(", jl):
        depth, i = 0, m.end() - 1
        while True:
            depth += {"(": 1, ")": -1}.get(jl[i], 0)
            if depth == 0:
                break
            i += 1
        args = _split_top(jl[m.end():i])
        name = re.match(r"\(:([A-Za-z0-9_]+)", args[0]).group(1)
        ret, types = args[1], args[2].strip()
        assert types.startswith("(") and types.endswith(")"), name
        jtypes = _split_top(types[1:-1])
        assert name in decls, name
        cret, cparams = decls[name]
        assert len(jtypes) == len(cparams), (name, jtypes, cparams)
        for jt, ct in zip(jtypes, cparams):
            ctype = re.sub(r"\b[A-Za-z_][A-Za-z0-9_]*$", "", ct).strip() or ct
            assert kind_jl(jt) == kind_c(ctype), (name, jt, ct)
        assert kind_jl(ret) == kind_c(cret), (name, ret, cret)
        seen += 1
    assert seen >= 15


def test_julia_rrule_extension_is_declared():
    """The ChainRulesCore rrule for amg_solve_diff lives in a package
    extension (loaded with ChainRulesCore): Project.toml declares it, the
    extension defines the rrule and its pullback calls the device adjoint."""
    jdir = ROOT / "draugr.jl_b200" / "julia"
    proj = (jdir / "Project.toml").read_text()
    assert 'DraugrB200ChainRulesCoreExt = "ChainRulesCore"' in proj and "[weakdeps]" in proj
    ext = (jdir / "ext" / "DraugrB200ChainRulesCoreExt.jl").read_text()
    assert "ChainRulesCore.rrule(::typeof(DraugrB200.amg_solve_diff)" in ext
    assert "DraugrB200.amg_solve_adjoint(" in ext
    src = (jdir / "src" / "DraugrB200.jl").read_text()
    for fn in ("function amg_solve_diff(", "function amg_solve_adjoint(", "function amg_fgmres!(",
               "function amg_refine!("):
        assert fn in src, fn
