"""ORACLE — test infrastructure, not part of the product.

ctypes harness around liboracle.so (oracle.c), the CPU restatement of
Draugr.jl's solve-phase arithmetic.  Only tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline / reference arms use it, as the checker or as
the timed CPU reference; the library in draugr.jl_b200/ never calls it.

OracleHierarchy takes the hierarchy *structure* a product hierarchy exports
(A, P, transpose map, colours of every level and the coarsest LU) — the
shared input of both sides — and runs the reference's cycle, stationary
solve, a textbook PCG and the reference's triple-map Galerkin resetup on it.
"""

from __future__ import annotations

import ctypes as C
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
_lib = None


def build() -> pathlib.Path:
    subprocess.run(["make", "-C", str(HERE)], check=True, capture_output=True)
    return LIB_PATH


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        _lib = C.CDLL(str(LIB_PATH))
        _declare(_lib)
    return _lib


P = C.c_void_p
i32, i64, f64 = C.c_int, C.c_int64, C.c_double


class OLevel(C.Structure):
    _fields_ = [("n", i32), ("nc", i32), ("A_rp", P), ("A_ci", P), ("A_v", P), ("P_rp", P),
                ("P_ci", P), ("P_v", P), ("T_off", P), ("T_rows", P), ("T_pnz", P),
                ("smoother", i32), ("omega", f64), ("invd", P), ("ncolors", i32),
                ("color_off", P), ("color_order", P), ("r", P), ("xc", P), ("bc", P),
                ("tmp", P), ("nz_off", P), ("tpi", P), ("tai", P), ("tpj", P),
                ("cheb_degree", i32), ("cheb_v0", P), ("cheb_coef", P), ("cheb_d", P),
                ("ilu_diag", P), ("ilu_L", P), ("ilu_U", P), ("spai1_M", P)]


class OHier(C.Structure):
    _fields_ = [("nlevels", i32), ("lv", C.POINTER(OLevel)), ("nc", i32), ("dense", P),
                ("lu", P), ("piv", P), ("cx", P), ("cb", P), ("solve_r", P), ("coarse_v", P),
                ("coarse_rp", P), ("coarse_ci", P)]


def _declare(lib):
    sig = {
        "orc_spmv": (None, [i32, P, P, P, P, P]),
        "orc_residual": (None, [i32, P, P, P, P, P, P]),
        "orc_invdiag": (None, [i32, P, P, P, P]),
        "orc_l1_invdiag": (None, [i32, P, P, P]),
        "orc_spai0": (None, [i32, P, P, P, P]),
        "orc_spectral_radius": (f64, [i32, P, P, P, P, P, i32, P]),
        "orc_cheb_coef": (None, [f64, i32, P]),
        "orc_ilu0_factor": (None, [i32, P, P, P, P, P, P]),
        "orc_serial_gs_invdiag": (None, [i32, P, P, P, P]),
        "orc_spai1": (None, [i32, P, P, P, P]),
        "orc_spai1_smooth": (None, [i32, P, P, P, P, P, P, i32, P]),
        "orc_serial_gs": (None, [i32, P, P, P, P, P, P, i32]),
        "orc_ilu0_smooth": (None, [i32, P, P, P, P, P, P, P, P, i32, P]),
        "orc_chebyshev": (None, [i32, P, P, P, P, P, i32, P, P, i32, P, P]),
        "orc_spai0_smooth": (None, [i32, P, P, P, P, P, P, i32, P]),
        "orc_jacobi": (None, [i32, P, P, P, P, f64, P, P, i32, P]),
        "orc_greedy_coloring": (i32, [i32, P, P, P]),
        "orc_color_order": (None, [i32, P, i32, P, P]),
        "orc_gs": (None, [i32, P, P, P, P, i32, P, P, P, P, i32]),
        "orc_transpose_map": (None, [i32, i32, P, P, P, P, P]),
        "orc_restrict": (None, [i32, P, P, P, P, P, P]),
        "orc_prolongate": (None, [i32, P, P, P, P, P]),
        "orc_coarse_sparsity": (i64, [i32, i32, P, P, P, P, P, P, P, P, P, P, P, P, P]),
        "orc_galerkin": (None, [i32, P, P, P, P, P, P, P]),
        "orc_coarsest_dense": (None, [i32, i32, P, P, P, P, P, P, P]),
        "orc_csr_to_dense": (None, [i32, P, P, P, P]),
        "orc_lu_factor": (i32, [i32, P, P]),
        "orc_lu_solve": (None, [i32, P, P, P]),
        "orc_cycle": (None, [C.POINTER(OHier), P, P, i32, i32, i32]),
        "orc_solve": (i32, [C.POINTER(OHier), P, P, i32, i32, i32, f64, i32, P]),
        "orc_pcg": (i32, [C.POINTER(OHier), P, P, i32, i32, i32, f64, i32, P, P]),
        "orc_resetup": (i32, [C.POINTER(OHier), P, i64]),
        "orc_strength_abs": (None, [i32, P, P, P, f64, P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args


def ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


# ---------------------------------------------------------------- array-level helpers
def csr_parts(A):
    A = A.tocsr()
    return (A.shape[0], np.ascontiguousarray(A.indptr, np.int32),
            np.ascontiguousarray(A.indices, np.int32), np.ascontiguousarray(A.data, np.float64))


def spmv(n, rp, ci, v, x):
    y = np.zeros(n)
    load().orc_spmv(n, ptr(rp), ptr(ci), ptr(v), ptr(np.ascontiguousarray(x, np.float64)), ptr(y))
    return y


def residual(n, rp, ci, v, x, b):
    r = np.zeros(n)
    load().orc_residual(n, ptr(rp), ptr(ci), ptr(v), ptr(np.ascontiguousarray(x, np.float64)),
                        ptr(np.ascontiguousarray(b, np.float64)), ptr(r))
    return r


def invdiag(n, rp, ci, v, l1=False):
    d = np.zeros(n)
    if l1:
        load().orc_l1_invdiag(n, ptr(rp), ptr(v), ptr(d))
    else:
        load().orc_invdiag(n, ptr(rp), ptr(ci), ptr(v), ptr(d))
    return d


def spai0(n, rp, ci, v):
    """SPAI(0) diagonal m_i = a_ii / sum_j a_ij^2 (spai0_kernel!)."""
    m = np.zeros(n)
    load().orc_spai0(n, ptr(rp), ptr(ci), ptr(v), ptr(m))
    return m


def spai0_smooth(n, rp, ci, v, m, x, b, steps):
    """`steps` SPAI(0) sweeps x <- x + m (b - A x) (smooth!(::SPAI0Smoother))."""
    x = np.array(x, dtype=np.float64)
    tmp = np.zeros(n)
    load().orc_spai0_smooth(n, ptr(rp), ptr(ci), ptr(v), ptr(np.ascontiguousarray(m, np.float64)), ptr(x),
                            ptr(np.ascontiguousarray(b, np.float64)), steps, ptr(tmp))
    return x


def spectral_radius(n, rp, ci, v, invd, v0, niter=10):
    """Power-iteration estimate of the spectral radius of D^-1 A from the
    normalised start vector v0 (_estimate_spectral_radius)."""
    w = np.zeros(n)
    vv = np.array(v0, dtype=np.float64)
    return load().orc_spectral_radius(n, ptr(rp), ptr(ci), ptr(v), ptr(np.ascontiguousarray(invd, np.float64)),
                                      ptr(vv), niter, ptr(w))


def cheb_coef(rho, degree=3):
    """Chebyshev coefficient table (1/theta, 0, scale_r, scale_d, ...)."""
    c = np.zeros(2 * degree)
    load().orc_cheb_coef(float(rho), degree, ptr(c))
    return c


def spai1(n, rp, ci, v):
    """SPAI(1) values of M on A's pattern (_compute_spai1!, the reference's
    loop over every row for every row: small cases only)."""
    M = np.zeros(len(ci))
    load().orc_spai1(n, ptr(rp), ptr(ci), ptr(v), ptr(M))
    return M


def spai1_smooth(n, rp, ci, v, M, x, b, steps):
    """`steps` SPAI(1) steps x <- x + M (b - A x) (smooth!(::SPAI1Smoother))."""
    x = np.array(x, dtype=np.float64)
    r = np.zeros(n)
    load().orc_spai1_smooth(n, ptr(rp), ptr(ci), ptr(v), ptr(np.ascontiguousarray(M, np.float64)), ptr(x),
                            ptr(np.ascontiguousarray(b, np.float64)), steps, ptr(r))
    return x


def serial_gs_invdiag(n, rp, ci, v):
    """1/a_ii for the serial Gauss-Seidel smoother (_serial_gs_compute_invdiag!)."""
    d = np.zeros(n)
    load().orc_serial_gs_invdiag(n, ptr(rp), ptr(ci), ptr(v), ptr(d))
    return d


def serial_gs(n, rp, ci, v, invd, x, b, steps):
    """`steps` in-place forward Gauss-Seidel sweeps in row order (_serial_gs_sweep!)."""
    x = np.array(x, dtype=np.float64)
    load().orc_serial_gs(n, ptr(rp), ptr(ci), ptr(v), ptr(np.ascontiguousarray(invd, np.float64)), ptr(x),
                         ptr(np.ascontiguousarray(b, np.float64)), steps)
    return x


def ilu0_diag(n, rp, ci):
    """Position of each row's diagonal entry (_ilu0_diag_indices)."""
    d = np.zeros(n, np.int32)
    for i in range(n):
        row = ci[rp[i]:rp[i + 1]]
        d[i] = rp[i] + int(np.nonzero(row == i)[0][0])
    return d


def ilu0_factor(n, rp, ci, v, diag):
    """ILU(0) factors (L strictly lower, U upper with the diagonal) on A's
    pattern (_ilu0_factorize!)."""
    L, U = np.zeros(len(ci)), np.zeros(len(ci))
    load().orc_ilu0_factor(n, ptr(rp), ptr(ci), ptr(v), ptr(np.ascontiguousarray(diag, np.int32)), ptr(L),
                           ptr(U))
    return L, U


def ilu0_smooth(n, rp, ci, v, diag, L, U, x, b, steps):
    """`steps` ILU(0) smoothing steps (smooth!(::SerialILU0Smoother))."""
    x = np.array(x, dtype=np.float64)
    t = np.zeros(n)
    load().orc_ilu0_smooth(n, ptr(rp), ptr(ci), ptr(v), ptr(np.ascontiguousarray(diag, np.int32)),
                           ptr(np.ascontiguousarray(L, np.float64)), ptr(np.ascontiguousarray(U, np.float64)),
                           ptr(x), ptr(np.ascontiguousarray(b, np.float64)), steps, ptr(t))
    return x


def chebyshev(n, rp, ci, v, invd, coef, x, b, steps):
    """`steps` Chebyshev applications (smooth!(::ChebyshevSmoother))."""
    x = np.array(x, dtype=np.float64)
    coef = np.ascontiguousarray(coef, np.float64)
    r, d = np.zeros(n), np.zeros(n)
    load().orc_chebyshev(n, ptr(rp), ptr(ci), ptr(v), ptr(np.ascontiguousarray(invd, np.float64)), ptr(coef),
                         len(coef) // 2, ptr(x), ptr(np.ascontiguousarray(b, np.float64)), steps, ptr(r), ptr(d))
    return x


def jacobi(n, rp, ci, v, invd, omega, x, b, steps):
    x = np.array(x, dtype=np.float64)
    tmp = np.zeros(n)
    load().orc_jacobi(n, ptr(rp), ptr(ci), ptr(v), ptr(invd), omega, ptr(x),
                      ptr(np.ascontiguousarray(b, np.float64)), steps, ptr(tmp))
    return x


def greedy_coloring(n, rp, ci):
    colors = np.zeros(n, np.int32)
    nc = load().orc_greedy_coloring(n, ptr(rp), ptr(ci), ptr(colors))
    off = np.zeros(nc + 1, np.int32)
    order = np.zeros(n, np.int32)
    load().orc_color_order(n, ptr(colors), nc, ptr(off), ptr(order))
    return colors, nc, off, order


def gs(n, rp, ci, v, invd, ncol, off, order, x, b, steps):
    x = np.array(x, dtype=np.float64)
    load().orc_gs(n, ptr(rp), ptr(ci), ptr(v), ptr(invd), ncol, ptr(off), ptr(order), ptr(x),
                  ptr(np.ascontiguousarray(b, np.float64)), steps)
    return x


def transpose_map(nf, nc, prp, pci):
    nnz = int(prp[nf])
    off = np.zeros(nc + 1, np.int32)
    rows = np.zeros(nnz, np.int32)
    pnz = np.zeros(nnz, np.int32)
    load().orc_transpose_map(nf, nc, ptr(prp), ptr(pci), ptr(off), ptr(rows), ptr(pnz))
    return off, rows, pnz


def restrict(nc, off, rows, pnz, pv, r):
    bc = np.zeros(nc)
    load().orc_restrict(nc, ptr(off), ptr(rows), ptr(pnz), ptr(pv),
                        ptr(np.ascontiguousarray(r, np.float64)), ptr(bc))
    return bc


def prolongate(nf, prp, pci, pv, xc, x):
    x = np.array(x, dtype=np.float64)
    load().orc_prolongate(nf, ptr(prp), ptr(pci), ptr(pv), ptr(np.ascontiguousarray(xc, np.float64)),
                          ptr(x))
    return x


def coarse_sparsity(nf, nc, arp, aci, av, prp, pci, pv):
    """compute_coarse_sparsity: (c_rp, c_ci, c_v, nz_off, tpi, tai, tpj)."""
    lib = load()
    c_rp = np.zeros(nc + 1, np.int32)
    nt = lib.orc_coarse_sparsity(nf, nc, ptr(arp), ptr(aci), ptr(av), ptr(prp), ptr(pci), ptr(pv),
                                 ptr(c_rp), None, None, None, None, None, None)
    nnzc = int(c_rp[nc])
    c_ci = np.zeros(nnzc, np.int32)
    c_v = np.zeros(nnzc)
    nz_off = np.zeros(nnzc + 1, np.int64)
    tpi = np.zeros(max(nt, 1), np.int32)
    tai = np.zeros(max(nt, 1), np.int32)
    tpj = np.zeros(max(nt, 1), np.int32)
    lib.orc_coarse_sparsity(nf, nc, ptr(arp), ptr(aci), ptr(av), ptr(prp), ptr(pci), ptr(pv),
                            ptr(c_rp), ptr(c_ci), ptr(c_v), ptr(nz_off), ptr(tpi), ptr(tai), ptr(tpj))
    return c_rp, c_ci, c_v, nz_off, tpi, tai, tpj


def lu_factor(M):
    """Column-major LU of a dense matrix: (lu as an n x n array, piv, info)."""
    n = M.shape[0]
    a = np.ascontiguousarray(np.asarray(M, dtype=np.float64).T).ravel()  # column-major
    piv = np.zeros(n, np.int32)
    info = load().orc_lu_factor(n, ptr(a), ptr(piv))
    return a.reshape(n, n).T, piv, info


def strength_abs(n, rp, ci, v, theta):
    s = np.zeros(len(ci), np.uint8)
    load().orc_strength_abs(n, ptr(rp), ptr(ci), ptr(v), theta, ptr(s))
    return s


# ---------------------------------------------------------------- structure files
# The arrays OracleHierarchy reads from a hierarchy, per level and for the
# coarsest level, so that the structure can be written by one process and
# the reference's solve phase run on it in another that loads nothing but
# the oracle.
_LEVEL_ARRAYS = ("A_rowptr", "A_colval", "A_nzval", "P_rowptr", "P_colval", "P_nzval", "T_offsets",
                 "T_rows", "T_pnz", "invdiag", "color_offsets", "color_order", "omega")
_SMOOTHER_ARRAYS = {8: ("cheb_v0", "cheb_coef"), 4: ("spai1_M",), 9: ("ilu_diag", "ilu_L", "ilu_U"),
                    10: ("ilu_diag", "ilu_L", "ilu_U")}
_COARSE_ARRAYS = ("C_rowptr", "C_colval", "C_nzval")


def save_structure(h, path, **extra):
    """Write the hierarchy structure `h` exposes (nlevels, level_info,
    export) to an uncompressed .npz at `path`, with any extra arrays given
    as keyword arguments (e.g. the right-hand side)."""
    d = {"nlevels": np.array([h.nlevels], np.int64)}
    for l in list(range(h.nlevels)) + [-1]:
        info = np.asarray(h.level_info(l), np.int64)
        d[f"L{l}_info"] = info
        names = _COARSE_ARRAYS if l < 0 else _LEVEL_ARRAYS + _SMOOTHER_ARRAYS.get(int(info[4]), ())
        for nm in names:
            d[f"L{l}_{nm}"] = h.export(l, nm)
    for k, v in extra.items():
        d[f"extra_{k}"] = np.asarray(v)
    np.savez(path, **d)


class StructureFile:
    """A hierarchy structure read back from save_structure's file, with the
    nlevels / level_info / export interface OracleHierarchy takes."""

    def __init__(self, path):
        z = np.load(path)
        self._d = {k: z[k] for k in z.files}
        self.nlevels = int(self._d["nlevels"][0])

    def level_info(self, lvl):
        return self._d[f"L{lvl}_info"]

    def export(self, lvl, what):
        return self._d[f"L{lvl}_{what}"]

    def extra(self, name):
        return self._d[f"extra_{name}"]


# ---------------------------------------------------------------- hierarchy mirror
SMOOTHER_KIND = {0: "jacobi", 1: "colored_gs", 2: "serial_gs", 3: "spai0", 4: "spai1", 5: "l1_jacobi",
                 6: "l1_colored_gs", 7: "l1_serial_gs", 8: "chebyshev", 9: "ilu0", 10: "serial_ilu0"}


class OracleHierarchy:
    """The reference's solve phase on the structure of a product hierarchy.

    `h` is a draugr.Hierarchy (possibly host-only).  Level values are copied;
    with with_rmaps=True each level also gets the reference's Galerkin
    RestrictionMap (built by the oracle from that level's A and P) so that
    resetup() can run the reference's triple-map product.
    """

    def __init__(self, h, with_rmaps: bool = False):
        self._keep = []
        self.with_rmaps = with_rmaps
        nl = h.nlevels
        self.nlevels = nl
        levels = (OLevel * max(nl, 1))()
        self.levels_np = []
        for l in range(nl):
            info = h.level_info(l)
            n, nc = int(info[0]), int(info[2])
            d = dict(
                A_rp=h.export(l, "A_rowptr"), A_ci=h.export(l, "A_colval"),
                A_v=h.export(l, "A_nzval").copy(), P_rp=h.export(l, "P_rowptr"),
                P_ci=h.export(l, "P_colval"), P_v=h.export(l, "P_nzval"),
                T_off=h.export(l, "T_offsets"), T_rows=h.export(l, "T_rows"),
                T_pnz=h.export(l, "T_pnz"), invd=h.export(l, "invdiag").copy(),
                color_off=h.export(l, "color_offsets"), color_order=h.export(l, "color_order"),
                r=np.zeros(n), xc=np.zeros(nc), bc=np.zeros(nc), tmp=np.zeros(n))
            sk = int(info[4])
            if sk not in SMOOTHER_KIND:
                raise ValueError(f"smoother kind {sk} has no oracle")
            omega = float(h.export(l, "omega")[0])
            L = levels[l]
            L.n, L.nc, L.smoother, L.omega = n, nc, sk, omega
            if sk == 8:
                d.update(cheb_v0=h.export(l, "cheb_v0"), cheb_coef=h.export(l, "cheb_coef").copy(),
                         cheb_d=np.zeros(n))
                L.cheb_degree = len(d["cheb_coef"]) // 2
                L.cheb_v0, L.cheb_coef, L.cheb_d = ptr(d["cheb_v0"]), ptr(d["cheb_coef"]), ptr(d["cheb_d"])
            if sk == 4:
                d.update(spai1_M=h.export(l, "spai1_M").copy())
                L.spai1_M = ptr(d["spai1_M"])
            if sk in (9, 10):
                d.update(ilu_diag=h.export(l, "ilu_diag"), ilu_L=h.export(l, "ilu_L").copy(),
                         ilu_U=h.export(l, "ilu_U").copy())
                L.ilu_diag, L.ilu_L, L.ilu_U = ptr(d["ilu_diag"]), ptr(d["ilu_L"]), ptr(d["ilu_U"])
            L.ncolors = int(info[5])
            for k in ("A_rp", "A_ci", "A_v", "P_rp", "P_ci", "P_v", "T_off", "T_rows", "T_pnz",
                      "invd", "color_off", "color_order", "r", "xc", "bc", "tmp"):
                setattr(L, k, ptr(d[k]))
            self.levels_np.append(d)
        self.nc = int(h.level_info(-1)[0])
        self.coarse_rp = h.export(-1, "C_rowptr")
        self.coarse_ci = h.export(-1, "C_colval")
        self.coarse_v = h.export(-1, "C_nzval").copy()
        self.dense = np.zeros(self.nc * self.nc)
        load().orc_csr_to_dense(self.nc, ptr(self.coarse_rp), ptr(self.coarse_ci),
                                ptr(self.coarse_v), ptr(self.dense))
        self.lu = self.dense.copy()
        self.piv = np.zeros(self.nc, np.int32)
        info = load().orc_lu_factor(self.nc, ptr(self.lu), ptr(self.piv))
        if info:
            raise ZeroDivisionError(f"SingularException({info})")
        self.cx = np.zeros(self.nc)
        self.cb = np.zeros(self.nc)
        n0 = int(h.level_info(0)[0]) if nl else self.nc
        self.n = n0
        self.solve_r = np.zeros(n0)
        if with_rmaps:
            for l in range(nl - 1):
                d = self.levels_np[l]
                nf, ncl = levels[l].n, levels[l].nc
                c_rp, c_ci, c_v, nz_off, tpi, tai, tpj = coarse_sparsity(
                    nf, ncl, d["A_rp"], d["A_ci"], d["A_v"], d["P_rp"], d["P_ci"], d["P_v"])
                d.update(nz_off=nz_off, tpi=tpi, tai=tai, tpj=tpj, c_rp=c_rp, c_ci=c_ci)
                L = levels[l]
                L.nz_off, L.tpi, L.tai, L.tpj = ptr(nz_off), ptr(tpi), ptr(tai), ptr(tpj)
        H = OHier()
        H.nlevels = nl
        H.lv = C.cast(levels, C.POINTER(OLevel))
        H.nc = self.nc
        H.dense, H.lu, H.piv = ptr(self.dense), ptr(self.lu), ptr(self.piv)
        H.cx, H.cb, H.solve_r = ptr(self.cx), ptr(self.cb), ptr(self.solve_r)
        H.coarse_v, H.coarse_rp, H.coarse_ci = (ptr(self.coarse_v), ptr(self.coarse_rp),
                                                ptr(self.coarse_ci))
        self._levels = levels
        self.H = H

    # solve phase -------------------------------------------------------
    def cycle(self, x, b, pre=1, post=1, w=False):
        x = np.array(x, dtype=np.float64)
        b = np.ascontiguousarray(b, np.float64)
        load().orc_cycle(C.byref(self.H), ptr(x), ptr(b), pre, post, int(w))
        return x

    def solve(self, x, b, pre=1, post=1, w=False, tol=1e-10, maxiter=100):
        x = np.array(x, dtype=np.float64)
        b = np.ascontiguousarray(b, np.float64)
        rel = C.c_double(0)
        it = load().orc_solve(C.byref(self.H), ptr(x), ptr(b), pre, post, int(w), tol, maxiter,
                              C.byref(rel))
        return x, it, rel.value

    def pcg(self, x, b, pre=1, post=1, w=False, tol=1e-8, maxiter=500):
        x = np.array(x, dtype=np.float64)
        b = np.ascontiguousarray(b, np.float64)
        work = np.zeros(4 * self.n)
        rel = C.c_double(0)
        it = load().orc_pcg(C.byref(self.H), ptr(x), ptr(b), pre, post, int(w), tol, maxiter,
                            C.byref(rel), ptr(work))
        return x, it, rel.value

    def resetup(self, new_values):
        if self.nlevels > 1 and not self.with_rmaps:
            raise ValueError("resetup of a hierarchy with more than one level needs with_rmaps=True")
        v = np.ascontiguousarray(new_values, np.float64)
        info = load().orc_resetup(C.byref(self.H), ptr(v), len(v))
        if info:
            raise ZeroDivisionError(f"SingularException({info})")

    def level_values(self, l):
        return self.levels_np[l]["A_v"]
