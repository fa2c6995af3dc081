"""Seeded synthetic test problems (scipy CSR, sorted columns, float64).

poisson1d / poisson2d follow the fixtures of Draugr.jl's test suite
(test/runtests.jl:13-48: tridiagonal [-1 2 -1], 5-point with diagonal 4,
Dirichlet boundaries dropped).  The 3-D operators are the workloads the
benchmarks are quoted on:

* heterogeneous_diffusion_3d: 7-point finite-volume diffusion with a
  log-normal permeability κ = exp(g), g a Gaussian random field (white noise
  filtered by a Gaussian kernel whose standard deviation is the correlation
  length, rescaled to standard deviation σ), harmonic-mean face
  transmissibilities 2κaκb/(κa+κb), Dirichlet faces with 2κ.  SPD M-matrix.
* anisotropic_27pt: trilinear (Q1) finite elements of -∇·(κ diag(1,1,ε_z) ∇u)
  with one κ per element, n³ interior nodes, zero Dirichlet values on the
  surrounding node layer; (3n-2)³ nonzeros.
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def poisson1d(n: int) -> sp.csr_matrix:
    main = 2.0 * np.ones(n)
    off = -1.0 * np.ones(n - 1)
    return sp.diags([off, main, off], [-1, 0, 1], format="csr").sorted_indices()


def poisson2d(nx: int, ny: int | None = None) -> sp.csr_matrix:
    ny = nx if ny is None else ny
    T = lambda m: sp.diags([-np.ones(m - 1), 2 * np.ones(m), -np.ones(m - 1)], [-1, 0, 1])
    A = sp.kron(sp.identity(ny), T(nx)) + sp.kron(T(ny), sp.identity(nx))
    A = sp.csr_matrix(A)
    A.sort_indices()
    return A


def poisson3d(n: int) -> sp.csr_matrix:
    T = sp.diags([-np.ones(n - 1), 2 * np.ones(n), -np.ones(n - 1)], [-1, 0, 1])
    I = sp.identity(n)
    A = sp.kron(sp.kron(I, I), T) + sp.kron(sp.kron(I, T), I) + sp.kron(sp.kron(T, I), I)
    A = sp.csr_matrix(A)
    A.sort_indices()
    return A


def _stencil_csr(n3: int, offsets, vals, valid) -> sp.csr_matrix:
    """Assemble CSR from per-row stencil arrays (offsets ascending)."""
    offs = np.asarray(offsets, dtype=np.int64)
    V = np.stack(vals, axis=1)          # (N, S)
    M = np.stack(valid, axis=1)         # (N, S)
    rows = np.arange(n3, dtype=np.int64)[:, None]
    cols = rows + offs[None, :]
    counts = M.sum(axis=1)
    rp = np.zeros(n3 + 1, dtype=np.int64)
    np.cumsum(counts, out=rp[1:])
    ci = cols[M].astype(np.int32)
    v = V[M].astype(np.float64)
    return sp.csr_matrix((v, ci, rp.astype(np.int32)), shape=(n3, n3))


def gaussian_field(n: int, sigma: float, corr_len: float, rng: np.random.Generator) -> np.ndarray:
    """Gaussian random field on an n³ grid (x fastest), std sigma."""
    w = rng.standard_normal((n, n, n))
    k = np.fft.fftfreq(n)
    kz, ky, kx = np.meshgrid(k, k, k, indexing="ij")
    filt = np.exp(-2.0 * np.pi ** 2 * corr_len ** 2 * (kx ** 2 + ky ** 2 + kz ** 2))
    g = np.fft.ifftn(np.fft.fftn(w) * filt).real
    g -= g.mean()
    g *= sigma / g.std()
    return g  # indexed [z, y, x]


def heterogeneous_diffusion_3d(n: int, sigma: float = 3.0, corr_len: float = 8.0,
                               seed: int = 0) -> sp.csr_matrix:
    rng = np.random.default_rng(seed)
    kappa = np.exp(gaussian_field(n, sigma, corr_len, rng))  # [z, y, x]
    N = n ** 3

    def face(axis):
        a = kappa
        b = np.roll(kappa, -1, axis=axis)
        t = 2.0 * a * b / (a + b)  # between cell and its + neighbour along axis
        return t

    # transmissibilities to the +neighbour along x (axis 2), y (1), z (0)
    tx, ty, tz = face(2), face(1), face(0)
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    kb = 2.0 * kappa
    # minus / plus neighbours per axis, with Dirichlet boundary faces
    t_xp = np.where(x < n - 1, tx, kb)
    t_xm = np.where(x > 0, np.roll(tx, 1, axis=2), kb)
    t_yp = np.where(y < n - 1, ty, kb)
    t_ym = np.where(y > 0, np.roll(ty, 1, axis=1), kb)
    t_zp = np.where(z < n - 1, tz, kb)
    t_zm = np.where(z > 0, np.roll(tz, 1, axis=0), kb)
    diag = t_xp + t_xm + t_yp + t_ym + t_zp + t_zm
    f = lambda a: a.reshape(N)
    offsets = [-n * n, -n, -1, 0, 1, n, n * n]
    vals = [-f(t_zm), -f(t_ym), -f(t_xm), f(diag), -f(t_xp), -f(t_yp), -f(t_zp)]
    valid = [f(z > 0), f(y > 0), f(x > 0), np.ones(N, bool), f(x < n - 1), f(y < n - 1),
             f(z < n - 1)]
    return _stencil_csr(N, offsets, vals, valid)


_S = np.array([[1.0, -1.0], [-1.0, 1.0]])
_M = np.array([[2.0, 1.0], [1.0, 2.0]]) / 6.0


def q1_element_entry(lx, ly, lz, mx, my, mz, k=(1.0, 1.0, 1.0)):
    """Entry (local node l, local node m) of the Q1 stiffness of diag(k)."""
    return (k[0] * _S[lx, mx] * _M[ly, my] * _M[lz, mz]
            + k[1] * _M[lx, mx] * _S[ly, my] * _M[lz, mz]
            + k[2] * _M[lx, mx] * _M[ly, my] * _S[lz, mz])


def anisotropic_27pt(n: int, eps_z: float = 1e-3, kappa_elem: np.ndarray | None = None
                     ) -> sp.csr_matrix:
    """27-point Q1 operator; kappa_elem has shape (n+1,)*3 ([z, y, x]); the
    element (a, b, c) spans nodes a..a+1 (node indices -1..n, -1 and n are
    the Dirichlet layer)."""
    if kappa_elem is None:
        kappa_elem = np.ones((n + 1, n + 1, n + 1))
    N = n ** 3
    kk = (1.0, 1.0, eps_z)
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    offsets, vals, valid = [], [], []
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                acc = np.zeros((n, n, n))
                # elements containing node p and node p+d: per axis the element
                # index e = p-1+s, s in {0,1}, must contain both p and p+d
                for sz in (0, 1):
                    for sy in (0, 1):
                        for sx in (0, 1):
                            lz, ly, lx = 1 - sz, 1 - sy, 1 - sx   # local index of p
                            mz, my, mx = lz + dz, ly + dy, lx + dx  # local index of p+d
                            if not (0 <= mz <= 1 and 0 <= my <= 1 and 0 <= mx <= 1):
                                continue
                            w = q1_element_entry(lx, ly, lz, mx, my, mz, kk)
                            # element index (a,b,c) = p - 1 + s  ->  kappa_elem[p + s]
                            ke = kappa_elem[sz:sz + n, sy:sy + n, sx:sx + n]
                            acc += w * ke
                ok = ((x + dx >= 0) & (x + dx < n) & (y + dy >= 0) & (y + dy < n)
                      & (z + dz >= 0) & (z + dz < n))
                offsets.append(dz * n * n + dy * n + dx)
                vals.append(acc.reshape(N))
                valid.append(ok.reshape(N))
    order = np.argsort(offsets)
    return _stencil_csr(N, [offsets[i] for i in order], [vals[i] for i in order],
                        [valid[i] for i in order])


def _csr_with_jacobian(n, v_rc, vals, d_rc, d_cell, d_vals, ncells):
    """CSR matrix from value contributions (rows, cols, vals) and the sparse
    Jacobian J (nnz x ncells) of its values with respect to cell
    coefficients from derivative contributions (rows, cols, cells, dvals)."""
    A = sp.csr_matrix((vals, v_rc), shape=(n, n))
    A.sum_duplicates()
    A.sort_indices()
    rid = np.repeat(np.arange(n, dtype=np.int64), np.diff(A.indptr))
    keys = rid * n + A.indices  # ascending: CSR order
    dk = d_rc[0].astype(np.int64) * n + d_rc[1]
    pos = np.searchsorted(keys, dk)
    assert np.array_equal(keys[pos], dk)
    J = sp.csr_matrix((d_vals, (pos, d_cell)), shape=(A.nnz, ncells))
    J.sum_duplicates()
    return A, J


def _faces(shape):
    """Interior faces (a, b) along each axis of a cell grid, and boundary
    cells (one entry per boundary face)."""
    idx = np.arange(int(np.prod(shape))).reshape(shape)
    inner, bnd = [], []
    for axis in range(len(shape)):
        m = shape[axis]
        a = np.take(idx, np.arange(m - 1), axis=axis).ravel()
        b = np.take(idx, np.arange(1, m), axis=axis).ravel()
        inner.append((axis, a, b))
        for side in (0, m - 1):
            bnd.append(np.take(idx, [side], axis=axis).ravel())
    return inner, bnd


# Position in CSR order of every value contribution of _fv_system, per cell
# grid shape (the contributions' rows and columns depend only on the shape).
_FV_POSITIONS = {}


def _fv_system(kappa, flux=None, values_only=False):
    """Finite-volume operator of -div(kappa grad u) + div(w u) (upwind) with
    Dirichlet boundary on a unit-spaced cell grid; flux[axis] gives, per
    interior face (a, b) of that axis, the flux from a to b (None: no
    convection).  Returns (A, J), or with values_only the values of A in
    CSR order alone (the pattern depends only on the grid shape; the
    positions of the contributions are computed once per shape)."""
    shape = kappa.shape
    n = kappa.size
    k = kappa.ravel()
    inner, bnd = _faces(shape)
    vr, vcol, vv, dr, dcol, dcell, dv = [], [], [], [], [], [], []

    def val(r, c, x):
        vr.append(r); vcol.append(c); vv.append(x)

    def der(r, c, cell, x):
        dr.append(r); dcol.append(c); dcell.append(cell); dv.append(x)

    for axis, a, b in inner:
        ka, kb = k[a], k[b]
        T = 2 * ka * kb / (ka + kb)
        dTa = 2 * kb * kb / (ka + kb) ** 2
        dTb = 2 * ka * ka / (ka + kb) ** 2
        F = flux[axis] if flux is not None else np.zeros(len(a))
        out_a, out_b = np.maximum(F, 0.0), np.maximum(-F, 0.0)
        for r, c, sgn, cv in ((a, a, 1.0, out_a), (b, b, 1.0, out_b), (a, b, -1.0, out_b), (b, a, -1.0, out_a)):
            val(r, c, sgn * T + (cv if sgn > 0 else -cv))
            der(r, c, a, sgn * dTa)
            der(r, c, b, sgn * dTb)
    for c in bnd:
        val(c, c, 2 * k[c])
        der(c, c, c, np.full(len(c), 2.0))
    cat = np.concatenate
    if values_only:
        pos = _FV_POSITIONS.get(shape)
        if pos is None:
            keys = cat(vr).astype(np.int64) * n + cat(vcol)
            uniq, inv = np.unique(keys, return_inverse=True)
            _FV_POSITIONS[shape] = pos = (inv, len(uniq))
        return np.bincount(pos[0], weights=cat(vv), minlength=pos[1])
    return _csr_with_jacobian(n, (cat(vr), cat(vcol)), cat(vv), (cat(dr), cat(dcol)), cat(dcell), cat(dv), n)


def fv_diffusion_3d(kappa: np.ndarray, values_only: bool = False):
    """Cell-centred finite volumes for -div(kappa grad u) on the m^3 grid of
    kappa ([z, y, x]), harmonic face transmissibilities, Dirichlet boundary
    (boundary faces 2 kappa).  Symmetric.  Returns (A, J), J = d(values of
    A)/d(kappa) (nnz x m^3); with values_only, A's values in CSR order."""
    return _fv_system(kappa, values_only=values_only)


def convection_diffusion_2d(kappa: np.ndarray, peclet: float = 50.0, seed: int = 0,
                            values_only: bool = False):
    """Upwind finite volumes for -div(kappa grad u) + div(w u) on the m^2
    grid of kappa ([y, x]), Dirichlet boundary.  w is divergence-free, from a
    seeded smooth stream function that vanishes on the boundary (no flow
    through it), scaled so that the largest face flux is `peclet` (the cell
    Peclet number at kappa = 1).  Nonsymmetric M-matrix.  Returns (A, J);
    with values_only, A's values in CSR order."""
    m = kappa.shape[0]
    rng = np.random.default_rng(seed)
    yy, xx = np.meshgrid(np.linspace(0, 1, m + 1), np.linspace(0, 1, m + 1), indexing="ij")
    psi = np.zeros((m + 1, m + 1))
    for _ in range(6):
        kx, ky = rng.integers(1, 5, size=2)
        ph = rng.uniform(0, 2 * np.pi, size=2)
        psi += rng.normal() * np.sin(kx * np.pi * xx + ph[0]) * np.sin(ky * np.pi * yy + ph[1])
    psi *= np.sin(np.pi * xx) * np.sin(np.pi * yy)  # zero on the boundary
    fx = (psi[1:, 1:-1] - psi[:-1, 1:-1])  # x faces between cells (j, i) and (j, i+1): psi(top) - psi(bottom)
    fy = -(psi[1:-1, 1:] - psi[1:-1, :-1])  # y faces between (j, i) and (j+1, i)
    scale = peclet / max(np.abs(fx).max(), np.abs(fy).max(), 1e-300)
    # face order of _faces: axis 0 (y) faces, then axis 1 (x) faces, each raveled [y, x]
    flux = {0: (fy * scale).ravel(), 1: (fx * scale).ravel()}
    return _fv_system(kappa, flux, values_only)


def rhs(n: int, seed: int = 0) -> np.ndarray:
    """b ~ U(-1, 1), seeded."""
    return np.random.default_rng(seed).uniform(-1.0, 1.0, n)
