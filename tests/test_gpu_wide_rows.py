"""Rows whose columns span 65536 indices or more.

The row kernel streams 16-bit column offsets from each tile's smallest
column for most row forms; a row that alone spans 65536 columns or more
cannot be stored that way and is read from the 32-bit columns in global
memory instead (in column order by one thread when the form sums rows in
order, else by the whole block).  These matrices put a few such rows among
ordinary ones, in a form that sums in order (uneven rows averaging fewer
than 32 entries: bit-exact against the oracle) and in a tree form (rows of
more than 32 entries: 1e-12).
"""

import numpy as np
import pytest
import scipy.sparse as sp

import draugr
import oracle
from draugr import problems

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 1e-5


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / (nb if nb > 0 else 1.0)


def with_hubs(A, hubs, far, per_hub, seed):
    """A plus symmetric couplings of each hub row to `per_hub` columns at
    distance >= `far`, diagonal raised to keep A diagonally dominant."""
    rng = np.random.default_rng(seed)
    n = A.shape[0]
    rows, cols = [], []
    for i in hubs:
        js = rng.choice(np.arange(far, n), size=per_hub, replace=False)
        js = (i + js) % n
        rows += [i] * per_hub
        cols += list(js)
    C = sp.csr_matrix((np.full(len(rows), -0.05), (rows, cols)), shape=(n, n))
    C = C + C.T
    D = sp.diags(np.asarray(-C.sum(axis=1)).ravel() + 1e-3)
    B = (A + C + D).tocsr()
    B.sum_duplicates()
    B.sort_indices()
    return B


def banded(n, half, seed):
    """SPD matrix with 2*half+1 entries per row (the tree form)."""
    rng = np.random.default_rng(seed)
    offs = list(range(-half, half + 1))
    diags = [np.full(n - abs(o), -0.1 * (1 + rng.uniform())) if o else np.zeros(n) for o in offs]
    A = sp.diags(diags, offs, shape=(n, n), format="csr")
    A = A + A.T
    A = A + sp.diags(np.asarray(-A.sum(axis=1)).ravel() + 1.0)
    return A.tocsr()


def finest_ops(A, cfg):
    h = draugr.amg_setup(A, cfg)
    O = oracle.OracleHierarchy(h)
    d = O.levels_np[0]
    n = A.shape[0]
    rng = np.random.default_rng(5)
    x = rng.uniform(-1, 1, n)
    b = rng.uniform(-1, 1, n)
    out = {
        "spmv": (h.level_op(0, 0, x), h.level_op(0, 0, x, precision=1),
                 oracle.spmv(n, d["A_rp"], d["A_ci"], d["A_v"], x)),
        "residual": (h.level_op(0, 1, x, b), None,
                     oracle.residual(n, d["A_rp"], d["A_ci"], d["A_v"], x, b)),
    }
    L = O._levels[0]
    ref = oracle.jacobi(n, d["A_rp"], d["A_ci"], d["A_v"], d["invd"], L.omega, x, b, 2)
    out["jacobi"] = (h.level_op(0, 2, x, b, steps=2), h.level_op(0, 2, x, b, steps=2, precision=1), ref)
    return h, out


CFG = draugr.AMGConfig(coarsening=draugr.AggregationCoarsening(), max_coarse_size=50,
                       smoother=draugr.JacobiSmootherType())


def test_wide_rows_in_order_are_bit_exact():
    A = with_hubs(problems.poisson2d(300), hubs=[3, 4000, 45000, 89000], far=70000, per_hub=80, seed=1)
    rp = A.indptr
    span = max(A.indices[rp[i]:rp[i + 1]].max() - A.indices[rp[i]:rp[i + 1]].min() for i in (3, 4000))
    assert span >= 65536 and np.diff(rp).max() > 64 and A.nnz / A.shape[0] < 32
    h, out = finest_ops(A, CFG)
    assert int(h.level_info(0)[7]) == 1  # every row of A summed in column order
    for name, (g64, g32, ref) in out.items():
        assert np.array_equal(g64, ref), name
        if g32 is not None:
            assert rel(g32, ref) < TOL32, name


def test_wide_rows_tree_form():
    A = with_hubs(banded(90000, 20, seed=2), hubs=[7, 30000, 60000], far=70000, per_hub=60, seed=3)
    assert A.nnz / A.shape[0] > 32
    h, out = finest_ops(A, CFG)
    for name, (g64, g32, ref) in out.items():
        assert rel(g64, ref) < TOL64, name
        if g32 is not None:
            assert rel(g32, ref) < TOL32, name
