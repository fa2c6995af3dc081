"""The fused correction on the way up (prolongation, correction and the
first post-smoothing sweep as one pass over Q = P - w D^-1 (A P), with the
residual formed on the way down; the regrouped src/prolongation.jl:742-760
and src/smoothers.jl:78-94).  It runs on levels whose rows are summed in a
tree and whose A*P is no larger than A and P together, so the cycle is
checked against the oracle's at the FP64 tolerance of the tree-summed
levels, after setup and after partial resetups (which rebuild Q from the
new A*P and inverse diagonals)."""

import numpy as np
import pytest

import draugr
import oracle
from draugr import problems

pytestmark = pytest.mark.gpu

TOL64 = 1e-12


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / (nb if nb > 0 else 1.0)


def _fusable(h):
    out = []
    for l in range(1, h.nlevels):
        info = h.level_info(l)
        if int(info[7]) == 0 and int(info[4]) in (0, 5) and 0 <= int(info[6]) <= int(info[1]) + int(info[3]):
            out.append(l)
    return out


def test_fused_correction_cycles_after_setup_and_resetups():
    A = problems.heterogeneous_diffusion_3d(48, sigma=3.0, corr_len=8.0, seed=5)
    n = A.shape[0]
    cfg = draugr.hypre_default_config(agg_trunc_factor=0.2, smoother=draugr.L1JacobiSmootherType(),
                                      seed=5)
    h = draugr.amg_setup(A, cfg)
    assert _fusable(h), "no level qualifies for the fused correction at this size"
    O = oracle.OracleHierarchy(h, with_rmaps=True)
    rng = np.random.default_rng(3)
    b = problems.rhs(n, 9)
    x0 = rng.uniform(-1, 1, n)

    def check(tag):
        for w in (False, True):
            c2 = draugr.AMGConfig(**{**cfg.__dict__, "cycle_type": "W" if w else "V"})
            for start in (np.zeros(n), x0):
                x = start.copy()
                draugr.amg_cycle(x, b, h, c2)
                assert rel(x, O.cycle(start, b, 1, 1, w)) < TOL64, (tag, w)
        xo, ito, _ = O.pcg(np.zeros(n), b, 1, 1, False, 1e-8, 500)
        x, it, _ = draugr.pcg(np.zeros(n), b, h, cfg, tol=1e-8, maxiter=500, precision="fp64")
        assert abs(it - ito) <= 1, (tag, it, ito)
        xm, itm, _ = draugr.pcg(np.zeros(n), b, h, cfg, tol=1e-8, maxiter=500, precision="mixed")
        Acur = A if tag == "setup" else A2
        assert np.linalg.norm(b - Acur @ xm) / np.linalg.norm(b) < 1e-8, tag

    check("setup")
    for seed in (6, 7):
        A2 = problems.heterogeneous_diffusion_3d(48, sigma=3.0, corr_len=8.0, seed=seed)
        assert np.array_equal(A2.indptr, A.indptr) and np.array_equal(A2.indices, A.indices)
        draugr.amg_resetup(h, A2, cfg, partial=True)
        O.resetup(A2.data)
        check(f"resetup {seed}")
    h.free()
