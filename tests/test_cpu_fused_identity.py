"""The regrouping behind the fused correction on the way up, checked on the
host with a real hierarchy (no GPU).  With r = b - A x the residual formed
on the way down, the reference's prolongation and first post-smoothing step
(src/prolongation.jl:742-760, src/smoothers.jl:78-94)

    x' = x + P e,   x_new = x' + (w D^-1)(b - A x')

equal  x_new = x + (w D^-1) r + Q e  with  Q = P - (w D^-1)(A P).  The
device builds Q on the pattern of A P that the hierarchy keeps for partial
resetups, placing each entry of P at its position in that pattern, so the
pattern of P has to lie inside it: checked here level by level."""

import sys
from pathlib import Path

import numpy as np
import scipy.sparse as sp

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "draugr.jl_b200"))
import draugr  # noqa: E402
from draugr import problems  # noqa: E402


def _csr(h, l, name, nrows, ncols):
    rp = h.export(l, f"{name}_rowptr")
    ci = h.export(l, f"{name}_colval")
    v = h.export(l, f"{name}_nzval") if name != "AP" else np.ones(len(ci))
    return sp.csr_matrix((v, ci, rp), shape=(nrows, ncols))


def test_regrouped_correction_and_the_ap_pattern():
    A = problems.heterogeneous_diffusion_3d(20, sigma=2.0, corr_len=4.0, seed=3)
    cfg = draugr.hypre_default_config(agg_trunc_factor=0.2, smoother=draugr.L1JacobiSmootherType(), seed=3)
    h = draugr.amg_setup(A, cfg, on_device=False)
    rng = np.random.default_rng(5)
    checked = 0
    for l in range(1, h.nlevels):
        info = h.level_info(l)
        n, nc = int(info[0]), int(info[2])
        Al = _csr(h, l, "A", n, n)
        P = _csr(h, l, "P", n, nc)
        APpat = _csr(h, l, "AP", n, nc)
        # P's pattern inside the kept A P pattern, which equals A P's
        assert (abs(P) > 0).astype(int).multiply(APpat).nnz == P.nnz, l
        assert set(zip(*(Al @ P).nonzero())) <= set(zip(*APpat.nonzero())), l
        w = float(h.export(l, "omega")[0])
        d = h.export(l, "invdiag")
        Q = P - sp.diags(w * d) @ (Al @ P)
        x, b, e = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n), rng.uniform(-1, 1, nc)
        r = b - Al @ x
        xp = x + P @ e
        ref = xp + w * d * (b - Al @ xp)
        got = x + w * d * r + Q @ e
        assert np.linalg.norm(got - ref) <= 1e-12 * np.linalg.norm(ref), l
        checked += 1
    assert checked >= 2
    h.free()
