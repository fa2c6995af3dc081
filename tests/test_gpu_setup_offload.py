"""The setup offload (the first "next" step of the hot path's scope): a
setup for the device computes each level's Galerkin products, the patterns
of A·P and Pᵀ(AP) (src/galerkin.jl:11-183) and their values, on the GPU
and hands them back to the CPU coarsening of the next level.  The patterns
are sets and the values keep the CPU numeric product's per-entry order, so
the hierarchy must be the host-only setup's bit for bit: every level's
matrix, interpolation, A·P pattern, the coarsest matrix and its LU."""

import os
import subprocess
import sys

import numpy as np
import pytest

import draugr
from cases import CASES
from draugr import problems

pytestmark = pytest.mark.gpu

INT_ARRAYS = ("A_rowptr", "A_colval", "P_rowptr", "P_colval", "AP_rowptr", "AP_colval")
VAL_ARRAYS = ("A_nzval", "P_nzval", "invdiag")


def assert_same_hierarchy(hd, hh):
    assert hd.nlevels == hh.nlevels
    for l in range(hd.nlevels):
        for w in INT_ARRAYS + VAL_ARRAYS:
            a, b = hd.export(l, w), hh.export(l, w)
            assert a.shape == b.shape and np.array_equal(a, b), (l, w)
    for w in ("C_rowptr", "C_colval", "C_nzval", "C_lu", "C_piv"):
        assert np.array_equal(hd.export(-1, w), hh.export(-1, w)), w


@pytest.mark.parametrize("name", sorted(CASES))
def test_small_cases(name):
    make, cfg = CASES[name]
    A = make()
    hd = draugr.amg_setup(A, cfg)
    hh = draugr.amg_setup(A, cfg, on_device=False)
    assert_same_hierarchy(hd, hh)


@pytest.mark.parametrize("which", ["hetero_48", "aniso27_32"])
def test_larger_hierarchies(which):
    if which == "hetero_48":
        A = problems.heterogeneous_diffusion_3d(48, seed=3)
    else:
        A = problems.anisotropic_27pt(32, 1e-3)
    cfg = draugr.hypre_default_config(agg_trunc_factor=0.2, smoother=draugr.L1JacobiSmootherType(), seed=5)
    hd = draugr.amg_setup(A, cfg)
    hh = draugr.amg_setup(A, cfg, on_device=False)
    assert_same_hierarchy(hd, hh)
    # and the offloaded hierarchy solves as the host one does
    b = problems.rhs(A.shape[0], 1)
    x, it, _ = draugr.pcg(np.zeros(A.shape[0]), b, hd, cfg, tol=1e-8)
    assert np.linalg.norm(b - A @ x) / np.linalg.norm(b) < 1e-8


def test_switch_off():
    """DRAUGR_B200_GPU_SETUP=0 keeps the whole setup on the host."""
    code = ("import sys; sys.path.insert(0, 'draugr.jl_b200'); import numpy as np, draugr; "
            "from draugr import problems; A = problems.poisson3d(12); "
            "cfg = draugr.hypre_default_config(agg_trunc_factor=0.2, smoother=draugr.L1JacobiSmootherType()); "
            "h = draugr.amg_setup(A, cfg); print(h.nlevels)")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "-c", code], cwd=root, capture_output=True, text=True, timeout=300,
                         env=dict(os.environ, DRAUGR_B200_GPU_SETUP="0"))
    assert out.returncode == 0, out.stderr[-1000:]
    assert int(out.stdout.strip()) >= 1
