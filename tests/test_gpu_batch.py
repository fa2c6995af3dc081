"""Many independent systems solved at once (the C3 batching configuration,
reduced): 3D 7-point Poisson systems of uneven size, each with its own
hierarchy and CUDA stream, solved concurrently from a pool of host threads
(mixed-precision PCG).  Each solve's arithmetic is fixed by its own
hierarchy, so the concurrent results must equal the same solves run one
at a time, bit for bit, and reach 1e-8 (FP64-verified)."""

import dataclasses

import numpy as np
import pytest

import draugr
from draugr import problems

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def test_concurrent_solves_equal_sequential_ones():
    rng = np.random.default_rng(9)
    sides = rng.integers(12, 33, size=10)
    cfg = draugr.hypre_default_config(agg_trunc_factor=0.2, smoother=draugr.L1JacobiSmootherType(), seed=4)
    mats = [problems.poisson3d(int(s)) for s in sides]
    hs = [draugr.amg_setup(A, cfg) for A in mats]
    bs = [torch.tensor(rng.uniform(-1, 1, A.shape[0]), device="cuda") for A in mats]
    torch.cuda.synchronize()  # the hierarchies run on their own streams
    seq = []
    for h, b in zip(hs, bs):
        x = torch.zeros_like(b)
        torch.cuda.synchronize()
        _, it, _ = draugr.pcg(x, b, h, cfg, tol=1e-8, maxiter=500, precision="mixed")
        seq.append((x.cpu().numpy(), it))
    for workers in (4, 10):
        xs = [torch.zeros_like(b) for b in bs]
        torch.cuda.synchronize()
        out = draugr.pcg_batch(hs, xs, bs, cfg, tol=1e-8, maxiter=500, precision="mixed", workers=workers)
        torch.cuda.synchronize()
        for k, (A, b, x) in enumerate(zip(mats, bs, xs)):
            xn = x.cpu().numpy()
            assert out[k][0] == seq[k][1]
            assert np.array_equal(xn, seq[k][0]), k
            bn = b.cpu().numpy()
            assert np.linalg.norm(bn - A @ xn) / np.linalg.norm(bn) < 1e-8


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("side,k,coarse", [(20, 5, 50), (24, 32, 50), (16, 1, 50), (18, 32, 300), (17, 6, 50)])
def test_block_pcg_matches_single_solves(side, k, coarse, precision):
    """Many right-hand sides of one matrix (the C3 96^3 x 32 case, reduced):
    block PCG, one pass over each level matrix for all k columns, against
    k single-right-hand-side PCG solves.  Odd k takes the unfused outer
    iteration and one warp per row; k = 6 the fused outer iteration with one
    warp per row (6 columns do not split into pieces of 4); max_coarse_size
    300 gives a coarsest system of more than 64 unknowns (the
    one-thread-per-column solve)."""
    A = problems.poisson3d(side)
    n = A.shape[0]
    cfg = draugr.hypre_default_config(agg_trunc_factor=0.2, smoother=draugr.L1JacobiSmootherType(), seed=6)
    cfg = dataclasses.replace(cfg, max_coarse_size=coarse)
    h = draugr.amg_setup(A, cfg)
    rng = np.random.default_rng(side + k)
    Bn = rng.uniform(-1, 1, (n, k))
    B = torch.tensor(Bn, device="cuda")
    X = torch.zeros_like(B)
    torch.cuda.synchronize()
    X, its, rels = draugr.pcg_multi(X, B, h, cfg, tol=1e-8, maxiter=500, precision=precision)
    Xn = X.cpu().numpy()
    for c in range(k):
        x1, it1, _ = draugr.pcg(np.zeros(n), Bn[:, c].copy(), h, cfg, tol=1e-8, maxiter=500,
                                precision=precision)
        assert abs(its[c] - it1) <= 1, (c, its[c], it1)
        r = np.linalg.norm(Bn[:, c] - A @ Xn[:, c]) / np.linalg.norm(Bn[:, c])
        assert r < 1e-8 and abs(r - rels[c]) < 1e-12
        assert np.linalg.norm(Xn[:, c] - x1) / np.linalg.norm(x1) < 1e-6


@pytest.mark.parametrize("k,precision", [(8, "mixed"), (8, "fp64"), (32, "mixed")])
def test_block_launch_shapes_change_no_value(k, precision, monkeypatch):
    """The launch shapes of the block cycle's products (threads per row,
    blocks per SM) are picked by timing.  Every shape sums each column of a
    row in one thread in column order, so the default shapes, each forced
    number of threads per row (DRAUGR_B200_BLOCK_TUNE=4/8/16, up to four
    times the threads a row's columns need) and the timed pick give the same
    solve bit for bit."""
    A = problems.poisson3d(22)
    n = A.shape[0]
    cfg = draugr.hypre_default_config(agg_trunc_factor=0.2, smoother=draugr.L1JacobiSmootherType(), seed=4)
    h = draugr.amg_setup(A, cfg)
    B = torch.tensor(np.random.default_rng(k).uniform(-1, 1, (n, k)), device="cuda")
    runs = {}
    for setting in ["0", "4", "8", "16", ""]:
        monkeypatch.setenv("DRAUGR_B200_BLOCK_TUNE", setting)
        X = torch.zeros_like(B)
        torch.cuda.synchronize()
        X, its, rels = draugr.pcg_multi(X, B, h, cfg, tol=1e-8, maxiter=500, precision=precision)
        runs[setting] = (X.cpu().numpy(), list(its), list(rels))
    X0, its0, rels0 = runs["0"]
    assert max(its0) > 0
    for setting, (X, its, rels) in runs.items():
        assert its == its0, setting
        assert rels == rels0, setting
        assert np.array_equal(X, X0), setting
