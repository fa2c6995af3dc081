"""Independent systems merged into one batch (the C3 batching
configuration, reduced): every cycle stage, dot product and vector update
is one launch for all systems, each system keeping its own step sizes.

The merged hierarchy holds each system's rows unchanged (block-diagonal
matrices with shifted columns) and solves each system's coarsest level with
its own LU factors, so one V-cycle of the batch must give, system by
system, what one V-cycle of the system's own hierarchy gives (1e-12); the
batched AMG-PCG must reach 1e-8 on every system (FP64-verified), in the
iterations of the system's own AMG-PCG (+-1: the per-system dot products
are reduced in another order), with solutions within 1e-6 of the single
solves'."""

import numpy as np
import pytest

import draugr
from draugr import problems

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def systems():
    rng = np.random.default_rng(11)
    sides = [int(s) for s in rng.integers(12, 29, size=9)]
    cfg = draugr.hypre_default_config(agg_trunc_factor=0.2, smoother=draugr.L1JacobiSmootherType(), seed=6)
    mats = [problems.poisson3d(s) for s in sides[:-1]] + [problems.heterogeneous_diffusion_3d(sides[-1], seed=2)]
    hs = [draugr.amg_setup(A, cfg) for A in mats]
    bs = [rng.uniform(-1, 1, A.shape[0]) for A in mats]
    batch = draugr.batch_setup(hs, cfg)
    yield cfg, mats, hs, bs, batch
    batch.free()
    for h in hs:
        h.free()


def test_layout(systems):
    cfg, mats, hs, bs, batch = systems
    assert batch.nsystems == len(mats)
    assert list(np.diff(batch.offsets)) == [A.shape[0] for A in mats]
    depths = {h.nlevels for h in hs}
    assert batch.nlevels == max(depths)


def test_one_cycle_equals_the_systems_own_cycles(systems):
    cfg, mats, hs, bs, batch = systems
    b = torch.tensor(np.concatenate(bs), device="cuda")
    x = torch.zeros_like(b)
    draugr.amg_cycle(x, b, batch, cfg)
    xb = x.cpu().numpy()
    for s, (h, bb) in enumerate(zip(hs, bs)):
        xs = np.zeros_like(bb)
        draugr.amg_cycle(xs, bb, h, cfg)
        lo, hi = batch.offsets[s], batch.offsets[s + 1]
        assert rel(xb[lo:hi], xs) < 1e-12, s


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batched_pcg_matches_single_solves(systems, precision):
    cfg, mats, hs, bs, batch = systems
    b = torch.tensor(np.concatenate(bs), device="cuda")
    x = torch.zeros_like(b)
    _, its, rr = draugr.pcg_batched(x, b, batch, cfg, tol=1e-8, maxiter=500, precision=precision)
    xb = x.cpu().numpy()
    for s, (A, h, bb) in enumerate(zip(mats, hs, bs)):
        xs, it, _ = draugr.pcg(np.zeros_like(bb), bb, h, cfg, tol=1e-8, maxiter=500, precision=precision)
        lo, hi = batch.offsets[s], batch.offsets[s + 1]
        xr = xb[lo:hi]
        assert np.linalg.norm(bb - A @ xr) / np.linalg.norm(bb) < 1e-8, s
        assert rr[s] < 1e-8, s
        assert abs(int(its[s]) - it) <= 1, (s, its[s], it)
        assert rel(xr, xs) < 1e-6, s
    # again from the converged solution: no system moves
    _, its2, rr2 = draugr.pcg_batched(x, b, batch, cfg, tol=1e-8, precision=precision)
    assert not np.any(its2) and np.all(rr2 < 1e-8)


def test_zero_right_hand_side_of_one_system(systems):
    cfg, mats, hs, bs, batch = systems
    bl = [bb.copy() for bb in bs]
    bl[2][:] = 0.0
    b = torch.tensor(np.concatenate(bl), device="cuda")
    x = torch.ones_like(b)
    _, its, rr = draugr.pcg_batched(x, b, batch, cfg, tol=1e-8, precision="mixed")
    xb = x.cpu().numpy()
    lo, hi = batch.offsets[2], batch.offsets[3]
    assert its[2] == 0 and not np.any(xb[lo:hi])
    assert all(rr[s] < 1e-8 for s in range(batch.nsystems))


def test_rejects_mismatched_inputs(systems):
    cfg, mats, hs, bs, batch = systems
    b = torch.zeros(int(batch.offsets[-1]) + 1, dtype=torch.float64, device="cuda")
    with pytest.raises(draugr.DraugrError, match="DimensionMismatch"):
        draugr.pcg_batched(torch.zeros_like(b), b, batch, cfg)
    gs = draugr.hypre_default_config(agg_trunc_factor=0.2, smoother=draugr.ColoredGaussSeidelType())
    hg = draugr.amg_setup(problems.poisson3d(12), gs)
    with pytest.raises(draugr.DraugrError, match="Jacobi"):
        draugr.batch_setup([hg], gs)
    hg.free()
