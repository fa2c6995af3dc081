"""The row kernel's bounded wait, made to run out without a stuck copy.

Every row kernel (k_tile_rows) waits on an mbarrier for the bulk copy of
each tile.  A wait that gives up must not read the stage: the block flags
the error, lets the copies it has in flight land (a second bounded wait),
and leaves; the entry point returns -1.  The test lowers the wait limit to
zero polls through the test hook draugr_b200_set_tile_wait_limit, so every
wait gives up at once while the copies themselves complete normally, checks
the error, restores the limit and checks that the next calls on the same
device give the oracle's results (the context is intact, the error flag and
the reduction tickets are cleared)."""

import ctypes as C

import numpy as np
import pytest

import draugr
import oracle
from draugr import problems

pytestmark = pytest.mark.gpu


def test_wait_that_runs_out_reports_an_error_and_the_device_stays_usable():
    torch = pytest.importorskip("torch")
    lib = draugr.load()
    A = problems.heterogeneous_diffusion_3d(24, seed=9)
    n = A.shape[0]
    cfg = draugr.hypre_default_config(agg_trunc_factor=0.2, smoother=draugr.L1JacobiSmootherType())
    h = draugr.amg_setup(A, cfg)
    assert h.nlevels >= 2
    rng = np.random.default_rng(5)
    xh, bh = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    x = torch.tensor(xh, device="cuda")
    b = torch.tensor(bh, device="cuda")
    r = torch.zeros(n, dtype=torch.float64, device="cuda")
    rn = C.c_double(0)
    try:
        lib.draugr_b200_set_tile_wait_limit(0)
        rc = lib.draugr_b200_residual_device(h.handle, n, x.data_ptr(), b.data_ptr(), r.data_ptr(),
                                             C.byref(rn))
        assert rc == -1 and "timed out" in draugr.last_error()
        xc = torch.zeros(n, dtype=torch.float64, device="cuda")
        rc = lib.draugr_b200_cycle_device(h.handle, n, xc.data_ptr(), b.data_ptr(), draugr.config_handle(cfg))
        assert rc == -1 and "timed out" in draugr.last_error()
    finally:
        lib.draugr_b200_set_tile_wait_limit(-1)
    torch.cuda.synchronize()
    # the same calls with the default limit: the oracle's results
    assert lib.draugr_b200_residual_device(h.handle, n, x.data_ptr(), b.data_ptr(), r.data_ptr(),
                                           C.byref(rn)) == 0, draugr.last_error()
    ref = oracle.residual(n, np.ascontiguousarray(A.indptr, np.int32),
                          np.ascontiguousarray(A.indices, np.int32), A.data, xh, bh)
    got = r.cpu().numpy()
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))
    assert abs(rn.value - np.linalg.norm(ref)) <= 1e-12 * np.linalg.norm(ref)
    xc = np.zeros(n)
    draugr.amg_cycle(xc, bh, h, cfg)
    O = oracle.OracleHierarchy(h)
    want = O.cycle(np.zeros(n), bh)
    assert np.linalg.norm(xc - want) / np.linalg.norm(want) < 1e-12
    h.free()
