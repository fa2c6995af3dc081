"""draugr_b200_residual_noalloc: the residual entry point for callers that
cannot allocate device memory (their own pool owns every byte, so the
library may not call cudaMalloc for them).  It works on the caller's CSR
arrays and vectors with a static scratch array.  It must give what the
allocating entry point draugr_b200_residual_device gives for the same
matrix and vectors, call after call, and, since it sums every row in
column order with separately rounded products and sums, the oracle's
residual (the reference's residual_kernel!) bit for bit.  Collected last
(file name) so a run that stops at the first failure has run every other
test before it."""

import ctypes as C

import numpy as np
import pytest

import draugr
import oracle
from draugr import problems

pytestmark = pytest.mark.gpu

TOL = 1e-12  # the FP64 tolerance of the parity tests


def test_noalloc_residual_matches_allocating_entry_point():
    torch = pytest.importorskip("torch")
    A = problems.heterogeneous_diffusion_3d(32, seed=4)
    n, nnz = A.shape[0], A.nnz
    cfg = draugr.hypre_default_config(agg_trunc_factor=0.2, smoother=draugr.L1JacobiSmootherType())
    h = draugr.amg_setup(A, cfg)
    lib = draugr.load()
    dev = torch.device("cuda")
    rp_h = np.ascontiguousarray(A.indptr, np.int32)
    ci_h = np.ascontiguousarray(A.indices, np.int32)
    v_h = np.ascontiguousarray(A.data, np.float64)
    rp = torch.tensor(rp_h, device=dev)
    ci = torch.tensor(ci_h, device=dev)
    v = torch.tensor(v_h, device=dev)
    rng = np.random.default_rng(12)
    for call in range(2):
        x_h, b_h = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
        x = torch.tensor(x_h, dtype=torch.float64, device=dev)
        b = torch.tensor(b_h, dtype=torch.float64, device=dev)
        r_ref = torch.zeros(n, dtype=torch.float64, device=dev)
        r_na = torch.full((n,), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        rn_ref, rn_na = C.c_double(0), C.c_double(0)
        assert lib.draugr_b200_residual_device(h.handle, n, x.data_ptr(), b.data_ptr(),
                                               r_ref.data_ptr(), C.byref(rn_ref)) == 0, draugr.last_error()
        assert lib.draugr_b200_residual_noalloc(n, nnz, rp.data_ptr(), ci.data_ptr(), v.data_ptr(),
                                                x.data_ptr(), b.data_ptr(), r_na.data_ptr(),
                                                C.byref(rn_na), None) == 0, draugr.last_error()
        torch.cuda.synchronize()
        ref, got = r_ref.cpu().numpy(), r_na.cpu().numpy()
        assert np.all(np.isfinite(got))
        assert np.max(np.abs(got - ref)) <= TOL * np.max(np.abs(ref)), f"call {call}"
        assert abs(rn_na.value - rn_ref.value) <= TOL * rn_ref.value, f"call {call}"
        assert np.array_equal(got, oracle.residual(n, rp_h, ci_h, v_h, x_h, b_h)), f"call {call}"
    h.free()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    lib = draugr.load()
    dummy = C.c_double(0)
    p = C.cast(C.pointer(dummy), C.c_void_p)
    rc = lib.draugr_b200_residual_noalloc(4194305, 1, p, p, p, p, p, p, None, None)
    assert rc == -1
    assert "exceeds its maximum of 4194304 rows" in draugr.last_error()
