"""Python host mirror of Draugr.jl's AMG API on top of libdraugr_b200.so.

Names and argument meanings follow the reference (src/types.jl,
src/setup.jl, src/cycle.jl, src/resetup.jl):

    h = amg_setup(A, AMGConfig(...))             # amg_setup(A, config)
    x, niter = amg_solve(x, b, h, config)         # amg_solve!(x, b, h, config)
    amg_cycle(x, b, h, config)                    # amg_cycle!(x, b, h, config)
    amg_resetup(h, A_new, config, partial=True)   # amg_resetup!(h, A, config)

``x`` and ``b`` are float64 NumPy arrays (updated in place like the Julia
``!`` functions) or CUDA tensors (device pointers are passed straight to
the library).  Every call goes through the C ABI; errors raise DraugrError
with the library's last-error message.
"""

from __future__ import annotations

import ctypes as C
import json
from dataclasses import dataclass, field
from typing import Any

import numpy as np

from . import _lib

# ---------------------------------------------------------------- config types


@dataclass(frozen=True)
class DirectInterpolation:
    trunc_factor: float = 0.0


@dataclass(frozen=True)
class StandardInterpolation:
    trunc_factor: float = 0.0


@dataclass(frozen=True)
class ExtendedIInterpolation:
    trunc_factor: float = 0.0
    max_elements: int = 0
    norm_p: int = 1
    rescale: bool = False


@dataclass(frozen=True)
class AggregationCoarsening:
    theta: float = 0.25
    filtering: bool = False
    filter_tol: float = 0.1


@dataclass(frozen=True)
class PMISCoarsening:
    theta: float = 0.25
    interpolation: Any = DirectInterpolation()


@dataclass(frozen=True)
class HMISCoarsening:
    theta: float = 0.25
    interpolation: Any = DirectInterpolation()


@dataclass(frozen=True)
class RSCoarsening:
    theta: float = 0.25
    interpolation: Any = DirectInterpolation()


@dataclass(frozen=True)
class AggressiveCoarsening:
    theta: float = 0.25
    base: str = "pmis"
    interpolation: Any = ExtendedIInterpolation()


@dataclass(frozen=True)
class SmoothedAggregationCoarsening:
    theta: float = 0.25
    omega: float = 2.0 / 3.0
    filtering: bool = False
    filter_tol: float = 0.1


class _SmootherType:
    name = ""

    def __eq__(self, o):
        return type(self) is type(o)

    def __hash__(self):
        return hash(self.name)

    def __repr__(self):
        return type(self).__name__ + "()"


def _smoother(cls_name, json_name):
    return type(cls_name, (_SmootherType,), {"name": json_name})


JacobiSmootherType = _smoother("JacobiSmootherType", "jacobi")
L1JacobiSmootherType = _smoother("L1JacobiSmootherType", "l1_jacobi")
ColoredGaussSeidelType = _smoother("ColoredGaussSeidelType", "colored_gs")
L1ColoredGaussSeidelType = _smoother("L1ColoredGaussSeidelType", "l1_colored_gs")
SerialGaussSeidelType = _smoother("SerialGaussSeidelType", "serial_gs")
L1SerialGaussSeidelType = _smoother("L1SerialGaussSeidelType", "l1_serial_gs")
SPAI0SmootherType = _smoother("SPAI0SmootherType", "spai0")
SPAI1SmootherType = _smoother("SPAI1SmootherType", "spai1")
ChebyshevSmootherType = _smoother("ChebyshevSmootherType", "chebyshev")
ILU0SmootherType = _smoother("ILU0SmootherType", "ilu0")
SerialILU0SmootherType = _smoother("SerialILU0SmootherType", "serial_ilu0")


@dataclass(frozen=True)
class AbsoluteStrength:
    pass


@dataclass(frozen=True)
class SignedStrength:
    pass


def _interp_json(ip):
    if isinstance(ip, DirectInterpolation):
        return {"type": "direct", "trunc_factor": ip.trunc_factor}
    if isinstance(ip, StandardInterpolation):
        return {"type": "standard", "trunc_factor": ip.trunc_factor}
    return {"type": "extended_i", "trunc_factor": ip.trunc_factor,
            "max_elements": ip.max_elements, "norm_p": ip.norm_p, "rescale": ip.rescale}


def _coarsening_json(c):
    """(name, theta, interpolation-or-None, extras) of a coarsening."""
    if isinstance(c, AggregationCoarsening):
        return "aggregation", c.theta, None, {"aggregation_filtering": c.filtering,
                                              "filter_tol": c.filter_tol}
    if isinstance(c, SmoothedAggregationCoarsening):
        return "smoothed_aggregation", c.theta, None, {"sa_omega": c.omega,
                                                       "aggregation_filtering": c.filtering,
                                                       "filter_tol": c.filter_tol}
    if isinstance(c, PMISCoarsening):
        return "pmis", c.theta, c.interpolation, {}
    if isinstance(c, HMISCoarsening):
        return "hmis", c.theta, c.interpolation, {}
    if isinstance(c, RSCoarsening):
        return "rs", c.theta, c.interpolation, {}
    if isinstance(c, AggressiveCoarsening):
        if c.base not in ("hmis", "pmis"):
            raise ValueError("AggressiveCoarsening base must be 'hmis' or 'pmis'")
        return "aggressive_" + c.base, c.theta, c.interpolation, {}
    raise TypeError(f"unknown coarsening {c!r}")


@dataclass(frozen=True)
class AMGConfig:
    """AMG configuration with the defaults of AMGConfig() (src/types.jl:514-536)."""

    coarsening: Any = HMISCoarsening(0.5, ExtendedIInterpolation())
    smoother: Any = L1ColoredGaussSeidelType()
    max_levels: int = 20
    max_coarse_size: int = 50
    pre_smoothing_steps: int = 1
    post_smoothing_steps: int = 1
    jacobi_omega: float = 2.0 / 3.0
    verbose: int = 0
    initial_coarsening: Any = None
    initial_coarsening_levels: int = 0
    max_row_sum: float = 1.0
    cycle_type: str = "V"
    strength_type: Any = AbsoluteStrength()
    coarse_solve_on_cpu: bool = False
    seed: int | None = None

    def __post_init__(self):
        if self.cycle_type not in ("V", "W"):
            raise ValueError("cycle_type must be :V or :W")

    def to_json(self) -> str:
        name, theta, ip, extra = _coarsening_json(self.coarsening)
        d = {"coarsening": name, "theta": theta,
             "smoother": {"type": self.smoother.name, "omega": self.jacobi_omega},
             "max_levels": self.max_levels, "max_coarse_size": self.max_coarse_size,
             "pre_smoothing_steps": self.pre_smoothing_steps,
             "post_smoothing_steps": self.post_smoothing_steps,
             "verbose": int(self.verbose),
             "initial_coarsening_levels": self.initial_coarsening_levels,
             "max_row_sum": self.max_row_sum, "cycle": self.cycle_type.lower(),
             "strength": "signed" if isinstance(self.strength_type, SignedStrength) else "absolute",
             "coarse_solve_on_cpu": self.coarse_solve_on_cpu}
        if ip is not None:
            d["interpolation"] = _interp_json(ip)
        d.update(extra)
        ic = self.initial_coarsening if self.initial_coarsening is not None else self.coarsening
        iname, itheta, iip, iextra = _coarsening_json(ic)
        d["initial_coarsening"] = iname
        d["initial_theta"] = itheta
        if iip is not None:
            d["initial_interpolation"] = _interp_json(iip)
        if self.seed is not None:
            d["seed"] = int(self.seed)
        return json.dumps(d)


def hypre_default_config(theta: float = 0.5, agg_num_levels: int = 1,
                         agg_trunc_factor: float = 0.3, **kwargs) -> AMGConfig:
    """BoomerAMG-like setup (src/types.jl:569-584): HMIS, aggressive HMIS on
    the first agg_num_levels levels, extended+i with truncation."""
    interp = ExtendedIInterpolation(agg_trunc_factor)
    return AMGConfig(coarsening=HMISCoarsening(theta, interp),
                     initial_coarsening=AggressiveCoarsening(theta, "hmis", interp),
                     initial_coarsening_levels=agg_num_levels, **kwargs)


def config_fields(config: AMGConfig | str | None) -> dict:
    """Every field of the configuration as the library parsed it
    (draugr_b200_config_json): coarsening and initial coarsening as dicts,
    smoother, omega, level and step counts, cycle, strength and seed."""
    text = _lib.load().draugr_b200_config_json(config_handle(config))
    if text is None:
        raise _lib.DraugrError(f"config_fields: {_lib.last_error()}")
    return json.loads(text)


_cfg_cache: dict[str, int] = {}


def config_handle(config: AMGConfig | str | None) -> int:
    """Config handle (draugr_amg_config_from_json) for a config or JSON text."""
    js = "{}" if config is None else (config if isinstance(config, str) else config.to_json())
    h = _cfg_cache.get(js)
    if h is None:
        h = _lib.check(_lib.load().draugr_amg_config_from_json(js.encode()),
                       "draugr_amg_config_from_json")
        _cfg_cache[js] = h
    return h


# ---------------------------------------------------------------- matrices

def _csr_arrays(A):
    """(n, rowptr int32, colval int32, nzval float64) of a CSR-like input."""
    if hasattr(A, "tocsr"):
        A = A.tocsr()
        n = A.shape[0]
        if A.shape[0] != A.shape[1]:
            raise ValueError("matrix must be square")
        return (n, np.ascontiguousarray(A.indptr, dtype=np.int32),
                np.ascontiguousarray(A.indices, dtype=np.int32),
                np.ascontiguousarray(A.data, dtype=np.float64))
    n, rp, ci, v = A
    return (int(n), np.ascontiguousarray(rp, dtype=np.int32),
            np.ascontiguousarray(ci, dtype=np.int32), np.ascontiguousarray(v, dtype=np.float64))


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def _is_device(t) -> bool:
    return hasattr(t, "is_cuda") and bool(t.is_cuda)


# ---------------------------------------------------------------- hierarchy

class Hierarchy:
    """Handle of a hierarchy in the library (AMGHierarchy in the reference)."""

    def __init__(self, handle: int, n: int, config: AMGConfig | None):
        self.handle = handle
        self.n = n
        self.config = config

    @property
    def nlevels(self) -> int:
        return _lib.check(_lib.load().draugr_b200_num_levels(self.handle), "num_levels")

    def level_info(self, lvl: int) -> np.ndarray:
        info = np.zeros(10, dtype=np.int64)
        _lib.check(_lib.load().draugr_b200_level_info(self.handle, lvl, _ptr(info)), "level_info")
        return info

    def export(self, lvl: int, what: str) -> np.ndarray:
        lib = _lib.load()
        cnt = lib.draugr_b200_export(self.handle, lvl, what.encode(), None, 0)
        _lib.check(cnt, f"export {what}")
        is_int = what in ("A_rowptr", "A_colval", "P_rowptr", "P_colval", "T_offsets", "T_rows",
                          "T_pnz", "colors", "color_order", "color_offsets", "AP_rowptr",
                          "AP_colval", "C_rowptr", "C_colval", "C_piv", "ilu_diag", "ilu_fwd_order",
                          "ilu_fwd_offsets", "ilu_bwd_order", "ilu_bwd_offsets", "sgs_order",
                          "sgs_offsets", "cf")
        out = np.zeros(cnt, dtype=np.int32 if is_int else np.float64)
        _lib.check(lib.draugr_b200_export(self.handle, lvl, what.encode(), _ptr(out), cnt),
                   f"export {what}")
        return out

    def set_resetup_precision(self, fp64_levels: int) -> None:
        """Galerkin products of later partial resetups: the first
        `fp64_levels` from the top in FP64, the rest in FP32 (negative: all
        FP64, the default)."""
        _lib.check(_lib.load().draugr_b200_set_resetup_precision(self.handle, fp64_levels),
                   "set_resetup_precision")

    def galerkin_host(self, lvl: int, values) -> np.ndarray:
        """The next level's values from new values of level lvl, by the
        setup's numeric product on the host (draugr_b200_galerkin_host)."""
        lib = _lib.load()
        v = np.ascontiguousarray(values, np.float64)
        nnz_next = int(self.level_info(lvl + 1)[1] if lvl + 1 < self.nlevels else self.level_info(-1)[1])
        out = np.zeros(nnz_next)
        _lib.check(lib.draugr_b200_galerkin_host(self.handle, lvl, len(v), _ptr(v), nnz_next, _ptr(out)),
                   "galerkin_host")
        return out

    def summary(self) -> str:
        s = _lib.load().draugr_b200_summary(self.handle)
        return s.decode() if s else ""

    def device_bytes(self) -> int:
        return _lib.load().draugr_b200_device_bytes(self.handle)

    def level_op(self, lvl: int, op: int, in1, in2=None, steps: int = 1,
                 precision: int = 0) -> np.ndarray:
        """One level kernel on host arrays (see draugr_b200_level_op)."""
        info = self.level_info(lvl if op != 5 else -1)
        n = int(info[0])
        nout = {3: int(info[2]), 6: 2 * n}.get(op, n)
        in1 = np.ascontiguousarray(in1, dtype=np.float64)
        in2 = None if in2 is None else np.ascontiguousarray(in2, dtype=np.float64)
        out = np.zeros(nout, dtype=np.float64)
        _lib.check(_lib.load().draugr_b200_level_op(
            self.handle, lvl, op, precision, _ptr(in1), None if in2 is None else _ptr(in2),
            _ptr(out), steps), f"level_op {op}")
        return out

    def time_level_op(self, lvl: int, op: int = 2, precision: int = 0, reps: int = 20) -> float:
        ms = C.c_float(0.0)
        _lib.check(_lib.load().draugr_b200_time_level_op(self.handle, lvl, op, precision, reps,
                                                          C.byref(ms)), "time_level_op")
        return ms.value

    def set_stream(self, stream) -> None:
        """Run on a CUDA stream: a torch.cuda.Stream, a raw cudaStream_t
        (int) or None for the library's own stream."""
        raw = getattr(stream, "cuda_stream", stream)
        _lib.check(_lib.load().draugr_b200_set_stream(self.handle, raw), "set_stream")

    def free(self):
        if self.handle > 0:
            _lib.check(_lib.load().draugr_amg_free(self.handle), "draugr_amg_free")
            self.handle = -1

    def __del__(self):
        try:
            if self.handle > 0:
                _lib.load().draugr_amg_free(self.handle)
        except Exception:
            pass


def amg_setup(A, config: AMGConfig | None = None, allow_partial_resetup: bool = True,
              on_device: bool = True) -> Hierarchy:
    """Build the hierarchy (CPU) and upload it to the current CUDA device
    (amg_setup, src/setup.jl:47-87).  on_device=False keeps the structure
    on the host only (inspection without a GPU)."""
    config = config if config is not None else AMGConfig()
    n, rp, ci, v = _csr_arrays(A)
    lib = _lib.load()
    fn = lib.draugr_amg_setup if on_device else lib.draugr_b200_setup_host
    h = _lib.check(fn(n, len(ci), _ptr(rp), _ptr(ci), _ptr(v), config_handle(config), 0,
                      1 if allow_partial_resetup else 0), "amg_setup")
    return Hierarchy(h, n, config)


def amg_resetup(h: Hierarchy, A, config: AMGConfig | None = None, partial: bool = True,
                allow_partial_resetup: bool = True) -> Hierarchy:
    """New coefficients (amg_resetup!, src/resetup.jl:20-70).  A may also be
    a CUDA tensor of the new finest-level values (same pattern)."""
    config = config if config is not None else (h.config or AMGConfig())
    lib = _lib.load()
    if _is_device(A):
        _lib.check(lib.draugr_b200_resetup_values_device(h.handle, A.numel(), A.data_ptr()),
                   "amg_resetup")
        return h
    n, rp, ci, v = _csr_arrays(A)
    _lib.check(lib.draugr_amg_resetup(h.handle, n, len(ci), _ptr(rp), _ptr(ci), _ptr(v),
                                      config_handle(config), 0, 1 if partial else 0,
                                      1 if allow_partial_resetup else 0), "amg_resetup")
    if not partial:
        h.n = n
    return h


def amg_cycle(x, b, h: Hierarchy, config: AMGConfig | None = None):
    """One cycle improving x in place (amg_cycle!, src/cycle.jl:12-28)."""
    config = config if config is not None else (h.config or AMGConfig())
    lib = _lib.load()
    if _is_device(x):
        _lib.check(lib.draugr_b200_cycle_device(h.handle, x.numel(), x.data_ptr(), b.data_ptr(),
                                                config_handle(config)), "amg_cycle")
        return x
    _check_vec(x, b, h)
    _lib.check(lib.draugr_amg_cycle(h.handle, len(x), _ptr(x), _ptr(b), config_handle(config)),
               "amg_cycle")
    return x


def amg_solve(x, b, h: Hierarchy, config: AMGConfig | None = None, tol: float = 1e-10,
              maxiter: int = 100):
    """Stationary AMG iteration (amg_solve!, src/cycle.jl:110-160).
    Returns (x, niter); x is updated in place."""
    config = config if config is not None else (h.config or AMGConfig())
    lib = _lib.load()
    if _is_device(x):
        it = _lib.check(lib.draugr_b200_solve_device(h.handle, x.numel(), x.data_ptr(),
                                                     b.data_ptr(), config_handle(config), tol,
                                                     maxiter), "amg_solve")
        return x, it
    _check_vec(x, b, h)
    it = _lib.check(lib.draugr_amg_solve(h.handle, len(x), _ptr(x), _ptr(b),
                                         config_handle(config), tol, maxiter), "amg_solve")
    return x, it


def pcg(x, b, h: Hierarchy, config: AMGConfig | None = None, tol: float = 1e-8,
        maxiter: int = 500, precision: str = "fp64"):
    """AMG-preconditioned conjugate gradients (FP64 outer iteration).
    precision "fp64": FP64 cycle; "mixed": FP32 hierarchy and cycle.
    Returns (x, niter, relres)."""
    config = config if config is not None else (h.config or AMGConfig())
    prec = {"fp64": 0, "mixed": 1, "fp32": 1}[precision]
    lib = _lib.load()
    rel = C.c_double(0.0)
    if _is_device(x):
        it = _lib.check(lib.draugr_b200_pcg_device(h.handle, x.numel(), x.data_ptr(), b.data_ptr(),
                                                   config_handle(config), tol, maxiter, prec,
                                                   C.byref(rel)), "pcg")
        return x, it, rel.value
    _check_vec(x, b, h)
    it = _lib.check(lib.draugr_b200_pcg(h.handle, len(x), _ptr(x), _ptr(b), config_handle(config),
                                        tol, maxiter, prec, C.byref(rel)), "pcg")
    return x, it, rel.value


def bicgstab(x, b, h: Hierarchy, config: AMGConfig | None = None, tol: float = 1e-8,
             maxiter: int = 500, transpose: bool = False, precision: str = "fp64"):
    """BiCGStab preconditioned by one AMG cycle (nonsymmetric systems):
    precision="fp64" (FP64 cycle) or "mixed" (FP32 cycle, FP64 vectors,
    products and dots).  transpose=True solves A^T x = b with cycles on the
    transposed hierarchy (the adjoint system of a gradient).  Returns
    (x, niter, relres)."""
    config = config if config is not None else (h.config or AMGConfig())
    prec = {"fp64": 0, "mixed": 1}[precision]
    lib = _lib.load()
    rel = C.c_double(0.0)
    if _is_device(x):
        it = _lib.check(lib.draugr_b200_bicgstab_device(h.handle, x.numel(), x.data_ptr(), b.data_ptr(),
                                                        config_handle(config), tol, maxiter,
                                                        1 if transpose else 0, prec, C.byref(rel)), "bicgstab")
        return x, it, rel.value
    _check_vec(x, b, h)
    it = _lib.check(lib.draugr_b200_bicgstab(h.handle, len(x), _ptr(x), _ptr(b), config_handle(config),
                                             tol, maxiter, 1 if transpose else 0, prec, C.byref(rel)),
                    "bicgstab")
    return x, it, rel.value


def fgmres(x, b, h: Hierarchy, config: AMGConfig | None = None, tol: float = 1e-8, maxiter: int = 500,
           restart: int = 30, precision: str = "fp64"):
    """Flexible GMRES(restart) right-preconditioned by one AMG cycle (FP64,
    or precision="mixed": the FP32 cycle with FP64 Arnoldi), for symmetric
    and nonsymmetric systems.  x (numpy or CUDA tensor) holds the initial
    guess and is updated in place.  Returns (x, niter, relres)."""
    config = config if config is not None else (h.config or AMGConfig())
    prec = {"fp64": 0, "mixed": 1}[precision]
    lib = _lib.load()
    rel = C.c_double(0.0)
    if _is_device(x):
        it = _lib.check(lib.draugr_b200_fgmres_device(h.handle, x.numel(), x.data_ptr(), b.data_ptr(),
                                                      config_handle(config), tol, maxiter, restart, prec,
                                                      C.byref(rel)), "fgmres")
        return x, it, rel.value
    _check_vec(x, b, h)
    it = _lib.check(lib.draugr_b200_fgmres(h.handle, len(x), _ptr(x), _ptr(b), config_handle(config), tol,
                                           maxiter, restart, prec, C.byref(rel)), "fgmres")
    return x, it, rel.value


def refine(x, b, h: Hierarchy, config: AMGConfig | None = None, tol: float = 1e-8, max_outer: int = 20,
           inner_tol: float = 1e-4, inner_maxiter: int = 500, inner: str = "pcg", precision: str = "mixed"):
    """Iterative refinement: FP64 residual r = b - A x, the correction A d = r
    solved to inner_tol by AMG-PCG (inner="pcg") or FGMRES (inner="fgmres")
    with an FP64 or FP32 (precision="mixed") cycle, x += d, until the FP64
    relative residual is below tol.  Returns (x, steps, inner_iterations,
    relres)."""
    config = config if config is not None else (h.config or AMGConfig())
    prec = {"fp64": 0, "mixed": 1}[precision]
    meth = {"pcg": 0, "fgmres": 1}[inner]
    lib = _lib.load()
    rel = C.c_double(0.0)
    its = C.c_int32(0)
    if _is_device(x):
        st = _lib.check(lib.draugr_b200_refine_device(h.handle, x.numel(), x.data_ptr(), b.data_ptr(),
                                                      config_handle(config), tol, max_outer, inner_tol,
                                                      inner_maxiter, meth, prec, C.byref(rel), C.byref(its)),
                        "refine")
        return x, st, its.value, rel.value
    _check_vec(x, b, h)
    st = _lib.check(lib.draugr_b200_refine(h.handle, len(x), _ptr(x), _ptr(b), config_handle(config), tol,
                                           max_outer, inner_tol, inner_maxiter, meth, prec, C.byref(rel),
                                           C.byref(its)), "refine")
    return x, st, its.value, rel.value


def nz_gradient(h: Hierarchy, x, lam):
    """dL/da_ij = -lambda_i x_j for the finest matrix's nonzeros (CSR order),
    with x = A^-1 b and lambda = A^-T dL/dx (CUDA tensors); returns a new
    CUDA tensor of nnz entries."""
    import torch

    lib = _lib.load()
    nnz = int(h.level_info(0)[1]) if h.nlevels > 0 else int(h.level_info(-1)[1])
    grad = torch.empty(nnz, dtype=torch.float64, device=x.device)
    _lib.check(lib.draugr_b200_nz_gradient_device(h.handle, x.numel(), x.data_ptr(), lam.data_ptr(),
                                                  grad.data_ptr()), "nz_gradient")
    return grad


class _Solve:
    """Holder of the torch.autograd.Function (built on first use, so that the
    package imports without torch)."""
    fn = None


def amg_solve_diff(values, b, h: Hierarchy, config: AMGConfig | None = None, tol: float = 1e-12,
                   maxiter: int = 1000, symmetric: bool = False, precision: str = "fp64"):
    """x = A(values)^-1 b as a differentiable torch operation (the role of a
    ChainRulesCore rrule around solve).  values: CUDA tensor of the finest
    matrix's nonzeros (the setup pattern, CSR order); b: CUDA tensor.  The
    forward pass resets the hierarchy up with `values` and solves (PCG when
    symmetric, else BiCGStab); the backward pass solves the adjoint system
    A^T lambda = dL/dx on the transposed hierarchy (or with PCG when
    symmetric), then dL/db = lambda and dL/da_ij = -lambda_i x_j.  Only x is
    kept between the passes.  precision="mixed" runs both solves with the
    FP32 cycle (FP32 copies of the hierarchy and of its transpose) inside
    the FP64 Krylov iteration."""
    import torch

    if _Solve.fn is None:
        class Fn(torch.autograd.Function):
            @staticmethod
            def forward(ctx, values, b, h, config, tol, maxiter, symmetric, precision):
                amg_resetup(h, values.detach().contiguous(), config)
                x = torch.zeros_like(b)
                bb = b.detach().contiguous()
                if symmetric:
                    _, it, rel = pcg(x, bb, h, config, tol=tol, maxiter=maxiter, precision=precision)
                else:
                    _, it, rel = bicgstab(x, bb, h, config, tol=tol, maxiter=maxiter, precision=precision)
                ctx.h, ctx.config, ctx.tol, ctx.maxiter, ctx.symmetric = h, config, tol, maxiter, symmetric
                ctx.precision = precision
                ctx.save_for_backward(x)
                return x

            @staticmethod
            def backward(ctx, gx):
                (x,) = ctx.saved_tensors
                lam = torch.zeros_like(x)
                g = gx.contiguous()
                if ctx.symmetric:
                    pcg(lam, g, ctx.h, ctx.config, tol=ctx.tol, maxiter=ctx.maxiter, precision=ctx.precision)
                else:
                    bicgstab(lam, g, ctx.h, ctx.config, tol=ctx.tol, maxiter=ctx.maxiter, transpose=True,
                             precision=ctx.precision)
                gv = nz_gradient(ctx.h, x, lam)
                return gv, lam, None, None, None, None, None, None

        _Solve.fn = Fn
    config = config if config is not None else (h.config or AMGConfig())
    if precision not in ("fp64", "mixed"):
        raise ValueError("precision must be 'fp64' or 'mixed'")
    return _Solve.fn.apply(values, b, h, config, tol, maxiter, symmetric, precision)


def pcg_multi(X, B, h: Hierarchy, config: AMGConfig | None = None, tol: float = 1e-8,
              maxiter: int = 500, precision: str = "mixed"):
    """PCG for up to 32 right-hand sides of one matrix at once.  X, B: CUDA
    float64 tensors of shape (n, k), row-major (X holds the initial guesses
    and receives the solutions).  Each product with a level matrix serves
    all k columns in one pass over the matrix.  Returns (X, iterations per
    column, relative residual per column)."""
    config = config if config is not None else (h.config or AMGConfig())
    if X.dim() != 2 or X.shape != B.shape or not X.is_contiguous() or not B.is_contiguous():
        raise ValueError("X and B must be contiguous (n, k) tensors of the same shape")
    n, k = int(X.shape[0]), int(X.shape[1])
    prec = {"fp64": 0, "mixed": 1, "fp32": 1}[precision]
    its = (C.c_int32 * k)()
    rel = (C.c_double * k)()
    lib = _lib.load()
    _lib.check(lib.draugr_b200_pcg_block_device(h.handle, n, k, X.data_ptr(), B.data_ptr(),
                                                config_handle(config), tol, maxiter, prec, its, rel),
               "pcg_multi")
    return X, list(its), list(rel)


def pcg_batch(hierarchies, xs, bs, config: AMGConfig | None = None, tol: float = 1e-8,
              maxiter: int = 500, precision: str = "mixed", workers: int = 16):
    """PCG on many independent systems at once: each hierarchy runs on its
    own CUDA stream, driven by one host thread of a pool of `workers`, so
    the small kernels of many systems share the GPU.  xs / bs: per-system
    vectors (CUDA tensors or NumPy arrays), x updated in place.  Returns a
    list of (niter, relres, seconds) per system."""
    import time
    from concurrent.futures import ThreadPoolExecutor

    def one(k):
        t0 = time.perf_counter()
        _, it, rel = pcg(xs[k], bs[k], hierarchies[k], config, tol=tol, maxiter=maxiter,
                         precision=precision)
        return it, rel, time.perf_counter() - t0

    with ThreadPoolExecutor(max_workers=max(1, min(workers, len(hierarchies)))) as ex:
        return list(ex.map(one, range(len(hierarchies))))


class BatchHierarchy(Hierarchy):
    """Independent systems merged level by level (draugr_b200_batch_setup);
    `offsets[s]:offsets[s + 1]` are system s's rows in the batch's vectors."""

    def __init__(self, handle: int, offsets: np.ndarray, config: AMGConfig | None):
        super().__init__(handle, int(offsets[-1]), config)
        self.offsets = offsets

    @property
    def nsystems(self) -> int:
        return len(self.offsets) - 1


def batch_setup(hierarchies, config: AMGConfig | None = None) -> BatchHierarchy:
    """Merge the hierarchies of independent systems into one batch (one
    launch per cycle stage for all of them).  The hierarchies stay usable."""
    lib = _lib.load()
    hs = np.ascontiguousarray([h.handle for h in hierarchies], np.int32)
    b = _lib.check(lib.draugr_b200_batch_setup(len(hs), _ptr(hs)), "batch_setup")
    ns = _lib.check(lib.draugr_b200_batch_offsets(b, None), "batch_offsets")
    off = np.zeros(ns + 1, np.int64)
    _lib.check(lib.draugr_b200_batch_offsets(b, _ptr(off)), "batch_offsets")
    return BatchHierarchy(b, off, config if config is not None else hierarchies[0].config)


def pcg_batched(x, b, batch: BatchHierarchy, config: AMGConfig | None = None, tol: float = 1e-8,
                maxiter: int = 500, precision: str = "mixed"):
    """AMG-PCG on every system of a batch at once.  x, b: CUDA float64
    tensors holding all systems' vectors (batch.offsets); x holds the
    initial guesses.  Returns (x, iterations per system, relative residuals
    per system)."""
    config = config if config is not None else (batch.config or AMGConfig())
    prec = {"fp64": 0, "mixed": 1}[precision]
    ns = batch.nsystems
    its = np.zeros(ns, np.int32)
    rel = np.zeros(ns)
    _lib.check(_lib.load().draugr_b200_batch_pcg_device(batch.handle, x.numel(), x.data_ptr(), b.data_ptr(),
                                                        config_handle(config), tol, maxiter, prec, _ptr(its),
                                                        _ptr(rel)), "pcg_batched")
    return x, its, rel


class DraugrPreconditioner:
    """One AMG cycle from a zero guess as a preconditioner, the role of
    Draugr.jl's DraugrPreconditioner (src/preconditioner.jl:12-102).

    update(A) builds the hierarchy on first use and resets it up (partial,
    same pattern) afterwards, like preconditioner_update!; apply(x, y) /
    ldiv(x, y) zero x and run one cycle for right-hand side y, like
    preconditioner_apply! / ldiv!, on NumPy arrays or CUDA tensors (x is
    updated in place and returned); nrows is preconditioner_nrows.
    as_linear_operator() wraps apply for SciPy's Krylov solvers
    (scipy.sparse.linalg.cg / gmres / bicgstab take it as M), the Python
    counterpart of the LinearSolve.jl and Krylov.jl hooks."""

    def __init__(self, config: AMGConfig | None = None, **kwargs):
        self.config = config if config is not None else AMGConfig(**kwargs)
        self.hierarchy: Hierarchy | None = None
        self.dim: tuple[int, int] | None = None

    def update(self, A):
        if self.hierarchy is None:
            self.hierarchy = amg_setup(A, self.config)
        else:
            amg_resetup(self.hierarchy, A, self.config)
        self.dim = tuple(A.shape)
        return self

    def apply(self, x, y):
        if self.hierarchy is None:
            raise _lib.DraugrError("preconditioner applied before update(A)")
        if _is_device(x):
            x.zero_()
        else:
            x[:] = 0.0
        return amg_cycle(x, y, self.hierarchy, self.config)

    ldiv = apply

    @property
    def nrows(self) -> int:
        return 0 if self.dim is None else self.dim[0]

    def as_linear_operator(self):
        import scipy.sparse.linalg as spla

        n = self.nrows

        def mv(y):
            y = np.ascontiguousarray(np.asarray(y, dtype=np.float64).reshape(-1))
            return self.apply(np.empty(n), y)

        return spla.LinearOperator((n, n), matvec=mv, dtype=np.float64)


def _check_vec(x, b, h):
    for name, a in (("x", x), ("b", b)):
        if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous):
            raise TypeError(f"{name} must be a contiguous float64 NumPy array")
        if len(a) != h.n:
            raise ValueError(f"DimensionMismatch: len({name}) = {len(a)} != {h.n}")
