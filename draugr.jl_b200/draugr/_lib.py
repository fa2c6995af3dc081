"""Loader for libdraugr_b200.so (the CUDA library built in this package's
directory by ``make``).  Every Python entry point of the package goes through
this module; there is no fallback implementation, so a missing or unloadable
library is an error."""

from __future__ import annotations

import ctypes as C
import os
import pathlib

PKG_DIR = pathlib.Path(__file__).resolve().parent.parent  # draugr.jl_b200/
LIB_PATH = PKG_DIR / "libdraugr_b200.so"

i32, i64, f64, f32 = C.c_int32, C.c_int64, C.c_double, C.c_float
P = C.c_void_p

# name -> (restype, argtypes); one line per symbol of include/draugr_amg.h and
# include/draugr_b200.h
SIGNATURES = {
    "init_julia": (None, [C.c_int, P]),
    "shutdown_julia": (None, [C.c_int]),
    "draugr_amg_last_error": (C.c_char_p, []),
    "draugr_amg_config_from_json": (i32, [C.c_char_p]),
    "draugr_amg_setup": (i32, [i32, i32, P, P, P, i32, i32, i32]),
    "draugr_amg_resetup": (i32, [i32, i32, i32, P, P, P, i32, i32, i32, i32]),
    "draugr_amg_solve": (i32, [i32, i32, P, P, i32, f64, i32]),
    "draugr_amg_cycle": (i32, [i32, i32, P, P, i32]),
    "draugr_amg_free": (i32, [i32]),
    "draugr_amg_config_free": (i32, [i32]),
    "draugr_b200_setup_host": (i32, [i32, i32, P, P, P, i32, i32, i32]),
    "draugr_b200_num_levels": (i32, [i32]),
    "draugr_b200_level_info": (i32, [i32, i32, P]),
    "draugr_b200_export": (i64, [i32, i32, C.c_char_p, P, i64]),
    "draugr_b200_summary": (C.c_char_p, [i32]),
    "draugr_b200_config_json": (C.c_char_p, [i32]),
    "draugr_b200_device_bytes": (i64, [i32]),
    "draugr_b200_solve_device": (i32, [i32, i32, P, P, i32, f64, i32]),
    "draugr_b200_cycle_device": (i32, [i32, i32, P, P, i32]),
    "draugr_b200_resetup_values_device": (i32, [i32, i64, P]),
    "draugr_b200_residual_device": (i32, [i32, i32, P, P, P, P]),
    "draugr_b200_galerkin_host": (i32, [i32, i32, i64, P, i64, P]),
    "draugr_b200_set_resetup_precision": (i32, [i32, i32]),
    "draugr_b200_residual_noalloc": (i32, [i32, i32, P, P, P, P, P, P, P, P]),
    "draugr_b200_pcg": (i32, [i32, i32, P, P, i32, f64, i32, i32, P]),
    "draugr_b200_pcg_device": (i32, [i32, i32, P, P, i32, f64, i32, i32, P]),
    "draugr_b200_fgmres": (i32, [i32, i32, P, P, i32, f64, i32, i32, i32, P]),
    "draugr_b200_fgmres_device": (i32, [i32, i32, P, P, i32, f64, i32, i32, i32, P]),
    "draugr_b200_refine": (i32, [i32, i32, P, P, i32, f64, i32, f64, i32, i32, i32, P, P]),
    "draugr_b200_refine_device": (i32, [i32, i32, P, P, i32, f64, i32, f64, i32, i32, i32, P, P]),
    "draugr_b200_batch_setup": (i32, [i32, P]),
    "draugr_b200_batch_offsets": (i32, [i32, P]),
    "draugr_b200_batch_pcg_device": (i32, [i32, i32, P, P, i32, f64, i32, i32, P, P]),
    "draugr_b200_bicgstab": (i32, [i32, i32, P, P, i32, f64, i32, i32, i32, P]),
    "draugr_b200_bicgstab_device": (i32, [i32, i32, P, P, i32, f64, i32, i32, i32, P]),
    "draugr_b200_nz_gradient_device": (i32, [i32, i32, P, P, P]),
    "draugr_b200_pcg_block_device": (i32, [i32, i32, i32, P, P, i32, f64, i32, i32, P, P]),
    "draugr_b200_level_op": (i32, [i32, i32, i32, i32, P, P, P, i32]),
    "draugr_b200_time_level_op": (i32, [i32, i32, i32, i32, i32, P]),
    "draugr_b200_kernel_launches": (i64, []),
    "draugr_b200_set_stream": (i32, [i32, P]),
    "draugr_b200_set_tile_wait_limit": (None, [i32]),
}

_lib = None


class DraugrError(RuntimeError):
    """A library call returned -1; the message is draugr_amg_last_error()."""


def load(path: str | os.PathLike | None = None) -> C.CDLL:
    """Load the library once (RTLD_GLOBAL not needed) and declare signatures."""
    global _lib
    if _lib is not None:
        return _lib
    p = pathlib.Path(path) if path else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(
            f"{p} is missing: build it with `make -C {PKG_DIR}` (or __graft_entry__.build())")
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    s = load().draugr_amg_last_error()
    return s.decode() if s else ""


def check(rc: int, what: str) -> int:
    if rc < 0:
        raise DraugrError(f"{what}: {last_error()}")
    return rc
