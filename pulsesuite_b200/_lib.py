"""ctypes binding of the sm_100a library (include/pulsesuite_b200.h).

The library is required: there is no CPU fallback.  Loading fails loudly if
the shared object is missing or the process has no CUDA device.
"""

import ctypes
import os

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpulsesuite_b200.so")

_lib = None

vp, i32, i64, f64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_double

_SIGNATURES = {
    "psb_abi_version": ([], i32),
    "psb_last_error": ([], ctypes.c_char_p),
    "psb_device_arch": ([vp], i32),
    "psb_coulomb_vint": ([vp, i32, vp, i32, f64, f64, f64, f64, vp, vp], i32),
    "psb_coulomb_k0": ([vp, i32, f64, f64, vp, vp], i32),
    "psb_chi1d": ([vp, i32, f64, f64, f64, f64, vp, vp], i32),
    "psb_screen_f64": ([vp, i32, vp, vp, i32, vp, vp, i32, vp], i32),
    "psb_rhs_f64": ([vp, i32, vp, i64, vp, i32, vp, vp, i64, i32, i32, vp, vp], i32),
    "psb_calch_f64": ([vp, i32, vp, i64, vp, i32, vp, vp, i64, i32, i32, vp, vp], i32),
    "psb_rk4_f64": ([vp, i32, vp, i64, vp, i32, vp, i32, vp, i64, i32, i32, i32, f64, vp, i64,
                     i32, i32, vp, vp], i32),
    "psb_leapfrog_f64": ([vp, i32, vp, i64, vp, i32, vp, i32, vp, vp, i64, i32, i32, vp, i64,
                          i64, i32, f64, vp, i64, i32, i32, vp, vp], i32),
    "psb_f64_smem_bytes": ([i32, i32], i32),
    "psb_diag_derivs_f64": ([vp, vp, vp, vp, f64, vp, i64, vp], i32),
    "psb_probe_fp64_fma": ([i32, i32, vp, vp, vp], i32),
    "psb_full_work_bytes": ([i32], i64),
    "psb_full_step_f64": ([i32, i32, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, i64, vp], i32),
    "psb_full_sources_f64": ([i32, i32, vp, vp, vp, f64, f64, f64, f64, vp, vp, vp], i32),
    "psb_full_mb_scratch_bytes": ([i32], i64),
    "psb_full_batch_work_bytes": ([i32, i32], i64),
    "psb_spline_rows_c128": ([vp, i32, vp, i32, vp, i32, vp], i32),
    "psb_full_step_batch_f64": ([i32, i32, i32, i32, vp, f64, f64, i32, vp, vp, vp, vp, vp, vp,
                                 vp, vp, i64, vp], i32),
    "psb_full_sources_batch_f64": ([i32, i32, i32, vp, vp, vp, f64, f64, vp, vp, vp, vp], i32),
    "psb_mb_tables_f64": ([i32, vp, vp, f64, f64, f64, i32, vp, vp], i32),
    "psb_full_step_mb_f64": ([i32, i32, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, i64, vp],
                             i32),
    "psb_split_ws_bytes": ([i64], i64),
    "psb_split_set_wait_limit": ([ctypes.c_uint32], i32),
    "psb_split_smem_bytes": ([i32, i32], i32),
    "psb_split_max_nk": ([i32], i32),
    "psb_split_max_nk_resident": ([i32], i32),
    "psb_rk4_split": ([vp, i32, vp, i64, vp, i32, vp, i32, i32, i32, vp, i64, vp, i64, i32,
                       f64, vp, i64, i32, i32, vp, vp], i32),
    "psb_rk4_split_noalloc": ([vp, i32, vp, i64, vp, i32, vp, i32, i32, i32, vp, i64, i32, f64,
                               vp, i64, i32, i32, vp, vp], i32),
    "psb_rk4_split_wire": ([vp, i32, vp, i64, vp, i32, vp, i32, i32, i32, i32, vp, i64, vp, i64,
                            i32, f64, vp, i64, i32, i32, vp, vp], i32),
    "psb_split_wire_max_group": ([i32, i32], i32),
    "psb_split_wire_smem_bytes": ([i32, i32, i32], i32),
}


class PsbError(RuntimeError):
    pass


def load():
    """Load the library (building it first if this tree has no build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        from . import build

        build.build()
    lib = ctypes.CDLL(LIB_PATH)
    for name, (args, res) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    if lib.psb_abi_version() != abi.PSB_ABI_VERSION:
        raise PsbError("libpulsesuite_b200.so ABI version mismatch")
    _lib = lib
    return lib


def check(rc, what=""):
    if rc != abi.PSB_OK:
        msg = load().psb_last_error().decode(errors="replace")
        raise PsbError(f"{what} failed ({rc}): {msg}")


def call(name, *args):
    rc = getattr(load(), name)(*args)
    check(rc, name)
    return rc
