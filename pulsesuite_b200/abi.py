"""C-ABI struct layouts of ``include/pulsesuite_b200.h`` as numpy dtypes.

The host builds tables, wires and model constants as numpy structured
arrays with exactly the C layout, then copies them to device memory (torch
uint8 tensors) and passes raw pointers through ctypes.
"""

import ctypes

import numpy as np

PSB_ABI_VERSION = 1

PSB_OK = 0
PSB_ERR_INVALID = -1
PSB_ERR_CUDA = -2
PSB_ERR_SIZE = -3
PSB_ERR_NONFINITE = -4
PSB_ERR_UNSUPPORTED = -5
PSB_ERR_TIMEOUT = -6

PSB_MAX_NK = 1024

PSB_TAB_EXCITONS = 1
PSB_TAB_SCREENED = 2
PSB_TAB_SHARED_V = 4

# Blocks of a table in the packed tabdata array (each nk doubles).
TAB_VEH, TAB_VEE, TAB_VHH, TAB_EE, TAB_EH, TAB_CHIE, TAB_CHIH, TAB_QE, TAB_QH = range(9)
TAB_BLOCKS = 9

TABLE_DTYPE = np.dtype(
    [("nk", "<i4"), ("flags", "<i4"), ("off", "<i8"), ("L", "<f8"), ("dens_max", "<f8")],
    align=True,
)

WIRE_DTYPE = np.dtype(
    [
        ("table", "<i4"),
        ("npulse", "<i4"),
        ("off", "<i8"),
        ("gap", "<f8"),
        ("gamma", "<f8"),
        ("mscale", "<f8"),
        ("pscale", "<f8"),
        ("t", "<f8"),
        ("amp", "<f8", (2,)),
        ("t0", "<f8", (2,)),
        ("fwhm", "<f8", (2,)),
        ("phase", "<f8", (2,)),
        ("p_off", "<i8"),
        ("status", "<i4"),
        ("steps", "<i4"),
    ],
    align=True,
)

MODEL_DTYPE = np.dtype([("hbar", "<f8"), ("flags", "<i4"), ("reserved", "<i4")], align=True)

FULL_PARAMS_DTYPE = np.dtype(
    [("ehint", "<f8"), ("dcv", "<f8"), ("yw", "<f8"), ("sgnw", "<f8"), ("gap", "<f8"),
     ("gam_e", "<f8"), ("gam_h", "<f8"), ("hbar", "<f8"), ("dt", "<f8"), ("excitons", "<i4"),
     ("lf", "<i4")],
    align=True,
)

# PsbFullMB: flags, rates, and device pointers (as uint64)
FULL_MB_DTYPE = np.dtype(
    [("diag_dph", "<i4"), ("offdiag_dph", "<i4"), ("ehs", "<i4"), ("phonon", "<i4"),
     ("gam_e", "<f8"), ("gam_h", "<f8"), ("gam_eh", "<f8"), ("vscale", "<f8"),
     ("maps", "<u8"), ("iq", "<u8"), ("xe", "<u8"), ("xh", "<u8"), ("C", "<u8"), ("ph", "<u8"),
     ("eps", "<u8"), ("scratch", "<u8"), ("recomb", "<i4"), ("dctrans", "<i4"),
     ("dc_dk", "<f8"), ("dhw", "<f8"), ("rho0_den", "<f8"), ("n_hw", "<i4"), ("pad_", "<i4"),
     ("emis", "<u8"), ("Y", "<u8")],
    align=True,
)

PSB_SPLIT_WMAX = 16
PSB_SPLIT_NOALLOC_SCRATCH_BYTES = 8 * 1024 * 1024
PSB_SPLIT_NOALLOC_MAX_STATE = (PSB_SPLIT_NOALLOC_SCRATCH_BYTES - 32) // 64
SPLIT_GROUP_DTYPE = np.dtype(
    [("table", "<i4"), ("nw", "<i4"), ("wire", "<i4", (PSB_SPLIT_WMAX,))], align=True)

assert TABLE_DTYPE.itemsize == 32
assert WIRE_DTYPE.itemsize == 136
assert MODEL_DTYPE.itemsize == 16
assert FULL_PARAMS_DTYPE.itemsize == 80
assert FULL_MB_DTYPE.itemsize == 168
assert SPLIT_GROUP_DTYPE.itemsize == 72


def model_array(hbar):
    m = np.zeros(1, dtype=MODEL_DTYPE)
    m["hbar"] = hbar
    return m


def as_ptr(arr):
    """ctypes void pointer of a C-contiguous numpy array."""
    assert arr.flags["C_CONTIGUOUS"]
    return ctypes.c_void_p(arr.ctypes.data)
