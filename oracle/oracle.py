"""ctypes wrapper of the CPU oracle (``libsbe_oracle.so``).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA product path.  Only
tests/, ``__graft_entry__.smoke()`` and bench.py's cpu_baseline /
``--impl reference`` legs import this module; the product package never does.

Every function restates a reference function (see ``sbe_oracle.c`` for the
file:line citations); parity of the restatement with the reference itself is
pinned by ``tests/golden`` (vectors generated by importing the reference).
"""

import ctypes
import os
import subprocess

import numpy as np

from pulsesuite_b200 import abi, grid

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libsbe_oracle.so")

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.orc_k03_crude.restype = d
        L.orc_k03_crude.argtypes = [d]
        L.orc_k0.restype = d
        L.orc_k0.argtypes = [d]
        L.orc_i0.restype = d
        L.orc_i0.argtypes = [d]
        L.orc_vint_table.argtypes = [vp, i, vp, i, d, d, d, d, vp]
        L.orc_k0_table.argtypes = [vp, i, d, d, vp]
        L.orc_chi1d_table.argtypes = [vp, i, d, d, d, d, vp]
        L.orc_rhs.argtypes = [vp, i, vp, vp, i, vp, vp, vp, vp]
        L.orc_rhs.restype = i
        L.orc_rk4.argtypes = [vp, i, vp, vp, i, vp, i, d, vp, i, i, vp, i]
        L.orc_rk4.restype = i
        L.orc_leapfrog.argtypes = [vp, i, vp, vp, i, vp, vp, vp, i, i, d, vp, i, i, vp, i]
        L.orc_leapfrog.restype = i
        _lib = L
    return _lib


def _c(a, dtype=np.float64):
    return np.ascontiguousarray(a, dtype=dtype)


def k03_crude(x):
    return lib().orc_k03_crude(float(x))


def k0(x):
    return lib().orc_k0(float(x))


def vint_table(qy, y, alpha1, alpha2, delta0, prefactor):
    qy, y = _c(qy), _c(y)
    out = np.zeros(qy.size)
    lib().orc_vint_table(abi.as_ptr(qy), qy.size, abi.as_ptr(y), y.size, alpha1, alpha2, delta0,
                         prefactor, abi.as_ptr(out))
    return out


def k0_table(q, radius, prefactor):
    q = _c(q)
    out = np.zeros(q.size)
    lib().orc_k0_table(abi.as_ptr(q), q.size, radius, prefactor, abi.as_ptr(out))
    return out


def chi1d_table(qc, alpha, delta0, mass, scale):
    qc = _c(qc)
    out = np.zeros(qc.size)
    lib().orc_chi1d_table(abi.as_ptr(qc), qc.size, alpha, delta0, mass, scale, abi.as_ptr(out))
    return out


def grid_tables(g, screened=False):
    """Table block of one grid with V and chi evaluated by the oracle."""
    if g.vkind == "vint":
        qy = g.qy
        veh = vint_table(qy, g.y, g.alphae, g.alphah, g.delta0, g.vprefactor)
        vee = vint_table(qy, g.y, g.alphae, g.alphae, g.delta0, g.vprefactor)
        vhh = vint_table(qy, g.y, g.alphah, g.alphah, g.delta0, g.vprefactor)
    else:
        veh = k0_table(g.qy, g.radius, g.vprefactor)
        vee = veh.copy()
        vhh = veh.copy()
    chie = chih = None
    if screened:
        chie = chi1d_table(g.qe, g.alphae, g.delta0, g.me, g.chi_scale)
        chih = chi1d_table(g.qh, g.alphah, g.delta0, g.mh, g.chi_scale)
    return grid.table_block(g, veh, vee, vhh, chie, chih)


def rhs(tables, tabdata, wires, y, hbar, t=None):
    tables, wires = _c(tables, abi.TABLE_DTYPE), _c(wires, abi.WIRE_DTYPE)
    tabdata, y = _c(tabdata), _c(y)
    dy = np.zeros_like(y)
    model = abi.model_array(hbar)
    tt = None if t is None else _c(t)
    rc = lib().orc_rhs(abi.as_ptr(tables), tables.size, abi.as_ptr(tabdata), abi.as_ptr(wires),
                       wires.size, None if tt is None else abi.as_ptr(tt), abi.as_ptr(y),
                       abi.as_ptr(dy), abi.as_ptr(model))
    if rc:
        raise RuntimeError(f"orc_rhs failed: {rc}")
    return dy


def rk4(tables, tabdata, wires, y, nsteps, dt, hbar, p_stride=0, p_cap=0, nthreads=0):
    """In place on wires (t, steps, status) and y; returns the P(t) records."""
    tables = _c(tables, abi.TABLE_DTYPE)
    tabdata = _c(tabdata)
    assert wires.flags["C_CONTIGUOUS"] and wires.dtype == abi.WIRE_DTYPE
    assert y.flags["C_CONTIGUOUS"] and y.dtype == np.float64
    P = None
    if p_stride > 0 and p_cap > 0:
        P = np.zeros(2 * (int(wires["p_off"].max()) + p_cap))
    model = abi.model_array(hbar)
    rc = lib().orc_rk4(abi.as_ptr(tables), tables.size, abi.as_ptr(tabdata), abi.as_ptr(wires),
                       wires.size, abi.as_ptr(y), nsteps, dt,
                       None if P is None else abi.as_ptr(P), p_stride, p_cap,
                       abi.as_ptr(model), nthreads)
    if rc:
        raise RuntimeError(f"orc_rk4 failed: {rc}")
    return None if P is None else P.view(np.complex128)


def leapfrog(tables, tabdata, wires, y1, y2, field, nsteps, dt, hbar, p_stride=0, p_cap=0,
             nthreads=0):
    tables = _c(tables, abi.TABLE_DTYPE)
    tabdata = _c(tabdata)
    field = _c(field)
    assert field.ndim == 2 and field.shape[0] == wires.size
    P = None
    if p_stride > 0 and p_cap > 0:
        P = np.zeros(2 * (int(wires["p_off"].max()) + p_cap))
    model = abi.model_array(hbar)
    rc = lib().orc_leapfrog(abi.as_ptr(tables), tables.size, abi.as_ptr(tabdata),
                            abi.as_ptr(wires), wires.size, abi.as_ptr(y1), abi.as_ptr(y2),
                            abi.as_ptr(field), field.shape[1], nsteps, dt,
                            None if P is None else abi.as_ptr(P), p_stride, p_cap,
                            abi.as_ptr(model), nthreads)
    if rc:
        raise RuntimeError(f"orc_leapfrog failed: {rc}")
    return None if P is None else P.view(np.complex128)
