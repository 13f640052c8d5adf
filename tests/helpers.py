"""Shared test helpers: golden loading and single-wire set-up."""

import os

import numpy as np
from scipy.constants import hbar

from pulsesuite_b200 import abi
from pulsesuite_b200 import grid as pgrid

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden(name):
    with np.load(os.path.join(GOLDEN, name + ".npz")) as f:
        return {k: f[k] for k in f.files}


def golden_exists(name):
    return os.path.exists(os.path.join(GOLDEN, name + ".npz"))


def grid_from(d, vkind):
    g = pgrid.Grid(nk=int(d["nk"]), dk=float(d["dk"]), kr=d["kr"], L=float(d["L"]),
                   me=float(d["me"]), mh=float(d["mh"]), epsr=float(d["epsr"]),
                   delta0=float(d["delta0"]), alphae=float(d["alphae"]),
                   alphah=float(d["alphah"]), vkind=vkind, radius=float(d["radius"]),
                   y=d.get("y"), gap=float(d["gap"]), dcv=float(d["dcv"]),
                   ehint=float(d["ehint"]), area=float(d["area"]))
    return g


def relerr(x, ref):
    """Normwise relative error max|x - ref| / max|ref|."""
    x, ref = np.asarray(x), np.asarray(ref)
    den = np.max(np.abs(ref))
    return float(np.max(np.abs(x - ref)) / (den if den > 0 else 1.0))


def one_wire(nk, gap=0.0, gamma=0.0, mscale=0.0, pscale=1.0, amp=0.0, t0=0.0, fwhm=1.0,
             phase=0.0, p_off=0):
    w = np.zeros(1, dtype=abi.WIRE_DTYPE)
    w["table"] = 0
    w["npulse"] = 1 if amp != 0.0 else 0
    w["off"] = 0
    w["gap"] = gap
    w["gamma"] = gamma
    w["mscale"] = mscale
    w["pscale"] = pscale
    w["amp"][0, 0] = amp
    w["t0"][0, 0] = t0
    w["fwhm"][0, :] = fwhm
    w["phase"][0, 0] = phase
    w["p_off"] = p_off
    return w


def rk4_golden_setup(d, screened=False):
    """Tables, wire and zero state for an rk4_* golden case."""
    g = grid_from(d, "k0")
    nk = g.nk
    v = d["V"]
    chie = chih = None
    if screened:
        from oracle import oracle as orc

        chie = orc.chi1d_table(g.qe, g.alphae, g.delta0, g.me, g.chi_scale)
        chih = orc.chi1d_table(g.qh, g.alphah, g.delta0, g.mh, g.chi_scale)
    blk = pgrid.table_block(g, v, v, v, chie, chih)
    tables, tabdata = pgrid.pack_tables([g], [blk], screened=screened)
    w = one_wire(nk, gap=float(d["gap_eff"]), gamma=float(d["gamma"]),
                 mscale=float(d["mscale"]), pscale=float(d["pscale"]), amp=float(d["amp"]),
                 t0=float(d["t0"]), fwhm=float(d["fwhm"]))
    y = np.zeros(4 * nk)
    return tables, tabdata, w, y


HBAR = hbar
