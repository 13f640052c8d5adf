"""Pin the CPU oracle against the reference's own outputs (tests/golden).

The goldens were produced by importing the reference (make_golden.py); these
tests need no GPU and no reference checkout.
"""

import numpy as np
import pytest
from helpers import HBAR, golden, golden_exists, grid_from, one_wire, relerr, rk4_golden_setup

from oracle import oracle as orc
from pulsesuite_b200 import grid as pgrid

TOL = 1e-12


def test_k0_matches_reference_cik01():
    d = golden("k0_ref")
    k0 = np.array([orc.k0(x) for x in d["x"]])
    assert np.max(np.abs(k0 - d["K03"]) / np.abs(d["K03"])) < 1e-13
    kj = np.array([orc.k03_crude(x) for x in d["x"]])
    np.testing.assert_array_equal(kj, d["K03_jit"])


@pytest.mark.parametrize("nk", [32, 114])
def test_reference_tables(nk):
    d = golden(f"tables_ref_nk{nk}")
    g = grid_from(d, "vint")
    ref = pgrid.reference_grid(L=float(d["L"]))
    np.testing.assert_array_equal(g.kr, ref.kr)
    np.testing.assert_array_equal(ref.y, d["y"])
    blk = orc.grid_tables(ref, screened=True).reshape(9, nk)
    # Vint tables (the q = 0 entry is never used by the SBE sums)
    for i, name in enumerate(["Veh", "Vee", "Vhh"]):
        assert relerr(blk[i][1:], d[name][1:]) < TOL
    assert relerr(blk[5], d["chie"]) < TOL
    assert relerr(blk[6], d["chih"]) < TOL
    np.testing.assert_array_equal(blk[7], d["qe"])
    np.testing.assert_array_equal(blk[8], d["qh"])
    assert ref.dens_max == pytest.approx(min(d["qe"][1], d["qh"][1]) / np.pi * 0.99, rel=1e-15)


@pytest.mark.parametrize("name", ["rhs_k0_nk16", "rhs_k0_nk32", "rhs_k0_nk64", "rhs_k0_nk128",
                                  "rhs_ref_nk32"])
def test_rhs(name):
    d = golden(name)
    nk = int(d["nk"])
    g = grid_from(d, "k0")
    cases = [(d["VC"], "dp", "dC", "dD")]
    if "VCs" in d:
        cases.append((d["VCs"], "dp_s", "dC_s", "dD_s"))
    for V, kp, kc, kd in cases:
        blk = pgrid.table_block(g, V[:, 0], V[:, 1], V[:, 2])
        tables, tabdata = pgrid.pack_tables([g], [blk])
        M = complex(d["M"])
        w = one_wire(nk, gap=float(d["gap_eff"]), gamma=float(d["gamma"]), mscale=1.0,
                     amp=abs(M), fwhm=1e30, phase=np.angle(-M))
        y = np.stack([d["p"].real, d["p"].imag, d["ne"], d["nh"]], 1).reshape(-1)
        dy = orc.rhs(tables, tabdata, w, y, HBAR, t=np.zeros(1)).reshape(nk, 4)
        assert relerr(dy[:, 0] + 1j * dy[:, 1], d[kp]) < TOL
        assert relerr(dy[:, 2], d[kc]) < TOL
        assert relerr(dy[:, 3], d[kd]) < TOL
        assert float(d["offdiag"]) == 0.0


def test_rhs_screened_from_tables():
    """Screening inside the oracle (chi tables + eps) reproduces the
    reference's CalcScreenedArrays V/eps for the same state."""
    d = golden("rhs_ref_nk32")
    nk = int(d["nk"])
    g = pgrid.reference_grid(L=float(d["L"]))
    blk = orc.grid_tables(g, screened=True).reshape(9, nk)
    blk[0:3] = d["VC"].T
    tables, tabdata = pgrid.pack_tables([g], [blk.reshape(-1)], screened=True)
    M = complex(d["M"])
    w = one_wire(nk, gap=float(d["gap_eff"]), gamma=float(d["gamma"]), mscale=1.0, amp=abs(M),
                 fwhm=1e30, phase=np.angle(-M))
    y = np.stack([d["p"].real, d["p"].imag, d["ne"], d["nh"]], 1).reshape(-1)
    dy = orc.rhs(tables, tabdata, w, y, HBAR, t=np.zeros(1)).reshape(nk, 4)
    assert relerr(dy[:, 0] + 1j * dy[:, 1], d["dp_s"]) < TOL
    assert relerr(dy[:, 2], d["dC_s"]) < TOL


@pytest.mark.parametrize("name,screened", [("rk4_c0_nk32", False), ("rk4_c0_nk64", False),
                                           ("rk4_screened_nk32", True)])
def test_rk4_trajectory(name, screened):
    d = golden(name)
    nk = int(d["nk"])
    tables, tabdata, w, y = rk4_golden_setup(d, screened=screened)
    n = int(d["nsteps"])
    P = orc.rk4(tables, tabdata, w, y, n, float(d["dt"]), HBAR, p_stride=1, p_cap=n)
    y = y.reshape(nk, 4)
    assert relerr(P, d["P"]) < TOL
    assert relerr(y[:, 0] + 1j * y[:, 1], d["p"]) < 1e-11
    assert relerr(y[:, 2], d["ne"]) < TOL
    assert relerr(y[:, 3], d["nh"]) < TOL
    assert int(w["steps"][0]) == n and w["status"][0] == 0


@pytest.mark.slow
def test_rk4_full_c0():
    if not golden_exists("rk4_c0_nk128_full"):
        pytest.skip("full c0 golden not generated")
    d = golden("rk4_c0_nk128_full")
    nk = int(d["nk"])
    tables, tabdata, w, y = rk4_golden_setup(d)
    n = int(d["nsteps"])
    P = orc.rk4(tables, tabdata, w, y, n, float(d["dt"]), HBAR, p_stride=1, p_cap=n)
    y = y.reshape(nk, 4)
    assert relerr(P, d["P"]) < TOL
    assert relerr(y[:, 0] + 1j * y[:, 1], d["p"]) < 1e-11
    assert relerr(y[:, 2], d["ne"]) < TOL


def leapfrog_setup(d):
    nk = int(d["nk"])
    scr = bool(d["screened"])
    g = grid_from(d, "vint")
    blk = pgrid.table_block(g, d["Veh"], d["Vee"], d["Vhh"], d["chie"], d["chih"])
    tables, tabdata = pgrid.pack_tables([g], [blk], screened=scr)
    w = one_wire(nk, gap=g.gap, gamma=2 * float(d["gam"]), mscale=float(d["mscale"]),
                 pscale=float(d["pscale"]))
    y1 = np.ascontiguousarray(d["y1_init"]).reshape(-1).copy()
    y2 = np.ascontiguousarray(d["y2_init"]).reshape(-1).copy()
    f = d["field"]
    field = np.stack([f.real, f.imag], 1).reshape(1, -1)
    return tables, tabdata, w, y1, y2, field, scr


@pytest.mark.parametrize("name", ["leapfrog_nk32", "leapfrog_screened_nk32"])
def test_leapfrog_trajectory(name):
    d = golden(name)
    nk = int(d["nk"])
    tables, tabdata, w, y1, y2, field, scr = leapfrog_setup(d)
    n = int(d["nsteps"])
    P = orc.leapfrog(tables, tabdata, w, y1, y2, field, n, float(d["dt"]), HBAR, p_stride=1,
                     p_cap=n)
    assert relerr(P, d["P"]) < TOL
    assert relerr(y2.reshape(nk, 4), d["y2"]) < 1e-11
    assert relerr(y1.reshape(nk, 4), d["y1"]) < 1e-11


def test_p_scalar_matches_reference_polarization():
    """P = pscale * sum_k p_k is the reference's QWPolarization3 output for a
    diagonal p (qwoptics.py:815-946): back in real space (iFFTG of the
    reference's Py) it equals Re(P) * window(r) * yw(1), with the wire window
    exp(-(r/(L/2))^150) of QWOptics.CalcQWWindow (qwoptics.py:634-655)."""
    d = golden("leapfrog_nk32")
    r = d["r"]
    window = np.exp(-((r / (float(d["L"]) / 2.0)) ** 150))
    expect = d["P"][-1].real * window * 1.0
    assert relerr(d["Py_space"], expect) < 1e-12
