"""GPU tests of the batched PSTD coupling: SBESolver.QWCalculatorAll steps
all wires of a Maxwell step in one launch set (psb_full_step_batch_f64,
psb_full_sources_batch_f64), replacing rhoPJ.QuantumWire's loop of
QWCalculator calls (rhoPJ.py:311-348).

  * against the reference's own runs (tests/golden, two wires that see the
    same field, as rhoPJ samples them): plain (screened and unscreened) and
    with the many-body terms (DiagDph, OffDiagDph, EHs, Phonon; with Recomb
    and DCTrans in a DC field, LF on and off), every step's Pxx, Pyy, Pzz,
    Rho and the final nine levels, 1e-10 normwise;
  * against the same solver stepped one QWCalculator call per wire: five
    wires with different fields, screened, all many-body flags, the
    wire-off gate switching on mid-batch -- outputs, counters and levels
    bitwise equal.
"""

import os

import numpy as np
import pytest
import torch
from helpers import golden, relerr
from test_gpu_manybody import MB
from test_gpu_solver_api import QW_PARAMS

from pulsesuite_b200 import SBEs

pytestmark = pytest.mark.gpu
TOL = 1e-10
KEYS = ("Pxx", "Pyy", "Pzz", "Rho")
LEVELS = ("YY1", "YY2", "YY3", "CC1", "CC2", "CC3", "DD1", "DD2", "DD3")
# Optics Excitons EHs Screened Phonon DCTrans LF FreePot DiagDph OffDiagDph
# Recomb PLSpec ignorewire Xqwparams LorentzDelta
PLAIN = "1\n1\n0\n{scr}\n0\n0\n1\n0\n0\n0\n0\n0\n0\n0\n0\n"


def make_solver(path, L, gam, nw, mb_text, edc=0.0, nrr=64):
    os.makedirs(path / "params", exist_ok=True)
    qw = QW_PARAMS.format(L=L, gam=gam).replace("0.0        # Edc", f"{edc!r}        # Edc")
    (path / "params" / "qw.params").write_text(qw)
    (path / "params" / "mb.params").write_text(mb_text)
    cwd = os.getcwd()
    os.chdir(path)
    try:
        rr = np.linspace(-5e-8, 5e-8, nrr)
        return SBEs.SBESolver(None, rr, 0.0, 1e7, 800e-9, nw, True)
    finally:
        os.chdir(cwd)


def golden_case(name):
    """(golden, mb.params text, Edc) of one reference QWCalculator run."""
    d = golden(name)
    edc = float(d["edc"]) if "edc" in d else 0.0
    if name in ("qwcalc_screened_nk32", "qwcalc_nk32"):
        return d, PLAIN.format(scr=int(name == "qwcalc_screened_nk32")), edc
    dc = name.startswith("qwcalc_mb_dc")
    return d, MB.format(scr=1, lor=0, rc=int(dc), dc=int(dc),
                        lf=int(not name.endswith("diag_nk32"))), edc


@pytest.mark.parametrize("name", ["qwcalc_screened_nk32", "qwcalc_nk32", "qwcalc_manybody_nk32",
                                  "qwcalc_mb_dc_lf_nk32", "qwcalc_mb_dc_diag_nk32"])
def test_all_wires_in_one_call_match_reference(cuda, tmp_path, name):
    d, mb_text, edc = golden_case(name)
    s = make_solver(tmp_path, float(d["L"]), float(d["gam"]), 2, mb_text, edc)
    rr, prof = d["rr"], d["prof"]
    n, nrr = int(d["nsteps"]), rr.size
    got = {k: np.zeros((n, 2, nrr), complex) for k in KEYS}
    for i in range(n):
        E = d["env"][i]
        o = [np.zeros((nrr, 2), complex) for _ in range(4)]
        s.QWCalculatorAll((0.3 * E * prof * (rr / 3e-8)).astype(complex),
                          (E * prof).astype(complex), (0.2 * E * prof).astype(complex),
                          np.zeros(nrr, complex), rr, None, float(d["dt"]), *o, [False], [False])
        for k, v in zip(KEYS, o):
            got[k][i] = v.T
    assert s.full is not None
    for k in ("Pyy", "Pzz", "Rho"):
        assert relerr(got[k], d[k]) < TOL, (k, relerr(got[k], d[k]))
    assert np.max(np.abs(got["Pxx"] - d["Pxx"])) < TOL * np.max(np.abs(d["Pyy"]))
    lv = s._level_arrays()
    for key in LEVELS:
        ref = np.transpose(d[key], (2, 0, 1))
        assert relerr(lv[key], ref) < TOL, (key, relerr(lv[key], ref))


def test_batch_equals_wire_by_wire_bitwise(cuda, tmp_path):
    nw, nrr, nsteps, dt = 5, 64, 40, 1e-17
    mb_text = MB.format(scr=1, lor=0, rc=1, dc=1, lf=1)
    a = make_solver(tmp_path / "a", 2.85e-8, 5e12, nw, mb_text, edc=2e6)
    b = make_solver(tmp_path / "b", 2.85e-8, 5e12, nw, mb_text, edc=2e6)
    rr = np.linspace(-5e-8, 5e-8, nrr)
    prof = np.exp(-((rr / 3e-8) ** 2))
    scale = np.array([0.7, 1.0, 1.3, 0.4, 1.1])       # a different field on every wire
    shift = np.array([-1e-8, 0.0, 5e-9, 1.5e-8, -5e-9])
    for i in range(nsteps):
        E = 2e8 * np.exp(-(((i * dt - 1e-16) / 1e-16) ** 2)) * np.cos(3.5e15 * i * dt)
        # wires 1-2 stay below the wire-off threshold in the first step, so
        # the gate switches the solver on at wire 3 of that step
        gate = np.where(np.arange(nw) < 2, 1e-5, 1.0) if i == 0 else np.ones(nw)
        pr = np.exp(-(((rr[:, None] - shift[None]) / 3e-8) ** 2)) * scale[None] * gate[None]
        Ex = (0.3 * E * pr * (rr[:, None] / 3e-8)).astype(complex)
        Ey = (E * pr).astype(complex)
        Ez = (0.2 * E * pr).astype(complex)
        Vr = np.zeros((nrr, nw), complex)
        oa = [np.zeros((nrr, nw), complex) for _ in range(4)]
        pa, da = [False], [False]
        a.QWCalculatorAll(Ex, Ey, Ez, Vr, rr, None, dt, *oa, pa, da)
        ob = [np.zeros((nrr, nw), complex) for _ in range(4)]
        pb, db = [False], [False]
        for w in range(nw):
            o = [np.zeros(nrr, complex) for _ in range(4)]
            b.QWCalculator(Ex[:, w], Ey[:, w], Ez[:, w], Vr[:, w], rr, None, dt, w + 1, *o, pb,
                           db)
            for x, y in zip(ob, o):
                x[:, w] = y
        for x, y in zip(oa, ob):
            assert np.array_equal(x, y), i
        assert (pa, da) == (pb, db)
        assert (a.xxx, a.jjj, a.t, a.wireoff) == (b.xxx, b.jjj, b.t, b.wireoff)
        if i == 0:
            assert np.all(oa[1][:, :2] == 0) and np.any(oa[1][:, 2] != 0)
    torch.cuda.synchronize()
    la, lb = a._level_arrays(), b._level_arrays()
    for key in LEVELS:
        assert np.array_equal(la[key], lb[key]), key
    assert np.max(np.abs(la["CC3"][0] - la["CC3"][1])) > 0  # the wires differ
