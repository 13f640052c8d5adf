"""GPU parity of the many-body terms of the full-matrix step
(psb_full_step_mb_f64, switched on by mb.params DiagDph, OffDiagDph, EHs,
Phonon, Recomb, DCTrans) against outputs of the reference itself
(tests/golden, generated by importing the reference):

  * units: on random levels of the reference's own grid, one step (dt = 0,
    so the new level equals the old one) leaves in its scratch the
    k-dependent dephasing rates (CalcGammaE / CalcGammaH), the off-diagonal
    dephasing kernels and term (CalcOffDiagDeph_E2 / _H2,
    OffDiagDephasing2), the in/out scattering rates (MBCE + MBPE,
    MBCH + MBPH, Lorentzian delta) and the spontaneous-emission rates
    (SpontEmission) of the reference's functions on the same inputs;
  * solver: QWCalculator with DiagDph, OffDiagDph, EHs, Phonon, screened,
    LF, fields along the wire (Gaussian delta), and the same with Recomb and
    DCTrans in a DC field, with LF (whole matrices shifted) and without
    (diagonals shifted): every step's Pxx, Pyy, Pzz, Rho and the final nine
    levels match the reference's run.

Tolerance 1e-10 normwise (measured ~1e-13 and below).
"""

import os

import numpy as np
import pytest
import torch
from helpers import golden, relerr
from test_gpu_solver_api import QW_PARAMS

from pulsesuite_b200 import SBEs

pytestmark = pytest.mark.gpu
TOL = 1e-10
# Optics Excitons EHs Screened Phonon DCTrans LF FreePot DiagDph OffDiagDph
# Recomb PLSpec ignorewire Xqwparams LorentzDelta
MB = "1\n1\n1\n{scr}\n1\n{dc}\n{lf}\n0\n1\n1\n{rc}\n0\n0\n0\n{lor}\n"


def make_solver(tmp_path, L, gam, screened, lorentz, nw=1, recomb=False, dctrans=False, lf=True,
                edc=0.0):
    os.makedirs(tmp_path / "params", exist_ok=True)
    qw = QW_PARAMS.format(L=L, gam=gam).replace("0.0        # Edc", f"{edc!r}        # Edc")
    (tmp_path / "params" / "qw.params").write_text(qw)
    (tmp_path / "params" / "mb.params").write_text(
        MB.format(scr=int(screened), lor=int(lorentz), rc=int(recomb), dc=int(dctrans),
                  lf=int(lf)))
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        rr = np.linspace(-5e-8, 5e-8, 64)
        return SBEs.SBESolver(None, rr, 0.0, 1e7, 800e-9, nw, True)
    finally:
        os.chdir(cwd)


def scratch_views(scratch, nk):
    """GamE, GamH, De, Dh, OffP, rates (+ Rsp) in psb_full_step_mb_f64's scratch
    (layout of its MBScratch: 256-byte aligned blocks in this order)."""
    def al(x):
        return (x + 255) // 256 * 256

    n2, nd = nk * nk, (2 * nk + 1) * nk
    de = al(2 * nk * 8)
    dh = al(de + nd * 8)
    offp = al(dh + nd * 8)
    x3 = al(offp + n2 * 16)
    rates = al(x3 + 3 * n2 * 16)
    b = scratch.cpu().numpy()
    f64 = lambda o, n: b[o:o + 8 * n].view(np.float64)  # noqa: E731
    return {"GamE": f64(0, nk), "GamH": f64(8 * nk, nk),
            "De": f64(de, nd).reshape(2 * nk + 1, nk), "Dh": f64(dh, nd).reshape(2 * nk + 1, nk),
            "OffP": b[offp:offp + 16 * n2].view(np.complex128).reshape(nk, nk),
            "rates": f64(rates, 5 * nk).reshape(5, nk)}


def test_manybody_terms_match_reference_functions(cuda, tmp_path):
    d = golden("manybody_units_nk32")
    s = make_solver(tmp_path, float(d["L"]), float(d["gam"]), screened=False, lorentz=True,
                    recomb=True)
    nk = s.Nk
    assert nk == int(d["nk"])
    s._enter_full()
    F = s.full
    F["L"][1][0].copy_(torch.as_tensor(np.stack([d["p1"], d["c1"], d["d1"]])))  # X1
    F["L"][2][0].copy_(torch.as_tensor(np.stack([d["p2"], d["c2"], d["d2"]])))  # X2
    nr = s.Nr
    Ex, Ey, Ez, Vr = (np.zeros(nr, complex) for _ in range(4))
    src = [np.zeros(nr, complex) for _ in range(5)]
    s._sbe_calculator(Ex, Ey, Ez, Vr, 0.0, *src, False, 1)
    torch.cuda.synchronize()
    v = scratch_views(F["mb"].scratch, nk)
    for k in ("GamE", "GamH", "De", "Dh", "OffP"):
        assert relerr(v[k], d[k]) < TOL, (k, relerr(v[k], d[k]))
    for i, k in enumerate(("WinE", "WoutE", "WinH", "WoutH", "Rsp")):
        assert relerr(v["rates"][i], d[k]) < TOL, (k, relerr(v["rates"][i], d[k]))


@pytest.mark.parametrize("name", ["qwcalc_manybody_nk32", "qwcalc_mb_dc_lf_nk32",
                                  "qwcalc_mb_dc_diag_nk32"])
def test_qwcalculator_many_body_matches_reference(cuda, tmp_path, name):
    d = golden(name)
    dc = name.startswith("qwcalc_mb_dc")
    s = make_solver(tmp_path, float(d["L"]), float(d["gam"]), screened=True, lorentz=False,
                    nw=2, recomb=dc, dctrans=dc, lf=not name.endswith("diag_nk32"),
                    edc=float(d["edc"]) if "edc" in d else 0.0)
    rr, prof = d["rr"], d["prof"]
    n, nrr = int(d["nsteps"]), rr.size
    got = {k: np.zeros((n, 2, nrr), complex) for k in ("Pxx", "Pyy", "Pzz", "Rho")}
    for i in range(n):
        E = d["env"][i]
        for w in (1, 2):
            o = [np.zeros(nrr, complex) for _ in range(4)]
            s.QWCalculator((0.3 * E * prof * (rr / 3e-8)).astype(complex),
                           (E * prof).astype(complex), (0.2 * E * prof).astype(complex),
                           np.zeros(nrr, complex), rr, None, float(d["dt"]), w, *o,
                           [False], [False])
            for k, v in zip(("Pxx", "Pyy", "Pzz", "Rho"), o):
                got[k][i, w - 1] = v
    assert s.full is not None and s.full["mb"] is not None
    for k in ("Pyy", "Pzz", "Rho"):
        assert relerr(got[k], d[k]) < TOL, (k, relerr(got[k], d[k]))
    assert np.max(np.abs(got["Pxx"] - d["Pxx"])) < TOL * np.max(np.abs(d["Pyy"]))
    lv = s._level_arrays()
    for key in ("YY1", "YY2", "YY3", "CC1", "CC2", "CC3", "DD1", "DD2", "DD3"):
        ref = np.transpose(d[key], (2, 0, 1))
        assert relerr(lv[key], ref) < TOL, (key, relerr(lv[key], ref))
