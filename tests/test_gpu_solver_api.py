"""GPU tests of the reference-named solver and Coulomb APIs
(pulsesuite_b200.SBEs.SBESolver + module shims, pulsesuite_b200.coulomb)
against outputs of the reference itself (tests/golden, generated by
importing the reference):

  * SBESolver built from the same params files, stepped through
    _sbe_calculator with a field at q = 0 of the wire, reproduces the
    reference's levels, P(t) and source terms (Px, Py, Pz; Re, Rh with LF)
    to 1e-10 normwise, and reads / writes the reference's backup files;
  * QWCalculator keeps the reference's wire-off gate and counters, and
    with fields along the wire (full Nk x Nk state, psb_full_step_f64)
    reproduces the reference's Pxx, Pyy, Pzz, Rho and levels;
  * InitializeCoulomb / CalcScreenedArrays / Eps1D / Vint / CalcChi1D /
    K03 reproduce the reference's Coulomb arrays to 1e-12.
"""

import os

import numpy as np
import pytest
from helpers import golden, relerr

from pulsesuite_b200 import SBEs, coulomb

pytestmark = pytest.mark.gpu
TOL = 1e-10

QW_PARAMS = """{L}     # L
5e-9       # Delta0
1.5        # gap
0.07       # me
0.45       # mh
100e-3     # HO
{gam}      # gam_e
{gam}      # gam_h
{gam}      # gam_eh
9.1        # epsr
36e-3      # Oph
3e-3       # Gph
0.0        # Edc
1000000    # jmax
20000      # ntmax
"""
MB = "1\n1\n0\n{scr}\n0\n0\n{lf}\n0\n0\n0\n0\n0\n0\n0\n0\n"


def make_solver(tmp_path, L, gam, screened=False, lf=False, nw=1):
    os.makedirs(tmp_path / "params", exist_ok=True)
    (tmp_path / "params" / "qw.params").write_text(QW_PARAMS.format(L=L, gam=gam))
    (tmp_path / "params" / "mb.params").write_text(MB.format(scr=int(screened), lf=int(lf)))
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        rr = np.linspace(-5e-7, 5e-7, 64)
        return SBEs.SBESolver(None, rr, 0.0, 1e7, 800e-9, nw, True)
    finally:
        os.chdir(cwd)


def diag_levels(s, w=1):
    p, c, d = s.levels(w)
    return np.stack([np.stack(p), np.stack(c), np.stack(d)])


@pytest.mark.parametrize("name", ["leapfrog_nk32", "leapfrog_screened_nk32"])
def test_solver_steps_match_reference_driver(cuda, tmp_path, name):
    d = golden(name)
    s = make_solver(tmp_path, float(d["L"]), float(d["gam"]), screened=bool(d["screened"]))
    assert s.Nk == int(d["nk"]) and s.NQ0 == int(d["NQ0"])
    np.testing.assert_allclose(s.r, d["r"], rtol=0, atol=0)
    lv = diag_levels(s)
    assert relerr(lv[1, 1].real, d["y1_init"][:, 2]) < TOL  # CC2: Fermi occupations
    nr, n = s.Nr, int(d["nsteps"])
    P = np.zeros(n, complex)
    srcs = [np.zeros(nr, complex) for _ in range(5)]
    for i in range(n):
        Ex, Ey, Ez, Vr = (np.zeros(nr, complex) for _ in range(4))
        Ey[s.NQ0] = d["field"][i]
        s._sbe_calculator(Ex, Ey, Ez, Vr, float(d["dt"]), *srcs, False, 1)
        p3 = s.levels(1)[0][2]
        P[i] = float(d["pscale"]) * np.sum(p3)
    assert relerr(P, d["P"]) < TOL
    lv = diag_levels(s)
    y2 = np.stack([lv[0, 2].real, lv[0, 2].imag, lv[1, 2].real, lv[2, 2].real], 1)
    y1 = np.stack([lv[0, 1].real, lv[0, 1].imag, lv[1, 1].real, lv[2, 1].real], 1)
    assert relerr(y2, d["y2"]) < TOL
    assert relerr(y1, d["y1"]) < TOL
    assert relerr(srcs[1], d["Py_last"]) < TOL


def test_solver_lf_sources_and_backup_files(cuda, tmp_path):
    d = golden("solver_lf_nk32")
    s = make_solver(tmp_path, float(d["L"]), float(d["gam"]), lf=True)
    assert s.Nk == int(d["nk"])
    assert abs(s.chiqw() - complex(d["chiw"])) <= 1e-12 * abs(complex(d["chiw"]))
    assert s.getqc() == pytest.approx(float(d["qc"]), rel=1e-14)
    assert s.QWArea() == pytest.approx(float(d["area"]), rel=1e-14)
    assert relerr(diag_levels(s), d["init"]) < TOL
    nr = s.Nr
    srcs = [np.zeros(nr, complex) for _ in range(5)]
    for i in range(int(d["nsteps"])):
        Ex, Ey, Ez, Vr = (np.zeros(nr, complex) for _ in range(4))
        Ey[s.NQ0] = d["field"][i]
        s._sbe_calculator(Ex, Ey, Ez, Vr, float(d["dt"]), *srcs, False, 1)
    assert relerr(diag_levels(s), d["final"]) < TOL
    for k, name in enumerate(["Py", "Pz", "Re", "Rh"], start=1):
        assert relerr(srcs[k], d[name]) < TOL, name
    # Px of a k-symmetric diagonal p cancels to rounding noise (alternating
    # dipole signs of Xcv, qwoptics.py:619-623): compared on the scale of Py
    assert np.max(np.abs(srcs[0] - d["Px"])) < TOL * np.max(np.abs(d["Py"]))
    # backup files: the reference's own text reads back to its levels ...
    bdir = tmp_path / "ref_backup"
    bdir.mkdir()
    keys = ("CC1", "CC2", "CC3", "DD1", "DD2", "DD3", "YY1", "YY2", "YY3")
    for key in keys:
        (bdir / f"{key}.7.dat").write_text(str(d[f"backup_{key}"]))
    s2 = make_solver(tmp_path, float(d["L"]), float(d["gam"]), lf=True)
    s2.read_sbes_data(7, directory=str(bdir) + "/")
    assert relerr(diag_levels(s2), d["final"]) < 1e-15
    # ... and what this solver writes for that state is the same text
    odir = tmp_path / "our_backup"
    s2.write_sbes_data(7, directory=str(odir) + "/")
    for key in keys:
        assert (odir / f"{key}.7.dat").read_text() == str(d[f"backup_{key}"]), key


def test_solver_module_shims_and_qwcalculator_gate(cuda, tmp_path):
    d = golden("leapfrog_nk32")
    s = make_solver(tmp_path, float(d["L"]), float(d["gam"]))
    SBEs._default_solver = s
    rr = np.linspace(-5e-7, 5e-7, 64)
    out = [np.ones(64, complex) for _ in range(4)]
    DoQWP, DoQWDl = [None], [None]
    weak = np.full(64, 1e3, complex)  # below 1e-3 of Emaxxx = 1e7: the wire stays off
    SBEs.QWCalculator(weak, weak, weak, weak * 0, rr, None, 1e-17, 1, *out, DoQWP, DoQWDl)
    assert all(np.all(o == 0) for o in out)
    assert DoQWP == [None] and s.xxx == 2 and s.t == pytest.approx(1e-17)
    assert s.full is None and s.wireoff
    strong = np.full(64, 1e5, complex)  # switches the wire on
    SBEs.QWCalculator(strong, strong, strong, weak * 0, rr, None, 1e-17, 1, *out, DoQWP,
                      DoQWDl)
    assert DoQWP == [True] and DoQWDl == [False] and not s.wireoff
    assert s.full is not None  # a field along the wire: full-matrix state
    assert SBEs.QWArea() == s.area and SBEs.getqc() == s.qc
    SBEs.ShutOffOptics()
    assert s.Optics is False


def test_solver_full_step_agrees_with_diagonal_step(cuda, tmp_path):
    """A q = 0 field keeps the state diagonal: stepping it on the full
    Nk x Nk state gives the diagonal kernel's numbers (1e-12), and the
    off-diagonal elements stay exactly zero."""
    d = golden("leapfrog_nk32")
    a = make_solver(tmp_path, float(d["L"]), float(d["gam"]), lf=True)
    b = make_solver(tmp_path, float(d["L"]), float(d["gam"]), lf=True)
    b._enter_full()
    nr = a.Nr
    for i in range(200):
        outs = []
        for s in (a, b):
            Ex, Ey, Ez, Vr = (np.zeros(nr, complex) for _ in range(4))
            Ey[s.NQ0] = d["field"][i]
            src = [np.zeros(nr, complex) for _ in range(5)]
            s._sbe_calculator(Ex, Ey, Ez, Vr, float(d["dt"]), *src, False, 1)
            outs.append(src)
    assert a.full is None
    assert relerr(diag_levels(b), diag_levels(a)) < 1e-12
    for x, y in zip(outs[1][1:], outs[0][1:]):  # Py, Pz, Re, Rh
        assert relerr(x, y) < 1e-12
    m = b.full["L"][2][0].cpu().numpy()
    for j in range(3):
        assert np.count_nonzero(m[j] - np.diag(np.diagonal(m[j]))) == 0


# ---------------------------------------------------------------------------
# coulomb.py names
# ---------------------------------------------------------------------------
def _kkp(kr, dk, nq0):
    return np.rint((kr[:, None] - kr[None, :]) / dk).astype(int) + nq0


@pytest.mark.parametrize("nk", [32, 114])
def test_coulomb_api_matches_reference(cuda, nk):
    d = golden(f"tables_ref_nk{nk}")
    kr, L = d["kr"], float(d["L"])
    me, mh = float(d["me"]), float(d["mh"])
    kkp = _kkp(kr, float(d["dk"]), int(d["NQ0"]))
    Ee = np.zeros(nk)
    coulomb.InitializeCoulomb(d["y"], kr, L, float(d["delta0"]), me, mh, Ee, Ee, 1e12, 1e12,
                              float(d["alphae"]), float(d["alphah"]), float(d["epsr"]),
                              d["Qr"], kkp, True)
    inst = coulomb._instance
    for name, arr in (("Veh", inst.Veh0), ("Vee", inst.Vee0), ("Vhh", inst.Vhh0)):
        assert relerr(arr[1:, 0], d[name][1:]) < 1e-12, name
    assert relerr(inst.Chi1De[:, 0], d["chie"]) < 1e-12
    assert relerr(inst.Chi1Dh[:, 0], d["chih"]) < 1e-12
    assert relerr(inst.qe[:, 0], d["qe"]) < 1e-15
    VC = np.zeros((nk, nk, 3))
    E1D = np.zeros((nk, nk))
    coulomb.CalcScreenedArrays(True, L, d["ne"].astype(complex), d["nh"].astype(complex), VC,
                               E1D)
    assert relerr(VC[1:, 0, :], d["VCs"][1:]) < 1e-12
    assert relerr(E1D[:, 0], d["E1D"]) < 1e-12
    for i, n1d in enumerate(d["dens"]):
        assert relerr(coulomb.Eps1D(n1d, nk)[:, 0], d["eps"][i]) < 1e-12
    pref = coulomb.e0**2 / (2 * np.pi * coulomb.eps0 * float(d["epsr"]) * L)
    k = nk // 3
    v = coulomb.Vint(d["Qr"][kkp[k, 0]], d["y"], float(d["alphae"]), float(d["alphah"]),
                     float(d["delta0"]))
    assert v * pref == pytest.approx(float(d["Veh"][k]), rel=1e-12)


def test_coulomb_k03_matches_reference(cuda):
    d = golden("k0_ref")
    for x, ref in zip(d["x"][::17], d["K03"][::17]):
        assert coulomb.K03(x) == pytest.approx(float(ref), rel=1e-12)


@pytest.mark.parametrize("name,screened", [("qwcalc_screened_nk32", True),
                                           ("qwcalc_nk32", False)])
def test_qwcalculator_full_matrix_matches_reference(cuda, tmp_path, name, screened):
    """QWCalculator as the PSTD caller drives it (rhoPJ.py:311-348): fields
    along the wire with a spatial profile, two wires, LF on.  The window of
    Prop2QW gives the wire field every q component, so the state is full
    Nk x Nk; every step's Pxx, Pyy, Pzz, Rho and the final nine levels
    match the reference (1e-10 normwise)."""
    d = golden(name)
    s = make_solver(tmp_path, float(d["L"]), float(d["gam"]), screened=screened, lf=True, nw=2)
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
    assert s.full is not None
    for k in ("Pyy", "Pzz", "Rho"):
        assert relerr(got[k], d[k]) < TOL, k
    assert np.max(np.abs(got["Pxx"] - d["Pxx"])) < TOL * np.max(np.abs(d["Pyy"]))
    lv = s._level_arrays()
    for key in ("YY1", "YY2", "YY3", "CC1", "CC2", "CC3", "DD1", "DD2", "DD3"):
        ref = np.transpose(d[key], (2, 0, 1))  # [w, k1, k2]
        assert relerr(lv[key], ref) < TOL, key
    # the full state round-trips through the reference's backup format
    s.write_sbes_data(3, directory=str(tmp_path / "bk") + "/")
    s2 = make_solver(tmp_path, float(d["L"]), float(d["gam"]), screened=screened, lf=True, nw=2)
    s2.read_sbes_data(3, directory=str(tmp_path / "bk") + "/")
    lv2 = s2._level_arrays()
    for key in lv:
        assert relerr(lv2[key], lv[key]) < 1e-15, key
