"""GPU tests of the reference-named SBE facade (pulsesuite_b200.SBEs) against
the reference's own CalcH + dpdt/dCdt/dDdt outputs (tests/golden, generated
by importing the reference): plain FP64, tolerance 1e-10 normwise."""

import numpy as np
import pytest
from helpers import golden, golden_exists, grid_from, relerr

from pulsesuite_b200 import SBEs

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _run(d, g, VC):
    nk = g.nk
    SBEs.configure(g.Ee, g.Eh, float(d["gap_eff"]))
    Meh = np.diag(np.full(nk, complex(d["M"])))
    C = np.diag(d["ne"].astype(complex))
    D = np.diag(d["nh"].astype(complex))
    P = np.diag(d["p"].astype(complex))
    Z = np.zeros((nk, nk), complex)
    Heh, Hee, Hhh = (np.zeros((nk, nk), complex) for _ in range(3))
    SBEs.CalcH(Meh, Z, Z, C, D, P, VC, Heh, Hee, Hhh)
    G = np.full(nk, float(d["gamma"]) / 2.0)
    dp = SBEs.dpdt(C, D, P, Heh, Hee, Hhh, G, G, Z)
    dC = SBEs.dCdt(C, D, P, Heh, Hee, Hhh, G, G, Z)
    dD = SBEs.dDdt(C, D, P, Heh, Hee, Hhh, G, G, Z)
    return np.diag(dp), np.diag(dC), np.diag(dD), dp


@pytest.mark.parametrize("name", ["rhs_ref_nk32", "rhs_k0_nk16", "rhs_k0_nk64"])
def test_facade_matches_reference_rhs(cuda, name):
    if not golden_exists(name):
        pytest.skip("golden missing")
    d = golden(name)
    g = grid_from(d, "k0")
    dp, dC, dD, full = _run(d, g, d["VC"])
    assert relerr(dp, d["dp"]) < TOL
    assert relerr(dC, d["dC"]) < TOL
    assert relerr(dD, d["dD"]) < TOL
    assert np.max(np.abs(full - np.diag(np.diag(full)))) == 0.0


def test_facade_screened_rhs(cuda):
    d = golden("rhs_ref_nk32")
    if "dp_s" not in d:
        pytest.skip("no screened case")
    g = grid_from(d, "k0")
    dp, dC, dD, _ = _run(d, g, d["VCs"])
    assert relerr(dp, d["dp_s"]) < TOL
    assert relerr(dC, d["dC_s"]) < TOL


def test_facade_rejects_offdiagonal_state(cuda):
    d = golden("rhs_k0_nk16")
    g = grid_from(d, "k0")
    nk = g.nk
    SBEs.configure(g.Ee, g.Eh, 0.0)
    P = np.diag(d["p"].astype(complex))
    P[0, 1] = 1e-3
    Z = np.zeros((nk, nk), complex)
    H = [np.zeros((nk, nk), complex) for _ in range(3)]
    with pytest.raises(NotImplementedError):
        SBEs.CalcH(Z, Z, Z, Z, Z, P, d["VC"], *H)
