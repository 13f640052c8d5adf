"""Host-made tables of the many-body terms (pulsesuite_b200.manybody), CPU
only, against the reference's own module state captured in
tests/golden/manybody_units_nk32.npz (made by importing the reference):

  * the photon-energy grid HOmega and weights square of InitializeEmission
    (emission.py:35-92, CalcHOmega :220-256): bit-identical;
  * the FFT wavenumbers Y of InitializeDC (dcfield.py:782-793): bit-identical;
  * the DC shift of one Transport call (dcfield.py:1240) and CalcHOmega's
    failure on a zero width.
"""

import numpy as np
import pytest
from helpers import golden

from pulsesuite_b200 import manybody


def test_emission_tables_match_reference():
    d = golden("manybody_units_nk32")
    hw, sq, dhw, den = manybody.emission_tables(float(d["dcv"]), float(d["epsr"]),
                                                float(d["gam_eh"]), float(d["ehint"]))
    assert np.array_equal(hw, d["HOmega"])
    assert np.array_equal(sq, d["square"])
    assert dhw == d["HOmega"][1] - d["HOmega"][0]
    assert den > 0.0
    # the sign of dcv does not matter (InitializeEmission takes |dcv|)
    assert np.array_equal(manybody.emission_tables(-float(d["dcv"]), float(d["epsr"]),
                                                   float(d["gam_eh"]), float(d["ehint"]))[1],
                          d["square"])


def test_emission_zero_width_raises():
    # CalcHOmega divides by min(kB T, hbar geh) / 20: a zero width fails there,
    # as the reference's Python-float division does
    with pytest.raises(ZeroDivisionError):
        manybody.emission_tables(1e-29, 9.1, 0.0, 1.0)


def test_dc_wavenumbers_match_reference():
    d = golden("manybody_units_nk32")
    assert np.array_equal(manybody.dc_wavenumbers(d["kr"]), d["Ydc"])


def test_dc_shift():
    assert manybody.dc_shift(0.0, 0.0, 1e-17) == 0.0
    from scipy.constants import e as e0
    from scipy.constants import hbar
    assert manybody.dc_shift(2e6, 5.0, 1e-17) == -e0 * (2e6 + 5.0) / hbar * 1e-17
