"""Host plumbing of the wire/propagation grids (pulsesuite_b200.wirespace)
against the reference's own outputs (tests/golden/glue.npz): the cubic
spline resampling and the centred transforms are the same arithmetic, so
they agree bit for bit."""

import numpy as np
from helpers import golden

from pulsesuite_b200 import wirespace as ws


def test_rescale_matches_reference():
    d = golden("glue")
    np.testing.assert_array_equal(ws.rescale_1d(d["x0"], d["z0"], d["x1"]), d["z1"])


def test_centred_transforms_match_reference():
    d = golden("glue")
    F = d["z0"].copy()
    ws.fftg(F)
    np.testing.assert_array_equal(F, d["fftg"])
    G = d["z0"].copy()
    ws.ifftg(G)
    np.testing.assert_array_equal(G, d["ifftg"])
    ws.fftg(G)  # round trip
    assert np.max(np.abs(G - d["z0"])) < 1e-14 * np.max(np.abs(d["z0"]))
