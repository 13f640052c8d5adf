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


def test_row_versions_equal_one_signal_calls():
    """prop2qw_rows / qw2prop_rows (all wires of a Maxwell step at once) give
    every row the bits of its own one-signal call."""
    rng = np.random.default_rng(5)
    RR = np.linspace(-5e-8, 5e-8, 64)
    r = np.linspace(-6e-8, 6e-8, 230)
    window = np.exp(-((r / 5e-8) ** 150))
    F = (rng.standard_normal((12, 64)) + 1j * rng.standard_normal((12, 64))) * 1e7
    rows = ws.prop2qw_rows(RR, F, r, window)
    for j in range(3):
        one = ws.prop2qw(RR, F[4 * j], F[4 * j + 1], F[4 * j + 2], F[4 * j + 3], r, window)
        for k in range(4):
            np.testing.assert_array_equal(rows[4 * j + k], one[k])
    for plasmonics in (False, True):
        S = rng.standard_normal((3, 5, 230)) + 1j * rng.standard_normal((3, 5, 230))
        got = ws.qw2prop_rows(r, S.copy(), RR, plasmonics)
        for j in range(3):
            a = [S[j, k].copy() for k in range(5)]
            one = ws.qw2prop(r, *a, RR, plasmonics)
            for k in range(5):
                np.testing.assert_array_equal(got[j, k], one[k])


def test_library_spline_equals_numpy_restatement():
    """psb_spline_rows_c128 (host code of the library, used by rescale_rows)
    gives the bits of the numpy restatement, down to two-point grids."""
    rng = np.random.default_rng(12)
    for n0, n1 in ((64, 230), (230, 64), (7, 20), (4, 9), (3, 5), (2, 4)):
        if n0 > 7:
            x0, x1 = np.linspace(-5e-8, 5e-8, n0), np.linspace(-6e-8, 6e-8, n1)
        else:
            x0, x1 = np.sort(rng.uniform(-1, 1, n0)), np.linspace(-1.2, 1.2, n1)
        Z = rng.standard_normal((9, n0)) + 1j * rng.standard_normal((9, n0))
        Z *= 10.0 ** rng.integers(-8, 9, (9, 1))
        Z[2] = Z[2].real
        np.testing.assert_array_equal(ws.rescale_rows(x0, Z, x1),
                                      ws.rescale_rows_numpy(x0, Z, x1))


def test_rho_post_rows_equals_one_wire_calls():
    rng = np.random.default_rng(13)
    A = rng.standard_normal((6, 230)) + 1j * rng.standard_normal((6, 230))
    N = rng.uniform(0, 1, (6, 114)) + 1j * rng.standard_normal((6, 114)) * 1e-3
    got = A.copy()
    ws.rho_post_rows(got, N, 5e-10)
    for j in range(0, 6, 2):
        re, rh = A[j].copy(), A[j + 1].copy()
        ws.rho_post(re, rh, N[j], N[j + 1], 5e-10)
        np.testing.assert_array_equal(got[j], re)
        np.testing.assert_array_equal(got[j + 1], rh)
