"""Field and source conversions between the propagation grid and the wire
grid of the reference's quantum-wire optics (host side, O(N) per call).

These are the reference's data-format plumbing around the SBE step, kept
alike so that a PSTD caller's fields and sources carry over:

  fftg / ifftg   the centred transforms FFTG / iFFTG (usefulsubs.py:2265-2334)
  rescale_1d     cubic-spline resampling of a complex array between grids
  (rescale_rows  the same for many signals at once),
                 zero outside the source range (spliner.py:153-188, with the
                 natural-end-correction spline of spline_dpc / seval_dpc,
                 spliner.py:1287-1396: the Forsythe-Malcolm-Moler spline)
  prop2qw        propagation-space fields -> windowed, real, transformed
                 wire-space fields (QWOptics.Prop2QW, qwoptics.py:673-721)
  qw2prop        wire-space sources -> propagation-space sources
                 (QWOptics.QW2Prop, qwoptics.py:723-812)
  *_rows         the same for many wires or fields at once: the splines and
                 transforms of all rows share one pass over the grid and give
                 each row the bits of its own one-signal call
  rho_post       the boundary offset, normalisation and transform of the
                 wire-space densities (QWRho5, qwoptics.py:1067-1078)

The SBE arithmetic itself (the O(Nk^2)/O(Nk^3) right-hand side and the
O(Nr Nk^2) source sums) runs in the sm_100a kernels.
"""

import numpy as np

QW_SMALL = 1e-100  # QWOptics._small (qwoptics.py:604)


def fftg(F):
    """FFTG in place: alternate-sign shift, FFT, shift, -F/N.  F is one
    signal or (m, n) rows of signals."""
    F[..., 1::2] = -F[..., 1::2]
    F[...] = np.fft.fft(F, axis=-1)
    F[..., 1::2] = -F[..., 1::2]
    F[...] = -F / float(F.shape[-1])


def ifftg(F):
    """iFFTG in place: alternate-sign shift, inverse FFT, shift, -F*N.  F is
    one signal or (m, n) rows of signals."""
    F[..., 1::2] = -F[..., 1::2]
    F[...] = np.fft.ifft(F, axis=-1)
    F[..., 1::2] = -F[..., 1::2]
    F[...] = -F * float(F.shape[-1])


def _locate(xx, x):
    """Index i with xx[i] <= x < xx[i+1] by bisection; 0 below the range and
    len(xx)-1 at or above its end."""
    n = len(xx)
    if x < xx[0]:
        return 0
    if x >= xx[n - 1]:
        return n - 1
    jl, ju = 0, n
    while ju - jl > 1:
        jm = (ju + jl) // 2
        if x >= xx[jm]:
            jl = jm
        else:
            ju = jm
    return jl


def _spline_rows(x, Y):
    """Coefficients (b, c, d), each (m, n), of the cubic splines through
    (x, Y[j]) for every row j: the Forsythe-Malcolm-Moler construction,
    whose end conditions match third derivatives of the cubics through the
    first and last four points.  Every element sees the same operations as
    a one-signal spline (the rows only share the loop over x)."""
    n = len(x)
    y = np.asarray(Y, dtype=np.complex128)
    m = y.shape[0]
    b = np.zeros((m, n), np.complex128)
    c = np.zeros((m, n), np.complex128)
    d = np.zeros((m, n), np.complex128)
    if n < 2:
        raise ValueError("Not enough points to spline.")
    if n < 3:
        b[:, 0] = (y[:, 1] - y[:, 0]) / (x[1] - x[0])
        b[:, 1] = b[:, 0]
        return b, c, d
    d[:, 0] = x[1] - x[0]
    c[:, 1] = (y[:, 1] - y[:, 0]) / d[:, 0]
    for i in range(1, n - 1):
        d[:, i] = x[i + 1] - x[i]
        b[:, i] = 2.0 * (d[:, i - 1] + d[:, i])
        c[:, i + 1] = (y[:, i + 1] - y[:, i]) / d[:, i]
        c[:, i] = c[:, i + 1] - c[:, i]
    b[:, 0] = -d[:, 0]
    b[:, n - 1] = -d[:, n - 2]
    c[:, 0] = 0.0
    c[:, n - 1] = 0.0
    if n != 3:
        c[:, 0] = c[:, 2] / (x[3] - x[1]) - c[:, 1] / (x[2] - x[0])
        c[:, n - 1] = c[:, n - 2] / (x[n - 1] - x[n - 3]) - c[:, n - 3] / (x[n - 2] - x[n - 4])
        c[:, 0] = c[:, 0] * d[:, 0] ** 2 / (x[3] - x[0])
        c[:, n - 1] = -c[:, n - 1] * d[:, n - 2] ** 2 / (x[n - 1] - x[n - 4])
    for i in range(1, n):
        t = d[:, i - 1] / b[:, i - 1]
        b[:, i] = b[:, i] - t * d[:, i - 1]
        c[:, i] = c[:, i] - t * c[:, i - 1]
    c[:, n - 1] = c[:, n - 1] / b[:, n - 1]
    for i in range(n - 2, -1, -1):
        c[:, i] = (c[:, i] - d[:, i] * c[:, i + 1]) / b[:, i]
    b[:, n - 1] = ((y[:, n - 1] - y[:, n - 2]) / d[:, n - 2]
                   + d[:, n - 2] * (c[:, n - 2] + 2.0 * c[:, n - 1]))
    for i in range(n - 1):
        b[:, i] = (y[:, i + 1] - y[:, i]) / d[:, i] - d[:, i] * (c[:, i + 1] + 2.0 * c[:, i])
        d[:, i] = (c[:, i + 1] - c[:, i]) / d[:, i]
        c[:, i] = 3.0 * c[:, i]
    c[:, n - 1] = 3.0 * c[:, n - 1]
    d[:, n - 1] = d[:, n - 2]
    return b, c, d


def _spline(x, y):
    """(b, c, d) of the cubic spline through (x, y): _spline_rows of one row."""
    b, c, d = _spline_rows(x, np.asarray(y, dtype=np.complex128)[None])
    return b[0], c[0], d[0]


def rescale_rows(x0, Z0, x1):
    """Every row of Z0 (m, len(x0)) resampled from grid x0 onto x1 by its
    cubic spline, (m, len(x1)); 0 outside [min x0, max x0].  Runs in the
    library's host code (psb_spline_rows_c128: the same operations as
    rescale_rows_numpy, the same bits)."""
    from . import _lib

    x0 = np.ascontiguousarray(x0, dtype=np.float64)
    x1 = np.ascontiguousarray(x1, dtype=np.float64)
    Z0 = np.ascontiguousarray(Z0, dtype=np.complex128)
    if Z0.ndim != 2 or Z0.shape[-1] != len(x0):
        raise ValueError("Bad sizes in rescale_1D_dpc")
    if len(x0) < 2:
        raise ValueError("Not enough points to spline.")
    out = np.empty((Z0.shape[0], len(x1)), np.complex128)
    _lib.call("psb_spline_rows_c128", x0.ctypes.data, len(x0), Z0.ctypes.data, Z0.shape[0],
              x1.ctypes.data, len(x1), out.ctypes.data)
    return out


def rescale_rows_numpy(x0, Z0, x1):
    """rescale_rows restated in numpy (the arithmetic psb_spline_rows_c128
    reproduces)."""
    x0 = np.asarray(x0, dtype=np.float64)
    Z0 = np.asarray(Z0, dtype=np.complex128)
    if Z0.shape[-1] != len(x0):
        raise ValueError("Bad sizes in rescale_1D_dpc")
    b, c, d = _spline_rows(x0, Z0)
    lo, hi = np.min(x0), np.max(x0)
    out = np.zeros((Z0.shape[0], len(x1)), np.complex128)
    for i, u in enumerate(np.asarray(x1, dtype=np.float64)):
        if lo <= u <= hi:
            j = _locate(x0, u)
            dx = u - x0[j]
            out[:, i] = Z0[:, j] + dx * (b[:, j] + dx * (c[:, j] + dx * d[:, j]))
    return out


def rescale_1d(x0, z0, x1):
    """z0 on grid x0 resampled onto x1 by the cubic spline; 0 outside
    [min x0, max x0]."""
    z0 = np.asarray(z0, dtype=np.complex128)
    if len(np.asarray(x0)) != len(z0):
        raise ValueError("Bad sizes in rescale_1D_dpc")
    return rescale_rows(x0, z0[None], x1)[0]


def prop2qw_rows(RR, F, R, window):
    """prop2qw of (m, len(RR)) rows of propagation-space fields at once:
    (m, len(R)) windowed, real, transformed wire-space fields."""
    f = rescale_rows(RR, F, R) * window
    f = np.real(f).astype(np.complex128)
    fftg(f)
    return f


def prop2qw(RR, Exx, Eyy, Ezz, Vrr, R, window):
    """Wire-space q-space fields (Ex, Ey, Ez, Vr) from the propagation-space
    fields along the wire: resampled onto the wire grid, windowed, real part,
    FFTG."""
    return list(prop2qw_rows(RR, np.stack([np.asarray(F, np.complex128)
                                           for F in (Exx, Eyy, Ezz, Vrr)]), R, window))


def rho_post(re, rh, ne, nh, dr):
    """QWRho5 after its sums: boundary offset removed (mean of the ten
    outermost points at each end), densities normalised to the carrier
    totals, FFTG; in place."""
    nr = len(re)
    for a, tot in ((re, np.sum(np.abs(ne)) + 1e-50), (rh, np.sum(np.abs(nh)) + 1e-50)):
        a[:] = a - np.real(np.sum(a[0:10]) + np.sum(a[nr - 10:nr])) / 20.0
        a[:] = a * tot / (np.sum(np.abs(a)) * dr + QW_SMALL)
        fftg(a)


def rho_post_rows(A, N, dr):
    """rho_post of many densities at once: rows of A (m, nr) with the
    occupations N (m, nk) they are normalised to; in place.  Each row's sums
    run over its own contiguous data (numpy's per-row reduction), so every
    row gets the bits of its own rho_post call."""
    nr = A.shape[-1]
    tot = np.sum(np.abs(N), axis=-1) + 1e-50
    A[...] = A - (np.real(np.sum(A[:, 0:10], axis=-1) + np.sum(A[:, nr - 10:nr], axis=-1))
                  / 20.0)[:, None]
    A[...] = A * tot[:, None] / (np.sum(np.abs(A), axis=-1) * dr + QW_SMALL)[:, None]
    fftg(A)


def qw2prop_rows(r, S, RR, plasmonics):
    """qw2prop of m wires at once: S (m, 5, len(r)) wire-space q-space
    sources Px, Py, Pz, re, rh (modified in place) -> (m, 5, len(RR))
    propagation-space Pxx, Pyy, Pzz, RhoE, RhoH.  The sums of the
    plasmonic normalisation are taken per wire, each over one contiguous
    signal, as the one-wire path takes them."""
    dr = r[1] - r[0]
    dRR = RR[1] - RR[0]
    m = S.shape[0]
    ifftg(S)
    total = None
    if plasmonics:
        # complex arithmetic throughout, as on the reference's complex arrays:
        # |x| stored as (|x|, 0), sums and divisions in complex128
        D = np.abs(S[:, 3:5]).astype(np.complex128)   # [m][2][nr], each row contiguous
        sums = np.sum(D, axis=-1)                     # per wire and density
        total = (sums[:, 0] * dr + sums[:, 1] * dr + QW_SMALL) / 2.0
        S[:, 3:5] = D * total[:, None, None] / (sums * dr + QW_SMALL)[:, :, None]
    out = rescale_rows(r, S.reshape(5 * m, -1), RR).reshape(m, 5, -1)
    if plasmonics:
        D = np.abs(out[:, 3:5]).astype(np.complex128)
        out[:, 3:5] = D * total[:, None, None] / (np.sum(D, axis=-1) * dRR + QW_SMALL)[:, :, None]
    return out


def qw2prop(r, Px, Py, Pz, re, rh, RR, plasmonics):
    """Propagation-space (Pxx, Pyy, Pzz, RhoE, RhoH) from the wire-space
    q-space sources (modified in place: transformed back and, with
    plasmonics, the densities made positive and normalised)."""
    S = np.stack([np.asarray(a, np.complex128) for a in (Px, Py, Pz, re, rh)])[None]
    out = qw2prop_rows(r, S, RR, plasmonics)
    for a, b in zip((Px, Py, Pz, re, rh), S[0]):
        a[:] = b
    return tuple(out[0])
