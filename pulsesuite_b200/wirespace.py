"""Field and source conversions between the propagation grid and the wire
grid of the reference's quantum-wire optics (host side, O(N) per call).

These are the reference's data-format plumbing around the SBE step, kept
alike so that a PSTD caller's fields and sources carry over:

  fftg / ifftg   the centred transforms FFTG / iFFTG (usefulsubs.py:2265-2334)
  rescale_1d     cubic-spline resampling of a complex array between grids,
                 zero outside the source range (spliner.py:153-188, with the
                 natural-end-correction spline of spline_dpc / seval_dpc,
                 spliner.py:1287-1396: the Forsythe-Malcolm-Moler spline)
  prop2qw        propagation-space fields -> windowed, real, transformed
                 wire-space fields (QWOptics.Prop2QW, qwoptics.py:673-721)
  qw2prop        wire-space sources -> propagation-space sources
                 (QWOptics.QW2Prop, qwoptics.py:723-812)
  rho_post       the boundary offset, normalisation and transform of the
                 wire-space densities (QWRho5, qwoptics.py:1067-1078)

The SBE arithmetic itself (the O(Nk^2)/O(Nk^3) right-hand side and the
O(Nr Nk^2) source sums) runs in the sm_100a kernels.
"""

import numpy as np

QW_SMALL = 1e-100  # QWOptics._small (qwoptics.py:604)


def fftg(F):
    """FFTG in place: alternate-sign shift, FFT, shift, -F/N."""
    F[1::2] = -F[1::2]
    F[:] = np.fft.fft(F)
    F[1::2] = -F[1::2]
    F[:] = -F / float(len(F))


def ifftg(F):
    """iFFTG in place: alternate-sign shift, inverse FFT, shift, -F*N."""
    F[1::2] = -F[1::2]
    F[:] = np.fft.ifft(F)
    F[1::2] = -F[1::2]
    F[:] = -F * float(len(F))


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


def _spline(x, y):
    """Coefficients (b, c, d) of the cubic spline through (x, y): the
    Forsythe-Malcolm-Moler construction, whose end conditions match third
    derivatives of the cubics through the first and last four points."""
    n = len(x)
    y = np.asarray(y, dtype=np.complex128)
    b = np.zeros(n, np.complex128)
    c = np.zeros(n, np.complex128)
    d = np.zeros(n, np.complex128)
    if n < 2:
        raise ValueError("Not enough points to spline.")
    if n < 3:
        b[0] = (y[1] - y[0]) / (x[1] - x[0])
        b[1] = b[0]
        return b, c, d
    d[0] = x[1] - x[0]
    c[1] = (y[1] - y[0]) / d[0]
    for i in range(1, n - 1):
        d[i] = x[i + 1] - x[i]
        b[i] = 2.0 * (d[i - 1] + d[i])
        c[i + 1] = (y[i + 1] - y[i]) / d[i]
        c[i] = c[i + 1] - c[i]
    b[0] = -d[0]
    b[n - 1] = -d[n - 2]
    c[0] = 0.0
    c[n - 1] = 0.0
    if n != 3:
        c[0] = c[2] / (x[3] - x[1]) - c[1] / (x[2] - x[0])
        c[n - 1] = c[n - 2] / (x[n - 1] - x[n - 3]) - c[n - 3] / (x[n - 2] - x[n - 4])
        c[0] = c[0] * d[0] ** 2 / (x[3] - x[0])
        c[n - 1] = -c[n - 1] * d[n - 2] ** 2 / (x[n - 1] - x[n - 4])
    for i in range(1, n):
        t = d[i - 1] / b[i - 1]
        b[i] = b[i] - t * d[i - 1]
        c[i] = c[i] - t * c[i - 1]
    c[n - 1] = c[n - 1] / b[n - 1]
    for i in range(n - 2, -1, -1):
        c[i] = (c[i] - d[i] * c[i + 1]) / b[i]
    b[n - 1] = (y[n - 1] - y[n - 2]) / d[n - 2] + d[n - 2] * (c[n - 2] + 2.0 * c[n - 1])
    for i in range(n - 1):
        b[i] = (y[i + 1] - y[i]) / d[i] - d[i] * (c[i + 1] + 2.0 * c[i])
        d[i] = (c[i + 1] - c[i]) / d[i]
        c[i] = 3.0 * c[i]
    c[n - 1] = 3.0 * c[n - 1]
    d[n - 1] = d[n - 2]
    return b, c, d


def rescale_1d(x0, z0, x1):
    """z0 on grid x0 resampled onto x1 by the cubic spline; 0 outside
    [min x0, max x0]."""
    x0 = np.asarray(x0, dtype=np.float64)
    z0 = np.asarray(z0, dtype=np.complex128)
    if len(x0) != len(z0):
        raise ValueError("Bad sizes in rescale_1D_dpc")
    b, c, d = _spline(x0, z0)
    lo, hi = np.min(x0), np.max(x0)
    out = np.zeros(len(x1), np.complex128)
    for i, u in enumerate(np.asarray(x1, dtype=np.float64)):
        if lo <= u <= hi:
            j = _locate(x0, u)
            dx = u - x0[j]
            out[i] = z0[j] + dx * (b[j] + dx * (c[j] + dx * d[j]))
    return out


def prop2qw(RR, Exx, Eyy, Ezz, Vrr, R, window):
    """Wire-space q-space fields (Ex, Ey, Ez, Vr) from the propagation-space
    fields along the wire: resampled onto the wire grid, windowed, real part,
    FFTG."""
    out = []
    for F in (Exx, Eyy, Ezz, Vrr):
        f = rescale_1d(RR, F, R) * window
        f = np.real(f).astype(np.complex128)
        fftg(f)
        out.append(f)
    return out


def rho_post(re, rh, ne, nh, dr):
    """QWRho5 after its sums: boundary offset removed (mean of the ten
    outermost points at each end), densities normalised to the carrier
    totals, FFTG; in place."""
    nr = len(re)
    for a, tot in ((re, np.sum(np.abs(ne)) + 1e-50), (rh, np.sum(np.abs(nh)) + 1e-50)):
        a[:] = a - np.real(np.sum(a[0:10]) + np.sum(a[nr - 10:nr])) / 20.0
        a[:] = a * tot / (np.sum(np.abs(a)) * dr + QW_SMALL)
        fftg(a)


def qw2prop(r, Px, Py, Pz, re, rh, RR, plasmonics):
    """Propagation-space (Pxx, Pyy, Pzz, RhoE, RhoH) from the wire-space
    q-space sources (modified in place: transformed back and, with
    plasmonics, the densities made positive and normalised)."""
    dr = r[1] - r[0]
    dRR = RR[1] - RR[0]
    for a in (Px, Py, Pz, re, rh):
        ifftg(a)
    total = None
    if plasmonics:
        re[:] = np.abs(re)
        rh[:] = np.abs(rh)
        total = (np.sum(re) * dr + np.sum(rh) * dr + QW_SMALL) / 2.0
        re[:] = re * total / (np.sum(re) * dr + QW_SMALL)
        rh[:] = rh * total / (np.sum(rh) * dr + QW_SMALL)
    Pxx, Pyy, Pzz, RhoE, RhoH = (rescale_1d(r, a, RR) for a in (Px, Py, Pz, re, rh))
    if plasmonics:
        RhoE = np.abs(RhoE).astype(np.complex128)
        RhoH = np.abs(RhoH).astype(np.complex128)
        RhoE = RhoE * total / (np.sum(RhoE) * dRR + QW_SMALL)
        RhoH = RhoH * total / (np.sum(RhoH) * dRR + QW_SMALL)
    return Pxx, Pyy, Pzz, RhoE, RhoH
