"""Tables of the flag-gated many-body terms of the full-matrix SBE step
(mb.params DiagDph, OffDiagDph, EHs, Phonon, Recomb, DCTrans) and the
PsbFullMB descriptor that hands them to psb_full_step_mb_f64.

The index maps and weights are made once per grid on the host, with the
reference's own arithmetic (they are exact integers or one-line formulas):
  dephasing maps k+q, k-q, k1', k1'-q, k1, k1-q and the weights xe, xh
      (InitializeDephasing, dephasing.py:471-538), and the index Vxx2 reads
      (dephasing.py:362-379);
  phonon matrices EP, HP and their transposes, the Bose occupation and the
      coupling scale (InitializePhonons, phonons.py:55-136, with the
      module's temperature 77 K and host dielectric constants 10 / 8.2);
  the photon-energy grid and weights of spontaneous emission
      (InitializeEmission, emission.py:35-92; CalcHOmega :220-256);
  the FFT wavenumbers of the DC shift (InitializeDC, dcfield.py:782-793);
the O(Nk^3) Coulomb scattering kernels Ceh, Cee, Chh (CalcMBArrays,
coulomb.py:367-499) on the GPU (psb_mb_tables_f64).
"""

import numpy as np
import torch
from scipy.constants import c as C0
from scipy.constants import e as E0
from scipy.constants import epsilon_0 as EPS0
from scipy.constants import hbar as HBAR
from scipy.constants import k as KB

from . import _lib, abi
from . import device as _dev

PHONON_TEMP = 77.0        # K (phonons.py:22)
PHONON_EPSR0 = 10.0       # host static dielectric constant (phonons.py:23)
PHONON_EPSRINF = 8.2      # host high-frequency dielectric constant (phonons.py:24)
EMISSION_TEMP = 77.0      # K (emission.py:29)


def dephasing_maps(ky, me, mh):
    """(maps [6][Nk][Nk] int32: k_p_q, k_m_q, k1p, k1p_m_q, k1, k1_m_q; xe; xh)
    as InitializeDephasing computes them (0-based indices; the kernels treat
    any value outside [0, Nk) as no partner)."""
    ky = np.asarray(ky, dtype=np.float64)
    nk = len(ky)
    dk = ky[1] - ky[0] if nk > 1 else 1.0
    kmax = ky[nk - 1] + dk
    kmin = ky[0] - dk
    nk0 = (nk - 1) // 2 + 1
    xe = me / HBAR**2 * np.abs(ky) / (np.abs(ky) + dk * 1e-5) ** 2 / dk
    xh = mh / HBAR**2 * np.abs(ky) / (np.abs(ky) + dk * 1e-5) ** 2 / dk
    K = ky[:, None]   # k (rows)
    Q = ky[None, :]   # q (columns)

    def idx(x):
        return (np.round(np.clip(x, kmin, kmax) / dk).astype(np.int64) + nk0 - 1).astype(np.int32)

    k_p_q = idx(K + Q)
    k_m_q = idx(K - Q)
    k1p_0 = ((me + mh) * Q - 2 * mh * K) / 2.0 / me
    k1p = idx(k1p_0)
    k1p_m_q = idx(k1p_0 - Q)
    k1_0 = ((me + mh) * Q - 2 * me * K) / 2.0 / mh
    k1 = idx(k1_0)
    k1_m_q = idx(k1_0 - Q)
    maps = np.stack([k_p_q, k_m_q, k1p, k1p_m_q, k1, k1_m_q]).astype(np.int32)
    return maps, xe, xh


def vxx2_index(ky):
    """round(|ky / dk|): the row of VC that Vxx2 reads for each q (dephasing.py:362)."""
    ky = np.asarray(ky, dtype=np.float64)
    dq = ky[1] - ky[0] if len(ky) > 1 else 1.0
    return np.round(np.abs(ky / dq)).astype(np.int32)


def phonon_tables(Ee, Eh, epsr, Gph, Oph):
    """(EP, EPT, HP, HPT, Vscale) of InitializePhonons."""
    Ee = np.asarray(Ee, dtype=np.float64)
    Eh = np.asarray(Eh, dtype=np.float64)
    nk = len(Ee)
    no = 1.0 / (np.exp(HBAR * Oph / KB / PHONON_TEMP) - 1.0)
    idel = np.ones((nk, nk))
    np.fill_diagonal(idel, 0.0)

    def mat(E):
        d = E[:, None] - E[None, :]   # E[k] - E[k1], [k, k1]
        den1 = (d - HBAR * Oph) ** 2 + (HBAR * Gph) ** 2
        den2 = (d + HBAR * Oph) ** 2 + (HBAR * Gph) ** 2
        return no / den1 + (no + 1.0) / den2

    EP = mat(Ee) * 2.0 * Gph * idel
    HP = mat(Eh) * 2.0 * Gph * idel
    vscale = HBAR * Oph * epsr * (1.0 / PHONON_EPSRINF - 1.0 / PHONON_EPSR0)
    return EP, np.ascontiguousarray(EP.T), HP, np.ascontiguousarray(HP.T), vscale


def emission_tables(dcv, epsr, geh, ehint):
    """(HOmega, square, dhw, rho0_den) of InitializeEmission with |dcv|:
    HOmega_n = (n + 1/2) dhw0 up to 4 (kB T + hbar geh), dhw0 = min(kB T,
    hbar geh) / 20; square = 3 dcv^2 ehint^2 / (eps0 sqrt(epsr) hbar)
    Lrtz(HOmega, hbar geh) exp(-HOmega / kB T); dhw = HOmega[1] - HOmega[0]
    as SpontIntegral takes it; rho0_den the denominator of rho0."""
    dcv = abs(dcv)
    kbt, hg = KB * EMISSION_TEMP, HBAR * geh
    hwmax = (kbt + hg) * 4.0
    dhw0 = min(kbt, hg) / 20.0
    nw = int(np.ceil(hwmax / dhw0))
    if nw < 10:
        raise ValueError("Error: temperature is too low in emission.py")
    hw = np.array([0.0 + (n + 0.5) * dhw0 for n in range(nw)])
    b = HBAR * geh
    lrtz = (b / np.pi) / (hw**2 + b**2)
    square = (3.0 * dcv**2 * ehint / EPS0 / np.sqrt(epsr) * ehint / HBAR * lrtz
              * np.exp(-hw / KB / EMISSION_TEMP))
    return hw, square, hw[1] - hw[0], C0**3 * np.pi**2 * HBAR**3


def dc_wavenumbers(ky):
    """Y of InitializeDC: GetKArray(nk, (nk - 1) dky), dky = ky[2] - ky[1]
    (FFT order, zero first)."""
    ky = np.asarray(ky, dtype=np.float64)
    nk = len(ky)
    dky = ky[2] - ky[1] if nk > 2 else ky[1] - ky[0] if nk > 1 else 1.0
    length = (nk - 1) * dky
    dl = 2.0 * np.pi / length if length > 0 else 1.0
    return np.array([float(i) * dl if i <= nk // 2 else float(i - nk) * dl for i in range(nk)])


def dc_shift(edc, eac, dt):
    """The k shift of one Transport call, -e0 (Edc + Eac) / hbar dt (dcfield.py:1240)."""
    return -E0 * (edc + eac) / HBAR * dt


class ManyBody:
    """Device tables and scratch of the many-body terms for one grid, and the
    PsbFullMB descriptor of a step."""

    def __init__(self, solver, Ee_dev, Eh_dev):
        s = solver
        nk = s.Nk
        self.flags = (bool(s.DiagDph), bool(s.OffDiagDph), bool(s.EHs), bool(s.Phonon))
        self.recomb, self.dctrans = bool(s.Recomb), bool(s.DCTrans)
        self.edc = float(s.Edc)
        maps, xe, xh = dephasing_maps(s.kr, s.me, s.mh)
        self.maps = torch.as_tensor(maps, device="cuda")
        self.iq = torch.as_tensor(vxx2_index(s.kr), device="cuda")
        self.xe = torch.as_tensor(xe, device="cuda")
        self.xh = torch.as_tensor(xh, device="cuda")
        self.C = None
        if s.EHs:
            self.C = torch.empty(3 * (nk + 1) ** 3, dtype=torch.float64, device="cuda")
            _lib.call("psb_mb_tables_f64", nk, _dev.ptr(Ee_dev), _dev.ptr(Eh_dev),
                      float(s.gam_e), float(s.gam_h), HBAR, int(bool(s.LorentzDelta)),
                      _dev.ptr(self.C), _dev.stream_ptr())
        EP, EPT, HP, HPT, self.vscale = phonon_tables(s.Ee, s.Eh, s.epsr, s.Gph, s.Oph)
        self.ph = torch.as_tensor(np.stack([EP, EPT, HP, HPT]), device="cuda")
        self.emis = None
        self.dhw = self.rho0_den = 0.0
        if self.recomb:
            hw, sq, self.dhw, self.rho0_den = emission_tables(s.dcv, s.epsr, s.gam_eh, s.ehint)
            self.emis = torch.as_tensor(np.stack([hw, sq]), device="cuda")
        self.Y = torch.as_tensor(dc_wavenumbers(s.kr), device="cuda")
        # one scratch region per wire (a batch step uses all of them)
        self.scratch = torch.empty(s.Nw * int(_lib.load().psb_full_mb_scratch_bytes(nk)),
                                   dtype=torch.uint8, device="cuda")
        self.gam = (float(s.gam_e), float(s.gam_h), float(s.gam_eh))

    def descriptor(self, eps=None, eac=0.0, dt=0.0):
        """PsbFullMB of one step: eps the screening of its V3, eac = Re Ex
        at q = 0 of the wire and dt its step (for the DC shift)."""
        d = np.zeros(1, dtype=abi.FULL_MB_DTYPE)
        d["diag_dph"], d["offdiag_dph"], d["ehs"], d["phonon"] = map(int, self.flags)
        d["gam_e"], d["gam_h"], d["gam_eh"] = self.gam
        d["vscale"] = self.vscale

        def addr(t):
            assert t.is_cuda and t.is_contiguous()
            return t.data_ptr()

        d["maps"], d["iq"] = addr(self.maps), addr(self.iq)
        d["xe"], d["xh"] = addr(self.xe), addr(self.xh)
        d["C"] = addr(self.C) if self.C is not None else 0
        d["ph"] = addr(self.ph)
        d["eps"] = addr(eps) if eps is not None else 0
        d["scratch"] = addr(self.scratch)
        d["recomb"], d["dctrans"] = int(self.recomb), int(self.dctrans)
        d["dc_dk"] = dc_shift(self.edc, eac, dt)
        if self.emis is not None:
            d["dhw"], d["rho0_den"] = self.dhw, self.rho0_den
            d["n_hw"] = self.emis.shape[1]
            d["emis"] = addr(self.emis)
        d["Y"] = addr(self.Y)
        return d
