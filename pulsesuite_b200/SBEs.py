"""Reference-named SBE functions for diagonal states, on the GPU.

Drop-in for the kernel-level signatures of pulsesuite's ``SBEs`` module when
the states p, C, D and the drive are diagonal in k (a k-independent field
along the wire, the case of the batched configurations):

    configure(Ee, Eh, gap, excitons=True, lf=False, freepot=False)  # module state
    CalcH(Meh, Wee, Whh, C, D, p, VC, Heh, Hee, Hhh)   # in place (SBEs.py:669)
    dpdt(C, D, p, Heh, Hee, Hhh, GamE, GamH, OffP)     # -> (Nk, Nk) (SBEs.py:1850)
    dCdt(Cee, Dhh, Phe, Heh, Hee, Hhh, GamE, GamH, OffE)   # (SBEs.py:2221)
    dDdt(Cee, Dhh, Phe, Heh, Hee, Hhh, GamE, GamH, OffH)   # (SBEs.py:2513)

The reference's private backends take the band energies, gap and flags as
extra arguments (``_CalcH_jit(..., Nk, Ee, Eh, gap, excitons, lf,
freepot)``); the module-level calls read them from module state, set here by
``configure`` (keyword arguments of ``CalcH`` override it per call).

The exchange sums over k' (the O(Nk^2) part) run in the sm_100a FP64 kernel
through ``psb_calch_f64``; the O(Nk) elementwise derivatives in one launch of
``psb_diag_derivs_f64``.  Arrays may be numpy arrays or tensors; results come
back as numpy (in place for CalcH, as the reference does).  These module
functions take diagonal states only: an off-diagonal state (a k-dependent
field along the wire) raises NotImplementedError here; its full-matrix
right-hand side runs inside ``SBESolver`` (psb_full_step_f64 and the batched
psb_full_step_batch_f64), which moves to it by itself.

For time integration use ``batch.WireBatch`` (RK4 or the reference's
leapfrog over many wires); these functions exist for callers that step the
reference's own way one right-hand side at a time.
"""

import numpy as np
from scipy.constants import hbar as HBAR

from . import _lib, abi, device, wirespace

ii = 1j
hbar = HBAR

_state = {"Ee": None, "Eh": None, "gap": 0.0, "excitons": True, "lf": False,
          "freepot": False}


def configure(Ee, Eh, gap, excitons=True, lf=False, freepot=False):
    """Band energies (J), gap (J, rotating frame: gap - hbar omega_L) and the
    mb.params flags used by CalcH (the reference's InitializeSBE state)."""
    _state.update(Ee=np.asarray(Ee, dtype=np.float64), Eh=np.asarray(Eh, dtype=np.float64),
                  gap=float(gap), excitons=bool(excitons), lf=bool(lf), freepot=bool(freepot))


def _np(a):
    if hasattr(a, "detach"):
        return a.detach().cpu().numpy()
    return np.asarray(a)


def _diag_of(name, m, tol=0.0):
    """Diagonal of a square matrix that must be diagonal."""
    m = _np(m)
    if m.ndim == 1:
        return m
    d = np.diag(m)
    off = m - np.diag(d)
    if np.max(np.abs(off), initial=0.0) > tol * max(1.0, np.max(np.abs(d), initial=0.0)):
        raise NotImplementedError(f"{name} is not diagonal in k: these module functions take "
                                  "diagonal states; SBESolver steps full-matrix states")
    return d


def _v_rows(VC, nk):
    """V_n(q), q = 0..nk-1, n = (eh, ee, hh) from the reference's VC array
    (VC[q, 0, n], SBEs.py:829-834) or an (nk, 3) array of those rows."""
    v = _np(VC)
    if v.ndim == 3:
        v = v[:, 0, :]
    if v.shape[0] < nk or v.shape[1] != 3:
        raise ValueError("VC must be (Nq, Nq, 3) or (Nq, 3) with Nq >= Nk")
    return np.ascontiguousarray(v[:nk].T)


_TABLE_CACHE = {}


def _device_table(v, Ee, Eh, excitons):
    """Device table descriptor + tabdata for one grid, cached by content (a
    caller stepping one wire re-uses the same V rows and band energies on
    every call)."""
    import hashlib

    import torch

    nk = v.shape[1]
    key = hashlib.sha1(b"".join(np.ascontiguousarray(a, dtype=np.float64).tobytes()
                                for a in (v, Ee, Eh)) + bytes([bool(excitons)])).hexdigest()
    hit = _TABLE_CACHE.get(key)
    if hit is not None:
        return hit
    blk = np.zeros((abi.TAB_BLOCKS, nk))
    blk[0:3] = v
    blk[abi.TAB_EE] = Ee
    blk[abi.TAB_EH] = Eh
    tables = np.zeros(1, dtype=abi.TABLE_DTYPE)
    tables["nk"] = nk
    flags = abi.PSB_TAB_EXCITONS if excitons else 0
    if np.array_equal(v[0], v[1]) and np.array_equal(v[0], v[2]):
        flags |= abi.PSB_TAB_SHARED_V
    tables["flags"] = flags
    tables["L"] = 1.0
    if len(_TABLE_CACHE) >= 8:
        _TABLE_CACHE.pop(next(iter(_TABLE_CACHE)))
    hit = (device.to_device(tables), torch.as_tensor(blk.reshape(-1), device="cuda"), flags)
    _TABLE_CACHE[key] = hit
    return hit


def h_diagonals(p, ne, nh, VC, Ee, Eh, gap, excitons=True, stream=None):
    """Device computation of the renormalised H diagonals for one wire:
    returns complex Heh exchange part (without the drive) and real Hee, Hhh,
    each (Nk,) numpy."""
    import torch

    device.require_cuda()
    p = np.asarray(p, dtype=np.complex128)
    nk = p.size
    v = _v_rows(VC, nk)
    d_tab, d_td, flags = _device_table(v, Ee, Eh, excitons)
    w = np.zeros(1, dtype=abi.WIRE_DTYPE)
    w["gap"] = gap
    y = np.stack([p.real, p.imag, np.asarray(ne, np.float64), np.asarray(nh, np.float64)], 1)
    d_w = device.to_device(w)
    d_y = torch.as_tensor(np.ascontiguousarray(y), device="cuda")
    d_h = torch.empty_like(d_y)
    model = abi.model_array(HBAR)
    _lib.call("psb_calch_f64", device.ptr(d_tab), 1, device.ptr(d_td), d_td.numel(),
              device.ptr(d_w), 1, device.ptr(d_y), device.ptr(d_h), nk, nk,
              flags & (abi.PSB_TAB_SHARED_V | abi.PSB_TAB_SCREENED), abi.as_ptr(model),
              device.stream_ptr(stream))
    h = d_h.cpu().numpy()
    return h[:, 0] + 1j * h[:, 1], h[:, 2].copy(), h[:, 3].copy()


def CalcH(Meh, Wee, Whh, C, D, p, VC, Heh, Hee, Hhh, **kw):
    """Hamiltonian matrices of the SBEs (SBEs.py:669-935), written in place
    into Heh, Hee, Hhh, for diagonal C, D, p and Meh.  Keyword arguments Ee,
    Eh, gap, excitons, freepot override the module state of ``configure``."""
    st = dict(_state)
    st.update(kw)
    if st["Ee"] is None:
        raise ValueError("call configure(Ee, Eh, gap) first (InitializeSBE state)")
    c = _diag_of("C", C)
    d = _diag_of("D", D)
    pd = _diag_of("p", p)
    meh = _np(Meh)
    md = np.diag(meh) if meh.ndim == 2 else meh
    nk = pd.size
    if np.max(np.abs(c.imag), initial=0.0) > 0 or np.max(np.abs(d.imag), initial=0.0) > 0:
        raise ValueError("diagonal C and D are occupations and must be real")
    xeh, hee, hhh = h_diagonals(pd, c.real, d.real, VC, st["Ee"], st["Eh"], st["gap"],
                                excitons=st["excitons"])
    heh_full = np.array(meh, dtype=np.complex128, copy=True) if meh.ndim == 2 else np.diag(md)
    heh_full[np.arange(nk), np.arange(nk)] = md + xeh
    hee_full = np.diag(hee.astype(np.complex128))
    hhh_full = np.diag(hhh.astype(np.complex128))
    if st["freepot"]:
        hee_full = hee_full + _np(Wee)
        hhh_full = hhh_full + _np(Whh)
    for out, val in ((Heh, heh_full), (Hee, hee_full), (Hhh, hhh_full)):
        if hasattr(out, "copy_"):
            import torch

            out.copy_(torch.as_tensor(val))
        else:
            out[...] = val


def _gam(g, nk):
    g = _np(g)
    return np.full(nk, float(g)) if g.ndim == 0 else np.asarray(g, dtype=np.float64)


def _derivs(C, D, p, Heh, Hee, Hhh, GamE, GamH, Off):
    """(dp, dC, dD) diagonals from one launch of psb_diag_derivs_f64."""
    import torch

    device.require_cuda()
    pd = _diag_of("p", p)
    nk = pd.size
    c, d = _diag_of("C", C), _diag_of("D", D)
    heh, hee, hhh = (_diag_of(n, m) for n, m in (("Heh", Heh), ("Hee", Hee), ("Hhh", Hhh)))
    off = _np(Off)
    off = np.diag(off) if off.ndim == 2 else off
    g = _gam(GamE, nk) + _gam(GamH, nk)
    h = np.stack([heh, hee, hhh], 1).astype(np.complex128)
    st = np.stack([pd, c, d], 1).astype(np.complex128)
    # one host->device copy of the packed inputs, one kernel, one copy back
    off = np.ascontiguousarray(np.broadcast_to(np.asarray(off, dtype=np.complex128), (nk,)))
    packed = np.concatenate([h.view(np.float64).reshape(-1), st.view(np.float64).reshape(-1),
                             g, off.view(np.float64)])
    buf = torch.as_tensor(packed, device="cuda")
    out = torch.empty(6 * nk, dtype=torch.float64, device="cuda")
    base = buf.data_ptr()
    _lib.call("psb_diag_derivs_f64", base, base + 8 * 6 * nk, base + 8 * 12 * nk,
              base + 8 * 13 * nk, float(hbar), device.ptr(out), nk, device.stream_ptr())
    r = out.cpu().numpy().view(np.complex128).reshape(nk, 3)
    return r[:, 0].copy(), r[:, 1].copy(), r[:, 2].copy()


def dpdt(C, D, p, Heh, Hee, Hhh, GamE, GamH, OffP):
    """d p / dt (SBEs.py:1850-1975) for diagonal states: (Nk, Nk) with the
    diagonal i hbar dp_k/dt = (Hee_k + Hhh_k) p_k - Heh_k (C_k + D_k) + Heh_k
    - i hbar (GamE_k + GamH_k) p_k + OffP_kk."""
    return np.diag(_derivs(C, D, p, Heh, Hee, Hhh, GamE, GamH, OffP)[0])


def dCdt(Cee, Dhh, Phe, Heh, Hee, Hhh, GamE, GamH, OffE):
    """d C / dt (SBEs.py:2221-2337) for diagonal states: the diagonal is
    (Heh_k conj(p_k) - conj(Heh_k) p_k) / (i hbar) (the Hee commutator
    vanishes on the diagonal)."""
    return np.diag(_derivs(Cee, Dhh, Phe, Heh, Hee, Hhh, GamE, GamH, 0.0 * _np(Phe))[1])


def dDdt(Cee, Dhh, Phe, Heh, Hee, Hhh, GamE, GamH, OffH):
    """d D / dt (SBEs.py:2513-2636) for diagonal states: same diagonal as
    dCdt, (Heh_k conj(p_k) - conj(Heh_k) p_k) / (i hbar)."""
    return np.diag(_derivs(Cee, Dhh, Phe, Heh, Hee, Hhh, GamE, GamH, 0.0 * _np(Phe))[2])


# ===========================================================================
# The solver API of the reference (SBEs.py:4631-6078) for diagonal drives.
# ===========================================================================
from scipy.constants import c as _c0  # noqa: E402
from scipy.constants import e as _e0  # noqa: E402
from scipy.constants import epsilon_0 as _eps0  # noqa: E402
from scipy.constants import k as _kB  # noqa: E402
from scipy.constants import m_e as _me0  # noqa: E402

_twopi = 2.0 * np.pi
_TEMP_K = 77.0  # lattice temperature of the Fermi occupations (phonons.py:22)


def _fftg(F):
    """FFTG of usefulsubs.py:2278-2304: alternate-sign shift, FFT, shift, -F/N."""
    F[1::2] = -F[1::2]
    F[:] = np.fft.fft(F)
    F[1::2] = -F[1::2]
    F[:] = -F / float(len(F))


def _ifftg(F):
    """iFFTG of usefulsubs.py:2307-2334."""
    F[1::2] = -F[1::2]
    F[:] = np.fft.ifft(F)
    F[1::2] = -F[1::2]
    F[:] = -F * float(len(F))


def _k_array(n, length):
    """GetKArray (typespace.py:362-381): wavenumbers in FFT order."""
    dl = _twopi / length if length > 0 else 1.0
    return np.array([i * dl if i <= n // 2 else (i - n) * dl for i in range(n)], dtype=np.float64)


def _array0_index(x):
    """GetArray0Index (usefulsubs.py:1028-1060)."""
    dx = x[2] - x[1]
    xi = np.round((x + 0.1 * dx) / dx).astype(np.int32)
    hits = np.nonzero(xi == 0)[0]
    if hits.size == 0:
        raise ValueError("Zero index not found in array")
    return int(hits[0])


def _fermi(En):
    """FermiDistr (phonons.py:317-341) at the module temperature."""
    return 1.0 / (np.exp(En / _kB / _TEMP_K) + 1.0)


def yw(w):
    """Wire sign factor (-1)^floor((w-1)/2) (qwoptics.py:1099-1112)."""
    return (-1) ** int(np.floor((w - 1) / 2.0))


def QWChi1(lam, dky, Ee, Eh, area, geh, dcv):
    """Linear susceptibility of the wire (qwoptics.py:1115-1152)."""
    ww = _twopi * _c0 / lam
    d1 = Ee + Eh - ii * HBAR * geh - HBAR * ww
    d2 = Ee + Eh + ii * HBAR * geh + HBAR * ww
    return 4 * dcv**2 / _eps0 / area * dky / _twopi * np.sum((Ee + Eh) / (d1 * d2))


class SBESolver:
    """The reference's ``SBESolver`` (SBEs.py:4631) on the GPU, for states and
    drives that are diagonal in k.

    Same constructor and parameter files: ``params/qw.params`` and
    ``params/mb.params`` are read from the working directory in the
    reference's line order (SBEs.py:4990-5038), and the k grid, wire-space
    grid, material constants and initial Fermi occupations are derived as in
    SBEs.py:4766-4885.  The Nw wires live in one ``WireBatch`` (plain FP64
    kernels): the reference's two stored levels (YY2/CC2/DD2 and
    YY3/CC3/DD3, SBEs.py:5073-5092) are the batch's y1 and y, and each step
    is one launch of ``psb_leapfrog_f64`` for the wire (the reference's
    integrator, SBEs.py:5685-5718), with the unscreened or per-step screened
    Coulomb table (mb.params Screened) of ``psb_coulomb_vint``.

    What is supported is the reference's diagonal sub-case: Optics and
    Excitons with the field entering only at q = 0 of the wire
    (``Ey[NQ0]``: a field uniform along the wire, dipole coupling Ycv), in
    which the reference's full-matrix state stays exactly diagonal.  A
    field with other q components (``QWCalculator`` windows the field along
    the wire, which gives it every q) moves the solver to the full Nk x Nk
    state, and so do the many-body flags DiagDph, OffDiagDph, EHs, Phonon,
    Recomb and DCTrans (k-dependent and off-diagonal dephasing,
    carrier-carrier and LO-phonon relaxation, spontaneous emission, DC-field
    transport: psb_full_step_mb_f64).  No data files are written (the
    reference's diagnostics under dataQW/ are not reproduced).
    """

    _MANY_BODY = ("DiagDph", "OffDiagDph", "EHs", "Phonon", "Recomb", "DCTrans")

    def __init__(self, q, rr, r0, Emaxxx, lam, Nw, QW, backend="auto"):
        # defaults of SBEs.py:4638-4671, overwritten by the params files
        self.L, self.Delta0, self.gap = 100e-9, 5e-9, 1.5 * _e0
        self.me, self.mh, self.HO = 0.07 * _me0, 0.45 * _me0, 100e-3 * _e0
        self.gam_e = self.gam_h = self.gam_eh = 1.0 / 1e-12
        self.epsr, self.Edc, self.wL = 9.1, 0.0, 0.0
        self.Optics = self.Excitons = self.EHs = self.Screened = self.Phonon = True
        self.DCTrans, self.LF, self.FreePot = False, True, False
        self.DiagDph = self.OffDiagDph = True
        self.OBE = self.Recomb = self.ReadDC = self.PLSpec = self.ignorewire = False
        self.Xqwparams = False
        self.jmax, self.ntmax = 1000, 100000
        self.small = 1e-200
        self.Nw = int(Nw)
        self.wireoff = True
        self.xxx = self.jjj = 1
        self.t = 0.0
        self.start = False
        self._backend = backend
        self.batch = None
        self.full = None
        self._many_body = False
        if not QW:
            return
        self._read_qw_params()
        self._read_mb_params()
        self._many_body = any(getattr(self, f) for f in self._MANY_BODY)
        self.Emax0 = float(Emaxxx)
        kmax = np.sqrt(1.2 * self.gap * 2.0 * self.me / (HBAR**2))
        self.dkr = _twopi / (2.0 * self.L)
        nk_odd = int(np.floor(kmax / self.dkr) * 2 + 1)
        self.Nr = nk_odd * 2
        self.Nk = nk_odd - 1
        dnk = (self.Nk - 1) // 2
        self.NK0 = dnk + 1
        self.kr = np.array([self.dkr * (-dnk + k - 0.5) for k in range(self.Nk)])
        self.r = np.linspace(-self.L, self.L, self.Nr)
        Qr = np.roll(_k_array(self.Nr, 2 * self.L), self.Nr // 2)
        Qr[0] = -Qr[0]
        self.Qr = Qr
        self.NQ0 = _array0_index(Qr)
        self.dr = (self.r[2] - self.r[1]) * (self.Nr - 1) / float(self.Nr)
        self.dcv = np.sqrt((_e0 * HBAR) ** 2 / (6.0 * _me0 * self.gap) * (_me0 / self.me - 1.0))
        self.alphae = np.sqrt(self.me * self.HO) / HBAR
        self.alphah = np.sqrt(self.mh * self.HO) / HBAR
        self.ehint = np.sqrt(2.0 * self.alphae * self.alphah /
                             (self.alphae**2 + self.alphah**2))
        self.gam_eh = (self.gam_e + self.gam_h) / 2.0
        self.qc = 2.0 * self.alphae * self.alphah / (self.alphae + self.alphah)
        self.area = np.sqrt(2.0 * np.pi) / np.sqrt(self.alphae**2 + self.alphah**2) * self.Delta0
        self.Ee = HBAR**2 * self.kr**2 / (2.0 * self.me)
        self.Eh = HBAR**2 * self.kr**2 / (2.0 * self.mh)
        self.window = np.exp(-((self.r / (self.L / 2.0)) ** 150))  # qwoptics.py:636-655
        self.chiw = QWChi1(lam, self.dkr, self.Ee + self.gap, self.Eh, self.area, self.gam_eh,
                           self.dcv)
        self._build_batch()
        self.start = True

    # -- parameter files (SBEs.py:4990-5038) ---------------------------------
    def _read_qw_params(self):
        with open("params/qw.params", "r", encoding="utf-8") as f:
            vals = [f.readline().split()[0] for _ in range(15)]
        self.L, self.Delta0 = float(vals[0]), float(vals[1])
        self.gap = float(vals[2]) * _e0
        self.me, self.mh = float(vals[3]) * _me0, float(vals[4]) * _me0
        self.HO = float(vals[5]) * _e0
        self.gam_e, self.gam_h, self.gam_eh = float(vals[6]), float(vals[7]), float(vals[8])
        self.epsr = float(vals[9])
        self.Oph = float(vals[10]) * _e0 / HBAR
        self.Gph = float(vals[11]) * _e0 / HBAR
        self.Edc = float(vals[12])
        self.jmax, self.ntmax = int(vals[13]), int(vals[14])

    def _read_mb_params(self):
        names = ("Optics", "Excitons", "EHs", "Screened", "Phonon", "DCTrans", "LF", "FreePot",
                 "DiagDph", "OffDiagDph", "Recomb", "PLSpec", "ignorewire", "Xqwparams",
                 "LorentzDelta")
        with open("params/mb.params", "r", encoding="utf-8") as f:
            for n in names:
                setattr(self, n, bool(int(f.readline().split()[0])))

    # -- device state ----------------------------------------------------------
    def _build_batch(self):
        import torch

        from . import coulomb
        from . import grid as pgrid
        from .batch import WireBatch

        g = pgrid.Grid(nk=self.Nk, dk=self.dkr, kr=self.kr, L=self.L, me=self.me, mh=self.mh,
                       epsr=self.epsr, delta0=self.Delta0, alphae=self.alphae,
                       alphah=self.alphah, vkind="vint", y=self.r, gap=self.gap, dcv=self.dcv,
                       ehint=self.ehint, area=self.area)
        self.grid = g
        blk = coulomb.table_block(g, screened=self.Screened)
        host = np.zeros((abi.TAB_BLOCKS, self.Nk))
        host[0:3] = blk.reshape(abi.TAB_BLOCKS, self.Nk)[0:3].cpu().numpy()
        tables, _ = pgrid.pack_tables([g], [host.reshape(-1)], screened=self.Screened,
                                      excitons=self.Excitons)
        w = np.zeros(self.Nw, dtype=abi.WIRE_DTYPE)
        w["table"] = 0
        w["npulse"] = 0
        w["gap"] = self.gap
        w["gamma"] = self.gam_e + self.gam_h
        w["pscale"] = 2.0 * self.ehint / self.area / self.L * self.dcv
        # M = -ehint Ycv Ey[NQ0] yw(w) (SBEs.py:5165-5175, Ycv = dcv)
        w["mscale"] = [self.ehint * self.dcv * yw(i + 1) for i in range(self.Nw)]
        self.batch = WireBatch([g], w, screened=self.Screened, excitons=self.Excitons, p_cap=1,
                               tables=tables, tabdata=blk.contiguous())
        # CC = DD = diag FermiDistr(Ee + gap/2) on every level (SBEs.py:4857-4868)
        f = _fermi(self.Ee + self.gap / 2.0)
        y = np.zeros((self.Nw, self.Nk, 4))
        y[:, :, 2] = f
        y[:, :, 3] = f
        self.batch.set_state(y.reshape(-1, 4), y.reshape(-1, 4))
        self.y0 = self.batch.y1.clone()  # level 1 (YY1/CC1/DD1)
        self._field = torch.zeros((self.Nw, 2), dtype=torch.float64, device="cuda")
        self._steps_col = abi.WIRE_DTYPE.fields["steps"][1] // 4
        self._wires_i32 = self.batch.d_wires.view(torch.int32).view(self.Nw, -1)

    def levels(self, w):
        """Diagonals (p, ne, nh) of the three stored levels of wire w (1-based),
        numpy, as (YY1, YY2, YY3), (CC1, CC2, CC3), (DD1, DD2, DD3)."""
        if self.full is not None:
            m = [lv[w - 1].cpu().numpy() for lv in self.full["L"]]  # (3, Nk, Nk) each
            return tuple([np.diagonal(a[j]).copy() for a in m] for j in range(3))
        s = self.batch.wire_slice(w - 1)
        out = []
        for lv in (self.y0, self.batch.y1, self.batch.y):
            a = lv[s].cpu().numpy()
            out.append(a)
        return ([a[:, 0] + 1j * a[:, 1] for a in out], [a[:, 2] + 0j for a in out],
                [a[:, 3] + 0j for a in out])

    # -- the step ---------------------------------------------------------------
    def _is_diagonal(self, Ex, Ey, Ez):
        if not self.Optics:
            return True
        lo, hi = self.NQ0 - (self.Nk - 1), self.NQ0 + self.Nk
        win = slice(max(lo, 0), hi)
        ey = np.array(Ey[win], dtype=np.complex128, copy=True)
        ey[self.NQ0 - win.start] = 0.0
        return not (np.any(np.asarray(Ex)[win] != 0) or np.any(np.asarray(Ez)[win] != 0)
                    or np.any(ey != 0))

    def _enter_full(self):
        """Move the state to full Nk x Nk matrices (the diagonal levels
        embedded) and set up the full-matrix step's device buffers."""
        import torch

        from . import device as _dev

        nk, nw = self.Nk, self.Nw
        levels = []
        for lv in (self.y0, self.batch.y1, self.batch.y):
            a = lv.view(nw, nk, 4)
            m = torch.zeros((nw, 3, nk, nk), dtype=torch.complex128, device="cuda")
            idx = torch.arange(nk, device="cuda")
            m[:, 0, idx, idx] = torch.complex(a[:, :, 0], a[:, :, 1])
            m[:, 1, idx, idx] = torch.complex(a[:, :, 2], torch.zeros_like(a[:, :, 2]))
            m[:, 2, idx, idx] = torch.complex(a[:, :, 3], torch.zeros_like(a[:, :, 3]))
            levels.append(m)
        blk = self.batch.tabdata.view(abi.TAB_BLOCKS, nk)
        w1 = np.zeros(1, dtype=abi.WIRE_DTYPE)  # one-wire descriptor for the screening
        w1["table"] = 0
        self.full = {
            "L": levels,
            "work": torch.empty(int(_lib.load().psb_full_work_bytes(nk)), dtype=torch.uint8,
                                device="cuda"),
            "V0": blk[0:3].contiguous(),
            "Ee": blk[abi.TAB_EE].contiguous(),
            "Eh": blk[abi.TAB_EH].contiguous(),
            "kr": torch.as_tensor(self.kr, device="cuda"),
            "r": torch.as_tensor(self.r, device="cuda"),
            "window": torch.as_tensor(self.window, device="cuda"),
            "wire1": _dev.to_device(w1),
            "y1": torch.zeros((nk, 4), dtype=torch.float64, device="cuda"),
            "eps": torch.zeros((1, nk), dtype=torch.float64, device="cuda"),
            "out": torch.zeros((5, self.Nr), dtype=torch.complex128, device="cuda"),
        }
        self.full["mb"] = None
        if self._many_body:
            from . import manybody

            self.full["mb"] = manybody.ManyBody(self, self.full["Ee"], self.full["Eh"])

    def _full_step(self, Ex, Ey, Ez, dt, Px, Py, Pz, Re, Rh, w):
        import torch

        from . import device as _dev

        F = self.full
        nk, i = self.Nk, w - 1
        for a in (Px, Py, Pz, Re, Rh):
            a[:] = 0.0
        L1, L2, L3 = (lv[i] for lv in F["L"])
        # Coulomb table of this step: V0, or V0 / eps(q; n1D) from the current
        # occupations (CalcScreenedArrays, coulomb.py:1195-1230)
        V3 = F["V0"]
        if self.Screened:
            idx = torch.arange(nk, device="cuda")
            F["y1"][:, 2] = L3[1, idx, idx].real
            F["y1"][:, 3] = L3[2, idx, idx].real
            _lib.call("psb_screen_f64", _dev.ptr(self.batch.d_tables), 1,
                      _dev.ptr(self.batch.tabdata), _dev.ptr(F["wire1"]), 1, _dev.ptr(F["y1"]),
                      _dev.ptr(F["eps"]), nk, _dev.stream_ptr())
            V3 = (F["V0"] / F["eps"]).contiguous()
        fields = torch.as_tensor(np.stack([np.asarray(Ex, np.complex128),
                                           np.asarray(Ey, np.complex128),
                                           np.asarray(Ez, np.complex128)]), device="cuda")
        if not self.Optics:
            fields.zero_()
        prm = np.zeros(1, dtype=abi.FULL_PARAMS_DTYPE)
        prm["ehint"], prm["dcv"], prm["yw"], prm["sgnw"] = self.ehint, self.dcv, yw(w), (-1) ** w
        prm["gap"], prm["gam_e"], prm["gam_h"] = self.gap, self.gam_e, self.gam_h
        prm["hbar"], prm["dt"] = HBAR, dt
        prm["excitons"], prm["lf"] = int(self.Excitons), int(self.LF)
        if F["mb"] is not None:
            # many-body terms (SBEs.py:5225-5232, 5688-5695) with the eps the
            # table was screened with (E1D of CalcScreenedArrays)
            # DC shift of this step from the wire's q = 0 field (SBEs.py:5698-5702)
            mbd = F["mb"].descriptor(eps=F["eps"] if self.Screened else None,
                                     eac=float(np.real(np.asarray(Ex)[self.NQ0])), dt=dt)
            _lib.call("psb_full_step_mb_f64", nk, self.Nr, self.NQ0, _dev.ptr(V3),
                      _dev.ptr(F["Ee"]), _dev.ptr(F["Eh"]), _dev.ptr(fields), abi.as_ptr(prm),
                      abi.as_ptr(mbd), _dev.ptr(L1), _dev.ptr(L2), _dev.ptr(L3),
                      _dev.ptr(F["work"]), F["work"].numel(), _dev.stream_ptr())
        else:
            _lib.call("psb_full_step_f64", nk, self.Nr, self.NQ0, _dev.ptr(V3),
                      _dev.ptr(F["Ee"]), _dev.ptr(F["Eh"]), _dev.ptr(fields), abi.as_ptr(prm),
                      _dev.ptr(L1), _dev.ptr(L2), _dev.ptr(L3), _dev.ptr(F["work"]),
                      F["work"].numel(), _dev.stream_ptr())
        if not (self.Optics or self.LF):
            return
        _lib.call("psb_full_sources_f64", nk, self.Nr, _dev.ptr(F["kr"]), _dev.ptr(F["r"]),
                  _dev.ptr(F["window"]), float(self.L), float(self.dcv), float(yw(w)),
                  float((-1) ** w), _dev.ptr(L3), _dev.ptr(F["out"]), _dev.stream_ptr())
        out = F["out"].cpu().numpy()
        c3 = L3[1].diagonal().cpu().numpy() if self.LF else None
        d3 = L3[2].diagonal().cpu().numpy() if self.LF else None
        self._full_sources_post(out, c3, d3, Px, Py, Pz, Re, Rh)

    def _full_sources_post(self, out, c3, d3, Px, Py, Pz, Re, Rh):
        """Px, Py, Pz (QWPolarization3's factor and transform) and, with LF,
        Re, Rh (QWRho5's boundary offset, normalisation, transform) from the
        sums of psb_full_sources_f64 and the new diagonals c3, d3."""
        if self.Optics:
            for a, src in zip((Px, Py, Pz), out[:3]):
                a[:] = src * 2 * self.ehint / self.area / self.L
                wirespace.fftg(a)
        if self.LF:
            Re[:] = out[3]
            Rh[:] = out[4]
            wirespace.rho_post(Re, Rh, c3, d3, self.r[1] - self.r[0])
            Re[:] = 2.0 * _e0 * Re / self.area * self.ehint
            Rh[:] = 2.0 * _e0 * Rh / self.area * self.ehint

    def _full_batch_inputs(self, w0, fields, dt):
        """Device inputs of a batch step of wires w0 + 1 .. Nw: the fields
        [n][3][Nr] (zero without Optics) and the per-wire parameters [n][4]
        = yw(w), (-1)^w, the DC shift of the wire's q = 0 field, 0."""
        import torch

        from .manybody import dc_shift

        F = self.full
        n = self.Nw - w0
        fd = torch.as_tensor(np.ascontiguousarray(fields, dtype=np.complex128), device="cuda")
        if not self.Optics:
            fd.zero_()
        wpar = np.zeros((n, 4))
        for i in range(n):
            w = w0 + i + 1
            wpar[i, 0], wpar[i, 1] = yw(w), (-1) ** w
            if F["mb"] is not None:
                wpar[i, 2] = dc_shift(F["mb"].edc, float(np.real(fields[i][0][self.NQ0])), dt)
        return fd, torch.as_tensor(wpar, device="cuda")

    def _full_launch_batch(self, w0, fd, wpd, dt):
        """Launch the step and the source sums of wires w0 + 1 .. Nw on the
        current stream (psb_full_step_batch_f64, psb_full_sources_batch_f64)
        from device-resident fields fd and parameters wpd; the sums land in
        full["bout"][:n].  No host copies."""
        import torch

        from . import device as _dev

        F = self.full
        nk, nw = self.Nk, self.Nw
        n = nw - w0
        prm = np.zeros(1, dtype=abi.FULL_PARAMS_DTYPE)
        prm["ehint"], prm["dcv"] = self.ehint, self.dcv
        prm["gap"], prm["gam_e"], prm["gam_h"] = self.gap, self.gam_e, self.gam_h
        prm["hbar"], prm["dt"] = HBAR, dt
        prm["excitons"], prm["lf"] = int(self.Excitons), int(self.LF)
        if "bwork" not in F:
            F["bwork"] = torch.empty(int(_lib.load().psb_full_batch_work_bytes(nw, nk)),
                                     dtype=torch.uint8, device="cuda")
            F["bout"] = torch.zeros((nw, 5, self.Nr), dtype=torch.complex128, device="cuda")
        # the descriptor array must outlive the call (its dc_dk and eps are
        # per wire here: wpar, and the batch's own screening)
        mbd_arr = None if F["mb"] is None else F["mb"].descriptor()
        mbd = None if mbd_arr is None else abi.as_ptr(mbd_arr)
        tab = self.batch.tabdata.view(abi.TAB_BLOCKS, nk)
        t0 = self.batch.h_tables[0]
        L1, L2, L3 = (lv[w0:] for lv in F["L"])
        _lib.call("psb_full_step_batch_f64", n, nk, self.Nr, self.NQ0, _dev.ptr(tab),
                  float(t0["L"]), float(t0["dens_max"]), int(self.Screened), _dev.ptr(fd),
                  abi.as_ptr(prm), _dev.ptr(wpd), mbd, _dev.ptr(L1), _dev.ptr(L2),
                  _dev.ptr(L3), _dev.ptr(F["bwork"]), F["bwork"].numel(), _dev.stream_ptr())
        if self.Optics or self.LF:
            _lib.call("psb_full_sources_batch_f64", n, nk, self.Nr, _dev.ptr(F["kr"]),
                      _dev.ptr(F["r"]), _dev.ptr(F["window"]), float(self.L), float(self.dcv),
                      _dev.ptr(wpd), _dev.ptr(L3), _dev.ptr(F["bout"][:n]), _dev.stream_ptr())

    def _full_step_batch(self, w0, fields, dt):
        """One step of wires w0 + 1 .. Nw (1-based) on the full state in one
        launch set; fields [n][3][Nr] complex wire-space Ex, Ey, Ez.  Returns
        the five sources (Px, Py, Pz, Re, Rh) of each wire, [n][5][Nr], as
        _full_step writes them."""
        import torch

        n = self.Nw - w0
        fd, wpd = self._full_batch_inputs(w0, fields, dt)
        self._full_launch_batch(w0, fd, wpd, dt)
        srcs = np.zeros((n, 5, self.Nr), np.complex128)
        if not (self.Optics or self.LF):
            return srcs
        out = self.full["bout"][:n].cpu().numpy()
        if self.Optics:
            # QWPolarization3's factor and transform, all wires at once
            P = out[:, :3] * 2 * self.ehint / self.area / self.L   # contiguous [n][3][Nr]
            wirespace.fftg(P.reshape(3 * n, self.Nr))
            srcs[:, :3] = P
        if self.LF:
            L3 = self.full["L"][2][w0:]
            diag = torch.diagonal(L3[:, 1:3], dim1=-2, dim2=-1).cpu().numpy()  # [n][2][nk]
            # QWRho5's offset, normalisation and transform of every wire's
            # two densities at once (each row the bits of its own rho_post)
            A = np.ascontiguousarray(out[:, 3:5]).reshape(2 * n, self.Nr)
            wirespace.rho_post_rows(A, diag.reshape(2 * n, -1), self.r[1] - self.r[0])
            srcs[:, 3:5] = 2.0 * _e0 * A.reshape(n, 2, self.Nr) / self.area * self.ehint
        return srcs

    def _drive(self, Ex, Ey, Ez):
        """E = Ey[NQ0] after checking that no other q component reaches Meh."""
        if not self.Optics:
            return 0.0
        lo, hi = self.NQ0 - (self.Nk - 1), self.NQ0 + self.Nk
        win = slice(max(lo, 0), hi)
        ey = np.array(Ey[win], dtype=np.complex128, copy=True)
        ey[self.NQ0 - win.start] = 0.0
        if np.any(np.asarray(Ex)[win] != 0) or np.any(np.asarray(Ez)[win] != 0) or np.any(ey != 0):
            raise NotImplementedError(
                "the field has components other than Ey at q = 0 of the wire: the SBE state "
                "becomes non-diagonal, which needs the full-matrix right-hand side (not "
                "provided by pulsesuite_b200)")
        return complex(Ey[self.NQ0])

    def _sbe_calculator(self, Ex, Ey, Ez, Vr, dt, Px, Py, Pz, Re, Rh, WriteFields, w):
        """One leapfrog step of wire w (1-based) driven by the wire-space fields
        (SBEs.py:5624-5836), with its source terms written in place: Px, Py,
        Pz = QWPolarization3 of the new p (qwoptics.py:815-946) and, with LF,
        Re, Rh = QWRho5 of the new C, D (qwoptics.py:948-1078), all in q space.

        While the state is diagonal and the field reaches the wire only at
        q = 0 (``Ey[NQ0]``), the step runs in the diagonal kernel; any other
        field (or a non-diagonal state read from backup files) switches the
        solver, for good, to the full Nk x Nk state (psb_full_step_f64)."""
        if self.full is None and (self._many_body or not self._is_diagonal(Ex, Ey, Ez)):
            self._enter_full()
        if self.full is not None:
            return self._full_step(Ex, Ey, Ez, dt, Px, Py, Pz, Re, Rh, w)
        E = self._drive(Ex, Ey, Ez)
        for a in (Px, Py, Pz, Re, Rh):
            a[:] = 0.0
        b = self.batch
        i = w - 1
        s = b.wire_slice(i)
        self.y0[s].copy_(b.y1[s])  # YY1 <- YY2 (SBEs.py:5082-5092)
        self._field[i, 0] = E.real
        self._field[i, 1] = E.imag
        self._wires_i32[i, self._steps_col] = 0  # the field sample of this step is index 0
        import torch

        order = torch.tensor([i], dtype=torch.int32, device="cuda")
        from . import device as _dev

        _lib.call("psb_leapfrog_f64", *b._common(), _dev.ptr(order), 1, _dev.ptr(b.y1),
                  _dev.ptr(b.y), b.n_state, self.Nk, b.tab_flags, _dev.ptr(self._field), 2,
                  self._field.numel(), 1, float(dt), _dev.ptr(b.P), b.P.shape[0], 1,
                  b.p_cap, abi.as_ptr(b.model), _dev.stream_ptr())
        st = int(b.wires()["status"][i])
        if st != abi.PSB_OK:
            raise _lib.PsbError(f"wire {w}: step status {st}")
        y3 = b.y[s].cpu().numpy()
        if self.Optics:
            # diagonal p: P(r) = 2 ehint/(area L) window(r) sum_k Re(p_k X_kk) (qwoptics.py:85-127)
            pr = y3[:, 0]
            sgn = np.array([(-1.0) ** (k + 1) for k in range(self.Nk)])
            scale = 2 * self.ehint / self.area / self.L
            Px[:] = scale * self.window * np.sum(pr * self.dcv * sgn)
            Py[:] = scale * self.window * (np.sum(pr * self.dcv) * yw(w))
            Pz[:] = scale * self.window * (np.sum(-pr * self.dcv) * (-1) ** w)
            for a in (Px, Py, Pz):
                _fftg(a)
        if self.LF:
            self._rho(y3[:, 2], y3[:, 3], Re, Rh)
            Re[:] = 2.0 * _e0 * Re / self.area * self.ehint
            Rh[:] = 2.0 * _e0 * Rh / self.area * self.ehint

    def _rho(self, ne, nh, re, rh):
        """QWRho5 (qwoptics.py:948-1078) for diagonal C, D: the density along
        the wire is sum_k n_k window(r) / (2L), then the boundary offset is
        removed, the totals are restored and the result is transformed."""
        nr = self.Nr
        dr = self.r[1] - self.r[0]
        re[:] = np.sum(ne) * self.window / (2.0 * self.L)
        rh[:] = np.sum(nh) * self.window / (2.0 * self.L)
        for a, tot in ((re, np.sum(np.abs(ne)) + 1e-50), (rh, np.sum(np.abs(nh)) + 1e-50)):
            a[:] = a - np.real(np.sum(a[0:10]) + np.sum(a[nr - 10:nr])) / 20.0
            a[:] = a * tot / (np.sum(np.abs(a)) * dr + 1e-100)
            _fftg(a)

    def QWCalculator(self, Exx, Eyy, Ezz, Vrr, rr, q, dt, w, Pxx, Pyy, Pzz, Rho, DoQWP,
                     DoQWDl):
        """Per-time-step entry (SBEs.py:5838-6001): the step counters and the
        wire-off gate of the reference (while the field stays below 1e-3 of
        Emaxxx the wire is off and the outputs are zero), then the fields
        brought onto the wire (Prop2QW: spline resampling, window, real part,
        transform), one step of wire w, and its sources brought back onto
        the propagation grid (QW2Prop) in place: Pxx, Pyy, Pzz and
        Rho = RhoH - RhoE.  The window makes a field along the wire reach
        every q, so the step runs on the full Nk x Nk state.  The
        diagnostic files of the reference are not written."""
        for a in (Pxx, Pyy, Pzz, Rho):
            a[:] = 0.0
        if w == 1:
            if self.jjj == self.jmax:
                self.jjj = 0
            self.xxx += 1
            self.jjj += 1
            self.t += dt
        mag = np.max(np.sqrt(np.abs(Exx) ** 2 + np.abs(Eyy) ** 2 + np.abs(Ezz) ** 2))
        if self.wireoff and mag < 1e-3 * self.Emax0:
            return
        self.wireoff = False
        DoQWP[0] = self.Optics
        DoQWDl[0] = self.LF
        Ex, Ey, Ez, Vr = wirespace.prop2qw(rr, Exx, Eyy, Ezz, Vrr, self.r, self.window)
        src = [np.zeros(self.Nr, np.complex128) for _ in range(5)]
        self._sbe_calculator(Ex, Ey, Ez, Vr, dt, *src, False, w)
        Px_, Py_, Pz_, RhoE, RhoH = wirespace.qw2prop(self.r, *src, np.asarray(rr), self.LF)
        Pxx[:] = Px_
        Pyy[:] = Py_
        Pzz[:] = Pz_
        Rho[:] = RhoH - RhoE
        if self.ignorewire:
            for a in (Pxx, Pyy, Pzz, Rho):
                a[:] = 0.0

    def QWCalculatorAll(self, Exx, Eyy, Ezz, Vrr, rr, q, dt, Pxx, Pyy, Pzz, Rho, DoQWP,
                        DoQWDl):
        """All Nw wires of one Maxwell step at once: the loop of
        rhoPJ.QuantumWire (rhoPJ.py:311-348), where wire w + 1 gets the
        fields sampled along it and one QWCalculator call.  Exx, Eyy, Ezz,
        Vrr are (Nx,) arrays that every wire sees (rhoPJ samples all wires at
        one place) or (Nx, Nw) arrays, column w for wire w + 1; Pxx, Pyy,
        Pzz, Rho are (Nx, Nw) arrays written in place.  The counters, the
        wire-off gate and every wire's outputs are those of the Nw
        QWCalculator calls in wire order; the steps of the wires that run
        are one psb_full_step_batch_f64 and one psb_full_sources_batch_f64
        launch set (a wire's results are the same bits as its own call's)."""
        nw = self.Nw

        def col(a, w):
            a = np.asarray(a)
            return a if a.ndim == 1 else a[:, w]

        for a in (Pxx, Pyy, Pzz, Rho):
            a[...] = 0.0
        # the counters of the call for wire 1 (SBEs.py:5849-5854)
        if self.jjj == self.jmax:
            self.jjj = 0
        self.xxx += 1
        self.jjj += 1
        self.t += dt
        # wire-off gate of each call in order: once a wire switches the
        # solver on, every later wire runs
        w0 = nw
        for w in range(nw):
            mag = np.max(np.sqrt(np.abs(col(Exx, w)) ** 2 + np.abs(col(Eyy, w)) ** 2
                                 + np.abs(col(Ezz, w)) ** 2))
            if not (self.wireoff and mag < 1e-3 * self.Emax0):
                w0 = w
                break
        if w0 == nw:
            return
        self.wireoff = False
        DoQWP[0] = self.Optics
        DoQWDl[0] = self.LF
        n = nw - w0
        # Prop2QW of every wire's four fields in one pass (once when all
        # wires see the same field)
        if all(np.asarray(a).ndim == 1 for a in (Exx, Eyy, Ezz, Vrr)):
            f1 = wirespace.prop2qw_rows(rr, np.stack([np.asarray(a, np.complex128) for a in
                                                      (Exx, Eyy, Ezz, Vrr)]), self.r, self.window)
            wf = np.broadcast_to(f1, (n,) + f1.shape)
        else:
            F = np.stack([np.stack([np.asarray(col(a, w), np.complex128)
                                    for a in (Exx, Eyy, Ezz, Vrr)]) for w in range(w0, nw)])
            wf = wirespace.prop2qw_rows(rr, F.reshape(4 * n, -1), self.r,
                                        self.window).reshape(n, 4, -1)
        if self.full is None and not self._many_body and all(
                self._is_diagonal(f[0], f[1], f[2]) for f in wf):
            # fields only at q = 0: the diagonal kernel, wire by wire
            srcs = np.zeros((n, 5, self.Nr), np.complex128)
            for i, f in enumerate(wf):
                self._sbe_calculator(f[0], f[1], f[2], f[3], dt, *srcs[i], False, w0 + i + 1)
        else:
            if self.full is None:
                self._enter_full()
            srcs = self._full_step_batch(w0, np.ascontiguousarray(wf[:, :3]), dt)
        out = wirespace.qw2prop_rows(self.r, srcs, np.asarray(rr), self.LF)
        if self.ignorewire:
            return
        Pxx[:, w0:] = out[:, 0].T
        Pyy[:, w0:] = out[:, 1].T
        Pzz[:, w0:] = out[:, 2].T
        Rho[:, w0:] = (out[:, 4] - out[:, 3]).T

    # -- small accessors (SBEs.py:5516-5534) ---------------------------------------
    def chiqw(self):
        return self.chiw

    def getqc(self):
        return self.qc

    def QWArea(self):
        return self.area

    def ShutOffOptics(self):
        self.Optics = False

    # -- backup files (SBEs.py:5536-5585) -----------------------------------------
    _KEYS = ("CC1", "CC2", "CC3", "DD1", "DD2", "DD3", "YY1", "YY2", "YY3")

    def _level_arrays(self):
        """{key: (Nw, Nk) complex diagonals} of the nine stored arrays, or
        (Nw, Nk, Nk) matrices [w, k1, k2] once the state is full."""
        out = {}
        if self.full is not None:
            for n, lv in enumerate(self.full["L"], start=1):
                a = lv.cpu().numpy()
                out[f"YY{n}"], out[f"CC{n}"], out[f"DD{n}"] = a[:, 0], a[:, 1], a[:, 2]
            return out
        levels = [lv.view(self.Nw, self.Nk, 4).cpu().numpy()
                  for lv in (self.y0, self.batch.y1, self.batch.y)]
        for n, a in enumerate(levels, start=1):
            out[f"YY{n}"] = a[:, :, 0] + 1j * a[:, :, 1]
            out[f"CC{n}"] = a[:, :, 2] + 0j
            out[f"DD{n}"] = a[:, :, 3] + 0j
        return out

    def write_sbes_data(self, n, directory="dataQW/backup/"):
        """Write the nine coherence arrays in the reference's backup format:
        one file per array, per wire then k2 then k1 one line "re im" of
        arr[k1, k2, w] (full Nk x Nk, zero off the diagonal)."""
        import os

        os.makedirs(directory, exist_ok=True)
        arrs = self._level_arrays()
        for key in self._KEYS:
            a = arrs[key]
            lines = []
            for w in range(self.Nw):
                for k2 in range(self.Nk):
                    for k1 in range(self.Nk):
                        if a.ndim == 3:
                            val = complex(a[w, k1, k2])
                        else:
                            val = complex(a[w, k1]) if k1 == k2 else 0j
                        lines.append(f"{np.real(val)} {np.imag(val)}\n")
            with open(os.path.join(directory, f"{key}.{n}.dat"), "w", encoding="utf-8") as f:
                f.write("".join(lines))

    def read_sbes_data(self, Nt, directory="dataQW/backup/"):
        """Read backup files written by the reference (or write_sbes_data);
        off-diagonal coherences switch the solver to the full Nk x Nk state."""
        import os

        import torch

        vals, mats, offdiag = {}, {}, False
        for key in self._KEYS:
            with open(os.path.join(directory, f"{key}.{Nt}.dat"), "r", encoding="utf-8") as f:
                raw = np.array([float(x) for x in f.read().split()], dtype=np.float64)
            m = (raw[0::2] + 1j * raw[1::2]).reshape(self.Nw, self.Nk, self.Nk)  # [w, k2, k1]
            mats[key] = np.ascontiguousarray(np.transpose(m, (0, 2, 1)))  # [w, k1, k2]
            vals[key] = np.einsum("wkk->wk", m)
            off = m.copy()
            idx = np.arange(self.Nk)
            off[:, idx, idx] = 0.0
            offdiag |= bool(np.any(off != 0))
        if offdiag or self.full is not None:
            if self.full is None:
                self._enter_full()
            for n, lv in enumerate(self.full["L"], start=1):
                m = np.stack([mats[f"YY{n}"], mats[f"CC{n}"], mats[f"DD{n}"]], 1)
                lv.copy_(torch.as_tensor(m))
            return
        for n, lv in enumerate((self.y0, self.batch.y1, self.batch.y), start=1):
            y = np.stack([vals[f"YY{n}"].real, vals[f"YY{n}"].imag, vals[f"CC{n}"].real,
                          vals[f"DD{n}"].real], -1).reshape(-1, 4)
            lv.copy_(torch.as_tensor(y))


# Module-level shims of the reference (SBEs.py:6019-6078).
_default_solver = None


def InitializeSBE(q, rr, r0, Emaxxx, lam, Nw, QW):
    global _default_solver
    _default_solver = SBESolver(q, rr, r0, Emaxxx, lam, Nw, QW)


def QWCalculator(Exx, Eyy, Ezz, Vrr, rr, q, dt, w, Pxx, Pyy, Pzz, Rho, DoQWP, DoQWDl):
    _default_solver.QWCalculator(Exx, Eyy, Ezz, Vrr, rr, q, dt, w, Pxx, Pyy, Pzz, Rho, DoQWP,
                                 DoQWDl)


def QWCalculatorAll(Exx, Eyy, Ezz, Vrr, rr, q, dt, Pxx, Pyy, Pzz, Rho, DoQWP, DoQWDl):
    _default_solver.QWCalculatorAll(Exx, Eyy, Ezz, Vrr, rr, q, dt, Pxx, Pyy, Pzz, Rho, DoQWP,
                                    DoQWDl)


def chiqw():
    return _default_solver.chiqw()


def getqc():
    return _default_solver.getqc()


def QWArea():
    return _default_solver.QWArea()


def ShutOffOptics():
    _default_solver.ShutOffOptics()


def WriteSBEsData(n):
    _default_solver.write_sbes_data(n)


def ReadSBEsData(Nt):
    _default_solver.read_sbes_data(Nt)
