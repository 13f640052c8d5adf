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
through ``psb_calch_f64``; the O(Nk) elementwise derivatives run as device
tensor arithmetic.  Arrays may be numpy arrays or tensors; results come
back as numpy (in place for CalcH, as the reference does).  Off-diagonal
states (a k-dependent field along the wire) need the full-matrix right-hand
side, which this package does not provide: such inputs raise
NotImplementedError.

For time integration use ``batch.WireBatch`` (RK4 or the reference's
leapfrog over many wires); these functions exist for callers that step the
reference's own way one right-hand side at a time.
"""

import numpy as np
from scipy.constants import hbar as HBAR

from . import _lib, abi, device

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
        raise NotImplementedError(f"{name} is not diagonal in k: the full-matrix SBE "
                                  "right-hand side is not provided by pulsesuite_b200")
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


def h_diagonals(p, ne, nh, VC, Ee, Eh, gap, excitons=True, stream=None):
    """Device computation of the renormalised H diagonals for one wire:
    returns complex Heh exchange part (without the drive) and real Hee, Hhh,
    each (Nk,) numpy."""
    import torch

    device.require_cuda()
    p = np.asarray(p, dtype=np.complex128)
    nk = p.size
    v = _v_rows(VC, nk)
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
    w = np.zeros(1, dtype=abi.WIRE_DTYPE)
    w["gap"] = gap
    y = np.stack([p.real, p.imag, np.asarray(ne, np.float64), np.asarray(nh, np.float64)], 1)
    d_tab = device.to_device(tables)
    d_td = torch.as_tensor(blk.reshape(-1), device="cuda")
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


def _device_diag(*arrs):
    import torch

    device.require_cuda()
    return [torch.as_tensor(np.array(a, dtype=np.complex128), device="cuda") for a in arrs]


def dpdt(C, D, p, Heh, Hee, Hhh, GamE, GamH, OffP):
    """d p / dt (SBEs.py:1850-1975) for diagonal states: (Nk, Nk) with the
    diagonal i hbar dp_k/dt = (Hee_k + Hhh_k) p_k - Heh_k (C_k + D_k) + Heh_k
    - i hbar (GamE_k + GamH_k) p_k + OffP_kk."""
    pd = _diag_of("p", p)
    nk = pd.size
    c, d = _diag_of("C", C), _diag_of("D", D)
    heh, hee, hhh = (_diag_of(n, m) for n, m in (("Heh", Heh), ("Hee", Hee), ("Hhh", Hhh)))
    off = np.diag(_np(OffP)) if _np(OffP).ndim == 2 else _np(OffP)
    g = _gam(GamE, nk) + _gam(GamH, nk)
    tp, tc, td, th, te, tH, to, tg = _device_diag(pd, c, d, heh, hee, hhh, off, g)
    r = (tH * tp + te * tp - th * tc - th * td + th - ii * hbar * tg * tp + to) / (ii * hbar)
    return np.diag(r.cpu().numpy())


def dCdt(Cee, Dhh, Phe, Heh, Hee, Hhh, GamE, GamH, OffE):
    """d C / dt (SBEs.py:2221-2337) for diagonal states: the diagonal is
    (Heh_k conj(p_k) - conj(Heh_k) p_k) / (i hbar) (the Hee commutator
    vanishes on the diagonal)."""
    pd = _diag_of("p", Phe)
    heh = _diag_of("Heh", Heh)
    tp, th = _device_diag(pd, heh)
    r = (th * tp.conj() - th.conj() * tp) / (ii * hbar)
    return np.diag(r.cpu().numpy())


def dDdt(Cee, Dhh, Phe, Heh, Hee, Hhh, GamE, GamH, OffH):
    """d D / dt (SBEs.py:2513-2636) for diagonal states: same diagonal as
    dCdt, (Heh_k conj(p_k) - conj(Heh_k) p_k) / (i hbar)."""
    return dCdt(Cee, Dhh, Phe, Heh, Hee, Hhh, GamE, GamH, OffH)
