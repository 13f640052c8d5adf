"""Coulomb tables and static screening on the GPU (drop-in for the hot-path
part of pulsesuite/PSTD3D/coulomb.py).

The reference computes its unscreened V(q) once per grid with a Gaussian
confinement double integral (``Vint``, coulomb.py:69-177), the 1D
susceptibility with a Bessel K0 (``CalcChi1D``, coulomb.py:580-630) and the
screened V/eps per SBE step (``CalcScreenedArrays``, coulomb.py:1195-1230).
Here the integrals and Bessel tables are CUDA kernels (``psb_coulomb_vint``,
``psb_coulomb_k0``, ``psb_chi1d``) and the per-step screening is fused into
the SBE step kernel; the functions below keep the reference's names and
signatures for callers that use them directly.  The module singleton mirrors
coulomb.py:1339-1447 (one grid per process, as in the reference).
"""

import numpy as np
import torch
from scipy.constants import e as e0
from scipy.constants import epsilon_0 as eps0
from scipy.constants import hbar

from . import _lib, device
from . import grid as pgrid

pi = np.pi
twopi = 2.0 * np.pi


# ---------------------------------------------------------------------------
# GPU table builders.
# ---------------------------------------------------------------------------
def vint_gpu(qy, y, alpha1, alpha2, delta0, prefactor, stream=None):
    """prefactor * Vint(qy[i]) for all i (device tensor, float64)."""
    device.require_cuda()
    qy_d = torch.as_tensor(np.ascontiguousarray(qy, dtype=np.float64), device="cuda")
    y_d = torch.as_tensor(np.ascontiguousarray(y, dtype=np.float64), device="cuda")
    out = torch.empty_like(qy_d)
    _lib.call("psb_coulomb_vint", device.ptr(qy_d), qy_d.numel(), device.ptr(y_d), y_d.numel(),
              float(alpha1), float(alpha2), float(delta0), float(prefactor), device.ptr(out),
              device.stream_ptr(stream))
    return out


def k0_gpu(q, radius, prefactor, stream=None):
    device.require_cuda()
    q_d = torch.as_tensor(np.ascontiguousarray(q, dtype=np.float64), device="cuda")
    out = torch.empty_like(q_d)
    _lib.call("psb_coulomb_k0", device.ptr(q_d), q_d.numel(), float(radius), float(prefactor),
              device.ptr(out), device.stream_ptr(stream))
    return out


def chi1d_gpu(qc, alpha, delta0, mass, scale, stream=None):
    device.require_cuda()
    q_d = torch.as_tensor(np.ascontiguousarray(qc, dtype=np.float64), device="cuda")
    out = torch.empty_like(q_d)
    _lib.call("psb_chi1d", device.ptr(q_d), q_d.numel(), float(alpha), float(delta0),
              float(mass), float(scale), device.ptr(out), device.stream_ptr(stream))
    return out


def table_block(g, screened=False):
    """The 9*nk table block of one grid (C-ABI layout), V and chi evaluated on
    the GPU, returned as a device float64 tensor."""
    if g.vkind == "vint":
        qy = g.qy
        veh = vint_gpu(qy, g.y, g.alphae, g.alphah, g.delta0, g.vprefactor)
        vee = vint_gpu(qy, g.y, g.alphae, g.alphae, g.delta0, g.vprefactor)
        vhh = vint_gpu(qy, g.y, g.alphah, g.alphah, g.delta0, g.vprefactor)
    else:
        veh = k0_gpu(g.qy, g.radius, g.vprefactor)
        vee = veh
        vhh = veh
    nk = g.nk
    blk = torch.zeros((9, nk), dtype=torch.float64, device="cuda")
    blk[0] = veh
    blk[1] = vee
    blk[2] = vhh
    blk[3] = torch.as_tensor(g.Ee, device="cuda")
    blk[4] = torch.as_tensor(g.Eh, device="cuda")
    if screened:
        blk[5] = chi1d_gpu(g.qe, g.alphae, g.delta0, g.me, g.chi_scale)
        blk[6] = chi1d_gpu(g.qh, g.alphah, g.delta0, g.mh, g.chi_scale)
        blk[7] = torch.as_tensor(g.qe, device="cuda")
        blk[8] = torch.as_tensor(g.qh, device="cuda")
    return blk.reshape(-1)


# ---------------------------------------------------------------------------
# Reference-named API (coulomb.py) for direct callers.
# ---------------------------------------------------------------------------
def K03(x):
    """K0(x) of the reference (usefulsubs.py:1794-1820), on the GPU."""
    x = float(x)
    if x > 1e2:
        return 0.0
    return float(k0_gpu(np.array([1.0]), x, 1.0).cpu()[0])


def Vint(Qyk, y, alphae, alphah, Delta0):
    """coulomb.py:107-177 (GPU)."""
    return float(vint_gpu(np.array([Qyk]), y, alphae, alphah, Delta0, 1.0).cpu()[0])


def MakeQs(ky, ae, ah):
    """coulomb.py:302-333."""
    d = np.abs(ky[None, :] - ky[:, None])
    return np.maximum(d, ae / 2.0), np.maximum(d, ah / 2.0)


def CalcCoulombArrays(y, ky, er, alphae, alphah, L, Delta0, Qy, kkp, ReadArrays=False,
                      ScrewThis=False):
    """coulomb.py:502-577: unscreened (N, N) arrays via the GPU Vint kernel."""
    N = len(ky)
    NQ = len(Qy)
    Veh0, Vee0, Vhh0 = (np.zeros((N, N)) for _ in range(3))
    if ReadArrays or ScrewThis:
        return Veh0, Vee0, Vhh0
    pref = e0**2 / (twopi * eps0 * er * L)
    eh = vint_gpu(Qy, y, alphae, alphah, Delta0, pref).cpu().numpy()
    ee = vint_gpu(Qy, y, alphae, alphae, Delta0, pref).cpu().numpy()
    hh = vint_gpu(Qy, y, alphah, alphah, Delta0, pref).cpu().numpy()
    kkp = np.asarray(kkp)
    ok = (kkp >= 0) & (kkp < NQ)
    idx = np.where(ok, kkp, 0)
    Veh0[ok] = eh[idx][ok]
    Vee0[ok] = ee[idx][ok]
    Vhh0[ok] = hh[idx][ok]
    return Veh0, Vee0, Vhh0


def CalcChi1D(ky, alphae, alphah, Delta0, epsr, me, mh, qe, qh):
    """coulomb.py:580-630 via the GPU K0 kernel."""
    scale = e0**2 / (twopi * eps0 * epsr * hbar**2)
    ce = chi1d_gpu(np.asarray(qe).reshape(-1), alphae, Delta0, me, scale).cpu().numpy()
    ch = chi1d_gpu(np.asarray(qh).reshape(-1), alphah, Delta0, mh, scale).cpu().numpy()
    return ce.reshape(np.shape(qe)), ch.reshape(np.shape(qh))


class CoulombModule:
    """Process-level Coulomb state (coulomb.py:1079-1230) with GPU tables.

    Only the arrays of the SBE hot path are built (V0, chi, qe/qh); the
    carrier-scattering tables (MakeK3/CalcMBArrays) belong to the
    relaxation terms, which this package does not provide."""

    def __init__(self, y, ky, L, Delta0, me, mh, Ee, Eh, ge, gh, alphae, alphah, er, Qy, kkp,
                 screened, LorentzDelta=False):
        self.LorentzDelta = LorentzDelta
        self.L = L
        self.qe, self.qh = MakeQs(ky, alphae, alphah)
        self.Veh0, self.Vee0, self.Vhh0 = CalcCoulombArrays(y, ky, er, alphae, alphah, L, Delta0,
                                                            Qy, kkp)
        self.Chi1De, self.Chi1Dh = CalcChi1D(ky, alphae, alphah, Delta0, er, me, mh, self.qe,
                                             self.qh)

    def SetLorentzDelta(self, boolean):
        self.LorentzDelta = bool(boolean)

    def Eps1D(self, n1D, Nk=None):
        """coulomb.py:1172-1193 (device elementwise)."""
        ce = torch.as_tensor(self.Chi1De, device="cuda")
        ch = torch.as_tensor(self.Chi1Dh, device="cuda")
        qe = torch.as_tensor(self.qe, device="cuda")
        qh = torch.as_tensor(self.qh, device="cuda")
        e = (1.0 - ce * 2 * torch.log(torch.abs((qe - pi * n1D) / (qe + n1D)))
             - ch * 2 * torch.log(torch.abs((qh - pi * n1D) / (qh + n1D))))
        return e.cpu().numpy()

    def CalcScreenedArrays(self, screened, L, ne, nh, VC, E1D):
        """coulomb.py:1195-1230, in place on VC (N, N, 3) and E1D (N, N)."""
        VC[:, :, 0] = self.Veh0
        VC[:, :, 1] = self.Vee0
        VC[:, :, 2] = self.Vhh0
        E1D[:, :] = 1.0
        if screened:
            density_1D = np.sum(np.real(ne) + np.real(nh)) / 2.0 / L
            density_max = min(self.qe[1, 1], self.qh[1, 1]) / pi * 0.99
            density_1D = min(density_1D, density_max)
            E1D[:, :] = self.Eps1D(density_1D)
            VC[:, :, 0] = VC[:, :, 0] / E1D
            VC[:, :, 1] = VC[:, :, 1] / E1D
            VC[:, :, 2] = VC[:, :, 2] / E1D


_instance = None
_LorentzDelta = False


def SetLorentzDelta(boolean):
    global _LorentzDelta
    _LorentzDelta = bool(boolean)
    if _instance is not None:
        _instance.SetLorentzDelta(boolean)


def InitializeCoulomb(y, ky, L, Delta0, me, mh, Ee, Eh, ge, gh, alphae, alphah, er, Qy, kkp,
                      screened):
    """coulomb.py:1351-1374: create / replace the process singleton."""
    global _instance
    _instance = CoulombModule(y, ky, L, Delta0, me, mh, Ee, Eh, ge, gh, alphae, alphah, er, Qy,
                              kkp, screened, LorentzDelta=_LorentzDelta)


def _require_instance():
    if _instance is None:
        raise ValueError("CoulombModule not initialized. Call InitializeCoulomb first.")
    return _instance


def CalcScreenedArrays(screened, L, ne, nh, VC, E1D):
    _require_instance().CalcScreenedArrays(screened, L, ne, nh, VC, E1D)


def Eps1D(n1D, Nk):
    return _require_instance().Eps1D(n1D, Nk)


def grid_tables(grids, screened=False, excitons=True):
    """Device tables for a list of grids: (host table descriptors, device
    tabdata tensor)."""
    blocks = [table_block(g, screened) for g in grids]
    # descriptors from host copies of the V rows (flags need them)
    host = []
    for g, b in zip(grids, blocks):
        h = np.zeros((9, g.nk))
        h[0:3] = b.reshape(9, g.nk)[0:3].cpu().numpy()
        host.append(h.reshape(-1))
    tables, _ = pgrid.pack_tables(grids, host, screened=screened, excitons=excitons)
    tabdata = torch.cat(blocks) if blocks else torch.zeros(0, dtype=torch.float64, device="cuda")
    return tables, tabdata.contiguous()
