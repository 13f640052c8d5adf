"""k grids, material constants and Coulomb-table specifications.

Host-side set-up arithmetic (O(Nk) per grid) that mirrors the reference's
initialisation; the O(Nk * Ny^2) Coulomb integrals and the Bessel tables are
evaluated by the CUDA entry points (``coulomb.py`` in this package) and only
assembled here.

Two kinds of grid:

* ``reference_grid`` -- the grid ``SBESolver.__init__`` derives from
  ``params/qw.params`` (pulsesuite/PSTD3D/SBEs.py:4766-4835, 5040-5052), with
  the Gaussian-confinement Coulomb integral ``Vint`` (coulomb.py:69-177).
* ``wire_grid`` -- the synthetic quantum wire of the benchmark workloads:
  Nk points uniform on [-kmax, kmax] (half-offset like the reference grid),
  kmax = 3/a, and V(q) = e^2/(2 pi eps0 eps_b L) K0(|q| a).
"""

from dataclasses import dataclass, field

import numpy as np
from scipy.constants import e as e0
from scipy.constants import epsilon_0 as eps0
from scipy.constants import hbar
from scipy.constants import m_e as me0

from . import abi

pi = np.pi
twopi = 2.0 * np.pi


@dataclass
class Grid:
    """One k grid and the material constants its tables depend on."""

    nk: int
    dk: float
    kr: np.ndarray  # k points (1/m)
    L: float  # wire length (m); n1D = sum(ne+nh)/2/L and V ~ 1/L
    me: float  # kg
    mh: float  # kg
    epsr: float
    delta0: float  # wire thickness (m)
    alphae: float  # 1/m
    alphah: float  # 1/m
    vkind: str  # "vint" (reference) or "k0" (synthetic wire)
    radius: float = 0.0  # K0(|q| a) radius for vkind == "k0"
    y: np.ndarray = field(default=None)  # real-space grid for vkind == "vint"
    gap: float = 0.0
    dcv: float = 0.0
    ehint: float = 1.0
    area: float = 1.0

    # -- derived arrays ---------------------------------------------------
    @property
    def Ee(self):
        # SBEs.py:4834
        return hbar**2 * self.kr**2 / (2.0 * self.me)

    @property
    def Eh(self):
        # SBEs.py:4835
        return hbar**2 * self.kr**2 / (2.0 * self.mh)

    @property
    def qy(self):
        """Momentum transfer of V(q) at index distance q = 0..nk-1."""
        if self.vkind == "vint":
            # Qr[NQ0 + q] = q * dkr (GetKArray order, SBEs.py:5046-5052)
            return np.arange(self.nk, dtype=np.float64) * self.dk
        return np.abs(self.kr - self.kr[0])

    @property
    def vprefactor(self):
        # e0^2 / (2 pi eps0 epsr L), coulomb.py:546
        return e0**2 / (twopi * eps0 * self.epsr * self.L)

    @property
    def qe(self):
        # MakeQs at [q, 0] (coulomb.py:325-327)
        return np.maximum(np.abs(self.kr[0] - self.kr), self.alphae / 2.0)

    @property
    def qh(self):
        return np.maximum(np.abs(self.kr[0] - self.kr), self.alphah / 2.0)

    @property
    def chi_scale(self):
        # coulomb.py:626
        return e0**2 / (twopi * eps0 * self.epsr * hbar**2)

    @property
    def dens_max(self):
        # min(qe[1,1], qh[1,1]) / pi * 0.99  (coulomb.py:1222)
        return min(self.alphae / 2.0, self.alphah / 2.0) / pi * 0.99

    @property
    def pscale(self):
        # P = 2 ehint / (area L) * sum_k p_k * dcv  (qwoptics.py:941-943)
        return 2.0 * self.ehint / self.area / self.L * self.dcv


def reference_grid(L=100e-9, Delta0=5e-9, gap_eV=1.5, me_rel=0.07, mh_rel=0.45, HO_eV=100e-3,
                   epsr=9.1):
    """The k grid and constants of ``SBESolver.__init__`` (SBEs.py:4766-4835)."""
    gap = gap_eV * e0
    me = me_rel * me0
    mh = mh_rel * me0
    HO = HO_eV * e0
    kmax = np.sqrt(1.2 * gap * 2.0 * me / (hbar**2))
    dkr = twopi / (2.0 * L)
    nk_odd = int(np.floor(kmax / dkr) * 2 + 1)
    nr = nk_odd * 2
    nk = nk_odd - 1
    dnk = (nk - 1) // 2
    kr = np.array([dkr * (-dnk + k - 0.5) for k in range(nk)], dtype=np.float64)
    y = np.linspace(-(2 * L) / 2.0, (2 * L) / 2.0, nr)
    alphae = np.sqrt(me * HO) / hbar
    alphah = np.sqrt(mh * HO) / hbar
    ehint = np.sqrt(2.0 * alphae * alphah / (alphae**2 + alphah**2))
    dcv = np.sqrt((e0 * hbar) ** 2 / (6.0 * me0 * gap) * (me0 / me - 1.0))
    area = np.sqrt(2.0 * pi) / np.sqrt(alphae**2 + alphah**2) * Delta0
    return Grid(nk=nk, dk=dkr, kr=kr, L=L, me=me, mh=mh, epsr=epsr, delta0=Delta0,
                alphae=alphae, alphah=alphah, vkind="vint", y=y, gap=gap, dcv=dcv,
                ehint=ehint, area=area)


def wire_grid(nk, a=5e-9, me_rel=0.067, mh_rel=0.45, epsb=12.9, gap_eV=1.5, dcv_enm=0.5,
              Delta0=5e-9, HO_eV=100e-3):
    """Synthetic GaAs-like wire of radius a: nk points on [-3/a, 3/a],
    V(q) ~ K0(|q| a)/eps_b.  The screening constants (alpha, Delta0) use the
    reference's default confinement (HO = 100 meV, Delta0 = 5 nm)."""
    if nk % 2:
        raise ValueError("nk must be even")
    me = me_rel * me0
    mh = mh_rel * me0
    kmax = 3.0 / a
    dk = 2.0 * kmax / nk
    kr = dk * (np.arange(nk, dtype=np.float64) - (nk - 1) / 2.0)
    L = pi / dk
    HO = HO_eV * e0
    alphae = np.sqrt(me * HO) / hbar
    alphah = np.sqrt(mh * HO) / hbar
    return Grid(nk=nk, dk=dk, kr=kr, L=L, me=me, mh=mh, epsr=epsb, delta0=Delta0,
                alphae=alphae, alphah=alphah, vkind="k0", radius=a, gap=gap_eV * e0,
                dcv=dcv_enm * e0 * 1e-9, ehint=1.0, area=pi * a * a)


def table_block(grid, veh, vee, vhh, chie=None, chih=None):
    """Pack one grid's doubles in the tabdata block order of the C ABI."""
    nk = grid.nk
    blk = np.zeros((abi.TAB_BLOCKS, nk), dtype=np.float64)
    blk[abi.TAB_VEH] = veh
    blk[abi.TAB_VEE] = vee
    blk[abi.TAB_VHH] = vhh
    blk[abi.TAB_EE] = grid.Ee
    blk[abi.TAB_EH] = grid.Eh
    if chie is not None:
        blk[abi.TAB_CHIE] = chie
        blk[abi.TAB_CHIH] = chih
        blk[abi.TAB_QE] = grid.qe
        blk[abi.TAB_QH] = grid.qh
    return blk.reshape(-1)


def pack_tables(grids, blocks, screened=False, excitons=True):
    """Table descriptors + packed tabdata for a list of grids."""
    tables = np.zeros(len(grids), dtype=abi.TABLE_DTYPE)
    off = 0
    for i, (g, b) in enumerate(zip(grids, blocks)):
        tables[i]["nk"] = g.nk
        flags = 0
        if excitons:
            flags |= abi.PSB_TAB_EXCITONS
        if screened:
            flags |= abi.PSB_TAB_SCREENED
        v = np.asarray(b).reshape(abi.TAB_BLOCKS, g.nk)
        if np.array_equal(v[abi.TAB_VEH], v[abi.TAB_VEE]) and np.array_equal(
                v[abi.TAB_VEH], v[abi.TAB_VHH]):
            flags |= abi.PSB_TAB_SHARED_V
        tables[i]["flags"] = flags
        tables[i]["off"] = off
        tables[i]["L"] = g.L
        tables[i]["dens_max"] = g.dens_max
        off += b.size
    tabdata = np.concatenate(blocks) if blocks else np.zeros(0)
    return tables, np.ascontiguousarray(tabdata)


def gaussian_amplitude(theta, fwhm, mscale):
    """Field amplitude of a Gaussian envelope exp(-4 ln2 t^2/fwhm^2) whose
    pulse area int 2|M|/hbar dt equals theta (M = -mscale E)."""
    integral = fwhm * np.sqrt(pi / (4.0 * np.log(2.0)))
    return theta * hbar / (2.0 * mscale * integral)
