"""Synthetic workloads of the benchmark configurations (seeded).

All use the GaAs-like wire of ``grid.wire_grid`` (me 0.067, mh 0.45, gap
1.5 eV, dcv 0.5 e nm, eps_b 12.9, a = 5 nm, kmax = 3/a) driven in the
rotating frame: gap -> gap - hbar*omega_L (= -detuning) and
M_k(t) = -(ehint dcv / 2) E_env(t); dephasing T2 = 1/(gam_e + gam_h).
Pulse amplitudes follow from the pulse area theta = int 2|M|/hbar dt.

  c0  1 wire, Nk 128, 4000 steps of 1 fs, 50 fs pulse of area pi/2, T2 100 fs
  c1  1024 wires, Nk ~ U[64,512] rounded to 32; area U[0.1pi, 2pi];
      detuning U[-50,50] meV; FWHM U[20,200] fs; T2 U[50,300] fs; 3000 steps
  c2  16384 wires, Nk 512, screened; area U[0.2pi, 1.5pi]; 2000 steps
  c3  65536 wires (256 x 256 sites), Nk 256, pump (30 fs, area U[0.1pi, pi])
      + probe (15 fs, delay U[0, 200] fs, phase U[0, 2pi)); T2 100 fs;
      dt 0.5 fs; 4000 steps
  c4  serving stream, see serve.py
"""

from dataclasses import dataclass

import numpy as np

from . import abi
from . import grid as pgrid

EV = 1.602176634e-19


@dataclass
class Workload:
    name: str
    grids: list
    wires: np.ndarray
    nsteps: int
    dt: float
    screened: bool = False

    @property
    def nks(self):
        return np.array([self.grids[t].nk for t in self.wires["table"]], dtype=np.int64)

    @property
    def units_per_step(self):
        """wire*k units advanced by one time step of the whole batch."""
        return int(self.nks.sum())

    def flops_per_step(self):
        """Algorithmic FP64 flops of one RK4 step of the batch: per unit
        32 Nk + 150 (4 right-hand sides of 8 Nk exchange flops plus ~30
        elementwise flops each, plus the RK combination)."""
        nk = self.nks.astype(np.float64)
        return float(np.sum(nk * (32.0 * nk + 150.0)))


def _grids_for(nks):
    uniq = sorted(set(int(n) for n in nks))
    return uniq, [pgrid.wire_grid(n) for n in uniq]


def _fill(w, i, g, table, theta, fwhm, t0, det_eV, T2):
    mscale = g.ehint * g.dcv / 2.0
    w["table"][i] = table
    w["npulse"][i] = 1
    w["gap"][i] = -det_eV * EV
    w["gamma"][i] = 1.0 / T2
    w["mscale"][i] = mscale
    w["pscale"][i] = g.pscale
    w["amp"][i, 0] = pgrid.gaussian_amplitude(theta, fwhm, mscale)
    w["t0"][i, 0] = t0
    w["fwhm"][i, :] = fwhm


def config0():
    g = pgrid.wire_grid(128)
    w = np.zeros(1, dtype=abi.WIRE_DTYPE)
    _fill(w, 0, g, 0, 0.5 * np.pi, 50e-15, 150e-15, 0.0, 100e-15)
    return Workload("c0: 1 wire Nk=128, 4000 x 1 fs RK4", [g], w, 4000, 1e-15)


def config1(seed=1, nwires=1024, nsteps=3000):
    rng = np.random.default_rng(seed)
    nks = (np.round(rng.uniform(64, 512, nwires) / 32.0) * 32).astype(int)
    uniq, grids = _grids_for(nks)
    w = np.zeros(nwires, dtype=abi.WIRE_DTYPE)
    for i in range(nwires):
        fwhm = rng.uniform(20e-15, 200e-15)
        _fill(w, i, grids[uniq.index(nks[i])], uniq.index(nks[i]),
              rng.uniform(0.1 * np.pi, 2 * np.pi), fwhm, 3.0 * fwhm,
              rng.uniform(-50e-3, 50e-3), rng.uniform(50e-15, 300e-15))
    return Workload(f"c1: {nwires} wires, Nk U[64,512]/32, {nsteps} x 1 fs RK4", grids, w,
                    nsteps, 1e-15)


def config2(seed=2, nwires=16384, nsteps=2000):
    rng = np.random.default_rng(seed)
    g = pgrid.wire_grid(512)
    w = np.zeros(nwires, dtype=abi.WIRE_DTYPE)
    for i in range(nwires):
        _fill(w, i, g, 0, rng.uniform(0.2 * np.pi, 1.5 * np.pi), 50e-15, 150e-15, 0.0, 100e-15)
    return Workload(f"c2: {nwires} wires, Nk 512, screened, {nsteps} x 1 fs RK4", [g], w,
                    nsteps, 1e-15, screened=True)


def config3(seed=3, nwires=65536, nsteps=4000):
    rng = np.random.default_rng(seed)
    g = pgrid.wire_grid(256)
    mscale = g.ehint * g.dcv / 2.0
    w = np.zeros(nwires, dtype=abi.WIRE_DTYPE)
    w["table"] = 0
    w["npulse"] = 2
    w["gamma"] = 1.0 / 100e-15
    w["mscale"] = mscale
    w["pscale"] = g.pscale
    pump = rng.uniform(0.1 * np.pi, np.pi, nwires)
    delay = rng.uniform(0.0, 200e-15, nwires)
    phase = rng.uniform(0.0, 2 * np.pi, nwires)
    w["amp"][:, 0] = pgrid.gaussian_amplitude(pump, 30e-15, mscale)
    w["amp"][:, 1] = pgrid.gaussian_amplitude(0.1 * np.pi, 15e-15, mscale)
    w["t0"][:, 0] = 90e-15
    w["t0"][:, 1] = 90e-15 + delay
    w["fwhm"][:, 0] = 30e-15
    w["fwhm"][:, 1] = 15e-15
    w["phase"][:, 1] = phase
    return Workload(f"c3: {nwires} wires, Nk 256, pump+probe, {nsteps} x 0.5 fs RK4", [g], w,
                    nsteps, 0.5e-15)


CONFIGS = {"c0": config0, "c1": config1, "c2": config2, "c3": config3}
