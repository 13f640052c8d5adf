"""GPU parity of the split form with one Coulomb matrix per wire
(psb_rk4_split_wire) against the CPU oracle, through the C ABI.

  * statically screened tables (eps(q; n1D) of each wire's own stage
    densities, recomputed every right-hand side: coulomb.py:1172-1230),
    the configuration-2 shape at Nk 512 and an uneven batch up to Nk 1024;
  * the reference's own Coulomb matrices (CalcCoulombArrays,
    coulomb.py:502-577: distinct Veh, Vee, Vhh from the electron and hole
    confinement), unscreened and screened;
  * per-wire results independent of the group a wire shares a CTA with
    (bitwise), and the timeout path of the bounded waits.

Tolerances as for the shared-matrix split form: <= 1e-6 normwise in P(t),
<= 1e-5 in the final state (p on the scale of its peak over the run).
"""

import numpy as np
import pytest
from test_gpu_configs import TOL_P, TOL_STATE, _errors
from test_gpu_parity import uneven_case

from pulsesuite_b200 import _lib, abi, workloads
from pulsesuite_b200 import grid as pgrid
from pulsesuite_b200.batch import WireBatch

pytestmark = pytest.mark.gpu


def _check(b, grids, w, n, dt, screened, label):
    assert (b.wires()["status"] == 0).all()
    e = _errors(b, grids, w, n, dt, screened=screened)
    print(f"{label}: max P err {e[:, 0].max():.2e}, max state err {e[:, 1:].max():.2e}")
    assert e[:, 0].max() < TOL_P and e[:, 1:].max() < TOL_STATE, e
    return e


def test_split_wire_c2_screened_nk512(cuda):
    wl = workloads.config2(seed=41, nwires=6, nsteps=400)
    b = WireBatch(wl.grids, wl.wires, screened=True, p_cap=wl.nsteps, form="split")
    assert len(b.wire_launches) == 1 and not b.split_launches
    b.rk4(wl.nsteps, wl.dt)
    _check(b, wl.grids, wl.wires, wl.nsteps, wl.dt, True, "c2 screened split")


def test_split_wire_screened_uneven(cuda):
    nks = [64, 1024, 96, 512, 128, 256, 320, 32]
    n, dt = 300, 1e-15
    grids, w = uneven_case(nks, seed=42, screened=True, nsteps=n)
    b = WireBatch(grids, w, screened=True, p_cap=n, form="split")
    b.rk4(n, dt)
    _check(b, grids, w, n, dt, True, "screened uneven split")


def _reference_case(Ls, seed, n, dt):
    """Wires on the reference's own grids (distinct Veh, Vee, Vhh).  Their
    k grids reach 1.2 x the gap in kinetic energy, so RK4 needs dt well
    below 1 fs (|E/hbar| dt < 2.8; at 1 fs the oracle itself diverges)."""
    rng = np.random.default_rng(seed)
    grids = [pgrid.reference_grid(L=L) for L in Ls]
    w = np.zeros(2 * len(grids), dtype=abi.WIRE_DTYPE)
    for i in range(len(w)):
        t = i % len(grids)
        g = grids[t]
        fwhm = rng.uniform(20e-15, 60e-15)
        workloads._fill(w, i, g, t, rng.uniform(0.2 * np.pi, 1.5 * np.pi), fwhm,
                        n * dt * rng.uniform(0.3, 0.6), rng.uniform(-30e-3, 30e-3),
                        rng.uniform(60e-15, 250e-15))
    return grids, w


@pytest.mark.parametrize("screened", [False, True])
def test_split_wire_reference_tables(cuda, screened):
    n, dt = 800, 0.25e-15
    grids, w = _reference_case([100e-9, 250e-9, 420e-9], seed=43 + screened, n=n, dt=dt)
    nks = [g.nk for g in grids]
    assert max(nks) <= 512 and len(set(nks)) == 3
    b = WireBatch(grids, w, screened=screened, p_cap=n, form="split")
    assert not (b.h_tables["flags"] & abi.PSB_TAB_SHARED_V).any()
    assert len(b.wire_launches) >= 1 and not b.split_launches
    b.rk4(n, dt)
    _check(b, grids, w, n, dt, screened, f"reference tables (nk {nks}), screened={screened}")


def test_split_wire_group_independent_bitwise(cuda):
    """A wire's result does not depend on the wires it shares a CTA with,
    nor on the group size."""
    wl = workloads.config2(seed=44, nwires=8, nsteps=60)
    runs = []
    for sw in (None, {512: 1}, {512: 3}):
        b = WireBatch(wl.grids, wl.wires, screened=True, p_cap=wl.nsteps, form="split",
                      split_w=sw)
        b.rk4(wl.nsteps, wl.dt)
        runs.append((b.state(), np.stack([b.records(i) for i in range(len(wl.wires))])))
    alone = WireBatch(wl.grids, wl.wires[3:4], screened=True, p_cap=wl.nsteps, form="split")
    alone.rk4(wl.nsteps, wl.dt)
    for y, P in runs[1:]:
        assert np.array_equal(y, runs[0][0]) and np.array_equal(P, runs[0][1])
    s = runs[0]
    nk = wl.grids[0].nk
    assert np.array_equal(alone.state(), s[0][3 * nk:4 * nk])
    assert np.array_equal(alone.records(0), s[1][3])


def test_split_wire_timeout_reported(cuda):
    """Waits bounded to one poll run out: the CTAs stop and report
    PSB_ERR_TIMEOUT, the call returns, and the next call (default bound) is
    correct (its tensor memory allocations complete)."""
    lib = _lib.load()
    wl = workloads.config2(seed=45, nwires=4, nsteps=20)
    b = WireBatch(wl.grids, wl.wires, screened=True, p_cap=wl.nsteps, form="split")
    lib.psb_split_set_wait_limit(1)
    try:
        b.rk4(wl.nsteps, wl.dt)
        st = b.wires()["status"]
    finally:
        lib.psb_split_set_wait_limit(0)
    assert set(np.unique(st)) <= {abi.PSB_OK, abi.PSB_ERR_TIMEOUT}, st
    assert (st == abi.PSB_ERR_TIMEOUT).any(), st
    b2 = WireBatch(wl.grids, wl.wires, screened=True, p_cap=wl.nsteps, form="split")
    b2.rk4(wl.nsteps, wl.dt)
    _check(b2, wl.grids, wl.wires, wl.nsteps, wl.dt, True, "after timeout")
