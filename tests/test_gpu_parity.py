"""GPU parity: the sm_100a FP64 path against the reference goldens and the
CPU oracle, through the C ABI (WireBatch -> libpulsesuite_b200.so).

Tolerance (FP64 plain form): normwise relative error <= 1e-10 in p_k,
n_e,k, n_h,k and P(t) (max|x - ref| / max|ref|).
"""

import numpy as np
import pytest
import torch
from helpers import HBAR, golden, golden_exists, grid_from, one_wire, relerr
from test_oracle_golden import leapfrog_setup

from oracle import oracle as orc
from pulsesuite_b200 import abi, coulomb
from pulsesuite_b200 import grid as pgrid
from pulsesuite_b200.batch import WireBatch

pytestmark = pytest.mark.gpu

TOL = 1e-10


def batch_from_blocks(grids, blocks, wires, screened=False, p_cap=0):
    tables, tabdata = pgrid.pack_tables(grids, blocks, screened=screened)
    td = torch.as_tensor(tabdata, device="cuda")
    return WireBatch(grids, wires, screened=screened, p_cap=p_cap, tables=tables, tabdata=td)


# ---------------------------------------------------------------------------
# Coulomb tables on the GPU vs the reference.
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("nk", [32, 114])
def test_gpu_reference_tables(cuda, nk):
    d = golden(f"tables_ref_nk{nk}")
    g = pgrid.reference_grid(L=float(d["L"]))
    blk = coulomb.table_block(g, screened=True).reshape(9, nk).cpu().numpy()
    for i, name in enumerate(["Veh", "Vee", "Vhh"]):
        assert relerr(blk[i][1:], d[name][1:]) < 1e-13
    assert relerr(blk[5], d["chie"]) < 1e-13
    assert relerr(blk[6], d["chih"]) < 1e-13


def test_gpu_k0(cuda):
    d = golden("k0_ref")
    out = coulomb.k0_gpu(d["x"], 1.0, 1.0).cpu().numpy()
    assert np.max(np.abs(out - d["K03"]) / np.abs(d["K03"])) < 1e-12


def test_gpu_screen_eps(cuda):
    """psb_screen_f64 = Eps1D at the wire's own density (coulomb.py:1195-1230)."""
    d = golden("tables_ref_nk32")
    g = pgrid.reference_grid(L=float(d["L"]))
    nk = g.nk
    w = one_wire(nk)
    b = WireBatch([g], w, screened=True)
    y = np.zeros((nk, 4))
    y[:, 2] = d["ne"]
    y[:, 3] = d["nh"]
    b.set_state(y)
    eps = torch.zeros((1, nk), dtype=torch.float64, device="cuda")
    from pulsesuite_b200 import _lib, device

    _lib.call("psb_screen_f64", device.ptr(b.d_tables), 1, device.ptr(b.tabdata),
              device.ptr(b.d_wires), 1, device.ptr(b.y), device.ptr(eps), nk,
              device.stream_ptr())
    assert relerr(eps.cpu().numpy()[0], d["E1D"]) < 1e-13


# ---------------------------------------------------------------------------
# Right-hand side vs the reference.
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("name", ["rhs_k0_nk16", "rhs_k0_nk32", "rhs_k0_nk64", "rhs_k0_nk128",
                                  "rhs_ref_nk32"])
def test_gpu_rhs(cuda, name):
    d = golden(name)
    nk = int(d["nk"])
    g = grid_from(d, "k0")
    M = complex(d["M"])
    w = one_wire(nk, gap=float(d["gap_eff"]), gamma=float(d["gamma"]), mscale=1.0, amp=abs(M),
                 fwhm=1e30, phase=np.angle(-M))
    V = d["VC"]
    b = batch_from_blocks([g], [pgrid.table_block(g, V[:, 0], V[:, 1], V[:, 2])], w)
    y = np.stack([d["p"].real, d["p"].imag, d["ne"], d["nh"]], 1)
    b.set_state(y)
    dy = b.rhs().cpu().numpy()
    assert relerr(dy[:, 0] + 1j * dy[:, 1], d["dp"]) < 1e-13
    assert relerr(dy[:, 2], d["dC"]) < 1e-13
    assert relerr(dy[:, 3], d["dD"]) < 1e-13


def test_gpu_rhs_screened(cuda):
    d = golden("rhs_ref_nk32")
    nk = int(d["nk"])
    g = pgrid.reference_grid(L=float(d["L"]))
    blk = coulomb.table_block(g, screened=True).reshape(9, nk).cpu().numpy()
    blk[0:3] = d["VC"].T
    M = complex(d["M"])
    w = one_wire(nk, gap=float(d["gap_eff"]), gamma=float(d["gamma"]), mscale=1.0, amp=abs(M),
                 fwhm=1e30, phase=np.angle(-M))
    b = batch_from_blocks([g], [blk.reshape(-1)], w, screened=True)
    b.set_state(np.stack([d["p"].real, d["p"].imag, d["ne"], d["nh"]], 1))
    dy = b.rhs().cpu().numpy()
    assert relerr(dy[:, 0] + 1j * dy[:, 1], d["dp_s"]) < 1e-13
    assert relerr(dy[:, 2], d["dC_s"]) < 1e-13


# ---------------------------------------------------------------------------
# Time evolution vs the reference.
# ---------------------------------------------------------------------------
def rk4_golden_batch(d, screened=False):
    g = grid_from(d, "k0")
    v = d["V"]
    chie = chih = None
    if screened:
        blk = coulomb.table_block(g, screened=True).reshape(9, g.nk).cpu().numpy()
        chie, chih = blk[5], blk[6]
    blk = pgrid.table_block(g, v, v, v, chie, chih)
    w = one_wire(g.nk, gap=float(d["gap_eff"]), gamma=float(d["gamma"]),
                 mscale=float(d["mscale"]), pscale=float(d["pscale"]), amp=float(d["amp"]),
                 t0=float(d["t0"]), fwhm=float(d["fwhm"]))
    return batch_from_blocks([g], [blk], w, screened=screened, p_cap=int(d["nsteps"]))


@pytest.mark.parametrize("name,screened", [("rk4_c0_nk32", False), ("rk4_c0_nk64", False),
                                           ("rk4_screened_nk32", True)])
def test_gpu_rk4_vs_reference(cuda, name, screened):
    d = golden(name)
    b = rk4_golden_batch(d, screened)
    n = int(d["nsteps"])
    b.rk4(n, float(d["dt"]), p_stride=1)
    y = b.state()
    assert relerr(b.records(0), d["P"]) < TOL
    assert relerr(y[:, 0] + 1j * y[:, 1], d["p"]) < TOL
    assert relerr(y[:, 2], d["ne"]) < TOL
    assert relerr(y[:, 3], d["nh"]) < TOL
    w = b.wires()
    assert w["steps"][0] == n and w["status"][0] == 0
    assert w["t"][0] == pytest.approx(n * float(d["dt"]), rel=1e-12)


def test_gpu_rk4_full_config0(cuda):
    """Config 0 in full: Nk=128, 4000 RK4 steps of 1 fs, 50 fs pulse of area
    pi/2, T2 = 100 fs, against the reference's own RHS + rk4_dpc."""
    if not golden_exists("rk4_c0_nk128_full"):
        pytest.skip("full c0 golden not generated")
    d = golden("rk4_c0_nk128_full")
    b = rk4_golden_batch(d)
    n = int(d["nsteps"])
    # in chunks, as a server advances it between launches
    P = []
    for _ in range(4):
        b.rk4(n // 4, float(d["dt"]), p_stride=1)
        P.append(b.records(0)[: n // 4])
    y = b.state()
    assert relerr(np.concatenate(P), d["P"]) < TOL
    assert relerr(y[:, 0] + 1j * y[:, 1], d["p"]) < TOL
    assert relerr(y[:, 2], d["ne"]) < TOL


@pytest.mark.parametrize("name", ["leapfrog_nk32", "leapfrog_screened_nk32"])
def test_gpu_leapfrog_vs_reference(cuda, name):
    d = golden(name)
    nk = int(d["nk"])
    tables, tabdata, w, y1, y2, field, scr = leapfrog_setup(d)
    g = grid_from(d, "vint")
    b = WireBatch([g], w, screened=scr, p_cap=int(d["nsteps"]), tables=tables,
                  tabdata=torch.as_tensor(tabdata, device="cuda"))
    b.set_state(y2.reshape(nk, 4), y1.reshape(nk, 4))
    f = torch.as_tensor(field, device="cuda")
    n = int(d["nsteps"])
    b.leapfrog(f, n, float(d["dt"]), p_stride=1)
    assert relerr(b.records(0), d["P"]) < TOL
    assert relerr(b.state(), d["y2"]) < TOL
    assert relerr(b.y1.cpu().numpy(), d["y1"]) < TOL


# ---------------------------------------------------------------------------
# Uneven batches vs the oracle; alone vs in the mix; failure isolation.
# ---------------------------------------------------------------------------
def uneven_case(nks, seed=3, screened=False, nsteps=300):
    rng = np.random.default_rng(seed)
    uniq = sorted(set(nks))
    grids = [pgrid.wire_grid(nk) for nk in uniq]
    w = np.zeros(len(nks), dtype=abi.WIRE_DTYPE)
    for i, nk in enumerate(nks):
        g = grids[uniq.index(nk)]
        fwhm = rng.uniform(20e-15, 200e-15)
        mscale = g.ehint * g.dcv / 2.0
        w["table"][i] = uniq.index(nk)
        w["npulse"][i] = 1
        w["gap"][i] = -rng.uniform(-50e-3, 50e-3) * 1.602176634e-19
        w["gamma"][i] = 1.0 / rng.uniform(50e-15, 300e-15)
        w["mscale"][i] = mscale
        w["pscale"][i] = g.pscale
        w["amp"][i, 0] = pgrid.gaussian_amplitude(rng.uniform(0.1 * np.pi, 2 * np.pi), fwhm,
                                                  mscale)
        w["t0"][i, 0] = 0.6 * nsteps * 1e-15 * rng.uniform(0.3, 1.0)
        w["fwhm"][i, :] = fwhm
    return grids, w


def oracle_run(grids, w, nsteps, dt, screened=False, y0=None):
    blocks = [orc.grid_tables(g, screened=screened) for g in grids]
    tables, tabdata = pgrid.pack_tables(grids, blocks, screened=screened)
    ww = w.copy()
    nks = tables["nk"][ww["table"]]
    ww["off"] = np.concatenate([[0], np.cumsum(nks)[:-1]])
    ww["p_off"] = np.arange(len(ww)) * nsteps
    y = np.zeros(4 * int(nks.sum())) if y0 is None else y0.reshape(-1).copy()
    P = orc.rk4(tables, tabdata, ww, y, nsteps, dt, HBAR, p_stride=1, p_cap=nsteps)
    return y.reshape(-1, 4), P.reshape(len(ww), nsteps), ww


@pytest.mark.parametrize("screened", [False, True])
def test_gpu_uneven_batch_vs_oracle(cuda, screened):
    nks = [64, 512, 96, 128, 320, 64, 256, 480, 160, 32, 1024, 114]
    grids, w = uneven_case(nks, screened=screened, nsteps=200)
    n, dt = 200, 1e-15
    b = WireBatch(grids, w, screened=screened, p_cap=n)
    b.rk4(n, dt, p_stride=1)
    y = b.state()
    yo, Po, ww = oracle_run(grids, w, n, dt, screened=screened)
    for i in range(len(nks)):
        s = b.wire_slice(i)
        assert relerr(b.records(i), Po[i]) < TOL, i
        assert relerr(y[s, 0] + 1j * y[s, 1], yo[s, 0] + 1j * yo[s, 1]) < TOL, i
        assert relerr(y[s, 2], yo[s, 2]) < TOL, i
    assert (b.wires()["status"] == 0).all()


def test_gpu_alone_vs_mix_bitwise(cuda):
    nks = [64, 512, 96, 128, 320, 64, 256]
    grids, w = uneven_case(nks, seed=5, nsteps=100)
    n, dt = 100, 1e-15
    mix = WireBatch(grids, w, p_cap=n)
    mix.rk4(n, dt)
    ymix = mix.state()
    for i in (0, 1, 4):
        one = w[i:i + 1].copy()
        one["table"] = 0
        alone = WireBatch([grids[int(w["table"][i])]], one, p_cap=n)
        alone.rk4(n, dt)
        np.testing.assert_array_equal(alone.state(), ymix[mix.wire_slice(i)])
        np.testing.assert_array_equal(alone.records(0), mix.records(i))


def test_gpu_nonfinite_wire_isolated(cuda):
    """A wire whose state is NaN is flagged PSB_ERR_NONFINITE; the others are
    untouched (bitwise equal to a clean run)."""
    nks = [64, 128, 64]
    grids, w = uneven_case(nks, seed=9, nsteps=50)
    clean = WireBatch(grids, w, p_cap=50)
    clean.rk4(50, 1e-15)
    bad = WireBatch(grids, w, p_cap=50)
    y0 = np.zeros((bad.n_state, 4))
    y0[bad.wire_slice(1).start + 3, 0] = np.nan
    bad.set_state(y0)
    bad.rk4(50, 1e-15)
    st = bad.wires()["status"]
    assert st[1] == abi.PSB_ERR_NONFINITE and st[0] == 0 and st[2] == 0
    for i in (0, 2):
        np.testing.assert_array_equal(bad.state()[bad.wire_slice(i)],
                                      clean.state()[clean.wire_slice(i)])


def test_gpu_invalid_descriptor_rejected(cuda):
    """A wire pointing at a table that does not exist is skipped with
    PSB_ERR_INVALID instead of reading out of bounds."""
    grids, w = uneven_case([64, 64], seed=1, nsteps=10)
    b = WireBatch(grids, w, p_cap=10)
    hw = b.h_wires.copy()
    hw["table"][1] = 7
    b.d_wires.copy_(torch.as_tensor(hw.view(np.uint8)))
    b.rk4(10, 1e-15)
    st = b.wires()["status"]
    assert st[0] == 0 and st[1] == abi.PSB_ERR_INVALID
