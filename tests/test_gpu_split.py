"""GPU parity of the split-precision tensor-core form (psb_rk4_split).

Tolerance (exchange sums as exact int8-digit products on the tensor cores,
FP64 right-hand side, FP32 stage point and RK accumulator, FP64 state):
normwise relative error <= 1e-6 in P(t) (the target of the split form) and
<= 1e-5 in the final p_k, n_e,k, n_h,k against the FP64 oracle / the
reference goldens.
"""

import numpy as np
import pytest
from helpers import golden, golden_exists, grid_from, one_wire, relerr
from test_gpu_parity import oracle_run, uneven_case

from pulsesuite_b200 import abi
from pulsesuite_b200 import grid as pgrid
from pulsesuite_b200.batch import WireBatch

pytestmark = pytest.mark.gpu

TOL = 1e-6
TOL_STATE = 1e-5


def test_split_small_single_wire(cuda):
    """One wire, Nk 64, 100 steps: the smallest case of the tcgen05 path."""
    grids, w = uneven_case([64], seed=11, nsteps=100)
    n, dt = 100, 1e-15
    b = WireBatch(grids, w, p_cap=n, form="split")
    b.rk4(n, dt)
    st = b.wires()
    assert st["status"][0] == 0, st["status"]
    assert st["steps"][0] == n
    yo, Po, _ = oracle_run(grids, w, n, dt)
    y = b.state()
    assert relerr(b.records(0), Po[0]) < TOL
    assert relerr(y[:, 0] + 1j * y[:, 1], yo[:, 0] + 1j * yo[:, 1]) < TOL_STATE
    assert relerr(y[:, 2], yo[:, 2]) < TOL_STATE


def test_split_uneven_batch_vs_oracle(cuda):
    nks = [64, 512, 96, 128, 320, 64, 256, 480, 160, 1024, 64, 512, 128, 96, 1024, 256,
           64, 64, 64, 64, 64, 64, 64, 64, 64, 64, 64, 64, 64, 64, 64, 64, 64]
    grids, w = uneven_case(nks, seed=21, nsteps=300)
    n, dt = 300, 1e-15
    b = WireBatch(grids, w, p_cap=n, form="split")
    b.rk4(n, dt)
    st = b.wires()
    assert (st["status"] == 0).all(), st["status"]
    y = b.state()
    yo, Po, _ = oracle_run(grids, w, n, dt)
    allerrs = []
    for i in range(len(nks)):
        s = b.wire_slice(i)
        allerrs.append([relerr(b.records(i), Po[i]),
                        relerr(y[s, 0] + 1j * y[s, 1], yo[s, 0] + 1j * yo[s, 1]),
                        relerr(y[s, 2], yo[s, 2]), relerr(y[s, 3], yo[s, 3])])
    e = np.array(allerrs)
    print(f"split: max P err {e[:, 0].max():.2e}, max state err {e[:, 1:].max():.2e}")
    assert e[:, 0].max() < TOL and e[:, 1:].max() < TOL_STATE, e


def test_split_full_config0_vs_reference(cuda):
    """Config 0 (Nk 128, 4000 RK4 steps of 1 fs) in the split form against
    the reference's own FP64 RHS + rk4_dpc."""
    if not golden_exists("rk4_c0_nk128_full"):
        pytest.skip("full c0 golden not generated")
    d = golden("rk4_c0_nk128_full")
    g = grid_from(d, "k0")
    v = d["V"]
    w = one_wire(g.nk, gap=float(d["gap_eff"]), gamma=float(d["gamma"]), mscale=float(d["mscale"]),
                 pscale=float(d["pscale"]), amp=float(d["amp"]), t0=float(d["t0"]),
                 fwhm=float(d["fwhm"]))
    import torch

    tables, tabdata = pgrid.pack_tables([g], [pgrid.table_block(g, v, v, v)])
    b = WireBatch([g], w, p_cap=1000, tables=tables, tabdata=torch.as_tensor(tabdata, device="cuda"),
                  form="split")
    n = int(d["nsteps"])
    P = []
    for _ in range(4):
        b.rk4(n // 4, float(d["dt"]))
        P.append(b.records(0)[: n // 4])
    y = b.state()
    assert relerr(np.concatenate(P), d["P"]) < TOL
    assert relerr(y[:, 0] + 1j * y[:, 1], d["p"]) < TOL_STATE
    assert relerr(y[:, 2], d["ne"]) < TOL_STATE


def test_split_alone_vs_mix_bitwise(cuda):
    nks = [128] * 12 + [512] * 3
    grids, w = uneven_case(nks, seed=31, nsteps=60)
    n, dt = 60, 1e-15
    mix = WireBatch(grids, w, p_cap=n, form="split")
    mix.rk4(n, dt)
    for i in (0, 5, 13):
        one = w[i:i + 1].copy()
        one["table"] = 0
        alone = WireBatch([grids[int(w["table"][i])]], one, p_cap=n, form="split")
        alone.rk4(n, dt)
        np.testing.assert_array_equal(alone.state(), mix.state()[mix.wire_slice(i)])
        np.testing.assert_array_equal(alone.records(0), mix.records(i))


def test_split_nonfinite_wire_isolated(cuda):
    nks = [128, 128, 128]
    grids, w = uneven_case(nks, seed=41, nsteps=40)
    clean = WireBatch(grids, w, p_cap=40, form="split")
    clean.rk4(40, 1e-15)
    bad = WireBatch(grids, w, p_cap=40, form="split")
    y0 = np.zeros((bad.n_state, 4))
    y0[bad.wire_slice(1).start + 7, 1] = np.inf
    bad.set_state(y0)
    bad.rk4(40, 1e-15)
    st = bad.wires()["status"]
    assert st[1] == abi.PSB_ERR_NONFINITE and st[0] == 0 and st[2] == 0
    for i in (0, 2):
        np.testing.assert_array_equal(bad.state()[bad.wire_slice(i)],
                                      clean.state()[clean.wire_slice(i)])


def test_split_routes_screened_tables_to_per_wire_kernel(cuda):
    """psb_rk4_split takes only unscreened tables with one shared matrix;
    the batch sends screened grids to psb_rk4_split_wire instead."""
    grids, w = uneven_case([64, 128], seed=1, nsteps=10)
    b = WireBatch(grids, w, screened=True, form="split")
    assert not b.split_launches and len(b.wire_launches) >= 1
    b.rk4(10, 1e-15)
    assert (b.wires()["status"] == 0).all()
