"""The bounded waits of the split kernel, made to run out on purpose.

psb_split_set_wait_limit(1) lets every on-chip hand-off wait (MMA issuer,
A-tile generators, drain warps) poll once before giving up, so the CTAs stop
at their first wait: each waits (bounded) for its MMAs in flight, frees its
tensor memory and marks its wires PSB_ERR_TIMEOUT.  The test checks the
status, then that the context and the library are still usable: with the
default limit restored a new batch runs and gives the same numbers as a
clean batch (had tensor memory not been freed, its allocation would fail to
complete).  No fault is raised and nothing is left hung: the failure is a
status the host reads.
"""

import numpy as np
import pytest
import torch
from test_gpu_parity import uneven_case

from pulsesuite_b200 import _lib, abi
from pulsesuite_b200.batch import WireBatch

pytestmark = pytest.mark.gpu


def test_split_wait_timeout_reports_and_recovers(cuda):
    lib = _lib.load()
    nks = [128] * 8 + [512] * 4
    grids, w = uneven_case(nks, seed=71, nsteps=40)
    b = WireBatch(grids, w, p_cap=40, form="split", tune=False)
    try:
        assert lib.psb_split_set_wait_limit(1) == abi.PSB_OK
        b.rk4(40, 1e-15)
        torch.cuda.synchronize()
    finally:
        lib.psb_split_set_wait_limit(0)
    st = b.wires()["status"]
    assert set(np.unique(st)) <= {abi.PSB_OK, abi.PSB_ERR_TIMEOUT}, st
    assert (st == abi.PSB_ERR_TIMEOUT).any(), st
    # the context is usable: two clean batches agree bit for bit
    c1 = WireBatch(grids, w, p_cap=40, form="split", tune=False)
    c2 = WireBatch(grids, w, p_cap=40, form="split", tune=False)
    c1.rk4(40, 1e-15)
    c2.rk4(40, 1e-15)
    torch.cuda.synchronize()
    assert (c1.wires()["status"] == 0).all()
    np.testing.assert_array_equal(c1.state(), c2.state())
