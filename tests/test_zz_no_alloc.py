"""psb_rk4_split_noalloc: the split RK4 step for callers that cannot
allocate device memory (code running under another framework's allocator,
or a host that owns every allocation and only lends this library its
inputs and outputs).  Its workspace is a fixed array inside the library.

The test drives the new entry point through the C ABI on a grid large
enough that the kernel really uses the workspace (stage state outside
shared memory), two calls in a row, and checks state, P(t) records and
wire status against psb_rk4_split with a caller workspace.  Both entry
points run the same kernel on the same layout, so the results must be
bitwise equal (tolerance 0).  It also checks that a batch beyond the
built-in limit is refused with PSB_ERR_SIZE.

The file name sorts last so that a run stopping at the first failure has
already run every other test.
"""

import numpy as np
import pytest
from test_gpu_parity import uneven_case

from pulsesuite_b200 import _lib, abi, device
from pulsesuite_b200.batch import WireBatch

pytestmark = pytest.mark.gpu


def _workspace_grid():
    """A grid size whose stage state does not fit shared memory (W = 4)."""
    lib = _lib.load()
    nk = (int(lib.psb_split_max_nk_resident(4)) // 64 + 1) * 64
    assert nk <= int(lib.psb_split_max_nk(4))
    return nk


def _noalloc_rk4(b, nsteps, dt):
    import torch

    stream = device.stream_ptr(torch.cuda.current_stream())
    for wg, groups, ng, nkmax in b.split_launches:
        _lib.call("psb_rk4_split_noalloc", *b._common(), device.ptr(groups), ng, wg, nkmax,
                  device.ptr(b.y), b.n_state, int(nsteps), float(dt), device.ptr(b.P),
                  b.P.shape[0], 1, b.p_cap, abi.as_ptr(b.model), stream)


def test_noalloc_matches_workspace_entry_point(cuda):
    nk = _workspace_grid()
    grids, w = uneven_case([nk, nk, nk], seed=51, nsteps=120)
    n, dt = 60, 1e-15
    ref = WireBatch(grids, w, p_cap=n, form="split")
    new = WireBatch(grids, w, p_cap=n, form="split")
    assert new.n_state <= abi.PSB_SPLIT_NOALLOC_MAX_STATE
    for call in range(2):
        ref.rk4(n, dt)
        _noalloc_rk4(new, n, dt)
        st_ref, st_new = ref.wires(), new.wires()
        assert (st_new["status"] == 0).all(), st_new["status"]
        np.testing.assert_array_equal(st_new["steps"], st_ref["steps"])
        np.testing.assert_array_equal(new.state(), ref.state())
        np.testing.assert_array_equal(new.P.cpu().numpy(), ref.P.cpu().numpy())
        np.testing.assert_array_equal(st_new["t"], st_ref["t"])


def test_noalloc_rejects_batch_beyond_limit(cuda):
    grids, w = uneven_case([64], seed=52, nsteps=10)
    b = WireBatch(grids, w, p_cap=4, form="split")
    wg, groups, ng, nkmax = b.split_launches[0]
    lib = _lib.load()
    rc = lib.psb_rk4_split_noalloc(*b._common(), device.ptr(groups), ng, wg, nkmax,
                                   device.ptr(b.y), abi.PSB_SPLIT_NOALLOC_MAX_STATE + 1, 4,
                                   1e-15, device.ptr(b.P), b.P.shape[0], 1, b.p_cap,
                                   abi.as_ptr(b.model), None)
    assert rc == abi.PSB_ERR_SIZE
    assert b"exceeds" in lib.psb_last_error()
