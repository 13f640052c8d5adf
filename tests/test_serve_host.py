"""Host-side logic of the serving loop (no GPU): request stream, slot pool
and HBM accounting."""

import numpy as np

from pulsesuite_b200 import serve


def test_poisson_stream_shape_and_determinism():
    a = serve.poisson_stream(rate=500.0, seconds=2.0, seed=7, chunk=50)
    b = serve.poisson_stream(rate=500.0, seconds=2.0, seed=7, chunk=50)
    assert [r.arrival for r in a] == [r.arrival for r in b]
    assert 700 < len(a) < 1300  # ~1000 arrivals
    arr = np.array([r.arrival for r in a])
    assert (np.diff(arr) > 0).all() and arr[-1] < 2.0
    nks = np.array([r.nk for r in a])
    assert set(nks) <= set(serve.C4_NKS)
    frac = [(nks == nk).mean() for nk in serve.C4_NKS]
    assert abs(frac[0] - 0.3) < 0.06 and abs(frac[4] - 0.05) < 0.03
    steps = np.array([r.nsteps for r in a])
    assert (steps % 50 == 0).all() and steps.min() >= 1000 and steps.max() <= 4000


def test_slot_pool_budget_and_reuse():
    pool = serve.SlotPool({64: 2, 512: 1}, budget_bytes=serve.request_bytes(512, 1000, "split") + 10)
    nb = serve.request_bytes(512, 1000, "split")
    s = pool.try_take(512, nb)
    assert s == 0
    assert pool.try_take(512, nb) is None          # no slot left
    small = serve.request_bytes(64, 1000, "split")
    assert pool.try_take(64, small) is None         # budget exhausted
    pool.give_back(512, s, nb)
    assert pool.used == 0
    assert pool.try_take(64, small) is not None
    assert pool.in_use(64) == 1 and pool.in_use(512) == 0


def test_request_bytes():
    assert serve.request_bytes(256, 1000, "plain") == 32 * 256 + 16 * 1000
    assert serve.request_bytes(256, 1000, "split") == 96 * 256 + 16 * 1000
