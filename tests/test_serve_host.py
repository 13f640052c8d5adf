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


def test_wires_per_cta_choice():
    # few solves: the longest CTA sets the tick, 4 wires per CTA keep it short
    assert serve.choose_wires_per_cta({1024: 10}, 148) == {1024: 4}
    # saturated: the total CTA time sets the tick, 8 wires per CTA lower it
    assert serve.choose_wires_per_cta({1024: 2000}, 148) == {1024: 8}
    sat = {64: 1800, 128: 1800, 256: 1200, 512: 900, 1024: 300}
    assert set(serve.choose_wires_per_cta(sat, 148).values()) == {8}
    # a Poisson-load mix: the largest grid keeps 4 (its CTA is the tick),
    # smaller grids take 8 where that frees SM time without lengthening it
    mix = {64: 300, 128: 300, 256: 200, 512: 150, 1024: 50}
    w = serve.choose_wires_per_cta(mix, 148)
    assert w[1024] == 4 and w[64] == 8
    # sizes where 8 wires do not fit stay at 4; empty sizes are left out
    assert serve.choose_wires_per_cta({1024: 2000, 64: 0}, 148, lambda nk: nk < 1024) == {1024: 4}
    assert serve.choose_wires_per_cta({}, 148) == {}
    # the cost model scales unlisted sizes by Nk^2 from the nearest entry
    assert abs(serve.split_cta_cost(2048, 4) - 4 * serve.SPLIT_CTA_MS[(1024, 4)]) < 1e-12


def test_wire_records_equal_one_request_records():
    """Admission builds a tick's descriptors in one pass (wire_records); each
    record has the bytes wire_record gives its request alone."""
    from pulsesuite_b200 import grid as pgrid

    reqs = serve.poisson_stream(rate=2000.0, seconds=0.3, seed=11, chunk=50)
    g = pgrid.wire_grid(128)
    offs = np.arange(len(reqs), dtype=np.int64) * 128
    p_offs = np.arange(len(reqs), dtype=np.int64) * 4000
    batch = serve.wire_records(reqs, g, table=1, offs=offs, p_offs=p_offs)
    one = np.concatenate([serve.wire_record(r, g, table=1, off=int(o), p_off=int(p))
                          for r, o, p in zip(reqs, offs, p_offs)])
    assert batch.dtype == one.dtype and batch.tobytes() == one.tobytes()
