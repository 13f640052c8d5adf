"""GPU tests of the continuous-batching solve server (serving configuration c4).

A small stream whose requests outnumber the slots, so requests are admitted
into the running batch as earlier ones retire.  Every result must (1) come
back with status 0, (2) equal, bit for bit, the same request served alone
(wires are independent in both step kernels), and (3) match the FP64 oracle
within the form's tolerance: plain <= 1e-10, split <= 1e-6 in P(t) and
<= 1e-5 in the final state (normwise relative).
"""

import numpy as np
import pytest
from helpers import relerr
from test_gpu_parity import oracle_run

from pulsesuite_b200 import grid as pgrid
from pulsesuite_b200 import serve

pytestmark = pytest.mark.gpu

NKS = (64, 128, 256, 512, 1024)
TOL = {"plain": (1e-10, 1e-10), "split": (1e-6, 1e-5)}


def small_stream(seed=5, n=14):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(n):
        nk = int(rng.choice(NKS, p=(0.3, 0.3, 0.2, 0.12, 0.08)))
        reqs.append(serve.SolveRequest(i, 0.0, nk, float(rng.uniform(0.3 * np.pi, 2 * np.pi)),
                                       float(rng.uniform(-50e-3, 50e-3)),
                                       float(rng.uniform(20e-15, 60e-15)),
                                       float(rng.uniform(50e-15, 300e-15)),
                                       int(rng.choice((100, 150, 200))), 1e-15))
    return reqs


def make_server(form, cap):
    return serve.Server(form=form, chunk=50, max_steps=200, capacity=cap, nks=NKS)


@pytest.mark.parametrize("form", ["split", "plain"])
def test_serve_mix_alone_and_oracle(cuda, form):
    reqs = small_stream()
    srv = make_server(form, {64: 2, 128: 2, 256: 1, 512: 1, 1024: 1})
    res = srv.run(reqs, realtime=False)
    assert len(res) == len(reqs)
    assert all(r.status == 0 for r in res), [r.status for r in res]
    assert all(r.nsteps == q.nsteps and r.nk == q.nk for r, q in zip(res, reqs))
    # more requests than slots: some were admitted only after others retired
    assert max(r.admitted for r in res) > 0.0 or len(reqs) <= 6
    tol_p, tol_s = TOL[form]
    big = [i for i, q in enumerate(reqs) if q.nk == 1024][:1]
    assert big, "the stream should hold an Nk 1024 request"
    for i in sorted({0, 3, 7, *big}):
        q = reqs[i]
        one = make_server(form, {nk: 1 for nk in NKS}).run([q], realtime=False)[0]
        np.testing.assert_array_equal(one.P, res[i].P)
        np.testing.assert_array_equal(one.y, res[i].y)
        g = pgrid.wire_grid(q.nk)
        w = serve.wire_record(q, g, table=0)
        yo, Po, _ = oracle_run([g], w, q.nsteps, q.dt)
        y = res[i].y
        assert relerr(res[i].P, Po[0]) < tol_p, (form, i)
        assert relerr(y[:, 0] + 1j * y[:, 1], yo[:, 0] + 1j * yo[:, 1]) < tol_s, (form, i)
        assert relerr(y[:, 2], yo[:, 2]) < tol_s, (form, i)


def test_serve_cancel_waiting_and_running(cuda):
    """A request cancelled while waiting returns at once with no steps; one
    cancelled while running retires at its next tick with the records it
    has, which equal the first records of the same request served alone;
    the other requests are unaffected."""
    reqs = [serve.SolveRequest(0, 0.0, 1024, 1.5 * np.pi, 0.01, 40e-15, 200e-15, 4000, 1e-15),
            serve.SolveRequest(1, 0.0, 64, 1.0 * np.pi, 0.0, 30e-15, 100e-15, 200, 1e-15),
            serve.SolveRequest(2, 0.0, 64, 1.2 * np.pi, 0.02, 30e-15, 100e-15, 200, 1e-15),
            serve.SolveRequest(3, 0.0, 64, 0.7 * np.pi, -0.02, 30e-15, 100e-15, 200, 1e-15)]
    srv = serve.Server(form="split", chunk=50, max_steps=4000, nks=(64, 1024),
                       capacity={64: 1, 1024: 1})
    # request 3 waits behind 1 and 2 (one Nk-64 slot) and is cancelled at
    # once; request 0 runs ~0.6 s and is cancelled after 0.1 s
    res = srv.run(reqs, realtime=False, cancels=[(0.0, 3), (0.1, 0)])
    st = {r.rid: r for r in res}
    assert st[3].status == serve.STATUS_CANCELLED and st[3].nsteps == 0
    assert st[0].status == serve.STATUS_CANCELLED
    assert 0 < st[0].nsteps < 4000 and st[0].nsteps % 50 == 0
    assert st[1].status == 0 and st[2].status == 0
    solo = serve.Server(form="split", chunk=50, max_steps=4000, nks=(64, 1024),
                        capacity={64: 1, 1024: 1}).run([reqs[0]], realtime=False)[0]
    np.testing.assert_array_equal(st[0].P, solo.P[:st[0].nsteps])
