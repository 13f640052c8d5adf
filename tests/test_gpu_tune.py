"""The split-form autotuner on the device: it measures per-CTA costs for
every allowed (Nk, W), caches them in its JSON file (a second tuner with the
same key measures nothing), and the batch engine's tuned groups give the
same numbers as any fixed width (results do not depend on W)."""

import numpy as np
import pytest
from test_gpu_parity import uneven_case

from pulsesuite_b200 import tune
from pulsesuite_b200.batch import WireBatch

pytestmark = pytest.mark.gpu


def test_tuner_measures_caches_and_chooses(cuda, tmp_path, monkeypatch):
    monkeypatch.setenv("PSB_TUNE_CACHE", str(tmp_path / "tune.json"))
    t = tune.SplitTuner(steps=5)
    table = t.table([64, 1024])
    assert set(table) == {(64, 4), (64, 8), (64, 16), (1024, 4), (1024, 8)}
    assert all(v > 0 for v in table.values())
    assert t.measured == 5
    t2 = tune.SplitTuner(steps=5)
    assert t2.table([64, 1024]) == table and t2.measured == 0
    for nk, n in ((64, 10), (64, 5000), (1024, 3)):
        w = t.best_width(nk, n)
        assert w in t.allowed(nk)
    # one wire of a large grid: the narrowest group has the shortest CTA
    assert t.best_width(1024, 1) == min(t.allowed(1024), key=lambda w: t.cost(1024, w))
    w = t.choose({64: 3000, 1024: 20})
    assert set(w) == {64, 1024}


def test_tuned_batch_matches_fixed_width(cuda):
    nks = [128] * 40 + [512] * 9
    grids, w = uneven_case(nks, seed=61, nsteps=80)
    tuned = WireBatch(grids, w, p_cap=80, form="split")
    fixed = WireBatch(grids, w, p_cap=80, form="split", tune=False, split_w={128: 4, 512: 4})
    tuned.rk4(80, 1e-15)
    fixed.rk4(80, 1e-15)
    np.testing.assert_array_equal(tuned.state(), fixed.state())
    np.testing.assert_array_equal(tuned.P.cpu().numpy(), fixed.P.cpu().numpy())
