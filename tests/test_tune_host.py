"""Host logic of the split-form autotuner (pulsesuite_b200.tune), no GPU:
the joint per-tick width choice and the per-grid choice from per-CTA costs."""

import math

from pulsesuite_b200 import tune


def fake_cost(nk, w):
    # a wider group costs more per CTA but less per wire (as measured)
    return {4: 1.0, 8: 1.4, 16: 3.0}[w] * (nk / 256.0) ** 2


def test_choose_widths_latency_vs_throughput():
    allowed = lambda nk: (4, 8, 16) if nk <= 512 else (4, 8)  # noqa: E731
    # few solves: the longest CTA sets the tick, the narrowest group wins
    assert tune.choose_widths({1024: 10}, 148, fake_cost, allowed) == {1024: 4}
    # saturated: the total sets the tick, the cheapest per wire wins
    w = tune.choose_widths({256: 20000}, 148, fake_cost, allowed)
    assert w == {256: 8}  # 1.4/8 per wire < 1.0/4 and < 3.0/16
    sat = {64: 1800, 128: 1800, 256: 1200, 512: 900, 1024: 300}
    w = tune.choose_widths(sat, 148, fake_cost, allowed)
    assert all(w[nk] == 8 for nk in (64, 128, 256, 512))
    assert tune.choose_widths({}, 148, fake_cost, allowed) == {}
    assert tune.choose_widths({64: 0}, 148, fake_cost, allowed) == {}


def test_best_width_counts_waves():
    t = object.__new__(tune.SplitTuner)
    t.sms = 148
    t.maxnk = {4: 1024, 8: 1024, 16: 512}
    t.cta_ms = {(nk, w): fake_cost(nk, w) for nk in (128, 1024) for w in (4, 8, 16)}
    t.use_file = False
    # 100 wires: 25 CTAs of 4 (one wave, 1.0) beat 13 CTAs of 8 (one wave, 1.4)
    assert t.best_width(128, 100) == 4
    # 4000 wires: 1000 CTAs of 4 = 7 waves (7.0) vs 500 of 8 = 4 waves (5.6)
    # vs 250 of 16 = 2 waves (6.0)
    assert t.best_width(128, 4000) == 8
    # 16 is not allowed above its largest grid
    assert t.allowed(1024) == (4, 8)
    assert t.best_width(1024, 100000) == 8
    assert math.isclose(t.cost(128, 8), fake_cost(128, 8))
