"""CUDA-graph capture of a batch step (WireBatch.capture): replaying the
graph advances the batch exactly like eager rk4 calls (bitwise), in both
forms, including the split form's side streams."""

import numpy as np
import pytest
import torch
from test_gpu_parity import uneven_case

from pulsesuite_b200.batch import WireBatch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("form", ["plain", "split"])
def test_graph_replay_matches_eager(cuda, form):
    nks = [64, 128, 128, 512, 1024, 256, 64]
    grids, w = uneven_case(nks, seed=81, nsteps=90)
    eager = WireBatch(grids, w, p_cap=30, form=form)
    graphed = WireBatch(grids, w, p_cap=30, form=form)
    for _ in range(3):
        eager.rk4(30, 1e-15)
    g = graphed.capture(30, 1e-15)  # one eager call, then the capture
    g.replay()
    g.replay()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(graphed.state(), eager.state())
    np.testing.assert_array_equal(graphed.P.cpu().numpy(), eager.P.cpu().numpy())
    we, wg = eager.wires(), graphed.wires()
    np.testing.assert_array_equal(we["steps"], wg["steps"])
    np.testing.assert_array_equal(we["t"], wg["t"])
