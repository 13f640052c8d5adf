"""Multi-rank host logic of bench.py on CPU (gloo, world size 2): each rank
draws its own shard of wires (weak scaling, no data-path collective), the
timed region is combined as the max over ranks and the whole-job value counts
every rank's units."""

import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    import sys

    import torch

    sys.path.insert(0, REPO)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench

    wl = bench.make_workload("c1", rank, 32)
    units = torch.tensor([float(wl.units_per_step)], dtype=torch.float64)
    fake_ms = torch.tensor([10.0 + rank], dtype=torch.float64)  # rank-dependent time
    dist.all_reduce(fake_ms, op=dist.ReduceOp.MAX)
    all_units = [torch.zeros(1, dtype=torch.float64) for _ in range(world)]
    dist.all_gather(all_units, units)
    first = torch.tensor(wl.wires["amp"][:4, 0].copy())
    firsts = [torch.zeros_like(first) for _ in range(world)]
    dist.all_gather(firsts, first)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, float(fake_ms.item()), [float(u.item()) for u in all_units],
           [f.numpy().tolist() for f in firsts]))


@pytest.mark.timeout(300)
def test_two_ranks_shard_and_max_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=240) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    # max over ranks, identical on every rank
    assert out[0][1] == out[1][1] == 11.0
    # each rank drew its own wires (different seeds), same size
    a, b = out[0][3]
    assert not np.allclose(a, b)
    units = out[0][2]
    assert len(units) == 2 and all(u > 0 for u in units)
