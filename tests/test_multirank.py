"""The N > 1 bench path on CPU: two gloo ranks run the timing reduction and seed
selection that bench.py uses under torchrun (replicas, max-over-ranks time)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    # each rank reports a different step time; every rank must see the max
    mine = [10.0 + rank, 5.0 * (world - rank), 1.0]
    got = bench.max_over_ranks(mine, world, device="cpu")
    seeds = [bench.rank_seed(k, rank) for k in range(3)]
    allseeds = [None] * world
    dist.all_gather_object(allseeds, seeds)
    out[rank] = (got, allseeds)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_two_rank_replica_timing(world):
    ctx = mp.get_context("spawn")
    port = _free_port()
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    for r in range(world):
        got, allseeds = res[r]
        assert got == [10.0 + world - 1, 5.0 * world, 1.0]
        flat = [s for ss in allseeds for s in ss]
        assert len(set(flat)) == len(flat)  # replicas never share a sample stream
