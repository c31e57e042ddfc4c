"""Multi-GPU host logic on CPU: two gloo ranks shard the tube batch the way
bench.py does under torchrun -- disjoint seeds per rank, no data-path
collective, and the timing reduced as the max over ranks."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

REPO = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, n_tubes, q):
    sys.path.insert(0, str(REPO))
    sys.path.insert(0, str(REPO / "vocalsim-2p5d-fdtd_b200" / "python"))
    import torch
    import torch.distributed as dist
    import bench
    import vocalsim_b200 as V
    from vocalsim_b200 import synthetic as S
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        seeds = bench.rank_tube_seeds(rank, n_tubes)
        cells = 0
        for sd in seeds:                      # host-side map build of this rank's tubes only
            L, A, _, _ = S.batch_tube(sd)
            cells += V.build_maps(V.params(cross_sectional_shape=2), V.Geometry(L, A))["dims"]["interior_cells"]
        gathered = [None] * world
        dist.all_gather_object(gathered, (seeds, cells))
        slowest = bench.max_over_ranks(10.0 * (rank + 1), world)
        q.put((rank, gathered, slowest))
    finally:
        dist.destroy_process_group()


def test_two_rank_tube_sharding():
    world, n = 2, 5
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, n, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, gathered, slowest in out:
        assert slowest == 20.0                       # max over ranks, not the local time
        seeds = [set(g[0]) for g in gathered]
        assert seeds[0].isdisjoint(seeds[1])
        assert sorted(seeds[0] | seeds[1]) == list(range(world * n))
        assert all(g[1] > 0 for g in gathered)
