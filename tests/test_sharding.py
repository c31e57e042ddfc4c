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


def test_lpt_partition_is_balanced_and_covers_each_tube_once():
    sys.path.insert(0, str(REPO / "vocalsim-2p5d-fdtd_b200" / "python"))
    from vocalsim_b200.sharding import lpt_partition
    rng = np.random.default_rng(3)
    costs = rng.integers(5_000, 20_000, size=256)
    for world in (1, 2, 3, 4, 8):
        parts = lpt_partition(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(int(costs[i]) for i in p) for p in parts]
        # LPT bound: no bin exceeds the mean by more than the largest single cost
        assert max(loads) - sum(loads) / world <= costs.max()
        assert max(loads) / min(loads) < 1.05
    assert lpt_partition([3, 1, 2], 5)[3:] == [[], []]


def _oracle_runner(ps, gs, steps):
    sys.path.insert(0, str(REPO / "oracle"))
    import oracle as O
    return np.stack([O.run(O.params(**p), O.Geometry(*g), steps, "f32") for p, g in zip(ps, gs)])


def _sharded_rank(rank, world, port, q):
    sys.path.insert(0, str(REPO))
    sys.path.insert(0, str(REPO / "vocalsim-2p5d-fdtd_b200" / "python"))
    import torch.distributed as dist
    from vocalsim_b200 import synthetic as S
    from vocalsim_b200.sharding import ShardedBatch
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        n = 5
        ps = [dict(cross_sectional_shape=2, source_type=2 if i == 3 else 1) for i in range(n)]
        gs = [S.batch_tube(i)[:2] for i in range(n)]
        costs = [10_000 + 1_000 * i for i in range(n)]
        sb = ShardedBatch(ps, gs, rank, world, costs=costs, runner=_oracle_runner)
        q.put((rank, sb.index, sb.run(120)))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharded_batch_gathers_the_traces_in_order():
    """Two gloo ranks split five tubes by LPT, each runs its share (here with
    the oracle as the runner, so no GPU is needed) and one all_gather returns
    the whole batch in the caller's order on both ranks: equal to the same
    tubes run in one process."""
    sys.path.insert(0, str(REPO / "vocalsim-2p5d-fdtd_b200" / "python"))
    from vocalsim_b200 import synthetic as S
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_sharded_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=180) for _ in range(world)), key=lambda x: x[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, idx0, tr0), (_, idx1, tr1) = out
    assert sorted(idx0 + idx1) == list(range(5)) and not set(idx0) & set(idx1)
    assert idx0 == [0, 1, 4] and idx1 == [2, 3]           # LPT of costs 10k..14k
    ps = [dict(cross_sectional_shape=2, source_type=2 if i == 3 else 1) for i in range(5)]
    gs = [S.batch_tube(i)[:2] for i in range(5)]
    ref = _oracle_runner(ps, gs, 120)
    assert np.array_equal(tr0, ref) and np.array_equal(tr1, ref)
