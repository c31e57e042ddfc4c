"""A caller's batch of tubes split across the GPUs of one node.

Tubes are independent (no per-step exchange), so a batch shards by tube:
every rank (one process per GPU, torch.distributed) takes a share of the
caller's tube list, runs it as one vs_batch on its own GPU, and the traces
come back to every rank in the caller's order with one all-gather.

  lpt_partition  longest-processing-time-first split of per-tube costs
                 (interior cells x steps) into `parts` bins: tubes in
                 decreasing cost, each to the currently lightest bin
  shard_batch    this rank's tube indices of a partition
  ShardedBatch   build + run this rank's share; gather(): the whole batch's
                 traces on every rank, in the caller's tube order

The gather pads every rank's (n_i, steps) block to the largest n_i, runs one
all_gather on the process group (NCCL over NVLink on GPUs, gloo on CPU) and
drops the padding.  Only the traces cross ranks; per-tube gradients of the
inversion are per-rank (Adam is per tube) and gather the same way.
"""
from __future__ import annotations

import heapq
from typing import Callable, Sequence

import numpy as np


def lpt_partition(costs: Sequence[float], parts: int) -> list[list[int]]:
    """Indices of `costs` split into `parts` bins by LPT; each bin keeps its
    indices in increasing order.  Ties go to the lowest bin index, so every
    rank computes the same partition."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, b) for b in range(parts)]
    bins: list[list[int]] = [[] for _ in range(parts)]
    for i in order:
        load, b = heapq.heappop(heap)
        bins[b].append(i)
        heapq.heappush(heap, (load + float(costs[i]), b))
    return [sorted(x) for x in bins]


def tube_costs(ps, gs) -> list[int]:
    """Interior cells of every tube (host map build only, no device work)."""
    from .solver import build_maps
    return [int(build_maps(p, g)["dims"]["interior_cells"]) for p, g in zip(ps, gs)]


def shard_batch(costs: Sequence[float], rank: int, world: int) -> list[int]:
    return lpt_partition(costs, world)[rank]


def gather_traces(local: np.ndarray, index: Sequence[int], n_total: int, group=None, device=None) -> np.ndarray:
    """All-gather every rank's (len(index), steps) traces; returns (n_total,
    steps) in the caller's order on every rank.  `device` is the torch device
    the collective runs on (a CUDA device for NCCL, None = CPU for gloo)."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    steps = local.shape[1] if local.ndim == 2 else 0
    n_local = torch.tensor([len(index)], dtype=torch.int64, device=device)
    sizes = [torch.zeros_like(n_local) for _ in range(world)]
    dist.all_gather(sizes, n_local, group=group)
    sizes = [int(s.item()) for s in sizes]
    width = max(sizes)
    buf = torch.zeros((width, steps + 1), dtype=torch.float32, device=device)
    if len(index):
        buf[:len(index), :steps] = torch.from_numpy(np.ascontiguousarray(local, np.float32)).to(buf.device)
        # the tube index rides along in the last column (exact in float32 below 2^24)
        buf[:len(index), steps] = torch.tensor(list(index), dtype=torch.float32, device=buf.device)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    out = np.zeros((n_total, steps), np.float32)
    seen = np.zeros(n_total, bool)
    for r, blk in enumerate(parts):
        blk = blk[:sizes[r]].cpu().numpy()
        for row in blk:
            i = int(row[steps])
            out[i] = row[:steps]
            seen[i] = True
    if not seen.all():
        raise RuntimeError("gather_traces: some tubes were not run by any rank")
    return out


class ShardedBatch:
    """This rank's LPT share of a caller's tube list, on this rank's GPU.

    runner(ps, gs, steps) -> (n, steps) traces runs a share; the default builds
    a vs_batch (vocalsim_b200.Batch) on the current CUDA device."""

    def __init__(self, ps, gs, rank: int, world: int, costs: Sequence[float] | None = None,
                 runner: Callable | None = None):
        if len(ps) != len(gs):
            raise ValueError("one geometry per parameter set")
        self.n = len(ps)
        self.costs = list(costs) if costs is not None else tube_costs(ps, gs)
        self.index = shard_batch(self.costs, rank, world)
        self.ps = [ps[i] for i in self.index]
        self.gs = [gs[i] for i in self.index]
        self._runner = runner
        self._batch = None

    def _default_run(self, steps: int) -> np.ndarray:
        from .solver import Batch
        if self._batch is None:
            self._batch = Batch(self.ps, self.gs)
        else:
            self._batch.reset()
        return self._batch.run(steps)

    def run_local(self, steps: int) -> np.ndarray:
        if not self.index:
            return np.zeros((0, steps), np.float32)
        if self._runner is not None:
            return np.asarray(self._runner(self.ps, self.gs, steps), np.float32)
        return self._default_run(steps)

    def run(self, steps: int, group=None, device=None) -> np.ndarray:
        """Traces of the whole batch (n, steps) on every rank."""
        return gather_traces(self.run_local(steps), self.index, self.n, group=group, device=device)

    def close(self) -> None:
        if self._batch is not None:
            self._batch.close()
            self._batch = None
