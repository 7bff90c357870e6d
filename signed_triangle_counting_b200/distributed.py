"""Counting on several GPUs: one process per GPU, torch.distributed for the
plumbing (NCCL between GPUs; gloo runs the same code on host tensors).

The reference counts on one machine with OpenMP, so nothing here has a
counterpart there; both paths reduce to the single-GPU counts exactly.

* ``count``: one graph.  Every rank builds the same forward CSR and counts
  its shard (``Context.count_shard``: a range of source vertices in (degree,
  id) order of about equal merge-model cost); one all-reduce of the four
  counters sums the shards.
* ``count_batch``: many graphs.  Graphs are assigned to ranks by LPT on their
  edge counts (``lpt_assign``); each rank counts its graphs as one batch and
  one all-reduce of a (G, 4) array, zero in the rows of other ranks' graphs,
  gives every rank every graph's counts.
"""
from __future__ import annotations

import heapq

import numpy as np

from . import GlobalTriCounts


def lpt_assign(costs, parts: int) -> list:
    """Longest-processing-time assignment of items to ``parts`` bins: items in
    order of decreasing cost (ties by index) each go to the bin with the least
    load so far (ties to the lowest bin).  Returns, per bin, its item indices
    in increasing order."""
    costs = np.asarray(costs, dtype=np.float64)
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, b) for b in range(parts)]
    bins = [[] for _ in range(parts)]
    for i in order:
        load, b = heapq.heappop(heap)
        bins[b].append(i)
        heapq.heappush(heap, (load + costs[i], b))
    return [sorted(b) for b in bins]


def _group_info(group):
    import torch.distributed as dist
    return dist.get_rank(group), dist.get_world_size(group)


def _reduce_sum(rows, group, device):
    import torch
    import torch.distributed as dist
    t = torch.as_tensor(np.asarray(rows, dtype=np.int64), device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()


def count(ctx, src, dst, sign, *, group=None, device=None, **kw) -> GlobalTriCounts:
    """Counts one graph across the ranks of ``group``; every rank passes the
    same edge list and receives the whole graph's counts.  ``device`` holds
    the reduction tensor (the rank's GPU under NCCL, None for gloo)."""
    rank, world = _group_info(group)
    c, _ = ctx.count_shard(src, dst, sign, rank, world, **kw)
    t = _reduce_sum([c.as_tuple()], group, device)[0]
    return GlobalTriCounts(*(int(x) for x in t))


def _take(a, idx_ranges):
    """Concatenates the slices [b, e) of ``a`` (numpy array or torch tensor)."""
    if hasattr(a, "is_cuda"):
        import torch
        parts = [a[b:e] for b, e in idx_ranges]
        return torch.cat(parts) if parts else a[:0]
    return np.concatenate([a[b:e] for b, e in idx_ranges]) if idx_ranges else a[:0]


def batch_shard(src, dst, sign, offsets, rank: int, world: int):
    """The graphs LPT assigns to ``rank`` of ``world``, packed back to back:
    returns (src, dst, sign, offsets, graph indices)."""
    offsets = np.asarray(offsets, dtype=np.int64)
    mine = lpt_assign(np.diff(offsets), world)[rank]
    spans = [(int(offsets[g]), int(offsets[g + 1])) for g in mine]
    sub_off = np.concatenate([[0], np.cumsum([e - b for b, e in spans])]).astype(np.uint64)
    return _take(src, spans), _take(dst, spans), _take(sign, spans), sub_off, mine


def gather_batch(counts, mine, G: int, *, group=None, device=None) -> list:
    """Every graph's counts on every rank from each rank's counts of its own
    graphs ``mine`` (one all-reduce of a (G, 4) array)."""
    rows = np.zeros((G, 4), dtype=np.int64)
    for g, c in zip(mine, counts):
        rows[g] = c.as_tuple()
    total = _reduce_sum(rows, group, device)
    return [GlobalTriCounts(*(int(x) for x in r)) for r in total]


def count_batch(ctx, src, dst, sign, offsets, *, group=None, device=None, **kw) -> list:
    """Counts graphs stored back to back (graph g owns entries
    [offsets[g], offsets[g + 1])) across the ranks of ``group``; every rank
    passes the same arrays and receives every graph's counts."""
    rank, world = _group_info(group)
    G = len(offsets) - 1
    s, d, g, sub_off, mine = batch_shard(src, dst, sign, offsets, rank, world)
    counts = ctx.count_batch_packed(s, d, g, sub_off, **kw) if mine else []
    return gather_batch(counts, mine, G, group=group, device=device)
