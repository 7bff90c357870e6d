"""Shard ranges and per-shard counts restated from the oracle's forward CSR
(test helper, shared by the CPU and GPU shard tests).

Rule under test: in rank space ((degree, id) order), vertex r costs
1 + sum over its forward arcs r -> v of (d+(r) + d+(v)), saturated at
2^32 - 1; with P(r) the cost of the ranks below r, shard s of S starts at the
first rank r with P(r) >= ceil(P(n) s / S).  A shard counts the triangles
whose lowest-ranked vertex lies in its range."""
import numpy as np

import oracle


def rank_space(el):
    a = oracle.ForwardCSR(el.src, el.dst, el.sign).arrays()
    off, edges = a["offsets"].astype(np.int64), a["edges"].astype(np.int64)
    fdeg, rank = a["fdeg"].astype(np.int64), a["rank"].astype(np.int64)
    return off, edges, fdeg, rank


def shard_ranges(el, shards):
    off, edges, fdeg, rank = rank_space(el)
    n = len(fdeg)
    tail = np.repeat(np.arange(n), np.diff(off))
    per_arc = fdeg[tail] + fdeg[edges]
    cost_id = 1 + np.bincount(tail, weights=per_arc, minlength=n).astype(np.int64)
    cost_id = np.minimum(cost_id, 2 ** 32 - 1)
    cost = np.zeros(n, np.int64)
    cost[rank] = cost_id
    pre = np.concatenate([[0], np.cumsum(cost)])
    total = int(pre[-1])
    bounds = [0]
    for s in range(1, shards):
        target = (total * s + shards - 1) // shards
        bounds.append(int(np.searchsorted(pre[:n], target, side="left")))
    bounds.append(n)
    return [(bounds[s], bounds[s + 1]) for s in range(shards)], rank


def shard_counts(el, shards):
    """Per shard: ((lo, hi), counts t0..t3) from the oracle's per-vertex counts."""
    ranges, rank = shard_ranges(el, shards)
    vc = oracle.ForwardCSR(el.src, el.dst, el.sign).vertex_counts()  # by id, (n, 4)
    by_rank = np.zeros_like(vc)
    by_rank[rank] = vc
    return [((lo, hi), tuple(int(x) for x in by_rank[lo:hi].sum(axis=0))) for lo, hi in ranges]
