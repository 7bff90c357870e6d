"""Multi-process paths on the host: LPT assignment of batch graphs, and the
two distributed counts run as world-size-2 gloo process groups whose ranks
count with the oracle (restating the shard rule) instead of a GPU."""
import os
import socket
import tempfile

import numpy as np
import pytest

import oracle
from signed_triangle_counting_b200 import GlobalTriCounts, distributed, synth

import _shard_ref


def test_lpt_assign_partitions_and_balances():
    rng = np.random.default_rng(5)
    costs = rng.integers(1, 1000, 300)
    for parts in (1, 2, 3, 8):
        bins = distributed.lpt_assign(costs, parts)
        assert len(bins) == parts
        flat = sorted(i for b in bins for i in b)
        assert flat == list(range(len(costs)))
        loads = [costs[b].sum() for b in bins]
        assert max(loads) <= costs.sum() / parts + costs.max()
        assert bins == distributed.lpt_assign(costs, parts)  # deterministic
    assert distributed.lpt_assign([5, 5, 5], 2) == [[0, 2], [1]]


class OracleContext:
    """Stands in for a GPU Context: the same interface, counted by the oracle."""

    def count_shard(self, src, dst, sign, shard, shards, **kw):
        el = synth.EdgeList(n=0, m=len(src), src=src, dst=dst, sign=sign)
        (rng, counts) = _shard_ref.shard_counts(el, shards)[shard]
        return GlobalTriCounts(*counts), rng

    def count_batch_packed(self, src, dst, sign, offsets, **kw):
        out = []
        for g in range(len(offsets) - 1):
            b, e = int(offsets[g]), int(offsets[g + 1])
            out.append(GlobalTriCounts(*oracle.count_arrays(src[b:e], dst[b:e], sign[b:e])))
        return out


def _graphs():
    el = synth.rmat(31, 11, 1 << 11, 16 << 11, p_pos=0.5)
    specs = synth.batch_specs(64)
    bel, offs = synth.batch_packed([s for s in specs if s["n"] < 20000][:6], 0, 6)
    return el, bel, offs


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        el, bel, offs = _graphs()
        ctx = OracleContext()
        c = distributed.count(ctx, el.src, el.dst, el.sign)
        rows = distributed.count_batch(ctx, bel.src, bel.dst, bel.sign, offs)
        np.save(os.path.join(out_dir, f"r{rank}.npy"),
                np.array([c.as_tuple()] + [r.as_tuple() for r in rows], dtype=np.int64))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.timeout(300)
def test_gloo_world2_counts_match_single_process():
    import torch.multiprocessing as mp
    with tempfile.TemporaryDirectory() as d:
        mp.spawn(_worker, args=(2, _free_port(), d), nprocs=2, join=True)
        res = [np.load(os.path.join(d, f"r{r}.npy")) for r in range(2)]
    np.testing.assert_array_equal(res[0], res[1])  # every rank holds every result
    el, bel, offs = _graphs()
    assert tuple(res[0][0]) == oracle.count_arrays(el.src, el.dst, el.sign)
    for g in range(len(offs) - 1):
        b, e = int(offs[g]), int(offs[g + 1])
        assert tuple(res[0][1 + g]) == oracle.count_arrays(bel.src[b:e], bel.dst[b:e], bel.sign[b:e])


def test_shard_rule_covers_rank_space_and_sums():
    el = synth.rmat(32, 10, 1 << 10, 16 << 10, p_pos=0.5)
    total = oracle.count_arrays(el.src, el.dst, el.sign)
    for shards in (1, 2, 3, 7):
        parts = _shard_ref.shard_counts(el, shards)
        assert parts[0][0][0] == 0
        for (a, b), (c, d) in zip([p[0] for p in parts], [p[0] for p in parts][1:]):
            assert b == c and a <= b
        assert tuple(sum(np.array(p[1]) for p in parts)) == total
