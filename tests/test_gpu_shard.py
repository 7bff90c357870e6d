"""GPU shards of one graph (the multi-GPU path on one device): each shard's
rank range and counts equal the restatement from the oracle, and the shards
add up to the whole count."""
import numpy as np
import pytest

import oracle
import signed_triangle_counting_b200 as stc
from signed_triangle_counting_b200 import synth

import _shard_ref

pytestmark = pytest.mark.gpu

GRAPHS = {
    "rmat": lambda: synth.rmat(41, 13, 1 << 13, 16 << 13, p_pos=0.5),
    "delaunay": lambda: synth.delaunay(42, 20000, 0.2, 0.6),
    "skew": lambda: synth.skew(43, 1 << 15, 1 << 16, 8, 1000, 10000, 0.8),
}


@pytest.mark.parametrize("name", sorted(GRAPHS))
def test_shards_match_oracle_and_sum(ctx, name):
    el = GRAPHS[name]()
    total = ctx.count(el.src, el.dst, el.sign).as_tuple()
    assert total == oracle.count_arrays(el.src, el.dst, el.sign)
    for shards in (1, 2, 3, 8):
        want = _shard_ref.shard_counts(el, shards)
        acc = np.zeros(4, np.int64)
        for s in range(shards):
            c, rng = ctx.count_shard(el.src, el.dst, el.sign, s, shards)
            assert rng == want[s][0], (shards, s)
            assert c.as_tuple() == want[s][1], (shards, s)
            acc += c.as_tuple()
        assert tuple(acc) == total


def test_shard_arguments_checked(ctx):
    el = GRAPHS["rmat"]()
    for shard, shards in ((0, 0), (2, 2), (0, 70000)):
        with pytest.raises(stc.StcError):
            ctx.count_shard(el.src, el.dst, el.sign, shard, shards)
