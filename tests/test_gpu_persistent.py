"""GPU tests of the persistent engine (device-planned worklists, one
persistent kernel on a device work queue, captured in a CUDA graph and
replayed): the same counts as the per-class kernels and the oracle, also when
a replay meets new data in the same buffers."""
import numpy as np
import pytest
import torch

import oracle
from signed_triangle_counting_b200 import synth

from test_gpu_parity import FAMILIES, STRATEGIES, _mixed_batch, small_graph

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("family", FAMILIES)
def test_persistent_single_graph(ctx, family):
    el = small_graph(family, seed=5)
    want = oracle.count_arrays(el.src, el.dst, el.sign)
    for strategy in STRATEGIES:
        for _ in range(2):  # capture, then replay
            got = ctx.count(el.src, el.dst, el.sign, strategy=strategy, persistent=True)
            assert got.as_tuple() == want, strategy


def test_persistent_vertex_counts(ctx):
    el = small_graph("rmat", seed=9)
    want = oracle.ForwardCSR(el.src, el.dst, el.sign).vertex_counts()
    np.testing.assert_array_equal(ctx.vertex_counts(el.src, el.dst, el.sign, persistent=True), want)


def test_replay_meets_new_data(ctx):
    # Same vertex count and edge count: the buffers (and the captured graph's
    # key) stay the same while the graph changes underneath.
    a = synth.er(101, 5000, 60000, 0.6)
    b = synth.er(102, 5000, 60000, 0.4)
    assert a.n == b.n and a.m == b.m
    wa = oracle.count_arrays(a.src, a.dst, a.sign)
    wb = oracle.count_arrays(b.src, b.dst, b.sign)
    assert wa != wb
    for el, want in ((a, wa), (b, wb), (a, wa), (b, wb)):
        assert ctx.count(el.src, el.dst, el.sign, persistent=True).as_tuple() == want


def test_persistent_on_a_torch_stream(ctx):
    el = small_graph("skew", seed=3)
    want = oracle.count_arrays(el.src, el.dst, el.sign)
    s = torch.cuda.Stream()
    dev = torch.device("cuda", 0)
    with torch.cuda.stream(s):
        src = torch.from_numpy(el.src.view(np.int32)).to(dev)
        dst = torch.from_numpy(el.dst.view(np.int32)).to(dev)
        sign = torch.from_numpy(el.sign).to(dev)
        for _ in range(2):
            assert ctx.count(src, dst, sign, persistent=True).as_tuple() == want
    torch.cuda.synchronize()


def test_batch_persistent_and_class_kernels_agree(ctx):
    graphs = _mixed_batch(40)
    offs = np.zeros(len(graphs) + 1, np.uint64)
    offs[1:] = np.cumsum([g.m for g in graphs])
    src = np.concatenate([g.src for g in graphs]).astype(np.uint32)
    dst = np.concatenate([g.dst for g in graphs]).astype(np.uint32)
    sign = np.concatenate([g.sign for g in graphs]).astype(np.int8)
    want = [oracle.count_arrays(g.src, g.dst, g.sign) for g in graphs]
    ctx.load_dispatch_model()
    for persistent in (True, False, True):
        for dispatch in ("fixed", "learned"):
            got = ctx.count_batch_packed(src, dst, sign, offs, dispatch=dispatch,
                                         persistent=persistent)
            assert [c.as_tuple() for c in got] == want, (persistent, dispatch)
    ctx.set_dispatch_model(None)
