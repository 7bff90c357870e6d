"""GPU tests of the persistent engine (device-planned worklists, one
persistent kernel on a device work queue, captured in a CUDA graph and
replayed; for a batch group, the whole build and count captured as one
graph): the same counts as the per-class kernels and the oracle, also when
a replay meets new data in the same buffers."""
import numpy as np
import pytest
import torch

import oracle
import signed_triangle_counting_b200 as stc
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


def _pack(graphs):
    offs = np.zeros(len(graphs) + 1, np.uint64)
    offs[1:] = np.cumsum([g.m for g in graphs])
    cat = lambda f, t: np.concatenate([getattr(g, f) for g in graphs]).astype(t)
    return cat("src", np.uint32), cat("dst", np.uint32), cat("sign", np.int8), offs


def _relabel(graphs, seed, grow=None):
    """Each graph with its ids permuted within its id space and signs
    re-drawn: same edge count, same id space and degree multiset.  With
    `grow` = (graph index, factor), that graph's ids are also multiplied by
    the factor, so the union outgrows the capacities of the first batch."""
    rng = np.random.default_rng(seed)
    out = []
    for i, g in enumerate(graphs):
        space = int(max(g.src.max(initial=0), g.dst.max(initial=0))) + 1 if g.m else 0
        perm = rng.permutation(space).astype(np.uint32) if space else np.zeros(0, np.uint32)
        src, dst = perm[g.src], perm[g.dst]
        if grow and grow[0] == i:
            src, dst = src * np.uint32(grow[1]), dst * np.uint32(grow[1])
        sign = np.where(rng.random(g.m) < 0.5, -1, 1).astype(np.int8)
        out.append(stc.EdgeList(int(max(src.max(initial=0), dst.max(initial=0))) + 1 if g.m else 0,
                                g.m, src, dst, sign))
    return out


def test_batch_pipeline_replays_over_new_data(ctx):
    """A batch group on the persistent engine: the first call builds
    uncapped, the second at capacities without capture, the third captures
    the whole pipeline (build and count) and every later call replays it,
    here over new contents of the same device buffers.  A batch that
    outgrows the capacities is counted again uncapped, exactly."""
    base = _mixed_batch(21)
    batches = {"a": base, "b": _relabel(base, 7), "c": _relabel(base, 8),
               "big": _relabel(base, 9, grow=(1, 400))}
    packed = {k: _pack(v) for k, v in batches.items()}
    want = {k: [oracle.count_arrays(g.src, g.dst, g.sign) for g in v] for k, v in batches.items()}
    assert want["a"] != want["b"]
    offs = packed["a"][3]
    for k in packed:
        assert np.array_equal(packed[k][3], offs)
    dev = torch.device("cuda", 0)
    src = torch.empty(len(packed["a"][0]), dtype=torch.int32, device=dev)
    dst = torch.empty_like(src)
    sign = torch.empty(len(packed["a"][0]), dtype=torch.int8, device=dev)
    replays = []
    for k in ("a", "b", "a", "b", "c", "big", "a", "b", "c"):
        s, d, g, _ = packed[k]
        src.copy_(torch.from_numpy(s.view(np.int32)))
        dst.copy_(torch.from_numpy(d.view(np.int32)))
        sign.copy_(torch.from_numpy(g))
        got = ctx.count_batch_packed(src, dst, sign, offs, persistent=True)
        assert [c.as_tuple() for c in got] == want[k], k
        st = ctx.last_stats()
        replays.append(st.groups_replayed)
        assert st.m_input == len(s)
        assert st.ms_count > 0
    # uncapped, capped, captured + replayed, replayed, replayed, overflow ->
    # uncapped, capped, captured + replayed, replayed
    assert replays == [0, 0, 1, 1, 1, 0, 0, 1, 1]
