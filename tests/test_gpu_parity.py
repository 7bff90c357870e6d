"""GPU parity: the CUDA path against the oracle and the reference's own outputs.

Every count is bit-exact (integer work).  Small cases compare with the oracle
directly; the seeded workloads compare with the reference's counts recorded in
golden.json; at full size, size-independent properties (sign-flip symmetry,
relabelling / edge-order / duplicate invariance) cover what a second counter
cannot afford to recompute.
"""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle
import signed_triangle_counting_b200 as stc
from signed_triangle_counting_b200 import _capi, synth

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
CLI = ROOT / "signed_triangle_counting_b200" / "stc"
STRATEGIES = ["auto", "merge", "hash", "search", "split", "head"]


def small_graph(family: str, seed: int = 1):
    if family == "er":
        return synth.er(seed, 2000, 30000, 0.7)
    if family == "rmat":
        return synth.rmat(seed, 13, 1 << 13, 16 << 13, p_pos=0.5)
    if family == "rmat_dense":
        return synth.rmat(seed, 9, 1 << 9, 64 << 9, p_pos=0.4)
    if family == "delaunay":
        return synth.delaunay(seed, 20000, 0.2, 0.6)
    if family == "skew":
        return synth.skew(seed, 1 << 16, 1 << 17, 8, 2000, 20000, 0.8)
    if family == "clique":
        k = 120
        a, b = np.triu_indices(k, 1)
        s = np.where(np.random.default_rng(seed).random(len(a)) < 0.5, 1, -1).astype(np.int8)
        return stc.EdgeList(n=k, m=len(a), src=a.astype(np.uint32), dst=b.astype(np.uint32), sign=s)
    raise ValueError(family)


FAMILIES = ["er", "rmat", "rmat_dense", "delaunay", "skew", "clique"]


def test_text_fixtures(ctx, golden, text_dir):
    for name in sorted(golden["text"]):
        g = golden["text"][name]["tc_serial"]
        el = stc.load_graph(text_dir / f"{name}.txt")
        for strategy in STRATEGIES:
            c = ctx.count_edge_list(el, strategy=strategy)
            assert c.as_tuple() == (g["t0"], g["t1"], g["t2"], g["t3"]), (name, strategy)
        assert ctx.last_stats().m_forward == g["forward_edges"], name


@pytest.mark.parametrize("family", FAMILIES)
@pytest.mark.parametrize("strategy", STRATEGIES)
def test_families_against_oracle(ctx, family, strategy):
    el = small_graph(family)
    want = oracle.count_arrays(el.src, el.dst, el.sign)
    assert sum(want) > 0
    assert ctx.count(el.src, el.dst, el.sign, strategy=strategy).as_tuple() == want


@pytest.mark.parametrize("family", FAMILIES)
def test_forward_csr_bit_exact(ctx, family):
    el = small_graph(family, seed=3)
    mine = ctx.build_forward_csr(el.src, el.dst, el.sign)
    want = oracle.ForwardCSR(el.src, el.dst, el.sign).arrays()
    assert (mine.n, mine.m) == (want["n"], want["m"])
    for k in ("offsets", "edges", "signs", "fdeg", "rank"):
        np.testing.assert_array_equal(getattr(mine, k), want[k], err_msg=k)


def test_count_from_reference_layout_csr(ctx):
    el = small_graph("rmat", seed=4)
    orc = oracle.ForwardCSR(el.src, el.dst, el.sign)
    a = orc.arrays()
    csr = stc.ForwardCSR(**a)
    for strategy in STRATEGIES:
        assert ctx.count_triangles(csr, strategy=strategy).as_tuple() == orc.count()


def test_malformed_csr_rejected(ctx):
    el = small_graph("er", seed=5)
    a = oracle.ForwardCSR(el.src, el.dst, el.sign).arrays()
    a["rank"] = a["rank"][::-1].copy()  # now some edges go from higher to lower rank
    with pytest.raises(stc.StcError) as e:
        ctx.count_triangles(stc.ForwardCSR(**a))
    assert e.value.status == _capi.STC_ERR_INVALID_ARGUMENT


def test_conflicting_duplicates_keep_first_occurrence(ctx):
    # Outside the reference's defined behaviour (its std::sort is unstable);
    # here the first occurrence in input order wins, as in the oracle.
    base = small_graph("er", seed=6)
    k = 5000
    src = np.concatenate([base.src, base.dst[:k]])
    dst = np.concatenate([base.dst, base.src[:k]])
    sign = np.concatenate([base.sign, -base.sign[:k]])
    want = oracle.count_arrays(src, dst, sign)
    assert want == oracle.count_arrays(base.src, base.dst, base.sign)
    assert ctx.count(src, dst, sign).as_tuple() == want


def test_self_loops_dropped(ctx):
    base = small_graph("er", seed=7)
    loops = np.arange(0, 2000, 3, dtype=np.uint32)
    src = np.concatenate([base.src, loops])
    dst = np.concatenate([base.dst, loops])
    sign = np.concatenate([base.sign, np.ones(len(loops), np.int8)])
    perm = np.random.default_rng(0).permutation(len(src))
    src, dst, sign = src[perm], dst[perm], sign[perm]
    assert ctx.count(src, dst, sign).as_tuple() == oracle.count_arrays(src, dst, sign)


def test_degenerate_inputs(ctx):
    z32, z8 = np.zeros(0, np.uint32), np.zeros(0, np.int8)
    assert ctx.count(z32, z32, z8).as_tuple() == (0, 0, 0, 0)
    one = np.array([3], np.uint32)
    assert ctx.count(one, one + 1, np.array([1], np.int8)).as_tuple() == (0, 0, 0, 0)
    assert ctx.count(one, one, np.array([-1], np.int8)).as_tuple() == (0, 0, 0, 0)
    # one triangle with ids at the top of the supported range
    top = (1 << 28) - 1
    t = ctx.count(np.array([top, top - 1, top], np.uint32), np.array([top - 1, 5, 5], np.uint32),
                  np.array([-1, -1, -1], np.int8))
    assert t.as_tuple() == (1, 0, 0, 0)


def _dense(src, dst):
    """The list relabelled to dense ids in the same order (the oracle's ids)."""
    ids, inv = np.unique(np.concatenate([src, dst]), return_inverse=True)
    return inv[: len(src)].astype(np.uint32), inv[len(src):].astype(np.uint32)


def test_large_ids_counted_as_dense(ctx):
    """Counts of totals take any uint32 id (the reference's parse does): ids
    at and above 2^31 - 1, up to 2^32 - 1, with duplicates and self-loops,
    give the counts of the same graph on dense ids."""
    rng = np.random.default_rng(17)
    for base in ((1 << 31) - 1, 1 << 31, (1 << 32) - 5000):
        el = synth.rmat(900 + base % 97, 11, 2000, 24000, p_pos=0.5)
        table = np.sort(rng.choice(np.arange(base, min(base + 4000, 1 << 32), dtype=np.uint64),
                                   el.n, replace=False)).astype(np.uint32)
        table[-1] = np.uint32((1 << 32) - 1)
        src, dst = table[el.src], table[el.dst]
        # a duplicate with the other sign, a self-loop on the largest id
        src = np.concatenate([src, src[:1], table[-1:]])
        dst = np.concatenate([dst, dst[:1], table[-1:]])
        sign = np.concatenate([el.sign, -el.sign[:1], np.array([1], np.int8)])
        ds, dd = _dense(src, dst)
        want = oracle.count_arrays(ds, dd, sign)
        assert ctx.count(src, dst, sign).as_tuple() == want, base
        # small ids mixed in
        src2 = np.concatenate([src, np.array([3, 4], np.uint32)])
        dst2 = np.concatenate([dst, np.array([4, int(table[0])], np.uint32)])
        sign2 = np.concatenate([sign, np.array([-1, 1], np.int8)])
        ds2, dd2 = _dense(src2, dst2)
        assert ctx.count(src2, dst2, sign2).as_tuple() == oracle.count_arrays(ds2, dd2, sign2)
    text = b"4294967295 5 1\n5 2147483647 -1\n2147483647 4294967295 1\n5 7 1\n"
    got = ctx.count_text(text)[0]
    assert got.as_tuple() == (0, 0, 1, 0)  # one triangle with one negative edge


def test_id_limit(ctx):
    """Per-vertex results are indexed by id: those calls keep ids below
    2^31 - 1."""
    for bad in ((1 << 31) - 1, 1 << 31, (1 << 32) - 1):
        with pytest.raises(stc.StcError) as e:
            ctx.vertex_counts(np.array([bad], np.uint32), np.array([1], np.uint32),
                              np.array([1], np.int8))
        assert e.value.status == _capi.STC_ERR_LIMIT


def test_vertex_counts(ctx):
    el = small_graph("rmat", seed=8)
    want = oracle.ForwardCSR(el.src, el.dst, el.sign).vertex_counts()
    got = ctx.vertex_counts(el.src, el.dst, el.sign)
    np.testing.assert_array_equal(got, want)


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref is not built")
@pytest.mark.parametrize("family", ["er", "rmat", "skew"])
def test_vertex_counts_equal_reference_cnt(ctx, family):
    # The reference's own per-source counts cnt[4n] (tc_serial.cpp:141-158),
    # taken from its unchanged count_triangles as differences of prefix
    # counts, against stc_vertex_counts vertex by vertex.
    if family == "er":
        el = synth.er(41, 1500, 12000, 0.7)
    elif family == "rmat":
        el = synth.rmat(42, 10, 1 << 10, 16 << 10)
    else:
        el = synth.skew(43, 1 << 11, 1 << 13, 4, 100, 600, 0.8)
    with oracle.RefKeptCSR(el.src, el.dst, el.sign) as ref:
        want = ref.vertex_counts().reshape(-1, 4)
    np.testing.assert_array_equal(ctx.vertex_counts(el.src, el.dst, el.sign), want)


def test_batch_graphs(ctx):
    graphs = [small_graph(f, seed=10 + i) for i, f in enumerate(FAMILIES)]
    got = ctx.count_batch([(g.src, g.dst, g.sign) for g in graphs])
    for g, c in zip(graphs, got):
        assert c.as_tuple() == oracle.count_arrays(g.src, g.dst, g.sign)


def test_device_generator_matches_host(ctx):
    import torch
    host = synth.rmat(99, 14, 1 << 14, 16 << 14, p_pos=0.3)
    m = host.m
    s = torch.empty(m, dtype=torch.int32, device="cuda")
    d = torch.empty(m, dtype=torch.int32, device="cuda")
    g = torch.empty(m, dtype=torch.int8, device="cuda")
    ctx.synth_rmat_device(99, 14, 1 << 14, 16 << 14, 0.57, 0.19, 0.19, 0.3, s, d, g)
    np.testing.assert_array_equal(s.cpu().numpy().view(np.uint32), host.src)
    np.testing.assert_array_equal(d.cpu().numpy().view(np.uint32), host.dst)
    np.testing.assert_array_equal(g.cpu().numpy(), host.sign)
    # torch device input goes through the same path
    assert ctx.count(s, d, g).as_tuple() == oracle.count_arrays(host.src, host.dst, host.sign)


def test_workloads_shrunk(ctx, golden):
    for key, w in sorted(golden["workloads"].items()):
        if w["shrink"] == 0:
            continue
        el = synth.workload(w["workload"], w["shrink"])
        for strategy in STRATEGIES:
            assert ctx.count(el.src, el.dst, el.sign, strategy=strategy).as_tuple() == tuple(w["t"]), \
                (key, strategy)


@pytest.mark.parametrize("k", [1, 2, 5])
def test_workloads_full_host_generated(ctx, golden, k):
    w = golden["workloads"].get(f"{k}/0")
    if w is None:
        pytest.skip("no full-size golden entry")
    el = synth.workload(k)
    assert el.m == w["m_input"]
    assert ctx.count(el.src, el.dst, el.sign).as_tuple() == tuple(w["t"])


def _rmat24(ctx):
    import torch
    n, samples = 1 << 24, 16 << 24
    s = torch.empty(samples, dtype=torch.int32, device="cuda")
    d = torch.empty(samples, dtype=torch.int32, device="cuda")
    g = torch.empty(samples, dtype=torch.int8, device="cuda")
    ctx.synth_rmat_device(synth.workload_seed(3), 24, n, samples, 0.57, 0.19, 0.19, 0.5, s, d, g)
    return s, d, g


def test_workload3_full_and_properties(ctx, golden):
    """Power-law workload at full size: reference counts, then sign-flip
    symmetry and invariance under relabelling, edge order and duplicates."""
    import torch
    w = golden["workloads"].get("3/0")
    s, d, g = _rmat24(ctx)
    c = ctx.count(s, d, g)
    if w is not None:
        assert c.as_tuple() == tuple(w["t"])
    # flipping every sign maps +++ <-> --- and ++- <-> +--
    flipped = ctx.count(s, d, -g)
    assert flipped.as_tuple() == (c.t3, c.t2, c.t1, c.t0)
    # relabel ids with a permutation, reverse half of the edges, shuffle them
    n = 1 << 24
    perm = torch.randperm(n, device="cuda", generator=torch.Generator("cuda").manual_seed(1)).int()
    s2, d2 = perm[s.long()], perm[d.long()]
    half = torch.arange(s.numel(), device="cuda") % 2 == 0
    s3 = torch.where(half, d2, s2)
    d3 = torch.where(half, s2, d2)
    order = torch.randperm(s.numel(), device="cuda", generator=torch.Generator("cuda").manual_seed(2))
    s3, d3, g3 = s3[order].contiguous(), d3[order].contiguous(), g[order].contiguous()
    assert ctx.count(s3, d3, g3).as_tuple() == c.as_tuple()
    # appending duplicates (same sign, either orientation) changes nothing
    k = 10_000_000
    s4 = torch.cat([s3, d3[:k]])
    d4 = torch.cat([d3, s3[:k]])
    g4 = torch.cat([g3, g3[:k]])
    assert ctx.count(s4, d4, g4).as_tuple() == c.as_tuple()


def test_cli_matches_reference_output(golden, text_dir):
    for name in ("k4_mixed", "crlf", "sign_tokens", "clique20", "rmat_s10", "workload1"):
        r = subprocess.run([str(CLI), str(text_dir / f"{name}.txt")], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        got = oracle.parse_program_output(r.stdout)
        s = golden["text"][name]["tc_serial"]
        mg = golden["text"][name]["tc_merge_sign_enu"]
        for k in ("n", "raw_edges", "forward_edges", "t0", "t1", "t2", "t3"):
            assert got[k] == s[k], (name, k)
        for k in ("balanced", "unbalanced", "total"):
            assert got[k] == mg[k], (name, k)


def _mixed_batch(count: int):
    graphs = []
    for i in range(count):
        kind = i % 7
        if kind == 0:
            el = synth.er(100 + i, 300 + 37 * i, 1500 + 90 * i, 0.3 + 0.01 * i)
        elif kind == 1:
            el = synth.rmat(100 + i, 9, 400 + i, 3000 + 50 * i, p_pos=0.5)
        elif kind == 2:
            el = synth.delaunay(100 + i, 500 + 40 * i, 0.2, 0.6)
        elif kind == 3:
            el = synth.skew(100 + i, 4096, 6000, 3, 100, 900, 0.8)
        elif kind == 4:  # empty graph
            el = stc.EdgeList(0, 0, np.zeros(0, np.uint32), np.zeros(0, np.uint32), np.zeros(0, np.int8))
        elif kind == 5:  # self-loops only, large ids
            ids = np.array([70000, 5, 9], np.uint32)
            el = stc.EdgeList(70001, 3, ids, ids.copy(), np.array([1, -1, 1], np.int8))
        else:  # reversed duplicates
            b = synth.er(100 + i, 200, 1200, 0.5)
            el = stc.EdgeList(b.n, 2 * b.m, np.concatenate([b.src, b.dst]),
                              np.concatenate([b.dst, b.src]), np.concatenate([b.sign, b.sign]))
        graphs.append(el)
    return graphs


def test_batch_packed_against_oracle(ctx):
    graphs = _mixed_batch(63)
    offs = np.zeros(len(graphs) + 1, np.uint64)
    offs[1:] = np.cumsum([g.m for g in graphs])
    src = np.concatenate([g.src for g in graphs]).astype(np.uint32)
    dst = np.concatenate([g.dst for g in graphs]).astype(np.uint32)
    sign = np.concatenate([g.sign for g in graphs]).astype(np.int8)
    for strategy in STRATEGIES:
        got = ctx.count_batch_packed(src, dst, sign, offs, strategy=strategy)
        for g, c in zip(graphs, got):
            assert c.as_tuple() == oracle.count_arrays(g.src, g.dst, g.sign), strategy


def test_batch_workload_full(ctx, golden):
    """The 4,096-graph workload against the reference's per-graph counts."""
    import torch
    b = golden.get("batch")
    if b is None:
        pytest.skip("no batch golden entry")
    specs = synth.batch_specs(b["G"])
    M = sum(b["m_input"])
    src = torch.empty(M, dtype=torch.int32, device="cuda")
    dst = torch.empty(M, dtype=torch.int32, device="cuda")
    sign = torch.empty(M, dtype=torch.int8, device="cuda")
    offs = np.zeros(b["G"] + 1, np.uint64)
    pos = 0
    for g0 in range(0, b["G"], 256):
        g1 = min(b["G"], g0 + 256)
        el, o = synth.batch_packed(specs, g0, g1)
        offs[g0:g1 + 1] = o + pos
        src[pos:pos + el.m] = torch.from_numpy(el.src.view(np.int32)).cuda()
        dst[pos:pos + el.m] = torch.from_numpy(el.dst.view(np.int32)).cuda()
        sign[pos:pos + el.m] = torch.from_numpy(el.sign).cuda()
        pos += el.m
    assert pos == M
    assert [int(x) for x in np.diff(offs)] == b["m_input"]
    got = ctx.count_batch_packed(src, dst, sign, offs)
    assert [list(c.as_tuple()) for c in got] == b["t"]


def test_complete_graph_closed_form(ctx):
    # A dense core too large for the oracle: K_8400 (35 M edges, forward
    # lists up to 8399 arcs, all in the giant class).  Signs are products of
    # vertex labels (a positive, b negative vertices), so every triangle is
    # balanced and the counts have closed forms: T3 = C(a,3) + C(b,3),
    # T1 = C(a,2) b + a C(b,2), T0 = T2 = 0.
    from math import comb
    k = 8400
    rng = np.random.default_rng(5)
    label = np.where(rng.random(k) < 0.6, 1, -1).astype(np.int8)
    a, b = np.triu_indices(k, 1)
    sign = (label[a] * label[b]).astype(np.int8)
    perm = rng.permutation(k).astype(np.uint32)
    na, nb = int((label > 0).sum()), int((label < 0).sum())
    want = (0, comb(na, 2) * nb + na * comb(nb, 2), 0, comb(na, 3) + comb(nb, 3))
    assert ctx.count(perm[a], perm[b], sign).as_tuple() == want
