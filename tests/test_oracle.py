"""The oracle (plain-C restatement) pinned against the reference's own outputs.

golden.json holds what the reference programs printed (tests/golden/make_golden.py
compiled them from the reference sources), so these tests pin the oracle without
needing the reference at run time.  Where oracle/_ref is present, the oracle is
also compared with the reference's forward CSR array by array.
"""
import numpy as np
import pytest

import oracle
from signed_triangle_counting_b200 import synth


def _fixture_names(golden):
    return sorted(golden["text"])


def test_golden_programs_agree(golden):
    # The four reference programs agree with each other on every fixture.
    for name, res in golden["text"].items():
        s = res["tc_serial"]
        for prog in ("tc_merge_sign_enu", "tc_hash_sign_enu", "tc_merge_sign_split"):
            assert res[prog]["balanced"] == s["t1"] + s["t3"], name
            assert res[prog]["unbalanced"] == s["t0"] + s["t2"], name


def test_oracle_text_fixtures(golden, text_dir):
    for name in _fixture_names(golden):
        g = golden["text"][name]["tc_serial"]
        el = oracle.load_graph(text_dir / f"{name}.txt")
        assert el["n"] == g["n"], name
        assert el["lines"] == g["raw_edges"], name
        csr = oracle.ForwardCSR(el["src"], el["dst"], el["sign"])
        assert csr.m == g["forward_edges"], name
        assert csr.count() == (g["t0"], g["t1"], g["t2"], g["t3"]), name
        for prog, fn in (("tc_merge_sign_enu", csr.count_merge), ("tc_hash_sign_enu", csr.count_hash)):
            r = golden["text"][name][prog]
            assert fn() == (r["balanced"], r["unbalanced"]), (name, prog)


def test_oracle_workloads_shrunk(golden):
    for key, w in golden["workloads"].items():
        if w["shrink"] == 0 and w["workload"] != 1:
            continue  # full sizes are checked on the GPU
        el = synth.workload(w["workload"], w["shrink"])
        assert el.m == w["m_input"]
        assert oracle.count_arrays(el.src, el.dst, el.sign) == tuple(w["t"]), key


def test_oracle_vertex_counts_sum_to_totals():
    el = synth.rmat(5, 11, 1 << 11, 8 << 11)
    csr = oracle.ForwardCSR(el.src, el.dst, el.sign)
    vc = csr.vertex_counts()
    assert tuple(int(x) for x in vc.sum(axis=0)) == csr.count()


def test_oracle_detects_a_planted_sign_flip():
    # A mistake planted in the oracle's input changes its answer: flipping one
    # edge that closes a triangle moves that triangle to another type.
    src = np.array([0, 1, 0], np.uint32)
    dst = np.array([1, 2, 2], np.uint32)
    sign = np.array([1, 1, 1], np.int8)
    assert oracle.count_arrays(src, dst, sign) == (0, 0, 0, 1)
    sign[2] = -1
    assert oracle.count_arrays(src, dst, sign) == (0, 0, 1, 0)


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built here")
@pytest.mark.parametrize("family", ["er", "rmat", "delaunay", "skew", "dups"])
def test_oracle_csr_equals_reference_csr(family):
    if family == "er":
        el = synth.er(21, 3000, 20000, 0.7)
    elif family == "rmat":
        el = synth.rmat(22, 12, 1 << 12, 16 << 12)
    elif family == "delaunay":
        el = synth.delaunay(23, 5000)
    elif family == "skew":
        el = synth.skew(24, 1 << 14, 1 << 15, 8, 100, 3000, 0.8)
    else:  # same-sign duplicates in both orientations
        base = synth.er(25, 500, 3000, 0.5)
        el = base
        el.src = np.concatenate([base.src, base.dst[:1000]])
        el.dst = np.concatenate([base.dst, base.src[:1000]])
        el.sign = np.concatenate([base.sign, base.sign[:1000]])
    mine = oracle.ForwardCSR(el.src, el.dst, el.sign).arrays()
    ref = oracle.ref_forward_csr(el.src, el.dst, el.sign)
    for k in ("n", "m"):
        assert mine[k] == ref[k]
    for k in ("offsets", "edges", "signs", "fdeg", "rank"):
        np.testing.assert_array_equal(mine[k], ref[k], err_msg=k)


@pytest.mark.parametrize("scale,n,samples,p", [(10, 1 << 10, 16 << 10, 0.5),
                                                (14, 1 << 14, 16 << 14, 0.5),
                                                (12, 3000, 8 << 12, 0.3)])
def test_oracle_rmat_generator_equals_package_generator(scale, n, samples, p):
    # The bench's CPU baseline feeds the reference with the oracle's
    # generator, which must give the package's edge list bit for bit.
    el = synth.rmat(1003, scale, n, samples, p_pos=p)
    src, dst, sign = oracle.synth_rmat(1003, scale, n, samples, p_pos=p)
    np.testing.assert_array_equal(src, el.src)
    np.testing.assert_array_equal(dst, el.dst)
    np.testing.assert_array_equal(sign, el.sign)


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built here")
@pytest.mark.parametrize("family", ["er", "rmat", "delaunay", "skew"])
def test_oracle_vertex_counts_equal_reference_cnt(family):
    # The reference's per-source counts cnt[4n] (tc_serial.cpp:141-158),
    # recovered from its own count_triangles as differences of prefix counts,
    # equal the oracle's restatement vertex by vertex.
    if family == "er":
        el = synth.er(31, 1500, 12000, 0.7)
    elif family == "rmat":
        el = synth.rmat(32, 10, 1 << 10, 16 << 10)
    elif family == "delaunay":
        el = synth.delaunay(33, 1500)
    else:
        el = synth.skew(34, 1 << 11, 1 << 13, 4, 100, 600, 0.8)
    with oracle.RefKeptCSR(el.src, el.dst, el.sign) as ref:
        want = ref.vertex_counts().reshape(-1, 4)
    got = oracle.ForwardCSR(el.src, el.dst, el.sign).vertex_counts()
    np.testing.assert_array_equal(got, want)
