"""Host-side checks that need no GPU: the C ABI library loads and exports what
include/*.h declares, the host text parser matches the oracle byte for byte,
the seeded generators have the properties the workloads promise, and the CLI's
error paths behave like the reference programs'."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle
import signed_triangle_counting_b200 as stc
from signed_triangle_counting_b200 import _capi, synth

ROOT = Path(__file__).resolve().parents[1]
CLI = ROOT / "signed_triangle_counting_b200" / "stc"


def declared_functions():
    names = set()
    for h in sorted((ROOT / "include").glob("*.h")):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for line in text.splitlines():
            if line.lstrip().startswith("static"):
                continue
            m = re.match(r"^\s*[A-Za-z_][\w\s\*]*?\b(stc_\w+)\s*\(", line)
            if m:
                names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    lib = _capi.lib()
    names = declared_functions()
    assert len(names) >= 25
    out = subprocess.run(["nm", "-D", "--defined-only", str(_capi.LIB_PATH)], capture_output=True,
                         text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if ln.strip()}
    missing = sorted(n for n in names if n not in exported)
    assert not missing, missing
    for n in names:
        getattr(lib, n)
    # and the ctypes table covers the header
    assert {s[0] for s in _capi.SIGNATURES} == names


def test_status_strings_and_abi_version():
    lib = _capi.lib()
    assert lib.stc_abi_version() == 2
    for s in range(0, 9):
        assert lib.stc_status_string(s)
    assert lib.stc_status_string(0) == b"ok"


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device path")
def test_context_without_device_reports_no_device():
    h = C.c_void_p()
    assert _capi.lib().stc_ctx_create(0, C.byref(h)) == _capi.STC_ERR_NO_DEVICE
    with pytest.raises(stc.StcError):
        stc.Context(0)


def test_null_arguments_are_rejected():
    lib = _capi.lib()
    out = _capi.stc_counts()
    assert lib.stc_count(None, None, None, None, 0, None, C.byref(out)) == 1
    assert lib.stc_load_edge_list(None, None) == 1
    el = _capi.stc_edge_list()
    assert lib.stc_load_edge_list(b"/nonexistent/graph.txt", C.byref(el)) == _capi.STC_ERR_IO


def test_host_parser_matches_oracle(golden, text_dir):
    for name in sorted(golden["text"]):
        path = text_dir / f"{name}.txt"
        mine = stc.load_graph(path)
        ref = oracle.load_graph(path)
        assert (mine.n, mine.lines, mine.m) == (ref["n"], ref["lines"], ref["m"]), name
        np.testing.assert_array_equal(mine.src, ref["src"])
        np.testing.assert_array_equal(mine.dst, ref["dst"])
        np.testing.assert_array_equal(mine.sign, ref["sign"])
        g = golden["text"][name]["tc_serial"]
        assert (mine.n, mine.lines) == (g["n"], g["raw_edges"]), name


def test_host_parser_large_buffer_threads():
    # Large enough for the multi-threaded path; includes self-loops and comments
    # that must vanish without leaving holes.
    rng = np.random.default_rng(3)
    n = 300_000
    u = rng.integers(0, 5000, n)
    v = rng.integers(0, 5000, n)
    s = np.where(rng.random(n) < 0.5, 1, -1)
    lines = []
    for i in range(n):
        if i % 1000 == 0:
            lines.append("# comment\n")
        lines.append(f"{u[i]} {v[i]} {s[i]}\n")
    data = "".join(lines).encode()
    mine = stc.parse_edge_text(data)
    ref = oracle.parse_text(data)
    assert (mine.n, mine.lines, mine.m) == (ref["n"], ref["lines"], ref["m"])
    assert mine.m < mine.lines  # self-loops were dropped
    np.testing.assert_array_equal(mine.src, ref["src"])
    np.testing.assert_array_equal(mine.dst, ref["dst"])
    np.testing.assert_array_equal(mine.sign, ref["sign"])


# ---------------------------------------------------------------- generators
def _canon(el):
    lo = np.minimum(el.src, el.dst).astype(np.uint64)
    hi = np.maximum(el.src, el.dst).astype(np.uint64)
    return (lo << np.uint64(32)) | hi


@pytest.mark.parametrize("k,shrink", [(1, 0), (2, 6), (3, 10), (5, 10)])
def test_workloads_deterministic_and_clean(k, shrink):
    a = synth.workload(k, shrink)
    synth.set_threads(3)
    b = synth.workload(k, shrink)
    synth.set_threads(0)
    for f in ("src", "dst", "sign"):
        np.testing.assert_array_equal(getattr(a, f), getattr(b, f))
    assert (a.src != a.dst).all()
    assert a.src.max() < a.n and a.dst.max() < a.n
    assert set(np.unique(a.sign).tolist()) <= {-1, 1}
    key = _canon(a)
    order = np.argsort(key, kind="stable")
    ks, ss = key[order], a.sign[order]
    same = ks[1:] == ks[:-1]
    assert (ss[1:][same] == ss[:-1][same]).all(), "duplicates with conflicting signs"


def test_er_is_distinct_and_sized():
    el = synth.workload(1)
    assert el.m == 100_000 and el.n == 10_000
    assert len(np.unique(_canon(el))) == el.m
    frac = (el.sign > 0).mean()
    assert 0.68 < frac < 0.72


def test_rmat_degree_skew():
    el = synth.rmat(9, 16, 1 << 16, 16 << 16)
    deg = np.bincount(np.concatenate([el.src, el.dst]), minlength=1 << 16)
    assert deg.max() > 50 * deg.mean()


# numpy restatement of stc_gen.h, to rebuild the Delaunay input points.
_M = np.uint64(0xFFFFFFFFFFFFFFFF)


def _mix64(z):
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def _draw(seed, stream, i):
    with np.errstate(over="ignore"):
        key = _mix64(np.uint64(seed) ^ _mix64(np.uint64(stream) * np.uint64(0xD1B54A32D192ED03)
                                              + np.uint64(0x632BE59BD9B4E019)))
        return _mix64(key + (np.asarray(i, np.uint64) + np.uint64(1)) * np.uint64(0x9E3779B97F4A7C15))


def _perm(seed, n, x):
    bits = 0
    while (1 << bits) < n:
        bits += 1
    h = max(1, (bits + 1) // 2)
    keys = [_draw(seed, 1, r) for r in range(4)]
    mask = np.uint64((1 << h) - 1)
    x = np.asarray(x, np.uint64).copy()
    todo = np.ones(len(x), bool)
    while todo.any():
        y = x[todo]
        L, R = y >> np.uint64(h), y & mask
        for r in range(4):
            F = _mix64(R ^ keys[r]) & mask
            L, R = R, L ^ F
        y = (L << np.uint64(h)) | R
        x[todo] = y
        todo[todo] = y >= np.uint64(n)
    return x


def test_delaunay_matches_scipy():
    spatial = pytest.importorskip("scipy.spatial")
    seed, n = 77, 20_000
    el = synth.delaunay(seed, n, 0.0, 0.6)
    i = np.arange(n, dtype=np.uint64)
    x = (_draw(seed, 7, 2 * i) >> np.uint64(36)).astype(np.float64)
    y = (_draw(seed, 7, 2 * i + np.uint64(1)) >> np.uint64(36)).astype(np.float64)
    tri = spatial.Delaunay(np.stack([x, y], 1))
    s = tri.simplices
    e = np.concatenate([s[:, [0, 1]], s[:, [1, 2]], s[:, [0, 2]]])
    p = _perm(seed, n, np.arange(n))
    a, b = p[e[:, 0]], p[e[:, 1]]
    want = np.unique((np.minimum(a, b) << np.uint64(32)) | np.maximum(a, b))
    got = np.unique(_canon(el))
    assert len(got) == el.m
    np.testing.assert_array_equal(got, want)


def test_delaunay_deletion_fraction():
    full = synth.delaunay(5, 50_000, 0.0, 0.6)
    cut = synth.delaunay(5, 50_000, 0.2, 0.6)
    assert 0.78 < cut.m / full.m < 0.82


def test_batch_specs_distribution():
    specs = synth.batch_specs(4096)
    ns = np.array([s["n"] for s in specs])
    kinds = np.bincount([s["kind"] for s in specs], minlength=3)
    ps = np.array([s["p_pos"] for s in specs])
    assert ns.min() >= 1000 and ns.max() <= 1_000_000
    assert 0.4 < np.mean(np.log10(ns) < 4.5) < 0.6  # log-uniform: median near 10^4.5
    assert kinds.min() > 1200
    assert ps.min() >= 0.3 and ps.max() <= 0.9
    assert specs == synth.batch_specs(4096)


# ---------------------------------------------------------------------- CLI
def test_cli_usage_error():
    r = subprocess.run([str(CLI)], capture_output=True, text=True)
    assert r.returncode == 1
    assert "usage:" in r.stderr


def test_cli_missing_file():
    r = subprocess.run([str(CLI), "/nonexistent/g.txt"], capture_output=True, text=True)
    assert r.returncode == 1
    assert "/nonexistent/g.txt" in r.stderr


def test_batch_packed_generator_matches_single_graphs():
    specs = synth.batch_specs(64)
    el, offs = synth.batch_packed(specs, 10, 22)
    assert len(offs) == 13 and offs[0] == 0 and offs[-1] == el.m
    for i, g in enumerate(range(10, 22)):
        one = synth.batch_graph(specs[g])
        a, b = int(offs[i]), int(offs[i + 1])
        np.testing.assert_array_equal(el.src[a:b], one.src)
        np.testing.assert_array_equal(el.dst[a:b], one.dst)
        np.testing.assert_array_equal(el.sign[a:b], one.sign)
