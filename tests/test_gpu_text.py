"""GPU text ingest: the device parser gives the host parser's edge list (the
reference grammar, MC/graph_io.h:72-212) byte for byte, and the whole path
from text gives the reference's counts, through the API and the CLI."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle
import signed_triangle_counting_b200 as stc

pytestmark = pytest.mark.gpu
CLI = Path(__file__).resolve().parents[1] / "signed_triangle_counting_b200" / "stc"


def same_edge_list(a, b):
    assert (a.n, a.lines, a.m) == (b.n, b.lines, b.m)
    np.testing.assert_array_equal(a.src, b.src)
    np.testing.assert_array_equal(a.dst, b.dst)
    np.testing.assert_array_equal(a.sign, b.sign)


def test_fixtures_parse_and_count(ctx, golden, text_dir):
    for name in sorted(golden["text"]):
        data = (text_dir / f"{name}.txt").read_bytes()
        same_edge_list(ctx.parse_edge_text_gpu(data), stc.parse_edge_text(data))
        g = golden["text"][name]["tc_serial"]
        c, lines, n = ctx.count_text(data)
        assert c.as_tuple() == (g["t0"], g["t1"], g["t2"], g["t3"]), name
        assert (n, lines) == (g["n"], g["raw_edges"]), name


def quirky_text(seed, lines):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(lines):
        r = rng.random()
        u, v = rng.integers(0, 50000, 2)
        s = rng.choice(["1", "-1", "+1", "0", "-", "+", "0.5", "-0.5", "abc", "-7", ""])
        if r < 0.03:
            out.append("# comment %d\n" % i)
        elif r < 0.05:
            out.append("% another\r\n")
        elif r < 0.07:
            out.append("\n")
        elif r < 0.08:
            out.append("\r\n")
        elif r < 0.09:
            out.append(" %d %d %s\n" % (u, v, s))        # leading blank: first id 0
        elif r < 0.10:
            out.append("%d\t%d\t%s\r\n" % (u, v, s))
        elif r < 0.11:
            out.append("%d %d 1\n" % (u, u))              # self-loop
        elif r < 0.12:
            out.append("99999999999 %d 1\n" % v)          # wraps around uint32
        else:
            out.append("%d %d %s\n" % (u, v, s))
    return "".join(out).encode()


@pytest.mark.parametrize("seed,lines", [(1, 1000), (2, 400_000)])
def test_quirky_text_matches_host(ctx, seed, lines):
    data = quirky_text(seed, lines)
    same_edge_list(ctx.parse_edge_text_gpu(data), stc.parse_edge_text(data))
    same_edge_list(ctx.parse_edge_text_gpu(data + b"5 6 -1"), stc.parse_edge_text(data + b"5 6 -1"))


def test_count_text_matches_oracle(ctx):
    data = quirky_text(3, 200_000)
    ref = oracle.parse_text(data)
    c, lines, n = ctx.count_text(data)
    assert c.as_tuple() == oracle.count_arrays(ref["src"], ref["dst"], ref["sign"])
    assert (lines, n) == (ref["lines"], ref["n"])


@pytest.mark.parametrize("flags", [[], ["--host-ingest"]])
def test_cli_both_ingests(golden, text_dir, flags):
    for name in sorted(golden["text"]):
        r = subprocess.run([str(CLI), *flags, str(text_dir / f"{name}.txt")], capture_output=True,
                           text=True)
        assert r.returncode == 0, (name, r.stderr)
        got = oracle.parse_program_output(r.stdout)
        s = golden["text"][name]["tc_serial"]
        for k in ("n", "raw_edges", "forward_edges", "t0", "t1", "t2", "t3"):
            assert got[k] == s[k], (name, k, flags)
