"""MatrixMarket input (stc_parse_mtx / stc_load_mtx): the coordinate format
the reference's GPU drivers read, both sign rules, and its error paths; the
edges must equal those of the same graph written as `u v sign` text."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle
import signed_triangle_counting_b200 as stc

ROOT = Path(__file__).resolve().parents[1]
CLI = ROOT / "signed_triangle_counting_b200" / "stc"

SYM = b"""%%MatrixMarket matrix coordinate real symmetric
% a comment
5 5 7
2 1 1.0
3 2 -2.5
3 1 0
4 4 3.0
5 4 -1e-50
5 1 1e-50
4 3 +7
"""


def edges(el):
    return sorted(zip(el.src.tolist(), el.dst.tolist(), el.sign.tolist()))


def test_symmetric_real_default_rule():
    el = stc.parse_mtx(SYM)
    assert (el.n, el.lines, el.m) == (5, 7, 6)  # the diagonal entry is dropped
    # w < 0 is negative; 0 and values that underflow float keep +1, and
    # -1e-50 reads as -0.0f, which is not below zero.
    assert edges(el) == [(0, 1, 1), (0, 2, 1), (0, 4, 1), (1, 2, -1), (2, 3, 1), (3, 4, 1)]


def test_zero_negative_rule():
    el = stc.parse_mtx(SYM, zero_negative=True)
    # w <= 0 is negative (GM/signed_tc.hxx:317), after conversion to float.
    assert edges(el) == [(0, 1, 1), (0, 2, -1), (0, 4, -1), (1, 2, -1), (2, 3, 1), (3, 4, -1)]


def test_general_pattern_and_integer():
    gen = b"%%MatrixMarket matrix coordinate pattern general\n3 3 4\n1 2\n2 1\n2 3\n3 3\n"
    el = stc.parse_mtx(gen)
    assert edges(el) == [(0, 1, 1), (0, 1, 1), (1, 2, 1)]  # both directions fold when built
    ints = b"%%MatrixMarket matrix coordinate integer general\r\n3 3 2\r\n1 3 -4\r\n3 2 0\r\n"
    assert edges(stc.parse_mtx(ints)) == [(0, 2, -1), (1, 2, 1)]


@pytest.mark.parametrize("bad", [
    b"1 2 1\n",                                                            # no banner
    b"%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n",         # array format
    b"%%MatrixMarket matrix coordinate complex general\n2 2 1\n1 2 1 0\n",  # complex field
    b"%%MatrixMarket matrix coordinate real skew-symmetric\n2 2 1\n2 1 1\n",
    b"%%MatrixMarket matrix coordinate real general\n2 2 1\n1 3 1\n",       # index out of range
    b"%%MatrixMarket matrix coordinate real general\n2 2 2\n1 2 1\n",       # fewer entries than nnz
    b"%%MatrixMarket matrix coordinate real general\n2 2 1\n1 2\n",         # missing value
])
def test_malformed_rejected(bad):
    with pytest.raises(stc.StcError):
        stc.parse_mtx(bad)


def test_same_edges_as_text_and_oracle():
    rng = np.random.default_rng(4)
    n, m = 3000, 200_000  # > 1 MB: the multi-threaded path
    i = rng.integers(1, n + 1, m)
    j = rng.integers(1, n + 1, m)
    w = np.round(rng.normal(size=m), 3)
    body = "".join(f"{a} {b} {c}\n" for a, b, c in zip(i, j, w))
    mtx = f"%%MatrixMarket matrix coordinate real general\n{n} {n} {m}\n{body}".encode()
    got = stc.parse_mtx(mtx)
    keep = i != j
    text = "".join(f"{a - 1} {b - 1} {-1 if c < 0 else 1}\n"
                   for a, b, c in zip(i[keep], j[keep], w[keep])).encode()
    want = oracle.parse_text(text)
    np.testing.assert_array_equal(got.src, want["src"])
    np.testing.assert_array_equal(got.dst, want["dst"])
    np.testing.assert_array_equal(got.sign, want["sign"])
    assert got.n == n and got.lines == m


def test_load_mtx_file_and_cli_errors(tmp_path):
    p = tmp_path / "g.mtx"
    p.write_bytes(SYM)
    assert edges(stc.load_mtx(p)) == edges(stc.parse_mtx(SYM))
    with pytest.raises(OSError):
        stc.load_mtx(tmp_path / "missing.mtx")
    bad = tmp_path / "bad.mtx"
    bad.write_bytes(b"%%MatrixMarket matrix coordinate real general\n2 2 1\n1 3 1\n")
    r = subprocess.run([str(CLI), str(bad)], capture_output=True, text=True)
    assert r.returncode == 1 and "invalid argument" in r.stderr
