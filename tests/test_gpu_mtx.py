"""GPU counts from MatrixMarket input under both sign rules, through the
Python API and the `stc` CLI (which also loads the shipped dispatch model)."""
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle
import signed_triangle_counting_b200 as stc
from signed_triangle_counting_b200 import synth

pytestmark = pytest.mark.gpu
CLI = Path(__file__).resolve().parents[1] / "signed_triangle_counting_b200" / "stc"


@pytest.fixture(scope="module")
def mtx_graph(tmp_path_factory):
    el = synth.delaunay(55, 30000, 0.2, 0.6)
    rng = np.random.default_rng(8)
    w = np.where(el.sign > 0, rng.uniform(0.5, 2.0, el.m), -rng.uniform(0.5, 2.0, el.m))
    w[rng.random(el.m) < 0.1] = 0.0  # zero weights: positive or negative by rule
    body = "".join(f"{b + 1} {a + 1} {x:.3f}\n" for a, b, x in zip(el.src, el.dst, w))
    n = int(max(el.src.max(), el.dst.max())) + 1
    path = tmp_path_factory.mktemp("mtx") / "g.mtx"
    path.write_text(f"%%MatrixMarket matrix coordinate real symmetric\n{n} {n} {el.m}\n{body}")
    pos = oracle.count_arrays(el.src, el.dst, np.where(w < 0, -1, 1).astype(np.int8))
    neg = oracle.count_arrays(el.src, el.dst, np.where(w <= 0, -1, 1).astype(np.int8))
    assert pos != neg
    return path, pos, neg


def test_mtx_counts_both_rules(ctx, mtx_graph):
    path, pos, neg = mtx_graph
    assert ctx.count_edge_list(stc.load_mtx(path)).as_tuple() == pos
    assert ctx.count_edge_list(stc.load_mtx(path, zero_negative=True)).as_tuple() == neg


def _cli_counts(out):
    v = {k: int(x) for k, x in re.findall(r"(T[0-3]) \(.*?\)\s*: (\d+)", out)}
    return (v["T0"], v["T1"], v["T2"], v["T3"])


def test_cli_reads_mtx(mtx_graph):
    path, pos, neg = mtx_graph
    r = subprocess.run([str(CLI), str(path)], capture_output=True, text=True, check=True)
    assert _cli_counts(r.stdout) == pos
    r = subprocess.run([str(CLI), "--zero-negative", "--dispatch", "learned", str(path)],
                       capture_output=True, text=True, check=True)
    assert _cli_counts(r.stdout) == neg
