"""Generates the golden fixtures under tests/golden/ from the reference itself.

The reference ships no test vectors, so the fixtures are produced by running
the reference's own CPU code, compiled unchanged from its sources by
oracle/Makefile into oracle/_ref/ (this needs the reference sources, i.e. the
machine where the repository is developed):

  text/*.txt       small `u v sign` files: grammar edge cases and seeded graphs
  golden.json      "text": per file, the parsed outputs of the four reference
                   programs (tc_serial, tc_merge_sign_enu, tc_hash_sign_enu,
                   tc_merge_sign_split), which must agree with each other;
                   "workloads": per-type counts of the seeded workloads from
                   the in-memory harness around tc_serial.cpp, at reduced
                   ("shrink") and full size;
                   "batch": per-graph counts of the 4,096-graph workload.

    python tests/golden/make_golden.py            # text + shrunken workloads
    python tests/golden/make_golden.py --full     # + full-size workloads
    OMP_NUM_THREADS=1 python tests/golden/make_golden.py --batch   # + the batch
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys
import time
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from signed_triangle_counting_b200 import synth  # noqa: E402

HERE = Path(__file__).resolve().parent
TEXT = HERE / "text"
GOLDEN = HERE / "golden.json"

# Grammar and structure edge cases (no self-loops, no MatrixMarket size line,
# no duplicates with conflicting signs: outside the reference's defined
# behaviour, MC/graph_io.h:147,191-192,244,251-256).
EDGE_CASES = {
    "empty": b"",
    "comments_only": b"# a comment\n% another\n",
    "triangle_ppp": b"0 1 1\n1 2 1\n0 2 1\n",
    "triangle_ppm": b"0 1 1\n1 2 1\n0 2 -1\n",
    "triangle_pmm": b"0 1 -1\n1 2 1\n0 2 -1\n",
    "triangle_mmm": b"0 1 -1\n1 2 -1\n0 2 -1\n",
    "k4_mixed": b"0 1 1\n0 2 -1\n0 3 1\n1 2 1\n1 3 -1\n2 3 -1\n",
    "reversed_duplicates": b"1 2 1\n2 1 1\n2 3 -1\n3 2 -1\n1 3 1\n3 1 1\n1 2 1\n",
    "crlf": b"0 1 1\r\n1 2 -1\r\n2 0 1\r\n2 3 1\r\n3 0 -1\r\n",
    "sign_tokens": (b"0 1 +1\n1 2 0\n2 0 0.5\n2 3 -1\n3 0 -0.5\n3 1 -\n0 4 +\n4 1\n"
                    b"4 2 abc\n4 3 -7\n"),
    # A whitespace-only line parses as the self-loop "0 0" (graph_io.h:183-192),
    # so blank lines here are truly empty (or a lone '\r').
    "blanks_tabs": b"\n\n0\t1\t1\n\n1  2   -1\n\r\n2 0 1\n\n",
    "leading_space": b" 1 2 1\n1 2 1\n0 2 -1\n",
    "no_trailing_newline": b"0 1 1\n1 2 1\n2 0 -1",
    "comment_lines_mixed": b"% header\n0 1 1\n# mid\n1 2 -1\n2 0 -1\n%tail\n",
    "star": b"".join(b"0 %d %d\n" % (i, 1 if i % 3 else -1) for i in range(1, 40)),
    "sparse_ids": b"1000000 5 1\n5 77 -1\n77 1000000 1\n77 300000 1\n300000 5 -1\n",
}


def clique_text(k: int, seed: int) -> bytes:
    rng = np.random.default_rng(seed)
    lines = []
    for a in range(k):
        for b in range(a + 1, k):
            s = 1 if rng.random() < 0.5 else -1
            lines.append(b"%d %d %d\n" % ((a, b, s) if rng.random() < 0.5 else (b, a, s)))
    return b"".join(lines)


def graph_text(el, shuffle_seed: int | None = None) -> bytes:
    idx = np.arange(el.m)
    if shuffle_seed is not None:
        np.random.default_rng(shuffle_seed).shuffle(idx)
    rows = np.stack([el.src[idx].astype(np.int64), el.dst[idx].astype(np.int64),
                     el.sign[idx].astype(np.int64)], axis=1)
    return "".join(f"{a} {b} {s}\n" for a, b, s in rows.tolist()).encode()


def seeded_texts() -> dict:
    out = {}
    out["clique20"] = clique_text(20, 7)
    out["er_1000_8000"] = graph_text(synth.er(11, 1000, 8000, 0.7))
    out["rmat_s10"] = graph_text(synth.rmat(12, 10, 1 << 10, 16 << 10, p_pos=0.5))
    out["delaunay_2000"] = graph_text(synth.delaunay(13, 2000, 0.2, 0.6))
    out["skew_small"] = graph_text(synth.skew(14, 4096, 12000, 4, 200, 2000, 0.8))
    out["workload1"] = graph_text(synth.workload(1))
    return out


def run_programs(path: Path) -> dict:
    res = {}
    for prog in oracle.REF_PROGRAMS:
        r = oracle.run_ref_program(prog, path, threads=4)
        res[prog] = {k: v for k, v in r.items() if k != "stdout" and not k.endswith("_s")}
    serial = res["tc_serial"]
    bal, unb = serial["t1"] + serial["t3"], serial["t0"] + serial["t2"]
    for prog in ("tc_merge_sign_enu", "tc_hash_sign_enu", "tc_merge_sign_split"):
        assert (res[prog]["balanced"], res[prog]["unbalanced"]) == (bal, unb), (path, prog, res)
    return res


def counts_digest(rows) -> str:
    h = hashlib.sha256()
    for r in rows:
        h.update(np.asarray(r, dtype=np.uint64).tobytes())
    return h.hexdigest()


def workload_entry(k: int, shrink: int) -> dict:
    t0 = time.time()
    el = synth.workload(k, shrink)
    tg = time.time() - t0
    t, sec = oracle.ref_count_arrays(el.src, el.dst, el.sign)
    print(f"workload {k} shrink {shrink}: n={el.n} m={el.m} gen {tg:.1f}s ref {sum(sec):.1f}s {t}",
          flush=True)
    return dict(workload=k, shrink=shrink, n=el.n, m_input=el.m, t=list(map(int, t)),
                ref_seconds=[round(x, 3) for x in sec])


def batch_entry(G: int, threads: int) -> dict:
    specs = synth.batch_specs(G)
    synth.set_threads(1)

    def one(i):
        el = synth.batch_graph(specs[i])
        t, _ = oracle.ref_count_arrays(el.src, el.dst, el.sign)
        return i, el.m, list(map(int, t))

    rows = [None] * G
    ms = [0] * G
    t0 = time.time()
    with ThreadPoolExecutor(threads) as ex:
        for i, m, t in ex.map(one, range(G)):
            rows[i] = t
            ms[i] = m
            if i % 256 == 0:
                print(f"batch graph {i}/{G} ({time.time() - t0:.0f}s)", flush=True)
    synth.set_threads(0)
    return dict(G=G, m_input=ms, t=rows, digest=counts_digest(rows))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--full", action="store_true")
    ap.add_argument("--batch", action="store_true")
    ap.add_argument("--batch-threads", type=int, default=os.cpu_count())
    a = ap.parse_args()
    if not oracle.ref_available():
        oracle.build()
    assert oracle.ref_available(), "oracle/_ref is missing: the reference sources are needed"
    golden = json.loads(GOLDEN.read_text()) if GOLDEN.exists() else {}

    if a.batch and not a.full:
        golden["batch"] = batch_entry(4096, a.batch_threads)
        GOLDEN.write_text(json.dumps(golden, indent=1))
        print("wrote", GOLDEN)
        return
    TEXT.mkdir(exist_ok=True)
    texts = dict(EDGE_CASES)
    texts.update(seeded_texts())
    golden["text"] = {}
    for name, data in texts.items():
        p = TEXT / f"{name}.txt"
        p.write_bytes(data)
        golden["text"][name] = run_programs(p)
    print(f"{len(texts)} text fixtures", flush=True)

    wl = dict(golden.get("workloads", {}))
    for k, shrinks in ((1, [0]), (2, [6, 3]), (3, [10, 8, 6]), (5, [10, 8])):
        for s in shrinks:
            wl[f"{k}/{s}"] = workload_entry(k, s)
    if a.full:
        for k in (2, 5, 3):
            wl[f"{k}/0"] = workload_entry(k, 0)
            golden["workloads"] = wl
            GOLDEN.write_text(json.dumps(golden, indent=1))
    golden["workloads"] = wl
    if a.batch:
        golden["batch"] = batch_entry(4096, a.batch_threads)
    GOLDEN.write_text(json.dumps(golden, indent=1))
    print("wrote", GOLDEN)


if __name__ == "__main__":
    main()
