"""ORACLE — test infrastructure, not product code.

Times the reference's own CPU programs at full size on the five workloads,
on the host this runs on, for the CPU-baseline table: the unchanged
tc_merge_sign_enu and tc_hash_sign_enu ("Signed_TC/Multicore
Implementations/", compiled by oracle/Makefile into oracle/_ref/) on text
files of workloads 1, 2, 3 and 5, with OpenMP on all host threads; workload
4 (4,096 graphs, about 50 GB as text) through the in-memory harness around
tc_serial.cpp instead.  For the power-law workload it also checks the bench's
sampled CPU rate against a full count: the harness's count_triangles over
all sources versus its time on the 1/64 id sample, scaled by merge work.

    python -m oracle.cpu_table [--workloads 1,2,3,5,4] [--out table.json] [--tmp DIR]

Prints one JSON object per workload and the host description (nproc, the
lscpu model name).  Inputs come from the package's seeded generators (the
reference ships no datasets).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402


def host() -> dict:
    model = ""
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True).stdout
        for ln in out.splitlines():
            if ln.startswith("Model name:"):
                model = ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return {"nproc": os.cpu_count(), "lscpu_model": model,
            "omp_threads": os.environ.get("OMP_NUM_THREADS", "all")}


def run_programs(name: str, src, dst, sign, tmp: Path) -> dict:
    path = tmp / f"{name}.txt"
    t0 = time.perf_counter()
    oracle.write_edge_text(path, src, dst, sign)
    row = {"workload": name, "m_input": int(len(src)), "text_bytes": path.stat().st_size,
           "write_s": time.perf_counter() - t0}
    try:
        for prog in ("tc_merge_sign_enu", "tc_hash_sign_enu"):
            r = oracle.run_ref_program(prog, path)
            row[prog] = {k: r.get(k) for k in ("count_s", "build_s", "total_s", "balanced",
                                               "unbalanced")}
            print(json.dumps({"progress": name, "program": prog, **row[prog]}), flush=True)
    finally:
        path.unlink(missing_ok=True)
    return row


def rmat_projection(scale: int = 24, div: int = 64) -> dict:
    """The bench's sample (sources with id < n / div) against a full count of
    the same kept CSR."""
    src, dst, sign = oracle.synth_rmat(1003, scale, 1 << scale, 16 << scale)
    with oracle.RefKeptCSR(src, dst, sign) as k:
        del src, dst, sign
        n_s = k.n // div
        arcs_s, work_s = k.prefix_size(n_s)
        arcs, work = k.prefix_size(k.n)
        _, t_s = k.count_prefix(n_s)
        full_counts, t_full = k.count_prefix(k.n)
        return {"edges": arcs, "build_s": k.build_s, "sort_s": k.sort_s,
                "count_s_full": t_full, "sample_count_s": t_s, "sample_edges": arcs_s,
                "count_s_projected": t_s * work / work_s, "counts": list(full_counts),
                "threads": k.threads}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--workloads", default="1,2,3,5,4")
    ap.add_argument("--out", default=None)
    ap.add_argument("--tmp", default=None)
    a = ap.parse_args()
    if not oracle.ref_available():
        raise SystemExit("oracle/_ref is missing: build it from the reference sources first")
    from signed_triangle_counting_b200 import synth
    res = {"host": host(), "rows": []}
    print(json.dumps(res["host"]), flush=True)
    tmp = Path(a.tmp or tempfile.mkdtemp(prefix="stc_cpu_table_"))
    for w in [int(x) for x in a.workloads.split(",")]:
        if w == 4:
            specs = synth.batch_specs(4096)
            row = {"workload": "4", "graphs": len(specs), "m_input": 0, "m_unique": 0,
                   "build_s": 0.0, "sort_s": 0.0, "count_s": 0.0}
            for g0 in range(0, len(specs), 256):
                el, offs = synth.batch_packed(specs, g0, min(len(specs), g0 + 256))
                for g in range(len(offs) - 1):
                    b, e = int(offs[g]), int(offs[g + 1])
                    _, sec, fe = oracle.ref_count_arrays(el.src[b:e], el.dst[b:e], el.sign[b:e],
                                                         with_edges=True)
                    row["build_s"] += sec[0]
                    row["sort_s"] += sec[1]
                    row["count_s"] += sec[2]
                    row["m_input"] += e - b
                    row["m_unique"] += fe
                print(json.dumps({"progress": "4", "graphs_done": min(len(specs), g0 + 256)}),
                      flush=True)
            row["program"] = "tc_serial.cpp via the in-memory harness, one graph at a time"
        else:
            el = synth.workload(w)
            row = run_programs(str(w), el.src, el.dst, el.sign, tmp)
            del el
            if w == 3:
                row["sample_check"] = rmat_projection()
        res["rows"].append(row)
        print(json.dumps(row), flush=True)
        if a.out:
            Path(a.out).write_text(json.dumps(res, indent=1) + "\n")


if __name__ == "__main__":
    main()
