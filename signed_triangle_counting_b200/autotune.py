"""Autotuner driver: tunes the staged classes' launch parameters (block-class
CTA threads, hash buckets per element, stream width) per workload with
``stc_autotune`` and keeps the results in a JSON file, one entry per
workload (the shipped file is ``tuning.json`` beside this module).

Each workload is tuned on a smaller instance of itself: RMAT scale 22 for the
scale-24 power-law graph, the first 512 graphs of the 4,096-graph batch, the
skew graph at a quarter of its size, the Delaunay mesh and the ER graph as
they are.

    python -m signed_triangle_counting_b200.autotune [--workloads 2 3 4 5] [--out PATH]
"""
from __future__ import annotations

import argparse
import json
import time
from pathlib import Path

import numpy as np

from . import synth

DEFAULT_TUNING = Path(__file__).resolve().parent / "tuning.json"
FORMAT_VERSION = 1
KEYS = ("block_threads", "hash_factor", "unroll")


def tuning_graph(workload: int):
    """The instance a workload is tuned on, as (src, dst, sign, description)."""
    if workload == 3:
        el = synth.rmat(synth.workload_seed(3) + 1, 22, 1 << 22, 16 << 22, p_pos=0.5)
        return el.src, el.dst, el.sign, "RMAT scale 22 (seed + 1)"
    if workload == 4:
        from .dispatcher import union
        specs = synth.batch_specs(4096)
        el, offs = synth.batch_packed(specs, 0, 512)
        s, d, g = union(el, offs, [x["n"] for x in specs[:512]])
        return s, d, g, "batch graphs 0..511 as one union"
    if workload == 5:
        el = synth.workload(5, 2)
        return el.src, el.dst, el.sign, "skew at shrink 2"
    el = synth.workload(workload)
    return el.src, el.dst, el.sign, f"workload {workload}"


def validate(t: dict) -> dict:
    if (t["block_threads"] not in (128, 256, 512) or len(t["hash_factor"]) != 3
            or len(t["unroll"]) != 3 or any(h not in (2, 4, 8) for h in t["hash_factor"])
            or any(u not in (1, 2, 4) for u in t["unroll"])):
        raise ValueError(f"invalid tuning {t}")
    return {k: t[k] for k in KEYS}


def save(path, entries: dict) -> None:
    doc = {"format": FORMAT_VERSION, "kind": "stc-tuning", "workloads": entries}
    Path(path).write_text(json.dumps(doc, indent=1) + "\n")


def load(path=None) -> dict:
    """Per-workload entries {"3": {"tuning": {...}, ...}, ...} of a tuning file."""
    doc = json.loads(Path(path or DEFAULT_TUNING).read_text())
    if doc.get("format") != FORMAT_VERSION or doc.get("kind") != "stc-tuning":
        raise ValueError(f"{path or DEFAULT_TUNING}: not a tuning file of format {FORMAT_VERSION}")
    for e in doc["workloads"].values():
        validate(e["tuning"])
    return doc["workloads"]


def tuning_for(workload: int, path=None):
    """The stored tuning of a workload, or None."""
    p = Path(path or DEFAULT_TUNING)
    if not p.exists():
        return None
    e = load(p).get(str(workload))
    return e["tuning"] if e else None


def _main() -> None:
    from . import Context
    ap = argparse.ArgumentParser(prog="python -m signed_triangle_counting_b200.autotune")
    ap.add_argument("--workloads", type=int, nargs="+", default=[2, 3, 4, 5])
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--out", default=str(DEFAULT_TUNING))
    a = ap.parse_args()
    import torch
    gpu = torch.cuda.get_device_name(0) if torch.cuda.is_available() else "?"
    ctx = Context(0)
    out = load(a.out) if Path(a.out).exists() else {}
    for w in a.workloads:
        s, d, g, desc = tuning_graph(w)
        ctx.set_tuning(None)
        t0 = time.time()
        t = ctx.autotune(s, d, g, reps=a.reps)
        out[str(w)] = {"tuning": t, "tuned_on": desc, "gpu": gpu, "reps": a.reps,
                       "seconds": round(time.time() - t0, 1)}
        print(json.dumps({"workload": w, **out[str(w)]}), flush=True)
    save(a.out, out)


if __name__ == "__main__":
    _main()
