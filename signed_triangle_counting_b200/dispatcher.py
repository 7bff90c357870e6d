"""Learned dispatcher: training data from the counter's own timings, training
on the device, model files, and regret against exhaustive per-cell timing.

The reference runs one intersection strategy per program (merge in
"Signed_TC/Multicore Implementations/tc_merge_sign_enu.cpp:12-44", hash in
"tc_hash_sign_enu.cpp:125-165"); this engine picks one per dispatch cell
(class of u's list, bucket |A'|, bucket |B|): MERGE, HASH, SEARCH and SPLIT
on the tail side, HEAD (A' streamed through the head's staged list) on the
head side.  All strategies give the same counts, so a dispatch table
changes only speed.

* ``record`` runs the timing recorder once per forced strategy: exhaustive
  per-cell timing of one graph (HEAD applies only to cells with |B| <= 4095;
  elsewhere its forced run times HASH, so its cost there is unavailable).
* ``samples`` turns a recording into training rows: the cell's features, the
  measured log2 cycles per arc of each strategy as targets, and a weight that
  grows with the cell's number of arcs.
* ``train`` fits the perceptron on the device (``stc_dispatcher_train``).
* ``regret`` scores any table against a recording: the time it would spend
  divided by the time of the per-cell best choice (1.0 = no regret).

    python -m signed_triangle_counting_b200.dispatcher train [--out PATH]
    python -m signed_triangle_counting_b200.dispatcher evaluate [--model PATH]
"""
from __future__ import annotations

import argparse
import json
import time
from pathlib import Path

import numpy as np

from . import _capi, dispatch_features, synth

STRATEGIES = ("merge", "hash", "search", "split", "head")  # output k is strategy code k + 1
STAGED_ONLY = (1, 3)  # outputs (HASH, SPLIT) that need the staged hash
SPLIT, HEAD = 3, 4    # outputs of the SPLIT and HEAD strategies
HEAD_MAX_BUCKET = 12  # HEAD applies to cells whose bucket |B| is at most this
GIANT = 3                                  # class index whose lists stage no hash
DEFAULT_STRATEGIES = ("merge", "hash", "search", "head")  # what the shipped model chooses from
DEFAULT_MODEL = Path(__file__).resolve().parent / "dispatch_model.json"
FORMAT_VERSION = 4


def record(ctx, src, dst, sign) -> dict:
    """Per-cell cycles of every strategy on one graph (one timed run per
    strategy).

    Returns {"cycles": (5, CELLS) float64, "arcs": (CELLS,) float64,
    "counts": GlobalTriCounts}; raises if the strategies disagree on the
    counts or on which arcs they timed."""
    cycles, arcs, counts = [], None, None
    for s in STRATEGIES:
        cy, ar, c = ctx.record_bucket_times(src, dst, sign, strategy=s)
        if counts is None:
            counts, arcs = c, ar
        elif c != counts or not np.array_equal(ar, arcs):
            raise RuntimeError(f"strategy {s} disagrees: {c} vs {counts}")
        cycles.append(cy.astype(np.float64))
    return {"cycles": np.stack(cycles), "arcs": arcs.astype(np.float64), "counts": counts}


def merge(records) -> dict:
    """Sums recordings of several graphs (cycles and arcs per cell)."""
    return {"cycles": sum(r["cycles"] for r in records), "arcs": sum(r["arcs"] for r in records)}


def cell_costs(rec) -> np.ndarray:
    """Mean cycles per arc, (5, CELLS); HASH and SPLIT are unavailable in the
    giant class (its arcs run MERGE), and HEAD in cells with bucket |B| > 12,
    so they cost infinity there; empty cells cost 0."""
    arcs = rec["arcs"]
    cost = np.divide(rec["cycles"], np.maximum(arcs, 1.0)[None, :])
    for k in STAGED_ONLY:
        cost[k, GIANT * 256:(GIANT + 1) * 256] = np.inf
    cost[HEAD, (np.arange(cost.shape[1]) & 15) > HEAD_MAX_BUCKET] = np.inf
    return cost


def samples(rec, min_arcs: int = 32, weight_power: float = 0.5):
    """Training rows of a recording: (features, targets, weights, cells).

    Only cells with at least ``min_arcs`` arcs are kept.  Targets = measured
    log2 cycles per arc of each strategy (NaN where unavailable); weight =
    arcs ** ``weight_power``, normalised to sum 1 (0.5 keeps the busiest
    cells first without letting a handful of them decide alone)."""
    arcs = rec["arcs"]
    cost = cell_costs(rec)
    cells = np.nonzero(arcs >= min_arcs)[0]
    c = cost[:, cells].T
    with np.errstate(divide="ignore"):
        targets = np.where(np.isfinite(c) & (c > 0), np.log2(np.where(c > 0, c, 1.0)), np.nan)
    w = arcs[cells] ** weight_power
    w = w / w.sum() if w.sum() > 0 else w
    X = dispatch_features()[cells]
    return X, targets.astype(np.float32), w.astype(np.float32), cells


def regret(rec, tables, strategies=DEFAULT_STRATEGIES) -> dict:
    """Cycles a dispatch table would spend on a recording, relative to the
    per-cell best of ``strategies`` (by default the four the shipped model
    chooses from).  ``tables``: strategy codes, (4, 16, 16) or flat."""
    t = np.asarray(tables).reshape(-1).astype(np.int64)
    arcs = rec["arcs"]
    cost = cell_costs(rec)
    best_cost = cost.copy()
    for k, name in enumerate(STRATEGIES):
        if name not in strategies:
            best_cost[k] = np.inf
    k = t - 1
    # The giant class runs MERGE where a table says HASH or SPLIT; a HEAD
    # cell beyond bucket |B| 12 runs HASH (MERGE in the giant class).
    giant = np.arange(len(t)) // 256 == GIANT
    k = np.where((k == HEAD) & ((np.arange(len(t)) & 15) > HEAD_MAX_BUCKET), 1, k)
    k = np.where(giant & np.isin(k, STAGED_ONLY), 0, k)
    used = arcs > 0
    chosen = cost[k, np.arange(len(t))]
    spent = float((arcs * np.where(used, chosen, 0.0)).sum())
    best = float((arcs * np.where(used, best_cost.min(axis=0), 0.0)).sum())
    return {"cycles": spent, "best_cycles": best, "ratio": spent / best if best else 1.0}


# Output bias that keeps a strategy out of every table (its predicted log2
# cost can never be the least).
EXCLUDED_BIAS = 1e30


def train(ctx, rec, *, epochs: int = 3000, lr: float = 0.02, weight_decay: float = 1e-3,
          seed: int = 1, min_arcs: int = 32, weight_power: float = 0.5, use_split: bool = False):
    """Trains on a recording and loads the model into ``ctx``; returns
    (params, info).  ``weighted_accuracy``: the weight of the training cells
    whose table entry is their measured fastest strategy.

    SPLIT is left out unless ``use_split``: the per-arc recorder measures it
    5-17% cheaper than HASH, but counted in the packed stream (forced on
    RMAT-24: 407.4 vs 406.1 ms) it gains nothing, and any table that uses it
    also pays for building the sign-split heads.  Left out, its targets are
    dropped and its output bias is set to EXCLUDED_BIAS."""
    X, T, w, cells = samples(rec, min_arcs, weight_power)
    if not use_split:
        T = T.copy()
        T[:, SPLIT] = np.nan
    params, loss = ctx.train_dispatcher(X, T, w, epochs=epochs, lr=lr, weight_decay=weight_decay,
                                        seed=seed)
    if not use_split:
        params = params.copy()
        params[len(params) - len(STRATEGIES) + SPLIT] = EXCLUDED_BIAS
    # The model overrides the fixed tables only on the cells its training
    # data covered.
    ctx.set_dispatch_model(params, cells)
    pred = ctx.dispatch_tables("learned").reshape(-1)[cells].astype(np.int64) - 1
    best = np.argmin(np.where(np.isnan(T), np.inf, T), axis=1)  # among the trained strategies
    acc = float((w * (pred == best)).sum())
    info = {"samples": int(len(cells)), "support": [int(c) for c in cells], "loss": loss,
            "weighted_accuracy": acc,
            "strategies": list(STRATEGIES if use_split else DEFAULT_STRATEGIES),
            "objective": "log2 cycles per arc, weighted squared error", "epochs": epochs,
            "lr": lr, "weight_decay": weight_decay, "seed": seed, "min_arcs": min_arcs,
            "weight_power": weight_power}
    return params, info


def save(path, params, meta: dict) -> None:
    doc = {"format": FORMAT_VERSION, "kind": "stc-dispatch-mlp",
           "layout": "W1[16][6], b1[16], W2[5][16], b2[5]; outputs: log2 cycles per arc "
                     "of merge, hash, search, split, head",
           "params": [float(x) for x in np.asarray(params, np.float32)]}
    doc.update(meta)
    Path(path).write_text(json.dumps(doc, indent=1) + "\n")


def load(path=None) -> dict:
    """Reads a model file; ``params`` comes back as a float32 array."""
    doc = json.loads(Path(path or DEFAULT_MODEL).read_text())
    if doc.get("format") != FORMAT_VERSION or doc.get("kind") != "stc-dispatch-mlp":
        raise ValueError(f"{path or DEFAULT_MODEL}: not a dispatch model of format {FORMAT_VERSION}")
    p = np.asarray(doc["params"], np.float32)
    if p.shape != (_capi.DISPATCH_MODEL_PARAMS,):
        raise ValueError("wrong number of model parameters")
    doc["params"] = p
    return doc


def union(el, offsets, ns):
    """One graph from graphs stored back to back (ids local to each graph):
    graph g's ids are shifted by the vertex counts of the graphs before it."""
    offsets = np.asarray(offsets, np.int64)
    vbase = np.concatenate([[0], np.cumsum(np.asarray(ns, np.int64))[:-1]])
    shift = np.repeat(vbase, np.diff(offsets)).astype(np.uint32)
    return el.src + shift, el.dst + shift, el.sign


def training_graphs(batch_graphs: int = 4096, group: int = 512):
    """The training inputs: the Delaunay mesh (1M points, 20% deleted) and
    the first ``batch_graphs`` graphs of the 4,096-graph batch, recorded as
    unions of ``group`` graphs."""
    d = synth.workload(2)
    yield "workload2", (d.src, d.dst, d.sign)
    del d
    specs = synth.batch_specs(4096)
    for g0 in range(0, batch_graphs, group):
        g1 = min(batch_graphs, g0 + group)
        el, offs = synth.batch_packed(specs, g0, g1)
        yield f"workload4[{g0}:{g1}]", union(el, offs, [s["n"] for s in specs[g0:g1]])


def _main() -> None:
    from . import Context
    ap = argparse.ArgumentParser(prog="python -m signed_triangle_counting_b200.dispatcher")
    ap.add_argument("mode", choices=["train", "evaluate"])
    ap.add_argument("--out", default=str(DEFAULT_MODEL))
    ap.add_argument("--model", default=None)
    ap.add_argument("--workload", type=int, default=3)
    ap.add_argument("--epochs", type=int, default=3000)
    ap.add_argument("--batch-graphs", type=int, default=4096)
    ap.add_argument("--with-split", action="store_true",
                    help="let the model choose the SPLIT strategy")
    ap.add_argument("--save-recording", default=None,
                    help="write the per-cell recordings to this .npz file")
    a = ap.parse_args()
    ctx = Context(0)
    import torch
    gpu = torch.cuda.get_device_name(0) if torch.cuda.is_available() else "?"
    if a.mode == "train":
        recs, names = [], []
        for name, (s, d, g) in training_graphs(a.batch_graphs):
            t0 = time.time()
            recs.append(record(ctx, s, d, g))
            names.append(name)
            print(json.dumps({"recorded": name, "m": int(len(s)), "s": round(time.time() - t0, 1)}),
                  flush=True)
        rec = merge(recs)
        if a.save_recording:
            np.savez(a.save_recording, names=np.array(names),
                     cycles=np.stack([r["cycles"] for r in recs]),
                     arcs=np.stack([r["arcs"] for r in recs]))
        params, info = train(ctx, rec, epochs=a.epochs, use_split=a.with_split)
        meta = {"gpu": gpu, "trained_on": names, **info,
                "train_regret_fixed": regret(rec, ctx.dispatch_tables("fixed"),
                                             info["strategies"])["ratio"],
                "train_regret_learned": regret(rec, ctx.dispatch_tables("learned"),
                                               info["strategies"])["ratio"]}
        save(a.out, params, meta)
        print(json.dumps(meta), flush=True)
    else:
        model = ctx.load_dispatch_model(a.model)
        el = synth.workload(a.workload)
        rec = record(ctx, el.src, el.dst, el.sign)
        if a.save_recording:
            np.savez(a.save_recording, names=np.array([f"workload{a.workload}"]),
                     cycles=rec["cycles"][None], arcs=rec["arcs"][None])
        out = {"gpu": gpu, "workload": a.workload, "model_trained_on": model.get("trained_on"),
               "fixed": regret(rec, ctx.dispatch_tables("fixed"),
                               model.get("strategies", DEFAULT_STRATEGIES)),
               "learned": regret(rec, ctx.dispatch_tables("learned"),
                                 model.get("strategies", DEFAULT_STRATEGIES)),
               "learned_vs_all": regret(rec, ctx.dispatch_tables("learned"), STRATEGIES),
               "counts": rec["counts"].as_tuple()}
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    _main()
