"""Benchmark: signed triangle counting on B200, one JSON line on rank 0.

A step is one pass of the whole counting path over one synthetic signed graph
resident in HBM: dedup, (degree, id) orientation, forward CSR with int8 signs
and the intersection engine, ending in the four per-type counts.  The default
workload is the power-law one: RMAT scale 24, edge factor 16,
(a, b, c, d) = (.57, .19, .19, .05), p(+) = .5, generated on the device
(268,435,456 samples, about 250M undirected edges after dedup).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload 3]
    python bench.py --impl reference ...      # the reference's CPU code

Metric: undirected edges (after dedup) counted per second, whole job.  With
N > 1 ranks the same workload is split across them (strong scaling): a single
graph into N rank-space shards of equal merge-model cost (every rank builds
the forward CSR; one NCCL all-reduce of the four counters), a batch into N
sets of graphs (LPT on edge counts; one all-reduce of the per-graph counts).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "edges/s (undirected edges after dedup, whole counting path)"
UNIT = "edges/s"
CPU_SAMPLE_DIV = 64  # the CPU baseline counts the sources with id < n / CPU_SAMPLE_DIV

WORKLOADS = {
    1: "ER G(n=10,000, m=100,000), p(+)=0.7",
    2: "Delaunay of 1,000,000 uniform points, 20% of edges deleted, p(+)=0.6",
    3: "RMAT scale 24, edge factor 16, (.57,.19,.19,.05), symmetrised + deduped, p(+)=0.5",
    4: "batch of 4,096 graphs: n log-uniform in [1e3, 1e6], ER deg 8 / RMAT ef 8 / Delaunay-20%, "
       "p(+) uniform in [0.3, 0.9]",
    5: "skew: 64Mi vertices, 128Mi samples, backbone + 32 hubs deg in [1e5,1e7], p(+)=0.8",
}


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-i", str(self.gpu), "-lms", "200"], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def load_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d["hbm_gbs"], "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def load_traffic(workload: int, rmat_scale: int = 24):
    """DRAM bytes (read + write) of one count stage as measured by ncu and
    committed with the profiles, or None where none was taken."""
    p = ROOT / "profiles" / "ncu_traffic.json"
    if not p.exists() or (workload == 3 and rmat_scale != 24):
        return None
    e = json.loads(p.read_text()).get(str(workload))
    return e["bytes_per_count"] if e else None


def golden_counts(workload: int):
    p = ROOT / "tests" / "golden" / "golden.json"
    if not p.exists():
        return None
    g = json.loads(p.read_text())
    if workload == 4:
        return g["batch"]["t"] if "batch" in g else None
    w = g.get("workloads", {}).get(f"{workload}/0")
    return tuple(w["t"]) if w else None


def make_device_workload(ctx, workload: int, seed_offset: int, torch, scale: int = 24):
    """Synthetic graph resident in HBM as (src, dst, sign) tensors."""
    from signed_triangle_counting_b200 import synth
    if workload == 3:
        n = 1 << scale
        samples = 16 << scale
        seed = synth.workload_seed(3) + seed_offset
        dev = torch.device("cuda", ctx.device)
        src = torch.empty(samples, dtype=torch.int32, device=dev)
        dst = torch.empty(samples, dtype=torch.int32, device=dev)
        sign = torch.empty(samples, dtype=torch.int8, device=dev)
        ctx.synth_rmat_device(seed, scale, n, samples, 0.57, 0.19, 0.19, 0.5, src, dst, sign)
        return src, dst, sign
    if workload == 4:
        specs = synth.batch_specs(4096)
        parts, offs, pos = [], [0], 0
        dev = torch.device("cuda", ctx.device)
        for g0 in range(0, len(specs), 256):
            el, o = synth.batch_packed(specs, g0, min(len(specs), g0 + 256))
            parts.append(el)
            offs.extend(int(x) + pos for x in o[1:])
            pos += el.m
        src = torch.empty(pos, dtype=torch.int32, device=dev)
        dst = torch.empty(pos, dtype=torch.int32, device=dev)
        sign = torch.empty(pos, dtype=torch.int8, device=dev)
        at = 0
        for el in parts:
            src[at:at + el.m] = torch.from_numpy(el.src.view("int32")).to(dev)
            dst[at:at + el.m] = torch.from_numpy(el.dst.view("int32")).to(dev)
            sign[at:at + el.m] = torch.from_numpy(el.sign).to(dev)
            at += el.m
        return src, dst, sign, offs
    el = synth.workload(workload)
    if seed_offset:
        raise SystemExit("only the RMAT workload has per-rank instances")
    dev = torch.device("cuda", ctx.device)
    return (torch.from_numpy(el.src.view("int32")).to(dev), torch.from_numpy(el.dst.view("int32")).to(dev),
            torch.from_numpy(el.sign).to(dev))


def cpu_reference_run(scale: int, steps: int, warmup: int, log=None) -> dict | None:
    """The reference's own CPU path on the power-law workload, with all host
    threads (OpenMP).  The input is the workload's edge list made by the
    oracle's restatement of the generator (bit-equal to the package's, and
    loading nothing from the package).  The reference's build_forward_csr
    and sort_adj_lists run once, at full size, and are timed there.  Each
    step then times its count_triangles (MC/tc_serial.cpp:138-170, unchanged)
    on a bounded sample of the same graph: the sources whose id is below
    n / CPU_SAMPLE_DIV, a uniform random vertex sample because the generator
    relabels ids by a seeded bijection.  A step's rate charges the sample its
    count time plus its share (by edges) of the full-size build and sort:
    sampled edges / (count s + (build s + sort s) * sampled edges / edges)."""
    import oracle
    if not oracle.ref_available():
        return None
    from oracle import RefKeptCSR, synth_rmat
    seed = 1000 + 3  # the power-law workload's seed
    t0 = time.perf_counter()
    src, dst, sign = synth_rmat(seed, scale, 1 << scale, 16 << scale, 0.57, 0.19, 0.19, 0.5)
    gen_s = time.perf_counter() - t0
    kept = RefKeptCSR(src, dst, sign)
    del src, dst, sign
    try:
        n_s = max(1, kept.n // CPU_SAMPLE_DIV)
        arcs_s, work_s = kept.prefix_size(n_s)
        arcs, work = kept.prefix_size(kept.n)
        prep_share = (kept.build_s + kept.sort_s) * arcs_s / max(1, arcs)
        vals, secs, counts = [], [], None
        for i in range(warmup + steps):
            counts, sec = kept.count_prefix(n_s)
            if log:
                log(f"cpu sample step {i}: {sec:.3f} s")
            if i >= warmup:
                secs.append(sec)
                vals.append(arcs_s / (sec + prep_share))
        count_s = statistics.median(secs)
        return dict(
            value=statistics.median(vals), step_seconds=secs, counts=counts,
            threads=kept.threads, edges=arcs, n=kept.n, sample_edges=arcs_s,
            build_s=kept.build_s, sort_s=kept.sort_s, gen_s=gen_s,
            count_edges_per_s=arcs_s / count_s,
            count_s_full_projected=count_s * work / max(1, work_s),
            sample=(f"RMAT scale {scale} (the workload's graph: {arcs} edges after dedup); "
                    f"timed per step: the reference's count_triangles over the {arcs_s} edges "
                    f"of the sources with id < n/{CPU_SAMPLE_DIV} ({n_s} of {kept.n} vertices, a "
                    f"uniform random vertex sample), plus the sample's edge share of its "
                    f"build_forward_csr ({kept.build_s:.2f} s) and sort_adj_lists "
                    f"({kept.sort_s:.2f} s), measured once at full size"))
    finally:
        kept.close()


def run_reference(args) -> None:
    world, rank, _ = _dist()
    if rank != 0:
        return
    import oracle
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref (the reference compiled from its sources) is missing"}))
        return
    r = cpu_reference_run(args.rmat_scale, args.steps, args.warmup)
    value = r["value"]
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": statistics.mean(r["step_seconds"]) * 1e3,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "u32/i8 (ids/signs), u64 counters", "data": "synthetic (seeded, generated on the host)",
        "config": dict(workload_config(3, args.rmat_scale), m_input=16 << args.rmat_scale,
                       m_unique=r["edges"], n=r["n"]),
        "run": {"parallelism": f"host OpenMP, {r['threads']} threads"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": r["threads"], "kind": "reference",
                         "sample": r["sample"]},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_stages": {k: r[k] for k in ("build_s", "sort_s", "gen_s", "count_edges_per_s",
                                               "count_s_full_projected", "sample_edges", "edges")},
        "sample_counts": list(r["counts"]),
    }
    print(json.dumps(out))


def workload_config(workload: int, rmat_scale: int = 24) -> dict:
    """The `config` both arms print for a workload."""
    if workload == 3 and rmat_scale != 24:
        name = f"RMAT scale {rmat_scale}, edge factor 16, (.57,.19,.19,.05), p(+)=0.5"
    else:
        name = WORKLOADS[workload]
    return {"workload": name}


def _time_form(fn, steps: int, stream, torch) -> float:
    """Three untimed passes (a batch on the persistent engine is built
    uncapped, then sized at capacities, then captured whole), then `steps`
    passes timed with CUDA events on `stream`; mean milliseconds per pass."""
    for _ in range(3):
        fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(steps):
        fn()
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / steps


def forms_run(ctx, args, stream, torch) -> dict:
    """The metric's second half, in the same run: the plain fixed-threshold
    form against the learned and batched forms, on the batched and the
    skewed workloads, each form timed over resident inputs (three untimed
    passes, then --forms-steps passes, CUDA events), counts checked against
    the reference's.

    batch: graphs [0, G) of the 4,096-graph batch (G = --forms-graphs; the
      graph recipes are drawn i.i.d., so a prefix is a random sample):
        plain_fixed      one call per graph, per-class kernels, fixed dispatch
        batched_fixed    all G graphs in one call, persistent engine replayed
                         from a CUDA graph, fixed dispatch
        learned_batched  as batched_fixed with the learned dispatch tables
    skew: the whole skewed graph, per-class kernels:
        plain_fixed      fixed dispatch
        learned          learned dispatch tables"""
    from signed_triangle_counting_b200 import autotune, synth
    dev = torch.device("cuda", ctx.device)
    model = ctx.load_dispatch_model()
    out = {"dispatch_model": model.get("trained_on"), "steps": args.forms_steps}
    sampler = ClockSampler(ctx.device)
    sampler.start()
    kw = dict(stream=stream.cuda_stream)

    # ---- batched workload
    G = args.forms_graphs
    specs = synth.batch_specs(4096)[:G]
    t0 = time.perf_counter()
    el, offs = synth.batch_packed(specs)
    gen_s = time.perf_counter() - t0
    src = torch.from_numpy(el.src.view("int32")).to(dev)
    dst = torch.from_numpy(el.dst.view("int32")).to(dev)
    sign = torch.from_numpy(el.sign).to(dev)
    del el
    spans = [(int(offs[g]), int(offs[g + 1])) for g in range(G)]
    ctx.set_tuning(autotune.tuning_for(4))
    res = {}

    def plain():
        res["plain"] = [ctx.count(src[b:e], dst[b:e], sign[b:e], dispatch="fixed",
                                  persistent=False, **kw) for b, e in spans]

    def batched(dispatch):
        def fn():
            res[dispatch] = ctx.count_batch_packed(src, dst, sign, offs, dispatch=dispatch,
                                                   persistent=True, **kw)
        return fn

    ms = {"plain_fixed": _time_form(plain, args.forms_steps, stream, torch),
          "batched_fixed": _time_form(batched("fixed"), args.forms_steps, stream, torch),
          "learned_batched": _time_form(batched("learned"), args.forms_steps, stream, torch)}
    edges = ctx.last_stats().m_unique
    want = golden_counts(4)
    got = {k: [list(c.as_tuple()) for c in res[r]]
           for k, r in (("plain_fixed", "plain"), ("batched_fixed", "fixed"),
                        ("learned_batched", "learned"))}
    exact = (all(v == want[:G] for v in got.values()) if want else None)
    out["batch"] = {
        "graphs": G, "m_input": int(offs[-1]), "m_unique": int(edges), "gen_s": gen_s,
        "exact": exact,
        "forms": {k: {"ms": v, "edges_per_s": edges / (v / 1e3)} for k, v in ms.items()},
        "ratio_learned_batched_vs_plain_fixed": ms["plain_fixed"] / ms["learned_batched"],
        "ratio_batched_fixed_vs_plain_fixed": ms["plain_fixed"] / ms["batched_fixed"],
        "ratio_learned_vs_fixed_batched": ms["batched_fixed"] / ms["learned_batched"],
    }
    del src, dst, sign

    # ---- skewed workload
    t0 = time.perf_counter()
    el = synth.workload(5)
    gen_s = time.perf_counter() - t0
    src = torch.from_numpy(el.src.view("int32")).to(dev)
    dst = torch.from_numpy(el.dst.view("int32")).to(dev)
    sign = torch.from_numpy(el.sign).to(dev)
    del el
    ctx.set_tuning(autotune.tuning_for(5))

    def single(dispatch):
        def fn():
            res[dispatch] = ctx.count(src, dst, sign, dispatch=dispatch, persistent=False, **kw)
        return fn

    ms = {"plain_fixed": _time_form(single("fixed"), args.forms_steps, stream, torch),
          "learned": _time_form(single("learned"), args.forms_steps, stream, torch)}
    st = ctx.last_stats()
    want = golden_counts(5)
    exact = (res["fixed"].as_tuple() == want and res["learned"].as_tuple() == want
             if want else None)
    out["skew"] = {
        "m_input": int(src.numel()), "m_unique": int(st.m_unique), "gen_s": gen_s, "exact": exact,
        "stage_ms": {"dedup": st.ms_dedup, "orient": st.ms_orient, "csr": st.ms_csr,
                     "count": st.ms_count},
        "forms": {k: {"ms": v, "edges_per_s": st.m_unique / (v / 1e3)} for k, v in ms.items()},
        "ratio_learned_vs_plain_fixed": ms["plain_fixed"] / ms["learned"],
    }
    del src, dst, sign
    ctx.set_dispatch_model(None)
    out["clocks"] = sampler.stop()
    return out


def run_gpu(args) -> None:
    import ctypes as C

    import torch
    import signed_triangle_counting_b200 as stc
    from signed_triangle_counting_b200 import _capi, distributed

    world, rank, local = _dist()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)
    ctx = stc.Context(local)
    model = ctx.load_dispatch_model() if args.dispatch == "learned" else None
    from signed_triangle_counting_b200 import autotune
    tuning = None if args.no_tuning else autotune.tuning_for(args.workload)
    if tuning:
        ctx.set_tuning(tuning)
    stream = torch.cuda.current_stream(local)
    # Every rank generates the same workload; with N > 1 ranks a single graph
    # is split into N shards of equal merge-model cost, a batch into N sets of
    # graphs (LPT on edge counts).
    wl = make_device_workload(ctx, args.workload, 0, torch, args.rmat_scale)
    src, dst, sign = wl[:3]
    offs = np.asarray(wl[3], np.uint64) if len(wl) > 3 else None
    G = len(offs) - 1 if offs is not None else 1
    mine = None
    if offs is not None and world > 1:
        src, dst, sign, offs_run, mine = distributed.batch_shard(src, dst, sign, offs, rank, world)
    else:
        offs_run = offs
    torch.cuda.synchronize()
    m_total_input = int(wl[0].numel())
    m_input = src.numel()
    persistent = args.engine == "persistent" or (args.engine == "auto" and offs is not None)
    kw = dict(strategy=args.strategy, dispatch=args.dispatch, stream=stream.cuda_stream,
              persistent=persistent)

    def step():
        if offs_run is not None:
            c = ctx.count_batch_packed(src, dst, sign, offs_run, **kw) if len(offs_run) > 1 else []
            if world > 1:
                c = distributed.gather_batch(c, mine, G, device=dev)
        elif world > 1:
            c = distributed.count(ctx, src, dst, sign, device=dev,
                                  **{k: v for k, v in kw.items() if k != "persistent"})
        else:
            c = ctx.count(src, dst, sign, **kw)
        return c, ctx.last_stats()

    counts, st = None, None
    for _ in range(args.warmup):
        counts, st = step()
    # Exact-count check of the whole job against the reference's counts.
    full = args.workload != 3 or args.rmat_scale == 24
    want = golden_counts(args.workload) if rank == 0 and full else None
    if offs is not None:
        exact = [list(c.as_tuple()) for c in counts] == want if want is not None else None
        counts_out = [int(sum(c.as_tuple()[k] for c in counts)) for k in range(4)]
    else:
        exact = (counts.as_tuple() == want) if want is not None else None
        counts_out = list(counts.as_tuple())

    # ---- timed region: inputs resident in HBM (larger than the 126 MB L2)
    sampler = ClockSampler(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    count_ms, launches, alg_bytes, probe_bytes = [], 0, 0, 0
    for _ in range(args.steps):
        counts, st = step()
        count_ms.append(st.ms_count)
        launches += st.kernel_launches
        alg_bytes = st.alg_bytes
        probe_bytes = st.probe_bytes
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    edges = st.m_unique  # this rank's graph (a single graph: the whole graph)
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        if offs is not None:  # a batch: every rank counted different graphs
            t = torch.tensor([edges], dtype=torch.int64, device=dev)
            dist.all_reduce(t)
            edges = int(t.item())
    value = edges * args.steps / (ms / 1e3)

    # ---- end to end through the C ABI from pinned host memory
    def host_copy(t):
        try:
            h = torch.empty(t.numel(), dtype=t.dtype, pin_memory=True)
        except RuntimeError:
            h = torch.empty(t.numel(), dtype=t.dtype)
        h.copy_(t)
        return h
    h_src, h_dst, h_sign = host_copy(src), host_copy(dst), host_copy(sign)
    pinned = h_src.is_pinned()
    torch.cuda.synchronize()
    o = stc.Context._opts(args.strategy, args.dispatch, False, True, stream.cuda_stream,
                          persistent)
    G_run = len(offs_run) - 1 if offs_run is not None else 1
    out = (_capi.stc_counts * max(1, G_run))()
    ptrs = [C.c_void_p(h.data_ptr()) for h in (h_src, h_dst, h_sign)]

    def e2e_step():
        if offs_run is not None:
            s_ = _capi.lib().stc_count_batch_packed(ctx._h, *ptrs, offs_run.ctypes.data_as(_capi.u64p),
                                                    G_run, C.byref(o), out)
            assert s_ == 0, stc.StcError(s_)
            if world > 1:
                distributed.gather_batch([stc.GlobalTriCounts(x.t0, x.t1, x.t2, x.t3)
                                          for x in out[:G_run]], mine, G, device=dev)
        elif world > 1:
            s_ = _capi.lib().stc_count_shard(ctx._h, *ptrs, m_input, C.byref(o), rank, world, out,
                                             None)
            assert s_ == 0, stc.StcError(s_)
            distributed._reduce_sum([[out[0].t0, out[0].t1, out[0].t2, out[0].t3]], None, dev)
        else:
            s_ = _capi.lib().stc_count(ctx._h, *ptrs, m_input, C.byref(o), out)
            assert s_ == 0, stc.StcError(s_)

    e2e_step()
    e2e_steps = max(1, min(args.steps, 5))
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(e2e_steps):
        e2e_step()
    f1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = f0.elapsed_time(f1)
    if world > 1:
        t = torch.tensor([e2e_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = edges * e2e_steps / (e2e_ms / 1e3)
    forms = (forms_run(ctx, args, stream, torch)
             if world == 1 and args.workload == 3 and not args.no_forms else None)

    if rank == 0:
        peaks = load_peaks()
        cms = statistics.mean(count_ms)
        achieved = probe_bytes / (cms / 1e3) / 1e9
        merge_achieved = alg_bytes / (cms / 1e3) / 1e9
        traffic = load_traffic(args.workload, args.rmat_scale)
        cpu = None
        if world == 1 and args.workload == 3 and not args.skip_cpu:
            r = cpu_reference_run(args.rmat_scale, steps=2, warmup=0)
            if r:
                cpu = {"value": r["value"], "unit": UNIT, "cores": r["threads"],
                       "kind": "reference", "sample": r["sample"],
                       "count_edges_per_s": r["count_edges_per_s"]}
        if world == 1:
            par = "1 GPU"
        elif offs is not None:
            par = (f"{world} GPUs: graphs assigned to ranks by LPT on edge counts, one all-reduce "
                   "of the per-graph counts")
        else:
            par = (f"{world} GPUs: every rank builds the forward CSR and counts one of {world} "
                   "rank-space shards of equal merge-model cost; one NCCL all-reduce of 4 counters")
        res = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "u32/i8 (ids/signs), u64 counters",
            "data": "synthetic (seeded, generated on the device)",
            "config": dict(workload_config(args.workload, args.rmat_scale),
                           m_input=int(m_total_input), m_unique=edges,
                           n=st.n if offs is None else None),
            "run": {"parallelism": par, "strategy": args.strategy, "dispatch": args.dispatch,
                    "dispatch_model": model.get("trained_on") if model else None,
                    "engine": "persistent (CUDA graph)" if persistent else "class kernels",
                    "tuning": tuning,
                    "l2": f"inputs {m_input * 9 / 1e9:.1f} GB per rank > 126 MB L2, no flush"},
            "exact": exact, "counts": counts_out,
            "stage_ms": {"dedup": st.ms_dedup, "orient": st.ms_orient, "csr": st.ms_csr,
                         "count": st.ms_count, "device_total": st.ms_total},
            "roofline": {"bound": "hbm", "kernel": "intersection engine (count)",
                         "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": achieved / peaks["hbm_gbs"], "peak_source": peaks["source"],
                         "traffic": traffic, "model": "probe: 5 min(|A'|, |B|) + 30 per arc",
                         "alg_bytes_per_launch": probe_bytes, "count_ms": cms,
                         "merge_model_bytes": alg_bytes,
                         "merge_model_achieved": merge_achieved,
                         "merge_model_frac": merge_achieved / peaks["hbm_gbs"]},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(m_input) * 9,
                    "d2h_bytes_per_step": 32 * G_run, "steps": e2e_steps,
                    "host_memory": "pinned" if pinned else "pageable"},
            "gpu_launches": launches,
            "clocks": clocks,
        }
        if forms:
            res["forms"] = forms
        print(json.dumps(res))
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["mine", "reference"], default="mine")
    ap.add_argument("--workload", type=int, default=3, choices=[1, 2, 3, 4, 5])
    ap.add_argument("--strategy", default="auto", choices=["auto", "merge", "hash", "search", "split"])
    ap.add_argument("--dispatch", default="fixed", choices=["fixed", "learned"])
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--no-tuning", action="store_true",
                    help="untuned launch parameters instead of the workload's autotuned ones")
    ap.add_argument("--no-forms", action="store_true",
                    help="skip the plain / batched / learned forms on the batch and skew workloads")
    ap.add_argument("--forms-graphs", type=int, default=1024,
                    help="graphs of the batch workload the forms are timed on")
    ap.add_argument("--forms-steps", type=int, default=3)
    ap.add_argument("--engine", default="auto", choices=["auto", "persistent", "classes"],
                    help="counting engine (auto: persistent for the batch, class kernels else)")
    ap.add_argument("--rmat-scale", type=int, default=24,
                    help="RMAT scale of workload 3 (24 = the benchmark; smaller for profiling)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
