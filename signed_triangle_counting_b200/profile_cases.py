"""Small, fixed cases of the counting path on cuda:0, for kernel profiles.

Each case builds its input once and runs the path `--reps` times, so that a
profiler can skip the first runs and capture one kernel of a later one
(`ncu -k regex:<kernel> -s <skip> -c <count>`).  Sizes are chosen to exceed
the 126 MB L2 while keeping a few GB on the device.

    python -m signed_triangle_counting_b200.profile_cases rmat  --scale 22
    python -m signed_triangle_counting_b200.profile_cases text  --scale 20
    python -m signed_triangle_counting_b200.profile_cases batch --graphs 512
    python -m signed_triangle_counting_b200.profile_cases skew  --shrink 2
    python -m signed_triangle_counting_b200.profile_cases mlp   --scale 16

rmat   the power-law workload at RMAT scale `--scale` (generated on the
       device); dedup, orientation, CSR and count kernels
text   the same graph at `--scale` as `u v sign` text in host memory,
       counted from text (GPU newline scan, line parse and compaction first)
batch  the first `--graphs` graphs of the 4,096-graph batch, in one call on
       the persistent engine
skew   the skewed workload with its sizes divided by 2**`--shrink`
mlp    the learned dispatcher: records per-cell cycles of every strategy on
       the power-law graph at `--scale`, then each rep trains the MLP
       (`k_mlp_train`, `--epochs`) and builds its tables (`k_mlp_tables`)
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import Context, synth


def _edge_text(el) -> bytes:
    """`u v sign` lines, sign 1 / -1."""
    s = np.where(el.sign < 0, "-1", "1")
    return "".join(f"{a} {b} {c}\n" for a, b, c in zip(el.src.tolist(), el.dst.tolist(),
                                                       s.tolist())).encode()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["rmat", "text", "batch", "skew", "mlp"])
    ap.add_argument("--scale", type=int, default=22)
    ap.add_argument("--graphs", type=int, default=512)
    ap.add_argument("--shrink", type=int, default=2)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--dispatch", default="fixed", choices=["fixed", "learned"])
    ap.add_argument("--epochs", type=int, default=3000)
    a = ap.parse_args()

    import torch
    from . import autotune

    ctx = Context(0)
    dev = torch.device("cuda", 0)
    info = {"case": a.case}
    if a.case == "rmat":
        n, samples = 1 << a.scale, 16 << a.scale
        src = torch.empty(samples, dtype=torch.int32, device=dev)
        dst = torch.empty(samples, dtype=torch.int32, device=dev)
        sign = torch.empty(samples, dtype=torch.int8, device=dev)
        ctx.synth_rmat_device(synth.workload_seed(3), a.scale, n, samples, 0.57, 0.19, 0.19, 0.5,
                              src, dst, sign)
        ctx.set_tuning(autotune.tuning_for(3))
        run = lambda: ctx.count(src, dst, sign, dispatch=a.dispatch)
    elif a.case == "text":
        el = synth.rmat(synth.workload_seed(3), a.scale, 1 << a.scale, 16 << a.scale, p_pos=0.5)
        data = _edge_text(el)
        info["text_bytes"] = len(data)
        ctx.set_tuning(autotune.tuning_for(3))
        run = lambda: ctx.count_text(data, dispatch=a.dispatch)[0]
    elif a.case == "batch":
        specs = synth.batch_specs(4096)[: a.graphs]
        el, offs = synth.batch_packed(specs)
        src = torch.from_numpy(el.src.view("int32")).to(dev)
        dst = torch.from_numpy(el.dst.view("int32")).to(dev)
        sign = torch.from_numpy(el.sign).to(dev)
        ctx.set_tuning(autotune.tuning_for(4))
        run = lambda: ctx.count_batch_packed(src, dst, sign, offs, dispatch=a.dispatch,
                                             persistent=True)
    elif a.case == "mlp":
        from . import dispatcher
        el = synth.rmat(synth.workload_seed(3), a.scale, 1 << a.scale, 16 << a.scale, p_pos=0.5)
        rec = dispatcher.record(ctx, el.src, el.dst, el.sign)
        params, _ = dispatcher.train(ctx, rec, epochs=a.epochs)
        info["params"] = int(len(params))
        run = lambda: dispatcher.train(ctx, rec, epochs=a.epochs)
    else:
        el = synth.workload(5, a.shrink)
        src = torch.from_numpy(el.src.view("int32")).to(dev)
        dst = torch.from_numpy(el.dst.view("int32")).to(dev)
        sign = torch.from_numpy(el.sign).to(dev)
        ctx.set_tuning(autotune.tuning_for(5))
        run = lambda: ctx.count(src, dst, sign, dispatch=a.dispatch)
    torch.cuda.synchronize()
    reps = []
    for _ in range(a.reps):
        t0 = time.perf_counter()
        run()
        torch.cuda.synchronize()
        st = ctx.last_stats()
        reps.append({"wall_ms": (time.perf_counter() - t0) * 1e3, "dedup_ms": st.ms_dedup,
                     "orient_ms": st.ms_orient, "csr_ms": st.ms_csr, "count_ms": st.ms_count,
                     "h2d_ms": st.ms_h2d, "launches": st.kernel_launches})
    st = ctx.last_stats()
    info.update(m_input=int(st.m_input), m_unique=int(st.m_unique), n=int(st.n),
                alg_bytes=int(st.alg_bytes), reps=reps)
    print(json.dumps(info))
    ctx.close()


if __name__ == "__main__":
    main()
