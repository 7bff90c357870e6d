"""Seeded synthetic signed graphs (include/stc_synth.h) as EdgeList objects.

Workloads (seed = 1000 + workload):
  1  ER G(10,000, 100,000), p(+) = 0.7
  2  Delaunay of 1,000,000 uniform points, 20 % of edges deleted, p(+) = 0.6
  3  RMAT scale 24, edge factor 16, (.57, .19, .19, .05), p(+) = 0.5
  4  batch of 4,096 graphs (ER / RMAT / Delaunay, n log-uniform in [1e3, 1e6])
  5  skew: 64 Mi vertices, 128 Mi samples, 32 hubs with degree in [1e5, 1e7], p(+) = 0.8
``shrink`` divides a workload's sizes by 2**shrink.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import EdgeList, _capi
from ._capi import lib

BATCH_KINDS = {0: "er", 1: "rmat", 2: "delaunay"}


def _take(g: _capi.stc_synth_graph) -> EdgeList:
    m = g.m
    try:
        if m:
            src = np.ctypeslib.as_array(g.src, (m,)).copy()
            dst = np.ctypeslib.as_array(g.dst, (m,)).copy()
            sign = np.ctypeslib.as_array(g.sign, (m,)).copy()
        else:
            src, dst, sign = np.zeros(0, np.uint32), np.zeros(0, np.uint32), np.zeros(0, np.int8)
        return EdgeList(n=int(g.n), m=int(m), src=src, dst=dst, sign=sign, lines=int(m))
    finally:
        lib().stc_synth_free(C.byref(g))


def _call(fn, *args) -> EdgeList:
    g = _capi.stc_synth_graph()
    st = fn(*args, C.byref(g))
    if st != 0:
        raise ValueError(f"generator rejected its arguments (status {st})")
    return _take(g)


def set_threads(threads: int) -> None:
    lib().stc_synth_set_threads(threads)


def workload_seed(workload: int) -> int:
    return int(lib().stc_synth_workload_seed(workload))


def workload(k: int, shrink: int = 0) -> EdgeList:
    return _call(lib().stc_synth_workload, k, shrink)


def er(seed: int, n: int, m: int, p_pos: float) -> EdgeList:
    return _call(lib().stc_synth_er, seed, n, m, p_pos)


def rmat(seed: int, scale: int, n: int, samples: int, a=0.57, b=0.19, c=0.19, p_pos=0.5) -> EdgeList:
    return _call(lib().stc_synth_rmat, seed, scale, n, samples, a, b, c, p_pos)


def delaunay(seed: int, n: int, delete_frac=0.2, p_pos=0.6) -> EdgeList:
    return _call(lib().stc_synth_delaunay, seed, n, delete_frac, p_pos)


def skew(seed: int, n: int, m_total: int, hubs=32, hub_deg_min=100_000, hub_deg_max=10_000_000,
         p_pos=0.8) -> EdgeList:
    return _call(lib().stc_synth_skew, seed, n, m_total, hubs, hub_deg_min, hub_deg_max, p_pos)


def batch_specs(G: int = 4096, seed: int | None = None) -> list:
    """Recipes of the batched workload's graphs as dicts."""
    seed = workload_seed(4) if seed is None else seed
    arr = (_capi.stc_batch_spec * G)()
    if lib().stc_synth_batch_specs(seed, G, arr) != 0:
        raise ValueError("bad batch arguments")
    return [dict(seed=s.seed, n=s.n, kind=s.kind, rmat_scale=s.rmat_scale, m_target=s.m_target,
                 p_pos=s.p_pos) for s in arr]


def batch_graph(spec: dict) -> EdgeList:
    s = _capi.stc_batch_spec(spec["seed"], spec["n"], spec["kind"], spec["rmat_scale"],
                             spec["m_target"], spec["p_pos"])
    return _call(lib().stc_synth_batch_graph, C.byref(s))


def _spec_array(specs):
    arr = (_capi.stc_batch_spec * max(1, len(specs)))()
    for i, sp in enumerate(specs):
        arr[i] = _capi.stc_batch_spec(sp["seed"], sp["n"], sp["kind"], sp["rmat_scale"],
                                      sp["m_target"], sp["p_pos"])
    return arr


def batch_packed(specs: list, g_begin: int = 0, g_end: int | None = None):
    """Graphs [g_begin, g_end) of a batch generated in parallel and packed back
    to back: (EdgeList of all their edges, offsets with g_end - g_begin + 1
    entries)."""
    g_end = len(specs) if g_end is None else g_end
    arr = _spec_array(specs)
    offs = np.zeros(g_end - g_begin + 1, np.uint64)
    g = _capi.stc_synth_graph()
    st = lib().stc_synth_batch_packed(arr, g_begin, g_end, C.byref(g),
                                      offs.ctypes.data_as(_capi.u64p))
    if st != 0:
        raise ValueError(f"batch generator failed (status {st})")
    return _take(g), offs
