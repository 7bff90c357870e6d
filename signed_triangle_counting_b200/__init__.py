"""B200-native signed triangle counting (host mirror of the reference interface).

The reference's CPU programs expose ``load_graph`` / ``build_forward_csr`` /
``count_triangles`` and a ``GlobalTriCounts`` result
("Signed_TC/Multicore Implementations/graph_io.h:100,231",
"tc_serial.cpp:11-31,138").  This module keeps those names and meanings over
the C ABI of ``libstc.so`` (include/stc.h); every counting call runs on the
GPU through hand-written sm_100a kernels and fails loudly when the native
library or a CUDA device is missing.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from pathlib import Path
from typing import Iterable, Optional, Sequence

import numpy as np

from . import _capi
from ._capi import lib

__all__ = [
    "GlobalTriCounts", "EdgeList", "ForwardCSR", "Stats", "StcError", "Context",
    "load_graph", "parse_edge_text", "load_mtx", "parse_mtx", "dispatch_features", "synth",
]


class StcError(RuntimeError):
    """A non-zero stc_status, with the context's last error message."""

    def __init__(self, status: int, message: str = ""):
        name = lib().stc_status_string(status).decode()
        super().__init__(f"{name} ({status})" + (f": {message}" if message else ""))
        self.status = status
        self.message = message


@dataclass(frozen=True)
class GlobalTriCounts:
    """Per-type triangle counts (tc_serial.cpp:11-31): t3 = +++, t2 = ++-,
    t1 = +--, t0 = ---."""

    t0: int
    t1: int
    t2: int
    t3: int

    def balanced(self) -> int:
        return self.t1 + self.t3

    def unbalanced(self) -> int:
        return self.t0 + self.t2

    def total(self) -> int:
        return self.t0 + self.t1 + self.t2 + self.t3

    def as_tuple(self) -> tuple:
        return (self.t0, self.t1, self.t2, self.t3)

    def format(self) -> str:
        """The block tc_serial prints (tc_serial.cpp:18-30)."""
        return (
            "\nTriangle counts\n"
            f"  T3 (+++ balanced)   : {self.t3}\n"
            f"  T1 (+-- balanced)   : {self.t1}\n"
            f"  T2 (++- unbalanced) : {self.t2}\n"
            f"  T0 (--- unbalanced) : {self.t0}\n"
            "  --------------------------------\n"
            f"  balanced total      : {self.balanced()}\n"
            f"  unbalanced total    : {self.unbalanced()}\n"
            f"  grand total         : {self.total()}\n")

    def print(self) -> None:
        print(self.format(), end="")


@dataclass
class EdgeList:
    """EdgeList (graph_io.h:14-20): src = min endpoint, dst = max endpoint."""

    n: int
    m: int
    src: np.ndarray
    dst: np.ndarray
    sign: np.ndarray
    lines: int = 0


@dataclass
class ForwardCSR:
    """ForwardCSR (graph_io.h:22-30) with lists sorted by neighbour id."""

    n: int
    m: int
    offsets: np.ndarray
    edges: np.ndarray
    signs: np.ndarray
    fdeg: np.ndarray
    rank: np.ndarray


@dataclass
class Stats:
    n: int
    m_input: int
    m_unique: int
    m_forward: int
    alg_bytes: int
    triangles: int
    ms_h2d: float
    ms_dedup: float
    ms_orient: float
    ms_csr: float
    ms_count: float
    ms_total: float
    kernel_launches: int
    groups_replayed: int
    probe_bytes: int


def _check(status: int, ctx=None) -> None:
    if status != _capi.STC_OK:
        msg = lib().stc_ctx_last_error(ctx).decode() if ctx else ""
        raise StcError(status, msg)


class _EdgeBuffers:
    """Owns the three malloc'd arrays of one stc_edge_list and frees them
    (stc_free_edge_list) once no numpy view of them is left."""

    def __init__(self, el: _capi.stc_edge_list):
        self._el = el

    def __del__(self):
        try:
            lib().stc_free_edge_list(C.byref(self._el))
        except Exception:
            pass


def _view(ptr, ctype, m: int, owner: _EdgeBuffers, dtype) -> np.ndarray:
    arr = (ctype * m).from_address(C.cast(ptr, C.c_void_p).value)
    arr._owner = owner  # the ctypes array, numpy's base, keeps the owner alive
    return np.frombuffer(arr, dtype=dtype)


def _edge_list_take(el: _capi.stc_edge_list) -> EdgeList:
    """An EdgeList over the library's arrays without copying them; the arrays
    are freed with the last view."""
    m = el.m
    owner = _EdgeBuffers(el)
    if not m:
        return EdgeList(n=el.n, m=0, src=np.zeros(0, np.uint32), dst=np.zeros(0, np.uint32),
                        sign=np.zeros(0, np.int8), lines=el.lines)
    return EdgeList(n=el.n, m=m, src=_view(el.src, C.c_uint32, m, owner, np.uint32),
                    dst=_view(el.dst, C.c_uint32, m, owner, np.uint32),
                    sign=_view(el.sign, C.c_int8, m, owner, np.int8), lines=el.lines)


def load_graph(path: str) -> EdgeList:
    """load_graph (graph_io.h:100-212): parses a `u v sign` file on the host."""
    el = _capi.stc_edge_list()
    st = lib().stc_load_edge_list(str(path).encode(), C.byref(el))
    if st == _capi.STC_ERR_IO:
        raise OSError(f"cannot read {path}")
    _check(st)
    return _edge_list_take(el)


def parse_edge_text(data: bytes) -> EdgeList:
    el = _capi.stc_edge_list()
    _check(lib().stc_parse_edge_text(data, len(data), C.byref(el)))
    return _edge_list_take(el)


def load_mtx(path: str, *, zero_negative: bool = False) -> EdgeList:
    """A MatrixMarket coordinate file as an edge list (stc_load_mtx): weight
    < 0 is negative, or <= 0 with ``zero_negative`` (the reference GPU
    drivers' rule, GM/signed_tc.hxx:317)."""
    el = _capi.stc_edge_list()
    st = lib().stc_load_mtx(str(path).encode(), _capi.MTX_ZERO_NEGATIVE if zero_negative else 0,
                            C.byref(el))
    if st == _capi.STC_ERR_IO:
        raise OSError(f"cannot read {path}")
    _check(st)
    return _edge_list_take(el)


def parse_mtx(data: bytes, *, zero_negative: bool = False) -> EdgeList:
    el = _capi.stc_edge_list()
    _check(lib().stc_parse_mtx(data, len(data), _capi.MTX_ZERO_NEGATIVE if zero_negative else 0,
                               C.byref(el)))
    return _edge_list_take(el)


def _host_arrays(src, dst, sign):
    src = np.ascontiguousarray(src, dtype=np.uint32)
    dst = np.ascontiguousarray(dst, dtype=np.uint32)
    sign = np.ascontiguousarray(sign, dtype=np.int8)
    if not (len(src) == len(dst) == len(sign)):
        raise ValueError("src, dst and sign must have the same length")
    return src, dst, sign


def _ptr(a) -> C.c_void_p:
    if hasattr(a, "data_ptr"):  # torch tensor
        return C.c_void_p(a.data_ptr())
    return C.c_void_p(a.ctypes.data)


class Context:
    """Owns an stc_ctx (device memory, stream) on one CUDA device."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        st = lib().stc_ctx_create(device, C.byref(h))
        _check(st)
        self._h = h
        self.device = device

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().stc_ctx_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _opts(strategy="auto", dispatch="fixed", device_input=False, timing=True,
              stream: Optional[int] = None, persistent=False) -> _capi.stc_opts:
        o = _capi.stc_opts()
        o.strategy = _capi.STRATEGY[strategy]
        o.dispatch = _capi.DISPATCH[dispatch]
        o.flags = ((_capi.F_DEVICE_INPUT if device_input else 0) | (_capi.F_TIMING if timing else 0)
                   | (_capi.F_PERSISTENT if persistent else 0))
        o.stream = C.c_void_p(stream) if stream else None
        return o

    def count(self, src, dst, sign, *, strategy="auto", dispatch="fixed", stream=None,
              timing=True, persistent=False) -> GlobalTriCounts:
        """Whole path (dedup, orientation, CSR, intersection) on the GPU.

        Host numpy arrays are copied to the device; torch CUDA tensors
        (uint32/int32 ids, int8 signs) are used in place.  ``persistent``
        counts with the persistent engine replayed from a CUDA graph."""
        dev = hasattr(src, "is_cuda") and src.is_cuda
        if dev:
            m = int(src.numel())
            ps, pd, pg = _ptr(src), _ptr(dst), _ptr(sign)
            if stream is None:  # stay ordered after the torch kernels that made the tensors
                import torch
                stream = torch.cuda.current_stream(src.device).cuda_stream
        else:
            src, dst, sign = _host_arrays(src, dst, sign)
            m = len(src)
            ps, pd, pg = _ptr(src), _ptr(dst), _ptr(sign)
        out = _capi.stc_counts()
        o = self._opts(strategy, dispatch, dev, timing, stream, persistent)
        _check(lib().stc_count(self._h, ps, pd, pg, m, C.byref(o), C.byref(out)), self._h)
        return GlobalTriCounts(out.t0, out.t1, out.t2, out.t3)

    def count_shard(self, src, dst, sign, shard: int, shards: int, *, strategy="auto",
                    dispatch="fixed", stream=None, timing=True):
        """Shard ``shard`` of ``shards`` of ``count`` (one graph on several
        GPUs): returns (counts, (lo, hi)), the counts of the triangles whose
        lowest-ranked vertex has its rank in [lo, hi).  The shards' counts add
        up to ``count``'s."""
        dev = hasattr(src, "is_cuda") and src.is_cuda
        if dev:
            m = int(src.numel())
            if stream is None:
                import torch
                stream = torch.cuda.current_stream(src.device).cuda_stream
        else:
            src, dst, sign = _host_arrays(src, dst, sign)
            m = len(src)
        out = _capi.stc_counts()
        rng = (C.c_uint64 * 2)()
        o = self._opts(strategy, dispatch, dev, timing, stream)
        _check(lib().stc_count_shard(self._h, _ptr(src), _ptr(dst), _ptr(sign), m, C.byref(o),
                                     shard, shards, C.byref(out), rng), self._h)
        return GlobalTriCounts(out.t0, out.t1, out.t2, out.t3), (int(rng[0]), int(rng[1]))

    def count_text(self, data, *, strategy="auto", dispatch="fixed", timing=True):
        """The whole path from `u v sign` text parsed on the GPU: bytes, a
        path, or a torch CUDA uint8 tensor.  Returns (counts, data lines, n)."""
        dev = hasattr(data, "is_cuda") and data.is_cuda
        if isinstance(data, (str, Path)):
            data = Path(data).read_bytes()
        info = _capi.stc_text_info()
        out = _capi.stc_counts()
        o = self._opts(strategy, dispatch, dev, timing)
        ptr = C.c_void_p(data.data_ptr()) if dev else C.c_char_p(bytes(data))
        size = int(data.numel()) if dev else len(data)
        _check(lib().stc_count_text(self._h, ptr, size, C.byref(o), C.byref(out), C.byref(info)),
               self._h)
        return GlobalTriCounts(out.t0, out.t1, out.t2, out.t3), info.lines, info.n

    def parse_edge_text_gpu(self, data: bytes) -> EdgeList:
        """The GPU text parser's edge list (same result as parse_edge_text)."""
        el = _capi.stc_edge_list()
        o = self._opts(timing=False)
        _check(lib().stc_parse_edge_text_gpu(self._h, C.c_char_p(data), len(data), C.byref(o),
                                             C.byref(el)), self._h)
        return _edge_list_take(el)

    def count_edge_list(self, el: EdgeList, **kw) -> GlobalTriCounts:
        return self.count(el.src, el.dst, el.sign, **kw)

    def build_forward_csr(self, src, dst, sign) -> ForwardCSR:
        """build_forward_csr + sort_adj_lists (graph_io.h:231-402,
        tc_serial.cpp:33-93) on the GPU, returned in the reference layout."""
        src, dst, sign = _host_arrays(src, dst, sign)
        out = _capi.stc_forward_csr()
        o = self._opts()
        _check(lib().stc_build_forward_csr(self._h, _ptr(src), _ptr(dst), _ptr(sign), len(src),
                                           C.byref(o), C.byref(out)), self._h)
        try:
            n, m = out.n, out.m
            return ForwardCSR(
                n=n, m=m,
                offsets=np.ctypeslib.as_array(out.offsets, (n + 1,)).copy(),
                edges=np.ctypeslib.as_array(out.edges, (m,)).copy() if m else np.zeros(0, np.uint32),
                signs=np.ctypeslib.as_array(out.signs, (m,)).copy() if m else np.zeros(0, np.int8),
                fdeg=np.ctypeslib.as_array(out.fdeg, (n,)).copy() if n else np.zeros(0, np.uint32),
                rank=np.ctypeslib.as_array(out.rank, (n,)).copy() if n else np.zeros(0, np.uint32))
        finally:
            lib().stc_free_forward_csr(C.byref(out))

    def count_triangles(self, csr: ForwardCSR, *, strategy="auto", dispatch="fixed") -> GlobalTriCounts:
        """count_triangles (tc_serial.cpp:138-170) over a reference-layout CSR."""
        offsets = np.ascontiguousarray(csr.offsets, np.uint64)
        edges = np.ascontiguousarray(csr.edges, np.uint32)
        signs = np.ascontiguousarray(csr.signs, np.int8)
        fdeg = np.ascontiguousarray(csr.fdeg, np.uint32)
        rank = np.ascontiguousarray(csr.rank, np.uint32)
        c = _capi.stc_forward_csr()
        c.n, c.m = csr.n, csr.m
        c.offsets = offsets.ctypes.data_as(_capi.u64p)
        c.edges = edges.ctypes.data_as(_capi.u32p)
        c.signs = signs.ctypes.data_as(_capi.i8p)
        c.fdeg = fdeg.ctypes.data_as(_capi.u32p)
        c.rank = rank.ctypes.data_as(_capi.u32p)
        out = _capi.stc_counts()
        o = self._opts(strategy, dispatch)
        _check(lib().stc_count_forward_csr(self._h, C.byref(c), C.byref(o), C.byref(out)), self._h)
        return GlobalTriCounts(out.t0, out.t1, out.t2, out.t3)

    def vertex_counts(self, src, dst, sign, *, strategy="auto", persistent=False) -> np.ndarray:
        """Per-source counts cnt[4n] (tc_serial.cpp:141-158) as an (n, 4) array."""
        src, dst, sign = _host_arrays(src, dst, sign)
        n_out = C.c_uint32()
        o = self._opts(strategy, persistent=persistent)
        n_bound = int(max(src.max(initial=0), dst.max(initial=0))) + 1 if len(src) else 0
        buf = np.zeros(4 * max(n_bound, 1), np.uint64)
        _check(lib().stc_vertex_counts(self._h, _ptr(src), _ptr(dst), _ptr(sign), len(src),
                                       C.byref(o), buf.ctypes.data_as(_capi.u64p), len(buf),
                                       C.byref(n_out)), self._h)
        return buf[: 4 * n_out.value].reshape(-1, 4)

    def count_batch(self, graphs: Sequence[tuple], *, strategy="auto", dispatch="fixed",
                    stream=None, persistent=True) -> list:
        """Counts independent graphs given as (src, dst, sign) triples."""
        keep = []
        arr = (_capi.stc_graph * max(1, len(graphs)))()
        dev = False
        for i, (s, d, g) in enumerate(graphs):
            dev = hasattr(s, "is_cuda") and s.is_cuda
            if not dev:
                s, d, g = _host_arrays(s, d, g)
            keep.append((s, d, g))
            arr[i].src = C.cast(_ptr(s), _capi.u32p)
            arr[i].dst = C.cast(_ptr(d), _capi.u32p)
            arr[i].sign = C.cast(_ptr(g), _capi.i8p)
            arr[i].m = int(s.numel()) if dev else len(s)
        outs = (_capi.stc_counts * max(1, len(graphs)))()
        if dev and stream is None:
            import torch
            stream = torch.cuda.current_stream(keep[0][0].device).cuda_stream
        o = self._opts(strategy, dispatch, dev, True, stream, persistent)
        _check(lib().stc_count_batch(self._h, arr, len(graphs), C.byref(o), outs), self._h)
        return [GlobalTriCounts(x.t0, x.t1, x.t2, x.t3) for x in outs[: len(graphs)]]

    def count_batch_packed(self, src, dst, sign, offsets, *, strategy="auto", dispatch="fixed",
                           stream=None, timing=True, persistent=True) -> list:
        """Counts graphs stored back to back (graph g owns entries
        [offsets[g], offsets[g + 1]), ids local to the graph); numpy arrays
        are host input, torch CUDA tensors device input."""
        offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
        G = len(offsets) - 1
        dev = hasattr(src, "is_cuda") and src.is_cuda
        if dev:
            if stream is None:
                import torch
                stream = torch.cuda.current_stream(src.device).cuda_stream
        else:
            src, dst, sign = _host_arrays(src, dst, sign)
        outs = (_capi.stc_counts * max(1, G))()
        o = self._opts(strategy, dispatch, dev, timing, stream, persistent)
        _check(lib().stc_count_batch_packed(self._h, _ptr(src), _ptr(dst), _ptr(sign),
                                            offsets.ctypes.data_as(_capi.u64p), G, C.byref(o),
                                            outs), self._h)
        return [GlobalTriCounts(x.t0, x.t1, x.t2, x.t3) for x in outs[:G]]

    # ------------------------------------------------------------ dispatcher
    def record_bucket_times(self, src, dst, sign, *, strategy="auto", dispatch="fixed"):
        """Timing recorder: counts like ``count`` with every arc timed alone.

        Returns (cycles, arcs, counts): per dispatch cell (``DISPATCH_CELLS``,
        index 256 class + 16 bucket|A'| + bucket|B|) the SM cycles spent on its
        arcs and their number, and the per-type counts."""
        src, dst, sign = _host_arrays(src, dst, sign)
        cycles = np.zeros(_capi.DISPATCH_CELLS, np.uint64)
        arcs = np.zeros(_capi.DISPATCH_CELLS, np.uint64)
        out = _capi.stc_counts()
        o = self._opts(strategy, dispatch)
        _check(lib().stc_record_bucket_times(self._h, _ptr(src), _ptr(dst), _ptr(sign), len(src),
                                             C.byref(o), cycles.ctypes.data_as(_capi.u64p),
                                             arcs.ctypes.data_as(_capi.u64p), C.byref(out)),
               self._h)
        return cycles, arcs, GlobalTriCounts(out.t0, out.t1, out.t2, out.t3)

    def train_dispatcher(self, features, targets, weights, *, epochs=3000, lr=0.02,
                         weight_decay=1e-3, seed=1):
        """Trains the dispatcher's perceptron on the device: features
        (samples, DISPATCH_FEATURES), targets (samples, DISPATCH_OUTPUTS)
        measured log2 cycles per arc of MERGE / HASH / SEARCH / SPLIT / HEAD (NaN =
        unavailable), weights
        (samples,).  Returns (parameters, final weighted squared error)."""
        X = np.ascontiguousarray(features, np.float32)
        T = np.ascontiguousarray(targets, np.float32)
        w = np.ascontiguousarray(weights, np.float32)
        if (X.ndim != 2 or X.shape[1] != _capi.DISPATCH_FEATURES
                or T.shape != (len(X), _capi.DISPATCH_OUTPUTS) or w.shape != (len(X),)):
            raise ValueError("features (S, DISPATCH_FEATURES), targets (S, DISPATCH_OUTPUTS), "
                             "weights (S,)")
        params = np.zeros(_capi.DISPATCH_MODEL_PARAMS, np.float32)
        loss = C.c_float()
        _check(lib().stc_dispatcher_train(self._h, X.ctypes.data_as(_capi.f32p),
                                          T.ctypes.data_as(_capi.f32p), w.ctypes.data_as(_capi.f32p),
                                          len(X), epochs, lr, weight_decay, seed,
                                          params.ctypes.data_as(_capi.f32p), C.byref(loss)), self._h)
        return params, float(loss.value)

    def set_dispatch_model(self, params, support=None) -> None:
        """Loads a model (``DISPATCH_MODEL_PARAMS`` floats) for dispatch="learned";
        ``support`` (DISPATCH_CELLS booleans, or cell indices) limits its
        overrides of the fixed tables to those cells.  None unloads it
        (learned then falls back to the fixed tables)."""
        if params is None:
            _check(lib().stc_ctx_set_dispatch_model(self._h, None, None), self._h)
            return
        p = np.ascontiguousarray(params, np.float32)
        if p.shape != (_capi.DISPATCH_MODEL_PARAMS,):
            raise ValueError(f"a model has {_capi.DISPATCH_MODEL_PARAMS} parameters")
        mask = None
        if support is not None:
            sup = np.asarray(support)
            if sup.dtype == bool or sup.shape == (_capi.DISPATCH_CELLS,) and sup.max(initial=0) <= 1:
                mask = np.ascontiguousarray(sup, np.uint8)
            else:
                mask = np.zeros(_capi.DISPATCH_CELLS, np.uint8)
                mask[sup.astype(np.int64)] = 1
            if mask.shape != (_capi.DISPATCH_CELLS,):
                raise ValueError("support: DISPATCH_CELLS booleans or cell indices")
        _check(lib().stc_ctx_set_dispatch_model(self._h, p.ctypes.data_as(_capi.f32p),
                                                mask.ctypes.data_as(_capi.u8p)
                                                if mask is not None else None), self._h)

    def load_dispatch_model(self, path=None) -> dict:
        """Loads a model file written by ``dispatcher.save`` (default: the
        model shipped with the package) and returns its metadata."""
        from . import dispatcher
        model = dispatcher.load(path)
        self.set_dispatch_model(model["params"], model.get("support"))
        return model

    def dispatch_tables(self, dispatch="fixed") -> np.ndarray:
        """The tables (class, bucket|A'|, bucket|B|) -> strategy code that a call
        with strategy="auto" and this dispatch uses, as a (4, 16, 16) array."""
        t = np.zeros(_capi.DISPATCH_CELLS, np.uint8)
        _check(lib().stc_dispatch_tables(self._h, _capi.DISPATCH[dispatch],
                                         t.ctypes.data_as(_capi.u8p)), self._h)
        return t.reshape(4, 16, 16)

    # ------------------------------------------------------------- tuning
    def set_tuning(self, tuning: Optional[dict]) -> None:
        """Sets the staged classes' launch parameters (a dict with
        block_threads, hash_factor[3], unroll[3]); None restores the defaults."""
        if tuning is None:
            _check(lib().stc_ctx_set_tuning(self._h, None), self._h)
            return
        t = _capi.stc_tuning()
        t.block_threads = int(tuning["block_threads"])
        for i in range(3):
            t.hash_factor[i] = int(tuning["hash_factor"][i])
            t.unroll[i] = int(tuning["unroll"][i])
        _check(lib().stc_ctx_set_tuning(self._h, C.byref(t)), self._h)

    def get_tuning(self) -> dict:
        t = _capi.stc_tuning()
        _check(lib().stc_ctx_get_tuning(self._h, C.byref(t)), self._h)
        return {"block_threads": t.block_threads, "hash_factor": list(t.hash_factor),
                "unroll": list(t.unroll)}

    def autotune(self, src, dst, sign, *, reps=3, strategy="auto", dispatch="fixed") -> dict:
        """Runs the autotuner on one graph (host arrays); the result is set on
        the context and returned."""
        src, dst, sign = _host_arrays(src, dst, sign)
        t = _capi.stc_tuning()
        o = self._opts(strategy, dispatch, timing=False)
        _check(lib().stc_autotune(self._h, _ptr(src), _ptr(dst), _ptr(sign), len(src), C.byref(o),
                                  reps, C.byref(t)), self._h)
        return {"block_threads": t.block_threads, "hash_factor": list(t.hash_factor),
                "unroll": list(t.unroll)}

    def last_stats(self) -> Stats:
        s = _capi.stc_stats()
        _check(lib().stc_ctx_last_stats(self._h, C.byref(s)))
        return Stats(**{f: getattr(s, f) for f, _ in _capi.stc_stats._fields_})

    def synth_rmat_device(self, seed: int, scale: int, n: int, samples: int, a: float, b: float,
                          c: float, p_pos: float, src, dst, sign) -> None:
        """Fills device arrays (torch tensors) with stc_synth_rmat's samples."""
        _check(lib().stc_synth_rmat_device(self._h, seed, scale, n, samples, a, b, c, p_pos,
                                           _ptr(src), _ptr(dst), _ptr(sign)), self._h)


def dispatch_features() -> np.ndarray:
    """Features of every dispatch cell, (DISPATCH_CELLS, DISPATCH_FEATURES)
    float32, as the dispatcher's inference kernel computes them."""
    f = np.zeros((_capi.DISPATCH_CELLS, _capi.DISPATCH_FEATURES), np.float32)
    _check(lib().stc_dispatch_features(f.ctypes.data_as(_capi.f32p)))
    return f


from . import synth  # noqa: E402  (needs the names above)
