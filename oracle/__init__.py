"""ORACLE — test infrastructure, not product code.

Python access to
  * liboracle.so — the plain-C restatement of the reference CPU path
    (stc_oracle.c, every function citing the reference lines it follows), and
  * _ref/ — the reference's own programs and an in-memory harness, compiled
    from the reference sources by oracle/Makefile (present only where those
    sources were available at build time; the built files travel with the
    repository snapshot).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
package, and only as the checker / the timed CPU baseline.
"""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
REF_DIR = HERE / "_ref"
REF_HARNESS = REF_DIR / "libref_harness.so"
REF_PROGRAMS = ("tc_serial", "tc_merge_sign_enu", "tc_hash_sign_enu", "tc_merge_sign_split")

u32p = C.POINTER(C.c_uint32)
u64p = C.POINTER(C.c_uint64)
i8p = C.POINTER(C.c_int8)


class _EdgeList(C.Structure):
    _fields_ = [("n", C.c_uint32), ("lines", C.c_uint64), ("m", C.c_uint64), ("src", u32p),
                ("dst", u32p), ("sign", i8p)]


class _CSR(C.Structure):
    _fields_ = [("n", C.c_uint32), ("m", C.c_uint64), ("offsets", u64p), ("edges", u32p),
                ("signs", i8p), ("fdeg", u32p), ("rank", u32p)]


_lib = None
_ref = None


def build() -> None:
    """Runs oracle/Makefile: the C restatement, and _ref/ when the
    STC_REFERENCE_DIR environment variable names the reference's
    "Signed_TC/Multicore Implementations" directory."""
    cmd = ["make", "-s", "-C", str(HERE)]
    ref = os.environ.get("STC_REFERENCE_DIR")
    if ref:
        cmd.append(f"REF={ref}")
    subprocess.run(cmd, check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        L.orc_parse_text.argtypes = [C.c_char_p, C.c_uint64, C.POINTER(_EdgeList)]
        L.orc_load_graph.argtypes = [C.c_char_p, C.POINTER(_EdgeList)]
        L.orc_edge_list_from_arrays.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64,
                                                C.POINTER(_EdgeList)]
        L.orc_free_edge_list.argtypes = [C.POINTER(_EdgeList)]
        L.orc_build_forward_csr.argtypes = [C.POINTER(_EdgeList), C.POINTER(_CSR)]
        L.orc_free_forward_csr.argtypes = [C.POINTER(_CSR)]
        L.orc_count_triangles.argtypes = [C.POINTER(_CSR), u64p]
        L.orc_vertex_counts.argtypes = [C.POINTER(_CSR), u64p]
        L.orc_count_merge.argtypes = [C.POINTER(_CSR), u64p, u64p]
        L.orc_count_hash.argtypes = [C.POINTER(_CSR), u64p, u64p]
        L.orc_count_arrays.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, u64p]
        L.orc_synth_rmat.argtypes = [C.c_uint64, C.c_uint32, C.c_uint64, C.c_uint64, C.c_double,
                                     C.c_double, C.c_double, C.c_double, C.c_void_p, C.c_void_p,
                                     C.c_void_p]
        L.orc_write_edge_text.argtypes = [C.c_char_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_uint64]
        _lib = L
    return _lib


def _arr(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def _el_to_py(el: _EdgeList) -> dict:
    m = el.m
    get = (lambda p, t: np.ctypeslib.as_array(p, (m,)).copy()) if m else (lambda p, t: np.zeros(0, t))
    return dict(n=el.n, lines=el.lines, m=m, src=get(el.src, np.uint32), dst=get(el.dst, np.uint32),
                sign=get(el.sign, np.int8))


def parse_text(data: bytes) -> dict:
    el = _EdgeList()
    rc = lib().orc_parse_text(data, len(data), C.byref(el))
    assert rc == 0
    try:
        return _el_to_py(el)
    finally:
        lib().orc_free_edge_list(C.byref(el))


def load_graph(path) -> dict:
    el = _EdgeList()
    rc = lib().orc_load_graph(str(path).encode(), C.byref(el))
    if rc:
        raise OSError(f"cannot read {path}")
    try:
        return _el_to_py(el)
    finally:
        lib().orc_free_edge_list(C.byref(el))


class ForwardCSR:
    """The oracle's ForwardCSR, kept in C memory for the counting calls."""

    def __init__(self, src, dst, sign):
        src, dst, sign = _arr(src, np.uint32), _arr(dst, np.uint32), _arr(sign, np.int8)
        el = _EdgeList()
        assert lib().orc_edge_list_from_arrays(src.ctypes.data, dst.ctypes.data, sign.ctypes.data,
                                               len(src), C.byref(el)) == 0
        self._c = _CSR()
        rc = lib().orc_build_forward_csr(C.byref(el), C.byref(self._c))
        lib().orc_free_edge_list(C.byref(el))
        assert rc == 0

    def __del__(self):
        if getattr(self, "_c", None) is not None:
            lib().orc_free_forward_csr(C.byref(self._c))
            self._c = None

    @property
    def n(self):
        return self._c.n

    @property
    def m(self):
        return self._c.m

    def arrays(self) -> dict:
        n, m = self._c.n, self._c.m
        g = lambda p, k, t: np.ctypeslib.as_array(p, (k,)).copy() if k else np.zeros(0, t)
        return dict(n=n, m=m, offsets=g(self._c.offsets, n + 1, np.uint64),
                    edges=g(self._c.edges, m, np.uint32), signs=g(self._c.signs, m, np.int8),
                    fdeg=g(self._c.fdeg, n, np.uint32), rank=g(self._c.rank, n, np.uint32))

    def count(self) -> tuple:
        t = (C.c_uint64 * 4)()
        lib().orc_count_triangles(C.byref(self._c), t)
        return tuple(t)

    def vertex_counts(self) -> np.ndarray:
        out = np.zeros(4 * max(1, self._c.n), np.uint64)
        lib().orc_vertex_counts(C.byref(self._c), out.ctypes.data_as(u64p))
        return out[: 4 * self._c.n].reshape(-1, 4)

    def count_merge(self) -> tuple:
        b, u = C.c_uint64(), C.c_uint64()
        lib().orc_count_merge(C.byref(self._c), C.byref(b), C.byref(u))
        return b.value, u.value

    def count_hash(self) -> tuple:
        b, u = C.c_uint64(), C.c_uint64()
        assert lib().orc_count_hash(C.byref(self._c), C.byref(b), C.byref(u)) == 0
        return b.value, u.value


def count_arrays(src, dst, sign) -> tuple:
    """(t0, t1, t2, t3) of the oracle for an edge list."""
    src, dst, sign = _arr(src, np.uint32), _arr(dst, np.uint32), _arr(sign, np.int8)
    t = (C.c_uint64 * 4)()
    assert lib().orc_count_arrays(src.ctypes.data, dst.ctypes.data, sign.ctypes.data, len(src), t) == 0
    return tuple(t)


def synth_rmat(seed: int, scale: int, n: int, samples: int, a=0.57, b=0.19, c=0.19,
               p_pos=0.5) -> tuple:
    """The package's seeded RMAT generator restated in C (synth_rmat.c):
    (src, dst, sign) arrays equal to signed_triangle_counting_b200.synth.rmat's
    for the same arguments, made without loading the package's library."""
    src = np.empty(samples, np.uint32)
    dst = np.empty(samples, np.uint32)
    sign = np.empty(samples, np.int8)
    rc = lib().orc_synth_rmat(seed, scale, n, samples, a, b, c, p_pos, src.ctypes.data,
                              dst.ctypes.data, sign.ctypes.data)
    if rc != 0:
        raise ValueError(f"orc_synth_rmat rejected its arguments ({rc})")
    return src, dst, sign


def write_edge_text(path, src, dst, sign) -> None:
    """`u v sign` lines (sign 1 / -1), the reference programs' input format."""
    src, dst, sign = _arr(src, np.uint32), _arr(dst, np.uint32), _arr(sign, np.int8)
    rc = lib().orc_write_edge_text(str(path).encode(), src.ctypes.data, dst.ctypes.data,
                                   sign.ctypes.data, len(src))
    if rc != 0:
        raise OSError(f"writing {path} failed ({rc})")


# ------------------------------------------------------- reference (_ref) --
def ref_available() -> bool:
    return REF_HARNESS.exists() and all((REF_DIR / p).exists() for p in REF_PROGRAMS)


def _ref_lib() -> C.CDLL:
    global _ref
    if _ref is None:
        L = C.CDLL(str(REF_HARNESS))
        L.stc_ref_count_arrays.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, u64p,
                                           C.POINTER(C.c_double), u64p]
        L.stc_ref_forward_csr.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64,
                                          u32p, u64p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_void_p]
        L.stc_ref_prepare.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64,
                                      C.POINTER(C.c_double), u32p, u64p]
        L.stc_ref_prefix_size.argtypes = [C.c_uint32, u64p, u64p]
        L.stc_ref_count_prefix.argtypes = [C.c_uint32, u64p, C.POINTER(C.c_double)]
        L.stc_ref_release.argtypes = []
        L.stc_ref_threads.argtypes = []
        _ref = L
    return _ref


def ref_count_arrays(src, dst, sign, with_edges: bool = False) -> tuple:
    """Reference's build_forward_csr + sort_adj_lists + count_triangles on
    arrays: ((t0, t1, t2, t3), (build_s, sort_s, count_s)[, forward_edges])."""
    src, dst, sign = _arr(src, np.uint32), _arr(dst, np.uint32), _arr(sign, np.int8)
    t = (C.c_uint64 * 4)()
    sec = (C.c_double * 3)()
    fe = C.c_uint64()
    rc = _ref_lib().stc_ref_count_arrays(src.ctypes.data, dst.ctypes.data, sign.ctypes.data,
                                         len(src), t, sec, C.byref(fe))
    assert rc == 0
    if with_edges:
        return tuple(t), tuple(sec), fe.value
    return tuple(t), tuple(sec)


def ref_forward_csr(src, dst, sign) -> dict:
    src, dst, sign = _arr(src, np.uint32), _arr(dst, np.uint32), _arr(sign, np.int8)
    n, m = C.c_uint32(), C.c_uint64()
    L = _ref_lib()
    assert L.stc_ref_forward_csr(src.ctypes.data, dst.ctypes.data, sign.ctypes.data, len(src),
                                 C.byref(n), C.byref(m), None, None, None, None, None) == 0
    N, M = n.value, m.value
    out = dict(n=N, m=M, offsets=np.zeros(N + 1, np.uint64), edges=np.zeros(max(M, 1), np.uint32),
               signs=np.zeros(max(M, 1), np.int8), fdeg=np.zeros(max(N, 1), np.uint32),
               rank=np.zeros(max(N, 1), np.uint32))
    assert L.stc_ref_forward_csr(src.ctypes.data, dst.ctypes.data, sign.ctypes.data, len(src),
                                 C.byref(n), C.byref(m), out["offsets"].ctypes.data,
                                 out["edges"].ctypes.data, out["signs"].ctypes.data,
                                 out["fdeg"].ctypes.data, out["rank"].ctypes.data) == 0
    out["edges"], out["signs"] = out["edges"][:M], out["signs"][:M]
    out["fdeg"], out["rank"] = out["fdeg"][:N], out["rank"][:N]
    return out


class RefKeptCSR:
    """The reference's forward CSR of one edge list, built and sorted once by
    its own build_forward_csr and sort_adj_lists and kept in the harness, so
    that count_triangles can be timed on samples of its sources.  One at a
    time per process."""

    def __init__(self, src, dst, sign):
        src, dst, sign = _arr(src, np.uint32), _arr(dst, np.uint32), _arr(sign, np.int8)
        sec = (C.c_double * 2)()
        n, fe = C.c_uint32(), C.c_uint64()
        L = _ref_lib()
        assert L.stc_ref_prepare(src.ctypes.data, dst.ctypes.data, sign.ctypes.data, len(src), sec,
                                 C.byref(n), C.byref(fe)) == 0
        self.n, self.m = n.value, fe.value
        self.build_s, self.sort_s = sec[0], sec[1]
        self.threads = int(L.stc_ref_threads())

    def prefix_size(self, n_sources: int) -> tuple:
        """(forward edges, merge work) of the sources with id < n_sources."""
        arcs, work = C.c_uint64(), C.c_uint64()
        assert _ref_lib().stc_ref_prefix_size(n_sources, C.byref(arcs), C.byref(work)) == 0
        return arcs.value, work.value

    def count_prefix(self, n_sources: int) -> tuple:
        """count_triangles over the sources with id < n_sources:
        ((t0, t1, t2, t3), seconds)."""
        t = (C.c_uint64 * 4)()
        sec = C.c_double()
        assert _ref_lib().stc_ref_count_prefix(n_sources, t, C.byref(sec)) == 0
        return tuple(t), sec.value

    def vertex_counts(self) -> np.ndarray:
        """The reference's per-source counts cnt[4n] (tc_serial.cpp:141-158),
        recovered as differences of prefix counts (one count per vertex: for
        small graphs only)."""
        out = np.zeros((self.n, 4), np.uint64)
        prev = np.zeros(4, np.uint64)
        for u in range(self.n):
            cur = np.array(self.count_prefix(u + 1)[0], np.uint64)
            out[u] = cur - prev
            prev = cur
        return out.reshape(-1)

    def close(self) -> None:
        _ref_lib().stc_ref_release()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


_NUM = r"(\d+)"
_PATTERNS = {
    "n": r"n=(\d+)\s+raw_edges=",
    "raw_edges": r"raw_edges=(\d+)",
    "forward_edges": r"forward_edges=(\d+)",
    "t3": r"T3 \(\+\+\+ balanced\)\s*:\s*(\d+)",
    "t1": r"T1 \(\+-- balanced\)\s*:\s*(\d+)",
    "t2": r"T2 \(\+\+- unbalanced\)\s*:\s*(\d+)",
    "t0": r"T0 \(--- unbalanced\)\s*:\s*(\d+)",
    "balanced": r"Balanced\s+=\s+(\d+)",
    "unbalanced": r"Unbalanced\s+=\s+(\d+)",
    "total": r"Total\s+=\s+(\d+)",
    "count_s": r"\[Triangle Counting Execution\] took ([0-9.]+) seconds",
    "build_s": r"\[Build Forward CSR\] took ([0-9.]+) seconds",
    "total_s": r"\[Total execution time\] took ([0-9.]+) seconds",
}


def parse_program_output(text: str) -> dict:
    out = {}
    for k, pat in _PATTERNS.items():
        mm = re.search(pat, text)
        if mm:
            out[k] = float(mm.group(1)) if k.endswith("_s") else int(mm.group(1))
    return out


def run_ref_program(name: str, path, threads: int | None = None, timeout: float = 3600) -> dict:
    """Runs one of the reference's compiled programs on a text file."""
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    r = subprocess.run([str(REF_DIR / name), str(path)], capture_output=True, text=True, env=env,
                       timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"{name} failed ({r.returncode}): {r.stderr[-500:]}")
    res = parse_program_output(r.stdout)
    res["stdout"] = r.stdout
    return res
