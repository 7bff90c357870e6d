"""Build recipe for libstc.so (sm_100a) and the `stc` command-line binary.

Everything is built in-tree: ``signed_triangle_counting_b200/libstc.so`` and
``signed_triangle_counting_b200/stc``; objects go to ``_build/``.  A source
is recompiled when it or any header is newer than its object.

    python -m signed_triangle_counting_b200.build [--force] [--verbose]
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = ROOT / "_build"
LIB = PKG / "libstc.so"
CLI = PKG / "stc"

NVCC = os.environ.get("STC_NVCC", "nvcc")
HOST_CXX = "/usr/bin/g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "-ccbin", HOST_CXX,
    "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
    f"-I{INCLUDE}", f"-I{CSRC}",
]
CXX_FLAGS = ["-O3", "-march=x86-64-v3", "-std=c++17", "-fPIC", "-Wall", "-Wno-unused-function",
             f"-I{INCLUDE}", f"-I{CSRC}"]

CUDA_SOURCES = ["capi.cu", "build.cu", "count.cu", "dispatch.cu", "text_gpu.cu"]
HOST_SOURCES = ["text_ingest.cpp", "mtx_ingest.cpp", "synth_host.cpp"]


def _headers() -> list[Path]:
    return sorted(list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h")))


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ... ({r.returncode})")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> Path:
    """Compiles libstc.so and the stc CLI; returns the library path."""
    BUILD.mkdir(exist_ok=True)
    headers = _headers()
    objs = []
    for src in CUDA_SOURCES:
        s = CSRC / src
        o = BUILD / (src + ".o")
        if force or _stale(o, [s] + headers):
            extra = ["-Xptxas", "-v"] if ptxas_verbose else []
            _run([NVCC, *NVCC_FLAGS, *extra, "-c", str(s), "-o", str(o)], verbose)
        objs.append(o)
    for src in HOST_SOURCES:
        s = CSRC / src
        o = BUILD / (src + ".o")
        if force or _stale(o, [s] + headers):
            _run([HOST_CXX, *CXX_FLAGS, "-c", str(s), "-o", str(o)], verbose)
        objs.append(o)
    if force or _stale(LIB, objs):
        _run([NVCC, *ARCH, "-ccbin", HOST_CXX, "-shared", "-o", str(LIB), *map(str, objs),
              "-lpthread"], verbose)
    cli_src = CSRC / "stc_cli.cpp"
    if force or _stale(CLI, [cli_src, LIB] + headers):
        _run([HOST_CXX, *CXX_FLAGS, str(cli_src), "-o", str(CLI), f"-L{PKG}", "-lstc",
              "-Wl,-rpath,$ORIGIN"], verbose)
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose, ptxas_verbose=a.ptxas_verbose))


if __name__ == "__main__":
    main()
