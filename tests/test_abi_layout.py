"""The Python mirror of the C ABI (ctypes structures in _capi.py) has the
C header's layout: every field at the offset and every struct at the size
that a C compiler gives them for include/stc.h and include/stc_synth.h.
A C program compiled here prints the offsets (no GPU, no libstc load)."""
import ctypes as C
import shutil
import subprocess
from pathlib import Path

import pytest

from signed_triangle_counting_b200 import _capi

ROOT = Path(__file__).resolve().parent.parent
STRUCTS = ["stc_counts", "stc_edge_list", "stc_forward_csr", "stc_graph", "stc_opts", "stc_stats",
           "stc_text_info", "stc_tuning", "stc_synth_graph", "stc_batch_spec"]


def _c_layout(tmp_path):
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "stc.h"', '#include "stc_synth.h"',
             'int main(void) {']
    for s in STRUCTS:
        lines.append(f'  printf("{s} size %zu\\n", sizeof({s}));')
        for name, _ in getattr(_capi, s)._fields_:
            lines.append(f'  printf("{s} {name} %zu\\n", offsetof({s}, {name}));')
    lines += ['  return 0;', '}']
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", f"-I{ROOT / 'include'}", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    return {tuple(ln.split()[:2]): int(ln.split()[2]) for ln in out.splitlines()}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_ctypes_mirror_matches_header(tmp_path):
    c = _c_layout(tmp_path)
    for s in STRUCTS:
        py = getattr(_capi, s)
        assert C.sizeof(py) == c[(s, "size")], s
        for name, _ in py._fields_:
            assert getattr(py, name).offset == c[(s, name)], (s, name)


def test_stats_field_names():
    names = [n for n, _ in _capi.stc_stats._fields_]
    assert "groups_replayed" in names and "probe_bytes" in names
