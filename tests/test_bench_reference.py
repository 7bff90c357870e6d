"""The bench's reference arm (the reference's own CPU code, compiled from its
sources into oracle/_ref) runs on the host alone and loads nothing from the
package: its one JSON line carries the keys, units and config of the device
arm, names the graph it sampled truly, and its sample's counts are those of
the oracle's restatement over the same sources."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

import oracle

ROOT = Path(__file__).resolve().parent.parent
SCALE = 16


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref is not built")
def test_reference_arm_json_line():
    probe = ("import runpy, sys; sys.argv = ['bench.py', '--impl', 'reference', '--rmat-scale', "
             f"'{SCALE}', '--steps', '2', '--warmup', '1']; runpy.run_path('bench.py', "
             "run_name='__main__'); "
             "print('LOADED', [m for m in sys.modules if m.startswith('signed_triangle')])")
    r = subprocess.run([sys.executable, "-c", probe], cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    # The reference arm imports nothing of the package (so maps none of its
    # native code).
    assert "LOADED []" in r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
                "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["unit"] == "edges/s" and d["higher_is_better"] is True and d["value"] > 0
    assert d["steps"] == 2 and d["warmup"] == 1
    cfg = d["config"]
    assert cfg["workload"].startswith(f"RMAT scale {SCALE},")
    assert cfg["m_input"] == 16 << SCALE
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == d["value"] and cb["cores"] >= 1
    assert cb["unit"] == d["unit"] and f"RMAT scale {SCALE} " in cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0

    # The same graph and sample through the oracle's restatement: the sample
    # is the sources with id < n / CPU_SAMPLE_DIV.
    sys.path.insert(0, str(ROOT))
    import bench
    src, dst, sign = oracle.synth_rmat(1003, SCALE, 1 << SCALE, 16 << SCALE)
    csr = oracle.ForwardCSR(src, dst, sign)
    assert cfg["m_unique"] == csr.m and cfg["n"] == csr.n
    n_s = csr.n // bench.CPU_SAMPLE_DIV
    want = csr.vertex_counts()[:n_s].sum(axis=0)
    assert [int(x) for x in want] == d["sample_counts"]
