"""The bench's reference arm (the reference's own CPU code, compiled from its
sources into oracle/_ref) runs on the host alone: its one JSON line carries
the keys and units of the device arm, and its counts are those of the
oracle's restatement on the same sample."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

import oracle

ROOT = Path(__file__).resolve().parent.parent


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref is not built")
def test_reference_arm_json_line():
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
                "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["unit"] == "edges/s" and d["higher_is_better"] is True and d["value"] > 0
    assert d["steps"] == 1 and d["warmup"] == 0
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == d["value"] and cb["cores"] >= 1
    assert cb["unit"] == d["unit"] and "RMAT scale 20" in cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    # The same sample through the oracle's restatement (single-threaded C,
    # about half a minute).
    sys.path.insert(0, str(ROOT))
    import bench
    from signed_triangle_counting_b200 import synth
    sc = bench.CPU_SAMPLE_SCALE
    el = synth.rmat(synth.workload_seed(3), sc, 1 << sc, 16 << sc, p_pos=0.5)
    assert tuple(d["counts"]) == oracle.count_arrays(el.src, el.dst, el.sign)
