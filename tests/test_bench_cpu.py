"""The bench's reference arm keeps the JSON-line contract (CPU: it times the reference's own
compiled CPU implementation; skipped where those modules are not built)."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def test_reference_arm_line(tmp_path):
    if not any((ROOT / "oracle" / "_ref").glob("em*.so")):
        pytest.skip("the reference's CPU modules are not built here")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--config", "c1",
                        "--steps", "3", "--warmup", "3"], capture_output=True, text=True, timeout=600, cwd=tmp_path)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["steps"] == 3 and d["warmup"] == 3 and d["higher_is_better"] is True
    assert d["value"] > 0 and abs(d["ms_per_step"] * d["value"] - 1000.0) < 1e-6 * 1000.0
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert "workload" in d["config"]


def test_warmup_below_three_is_raised_to_three(tmp_path):
    if not any((ROOT / "oracle" / "_ref").glob("em*.so")):
        pytest.skip("the reference's CPU modules are not built here")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--config", "c1",
                        "--steps", "1", "--warmup", "1"], capture_output=True, text=True, timeout=600, cwd=tmp_path)
    assert "--warmup must be >= 3" in (r.stdout + r.stderr)
    d = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("{")][0])
    assert d["warmup"] == 3
