"""The reference arm of bench.py on the host cores (no GPU): one JSON line
with the contract's keys, measured full solves of the reference algorithm at
16x16x8 that converge, and the operator samples of the larger grids."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "config",
              "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["value"] > 0 and d["unit"] == "solves/s" and d["higher_is_better"] is True
    assert d["converged"] is True and d["steps"] >= 5
    assert d["spread"]["min"] <= d["spread"]["median"] <= d["spread"]["max"]
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0
    ops = d["operator_apply_s"]
    assert ops["grid_64x64x16"]["median"] > 0 and ops["grid_128x128x32"]["median"] > 0
