"""bench.py's reference arm runs on the host cores alone (the float64 oracle
of the reference path timed on a bounded sample), so its JSON contract can be
checked without a GPU: one line with the fields the driver reads, the
reference arm's own `cpu_baseline`, and an `e2e` object with no host-device
traffic.  A small n keeps the sample to a few seconds.
"""

import json
import subprocess
import sys
from pathlib import Path

REPO = Path(__file__).resolve().parents[1]


def test_reference_arm_json_line():
    out = subprocess.run(
        [sys.executable, str(REPO / "bench.py"), "--impl", "reference", "--n", "3000", "--steps", "1",
         "--warmup", "0", "--ref-sample-s", "0.3"],
        cwd=REPO, capture_output=True, text=True, timeout=600, check=True)
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    for key in ("metric", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config"):
        assert key in d, key
    assert d["value"] > 0 and d["unit"] == "solves/s" and d["higher_is_better"] is True
    assert abs(d["ms_per_step"] - 1e3 / d["value"]) <= 1e-6 * d["ms_per_step"]
    assert "n=3000" in d["config"]["workload"] and "extrapolated" in d["config"]["method"]
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] in ("port", "reference") and cb["cores"] >= 1
    assert cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
