"""The bench's reference arm on the CPU: `bench.py --impl reference` runs the
reference's own RHO (oracle/_ref, built from its sources) on the workload's
configuration and prints one JSON line with the contract's keys.  A small
size keeps it to seconds; it needs no GPU."""
from __future__ import annotations

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libtbref.so")


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="oracle/_ref not built")
def test_reference_arm_json_line():
    out = subprocess.run(
        [sys.executable, "bench.py", "--impl", "reference", "--steps", "2", "--warmup", "1",
         "--log2-r", "16", "--log2-s", "18"],
        cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [x for x in out.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["unit"] == "Mtuples/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["n_gpus"] == 1 and d["steps"] == 2 and d["warmup"] == 1
    # PK-FK at 100% selectivity: every S row matches once
    assert d["matches"] == 1 << 18
    assert d["config"]["nR"] == 1 << 16 and d["config"]["nS"] == 1 << 18
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == d["value"] and cb["cores"] >= 1
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
