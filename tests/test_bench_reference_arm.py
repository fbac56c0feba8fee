"""bench.py's reference arm (the reference built from its sources, run on
the host cores) prints one well-formed JSON line; it needs no GPU."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_its_line():
    from oracle import ref_driver
    if not ref_driver.available():
        pytest.skip("reference build missing")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["dtype"] == "f64"
    assert line["e2e"]["value"] == line["value"] and line["cpu_baseline"]["kind"] == "reference"
