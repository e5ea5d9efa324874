"""The reference arm of bench.py (`--impl reference`) on the host cores: one JSON line with the
contract's keys, the requested steps and warm-ups, a cpu_baseline describing the run and an
e2e object without host-device bytes. Runs the reference's own CPU build (oracle/_ref) on a
bounded sample; no GPU."""

import json
import os
import subprocess
import sys

import pytest

from conftest import has_reference_build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(not has_reference_build(), reason="reference build missing")
def test_reference_arm_prints_one_contract_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--workload", "singlet", "--steps", "2", "--warmup", "1"],
                         cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["steps"] == 2 and d["warmup"] == 1
    for k in ("metric", "value", "unit", "n_gpus", "higher_is_better", "scaling", "dtype",
              "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["value"] > 0 and d["cpu_baseline"]["value"] == d["value"]
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["e2e"]["unit"] == d["unit"]
