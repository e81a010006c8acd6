"""The reference arm of bench.py runs the reference's own build alone.

`bench.py --impl reference` times oracle/_ref (the reference's sources,
compiled unmodified) from the reference's own 1LPT of the configuration's white
noise; no library of this repository's product may be mapped into that
process. Run here on the smallest configuration (c1, 2 steps) on the CPU.
"""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libhyowon_ref.so")),
                    reason="the reference build is not present")
def test_reference_arm_loads_only_the_reference_build():
    env = dict(os.environ, OMP_NUM_THREADS="2")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--config", "c1", "--steps", "2"], cwd=ROOT, env=env,
                         capture_output=True, text=True, timeout=300, check=True).stdout
    line = json.loads([ln for ln in out.splitlines() if ln.startswith("{")][-1])
    assert line["impl"] == "reference"
    assert line["native_libraries"] == ["oracle/_ref/libhyowon_ref.so"]
    assert line["value"] > 0 and line["steps"] == 2
    assert line["cpu_baseline"]["kind"] == "reference"
    assert line["e2e"]["h2d_bytes_per_step"] == 0
