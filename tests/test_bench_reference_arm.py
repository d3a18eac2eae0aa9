"""The bench's reference arm (`bench.py --impl reference`) times the
reference's algorithm through the CPU restatement alone: a short run prints
its JSON line, and the process never loads this library's libfd2.so (the
plan's geometry and flags come from the oracle's host restatements or the
reference's own fixture)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import runpy, sys
sys.argv = ['bench.py', '--impl', 'reference', '--beams', '8', '--steps', '1', '--warmup', '0', '--cpu-seconds', '1']
runpy.run_path('bench.py', run_name='__main__')
maps = open('/proc/self/maps').read()
print('MAPS', 'libfd2.so' in maps, 'liboracle' in maps)
"""


def test_reference_arm_runs_on_the_oracle_alone():
    out = subprocess.run([sys.executable, "-c", SCRIPT], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = out.stdout.strip().splitlines()
    line = json.loads([ln for ln in lines if ln.startswith("{")][-1])
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["e2e"]["h2d_bytes_per_step"] == 0
    assert "oracle's host restatement" in line["config"]["flags"]  # 8 beams: not the fixture's plan
    maps = [ln for ln in lines if ln.startswith("MAPS")][-1].split()
    assert maps[1] == "False", "the reference arm loaded libfd2.so"
    assert maps[2] == "True"
