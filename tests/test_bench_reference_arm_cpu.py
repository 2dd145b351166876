"""bench.py's reference arm on the CPU: one short step prints the contract's
JSON line (impl "reference", the GPU arm's metric and config, a
cpu_baseline describing the run, an e2e block with no host-device bytes),
and the process never loads the CUDA library."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WRAPPER = r"""
import runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0"]
try:
    runpy.run_path("bench.py", run_name="__main__")
except SystemExit as e:
    if e.code not in (None, 0):
        raise
with open("/proc/self/maps") as f:
    loaded = "libpaxpro_b200" in f.read()
print("CUDA_LIBRARY_LOADED=%d" % loaded)
"""


def test_reference_arm_line_and_no_cuda_library():
    r = subprocess.run([sys.executable, "-c", WRAPPER], cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert lines, r.stdout[-2000:]
    d = json.loads(lines[-1])
    assert d["impl"] == "reference"
    assert d["metric"] == "grid-pt*steps/s (plain FP64)"
    assert d["unit"] == "grid-pt*steps/s" and d["higher_is_better"] is True
    assert d["value"] > 0
    assert d["config"]["workload"].startswith("CrankNicholson Nx=4096 x 8000 steps + ADI 1024^2")
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["cpu_baseline"]["cores"] >= 1 and d["cpu_baseline"]["kind"] in ("reference", "port")
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert "CUDA_LIBRARY_LOADED=0" in r.stdout
