"""The propagator's sin/cos (paxpro_b200/csrc/pxp_sincos.h, Cody-Waite
reduction + Taylor series) stays within one unit of 2^-52 of long-double
sinl/cosl on the phase range of the configurations and beyond."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_sincos_within_one_ulp():
    exe = os.path.join(ROOT, "_build", "sincos_check")
    os.makedirs(os.path.dirname(exe), exist_ok=True)
    subprocess.run(["/usr/bin/g++", "-std=c++17", "-O2",
                    os.path.join(ROOT, "tests", "cpp", "sincos_check.cpp"), "-o", exe], check=True)
    for n, xmax in ((200000, 2000.0), (100000, 1.0e5)):
        out = subprocess.run([exe, str(n), str(xmax)], capture_output=True, text=True,
                             check=True).stdout.split()
        assert float(out[0]) <= 1.0, out
