"""Compile the C++ API examples of tests/cpp against include/ and the in-tree
library (used by the tests; the examples mirror the reference's usage)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "paxpro_b200", "lib")
OUT = os.path.join(ROOT, "_build", "cpp")


def build(name: str) -> str:
    os.makedirs(OUT, exist_ok=True)
    src = os.path.join(ROOT, "tests", "cpp", name + ".cpp")
    exe = os.path.join(OUT, name)
    cmd = ["/usr/bin/g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I" + os.path.join(ROOT, "include"),
           src, "-L" + LIBDIR, "-lpaxpro_b200", "-Wl,-rpath," + LIBDIR, "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(r.stderr)
    return exe
