"""Host-side table builders of the CUDA library, run without a GPU
(tests/cpp/host_tables.cpp):

* the ADI one-wave kernel's staged Thomas-factor tables: the run of chunks
  whose entries are bit for bit equal (the kernel reads the run's first
  chunk for all of them, so its results cannot change) is found, holds, and
  is maximal -- on the benchmark grid, padded grids and a strongly diagonal
  matrix;
* the FFTSolver3D line kernel's twiddle table: its length per size and
  every exponent."""
import subprocess

from tests.cpp_build import build


def test_host_table_builders():
    exe = build("host_tables")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().endswith("OK"), r.stdout
    assert "adi n=1024 nw=1024 run=[7,128)" in r.stdout
