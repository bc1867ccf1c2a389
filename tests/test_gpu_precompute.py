"""The GPU operator build's pieces against the host's, bit for bit, through
the library's own functions: the Jacobi sweeps in one cooperative launch and
in the per-sweep graph form that takes over when a cooperative launch is
refused, and the kernel spectra (tests/precompute_harness.cpp)."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "exafmm-rd_b200")


def test_jacobi_and_spectra_equal_host(pkg, tmp_path):
    pkg.rtfmm.lib()  # the library is built
    exe = str(tmp_path / "precompute_harness")
    subprocess.run(["/usr/local/cuda/bin/nvcc", "-std=c++17", "-O2", "-I", os.path.join(PKG, "csrc"),
                    os.path.join(ROOT, "tests", "precompute_harness.cpp"), "-o", exe, "-L", PKG, "-lrtfmm_b200",
                    "-Xlinker", "-rpath," + PKG, "-Xcompiler", "-fopenmp"], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    print(out.stdout)
    assert out.returncode == 0 and out.stdout.strip().endswith("OK"), out.stdout + out.stderr
