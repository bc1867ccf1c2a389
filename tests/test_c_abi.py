"""The C ABI from plain C99 (no GPU): tests/c_abi_host.c is compiled with gcc
against include/rtfmm_b200.h and linked to the library, then run.  It
creates a solver, sets up a body set on the host, reads the plan's sizes and
set-up times, saves the operator tables and checks the error paths; the
sizes must equal what the Python binding sees for the same bodies, and the
saved tables must load back."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def lcg_bodies(n, seed):
    # the C program's generator
    s = seed
    mask = (1 << 64) - 1
    vals = []
    for _ in range(4 * n):
        s = (s * 6364136223846793005 + 1442695040888963407) & mask
        vals.append((s >> 11) / 9007199254740992.0)
    v = np.array(vals).reshape(n, 4)
    x = v[:, :3].copy()
    q = 2 * v[:, 3] - 1
    return x, q - q.mean()


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_c99_caller(pkg, tmp_path):
    lib_dir = os.path.join(ROOT, "exafmm-rd_b200")
    exe = str(tmp_path / "c_abi_host")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c_abi_host.c"), "-o", exe, "-L", lib_dir, "-lrtfmm_b200",
                    "-Wl,-rpath," + lib_dir], check=True)
    ops = str(tmp_path / "ops.bin")
    out = subprocess.run([exe, ops], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    words = out.stdout.split()
    assert words[0] == "ok", out.stdout
    ncell, nleaf, n_p2p = (int(w) for w in words[1:4])
    x, q = lcg_bodies(2000, 7)
    f = pkg.LaplaceFMM(x, q, pkg.Argument(P=5, ncrit=32, images=2, cycle=1.0, x=(0.5, 0.5, 0.5),
                                          dipole_correction=0, divide_4pi=1))
    f.setup()
    info = f.info()
    assert (ncell, nleaf, n_p2p) == (info["ncell"], info["nleaf"], info["n_p2p"])
    pkg.clear_operator_cache()
    pkg.load_operators(ops)
    ns = 6 * 4 ** 2 + 2
    g = pkg.LaplaceFMM(x, q, pkg.Argument(P=5, ncrit=32, images=2, cycle=1.0, x=(0.5, 0.5, 0.5)))
    g.setup()
    assert np.array_equal(f.operator(1, 8 * ns * ns), g.operator(1, 8 * ns * ns))
    pkg.clear_operator_cache()
    f.close()
    g.close()
