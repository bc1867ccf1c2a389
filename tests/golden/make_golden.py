"""Generates pointwise golden vectors by running the reference's own FMM.

    bash oracle/build_ref.sh && python tests/golden/make_golden.py

Each fixture is the output of the reference's LaplaceFMM::solve
(3dpp/src/fmm.cpp:13-81; compiled from its sources by oracle/build_ref.sh)
on seeded synthetic bodies, and for one fixture also its EwaldSolver
(3dpp/src/ewald.cpp).  Positions are given in the reference's box (centre 0,
half edge cycle/2).  Stored per fixture: x (n,3), q (n,), phi (n,), grad (n,3)
[, ewald_phi, ewald_grad] and the flags, in golden_<name>.npz.
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
BIN = os.path.join(ROOT, "oracle", "_ref", "rtfmm_ref_pass")

FIXTURES = [
    # name, n, P, ncrit, images, dipole_correction, divide_4pi, ewald, body kind
    ("c1_small", 1500, 6, 64, 3, 0, 1, True, "uniform"),
    ("free_p8", 1200, 8, 32, 0, 0, 1, False, "uniform"),
    ("clustered_i2", 1600, 5, 24, 2, 1, 0, False, "blobs"),
]


def bodies(kind, n, seed):
    rng = np.random.default_rng(seed)
    if kind == "uniform":
        x = rng.random((n, 3))
        q = rng.random(n) * 2 - 1
    else:
        c = rng.random((4, 3))
        x = np.mod(c[rng.integers(0, 4, n)] + 0.03 * rng.standard_normal((n, 3)), 1.0)
        q = np.where(rng.random(n) < 0.5, -1.0, 1.0)
    return x - 0.5, q - q.mean()


def main():
    if not os.path.exists(BIN):
        sys.exit("build the reference first: bash oracle/build_ref.sh")
    for k, (name, n, P, ncrit, images, dip, d4, ew, kind) in enumerate(FIXTURES):
        x, q = bodies(kind, n, 100 + k)
        with tempfile.TemporaryDirectory() as td:
            fin, fout, few = (os.path.join(td, s) for s in ("in.bin", "out.bin", "ew.bin"))
            np.concatenate([x, q[:, None]], axis=1).astype(np.float64).tofile(fin)
            cmd = [BIN, "--in", fin, "--out", fout, "-n", str(n), "-P", str(P), "-m", str(ncrit),
                   "-i", str(images), "-c", "1", "--th_num", "8", "--dipole_correction", str(dip),
                   "--divide_4pi", str(d4)]
            if ew:
                cmd += ["--ewald", few]
            subprocess.run(cmd, check=True, capture_output=True,
                           env=dict(os.environ, OPENBLAS_NUM_THREADS="1"))
            r = np.fromfile(fout).reshape(n, 4)
            extra = {}
            if ew:
                e = np.fromfile(few).reshape(n, 4)
                extra = {"ewald_phi": e[:, 0], "ewald_grad": e[:, 1:]}
        np.savez_compressed(os.path.join(HERE, "golden_%s.npz" % name), x=x, q=q, phi=r[:, 0], grad=r[:, 1:],
                            P=P, ncrit=ncrit, images=images, cycle=1.0, dipole_correction=dip, divide_4pi=d4,
                            **extra)
        print("wrote golden_%s.npz" % name)


if __name__ == "__main__":
    main()
