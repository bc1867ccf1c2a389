"""Generates the sampled golden vectors of the headline workload by running
the reference's own FMM at full size.

    bash oracle/build_ref.sh && python tests/golden/make_golden_c2.py

Workload: N = 2^20 bodies i.i.d. uniform in [0,1)^3 with charges uniform in
[-1,1] shifted to zero net charge, drawn by numpy's default_rng(2) (positions
first, then charges), P = 8, ncrit = 256, 3 image levels, cycle 1, kernel
1/(4 pi r), no dipole correction.  The reference's LaplaceFMM::solve
(3dpp/src/fmm.cpp:13-81, compiled from its sources by oracle/build_ref.sh)
runs on all bodies, shifted into its box (centre 0, half edge 1/2); its
outputs are kept at 4096 sampled bodies, with whole-array sums, so that the
fixture stays small:

  idx (4096,) int64      sampled body indices (default_rng(21))
  phi, grad              the reference's potential and gradient there
  x_head                 the first 4 positions, to check that the bodies
                         regenerated from the seed are these
  phi_mean, phi_norm_mr  mean of phi over all bodies, and the L2 norm of
                         phi - mean (for mean-removed comparisons)
  grad_norm              L2 norm of the whole gradient
  fmm_kernels_s, threads the reference's FMM_kernels timer, and its threads
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
BIN = os.path.join(ROOT, "oracle", "_ref", "rtfmm_ref_pass")
N, P, NCRIT, IMAGES, SEED, NSAMPLE = 1 << 20, 8, 256, 3, 2, 4096


def bodies():
    rng = np.random.default_rng(SEED)
    x = rng.random((N, 3))
    q = rng.random(N) * 2 - 1
    return x, q - q.mean()


def sample_idx():
    return np.sort(np.random.default_rng(21).choice(N, NSAMPLE, replace=False))


def main():
    if not os.path.exists(BIN):
        sys.exit("build the reference first: bash oracle/build_ref.sh")
    threads = os.cpu_count() or 1
    x, q = bodies()
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        np.concatenate([x - 0.5, q[:, None]], axis=1).astype(np.float64).tofile(fin)
        cmd = [BIN, "--in", fin, "--out", fout, "-n", str(N), "-P", str(P), "-m", str(NCRIT), "-i", str(IMAGES),
               "-c", "1", "--th_num", str(threads), "--dipole_correction", "0", "--divide_4pi", "1"]
        out = subprocess.run(cmd, check=True, capture_output=True, text=True,
                             env=dict(os.environ, OPENBLAS_NUM_THREADS="1")).stdout
        r = np.fromfile(fout).reshape(N, 4)
    t = None
    for line in out.splitlines():
        if line.startswith("[FMM_kernels time measured"):
            t = float(line.split(":")[1].split()[0])
    idx = sample_idx()
    phi, grad = r[:, 0], r[:, 1:]
    np.savez_compressed(os.path.join(HERE, "golden_c2_sampled.npz"), idx=idx, phi=phi[idx], grad=grad[idx],
                        x_head=x[:4], phi_mean=phi.mean(), phi_norm_mr=np.linalg.norm(phi - phi.mean()),
                        grad_norm=np.linalg.norm(grad), fmm_kernels_s=t, threads=threads, N=N, P=P, ncrit=NCRIT,
                        images=IMAGES, seed=SEED)
    print("wrote golden_c2_sampled.npz (FMM_kernels %.3f s on %d threads)" % (t, threads))


if __name__ == "__main__":
    main()
