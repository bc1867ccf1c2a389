// GPU operator-build pieces against the host's, bit for bit: the Jacobi
// sweeps in one cooperative launch and as per-sweep graphs, and the kernel
// spectra.  Built and run by tests/test_gpu_precompute.py; prints one line
// per order and "OK" at the end, exits 1 on a difference.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "rtfmm_plan.h"
#include "rtfmm_precompute.h"

using namespace rtfmm_b200;

int main() {
  cudaStream_t st;
  if (cudaStreamCreate(&st) != cudaSuccess) return 2;
  int bad = 0;
  for (int P : {4, 6, 8}) {
    const int n = 6 * (P - 1) * (P - 1) + 2, m = n + (n & 1);
    // the check-to-equivalent matrix of build_operators, as columns of W
    std::vector<double> su;
    for (int i = 0; i < P; ++i)
      for (int j = 0; j < P; ++j)
        for (int k = 0; k < P; ++k)
          if (i == 0 || i == P - 1 || j == 0 || j == P - 1 || k == 0 || k == P - 1)
            for (int c : {i, j, k}) su.push_back(-1.0 + c * 2.0 / (P - 1));
    std::vector<double> W0((size_t)m * n, 0.0), V0((size_t)m * m, 0.0);
    for (int t = 0; t < n; ++t)
      for (int s = 0; s < n; ++s) {
        double d2 = 0;
        for (int k = 0; k < 3; ++k) {
          const double d = su[3 * t + k] * 2.95 - su[3 * s + k] * 1.05;
          d2 += d * d;
        }
        W0[(size_t)s * n + t] = 1.0 / std::sqrt(d2);
      }
    for (int j = 0; j < m; ++j) V0[(size_t)j * m + j] = 1.0;
    std::vector<double> Wh = W0, Vh = V0, Wc = W0, Vc = V0, Wg = W0, Vg = V0;
    jacobi_sweeps_host(n, Wh, Vh);
    const int sc = jacobi_sweeps_gpu(n, Wc, Vc, st, true);
    const int sg = jacobi_sweeps_gpu(n, Wg, Vg, st, false);
    const bool eq_c = !std::memcmp(Wh.data(), Wc.data(), 8 * Wh.size()) && !std::memcmp(Vh.data(), Vc.data(), 8 * Vh.size());
    const bool eq_g = !std::memcmp(Wh.data(), Wg.data(), 8 * Wh.size()) && !std::memcmp(Vh.data(), Vg.data(), 8 * Vh.size());
    // kernel spectra for a few offsets
    const int N = 2 * P - 1, Nf = N * N * (N / 2 + 1);
    const std::vector<int> offs = {2, 0, 0, -3, 1, 2, 4, -4, 0, 0, 0, -2};
    const int noff = (int)offs.size() / 3;
    std::vector<double> gh((size_t)noff * Nf * 2), gg(gh.size());
    const double r0 = 0.5, delta = 2 * r0 / (P - 1) * 1.05, gsize = r0 * 2 * 1.05;
    kernel_spectra_host(N, noff, offs.data(), r0, delta, gsize, gh.data());
    kernel_spectra_gpu(N, noff, offs.data(), r0, delta, gsize, gg.data(), st);
    const bool eq_s = !std::memcmp(gh.data(), gg.data(), 8 * gh.size());
    std::printf("P=%d sweeps one-launch %d graph %d equal %d %d spectra equal %d\n", P, sc, sg, eq_c, eq_g, eq_s);
    bad |= !(eq_c && eq_g && eq_s && sc > 0 && sg == -1);
  }
  std::printf(bad ? "FAILED\n" : "OK\n");
  return bad;
}
