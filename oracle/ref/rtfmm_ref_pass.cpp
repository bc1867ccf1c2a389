// Driver for the reference's own FMM (mumairsadiq/exafmm-rd, 3dpp), compiled
// from its unmodified sources by oracle/build_ref.sh.  Test infrastructure:
// it produces the reference outputs the oracle and the GPU path are checked
// against, and the CPU timings bench.py reports.
//
//   rtfmm_ref_pass --in bodies.bin [--out result.bin] [--ewald ewald.bin]
//                  <reference flags: -n N -P P -m ncrit -i images -c cycle ...>
//
// bodies.bin: n records of 4 doubles (x, y, z, q), positions in the
// reference's box (centre 0, half edge cycle/2).  result.bin: n records of 4
// doubles (p, fx, fy, fz) in input order, as LaplaceFMM::solve returns them
// (3dpp/src/fmm.cpp:13-81).  The reference prints its own stage timers.
#include <omp.h>

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "argument.h"
#include "body.h"
#include "ewald.h"
#include "fmm.h"

int main(int argc, char* argv[]) {
  std::string fin, fout, fewald;
  std::vector<char*> rest;
  rest.push_back(argv[0]);
  for (int i = 1; i < argc; ++i) {
    if (!std::strcmp(argv[i], "--in") && i + 1 < argc) {
      fin = argv[++i];
    } else if (!std::strcmp(argv[i], "--out") && i + 1 < argc) {
      fout = argv[++i];
    } else if (!std::strcmp(argv[i], "--ewald") && i + 1 < argc) {
      fewald = argv[++i];
    } else {
      rest.push_back(argv[i]);
    }
  }
  rtfmm::Argument args((int)rest.size(), rest.data());
  omp_set_dynamic(0);
  omp_set_num_threads(args.th_num);
  rtfmm::Bodies3 bs(args.n);
  FILE* f = std::fopen(fin.c_str(), "rb");
  if (!f) {
    std::fprintf(stderr, "cannot open %s\n", fin.c_str());
    return 2;
  }
  std::vector<double> buf(4 * (size_t)args.n);
  if (std::fread(buf.data(), sizeof(double), buf.size(), f) != buf.size()) {
    std::fprintf(stderr, "short read\n");
    return 2;
  }
  std::fclose(f);
  for (int i = 0; i < args.n; ++i) {
    bs[i].idx = i;
    bs[i].x = rtfmm::vec3r(buf[4 * i], buf[4 * i + 1], buf[4 * i + 2]);
    bs[i].q = buf[4 * i + 3];
    bs[i].p = 0;
    bs[i].f = rtfmm::vec3r(0, 0, 0);
  }
  rtfmm::LaplaceFMM fmm(bs, args);
  rtfmm::Bodies3 res = fmm.solve();
  auto dump = [&](const std::string& path, const rtfmm::Bodies3& r) {
    FILE* o = std::fopen(path.c_str(), "wb");
    for (int i = 0; i < args.n; ++i) {
      double v[4] = {r[i].p, r[i].f[0], r[i].f[1], r[i].f[2]};
      std::fwrite(v, sizeof(double), 4, o);
    }
    std::fclose(o);
  };
  if (!fout.empty()) dump(fout, res);
  if (!fewald.empty()) {
    rtfmm::EwaldSolver ewald(bs, args);
    rtfmm::Bodies3 e = ewald.solve();
    if (args.divide_4pi) rtfmm::scale_bodies(e);
    dump(fewald, e);
  }
  return 0;
}
