// Driver for the reference's own FMM (mumairsadiq/exafmm-rd, 3dpp), compiled
// from its unmodified sources by oracle/build_ref.sh.  Test infrastructure:
// it produces the reference outputs the oracle and the GPU path are checked
// against, and the CPU timings bench.py reports.
//
//   rtfmm_ref_pass --in bodies.bin [--out result.bin] [--ewald ewald.bin]
//                  [--repeat K]
//                  <reference flags: -n N -P P -m ncrit -i images -c cycle ...>
//
// --repeat K: build the tree, lists and operator tables once, exactly as
// LaplaceFMM::solve does (fmm.cpp:15-49), then run the solver's own hot block
// (its P2M, M2M, M2L, P2L, L2L, L2P, M2P and P2P methods, fmm.cpp:51-60) K
// times on zeroed cell matrices and body outputs, printing each pass's wall
// seconds as "[repeat_pass k seconds]"; the last pass's outputs get the
// solver's post-processing (fmm.cpp:75-80) and are written as with one
// solve().  The set-up at N = 2^20 costs the reference about ten times the
// pass (its M2L parent map is O(27 C^2)), so timing passes this way keeps a
// run of several steps within minutes.
//
// bodies.bin: n records of 4 doubles (x, y, z, q), positions in the
// reference's box (centre 0, half edge cycle/2).  result.bin: n records of 4
// doubles (p, fx, fy, fz) in input order, as LaplaceFMM::solve returns them
// (3dpp/src/fmm.cpp:13-81).  The reference prints its own stage timers.
#include <omp.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "argument.h"
#include "body.h"
#include "ewald.h"
#include "kernel.h"
#include "traverser.h"
#include "tree.h"
// The solver's stage methods and members are private; the repeat mode calls
// them directly (every other header is already included, so only the
// LaplaceFMM declaration is read this way).
#define private public
#include "fmm.h"
#undef private

int main(int argc, char* argv[]) {
  std::string fin, fout, fewald;
  int repeat = 0;
  std::vector<char*> rest;
  rest.push_back(argv[0]);
  for (int i = 1; i < argc; ++i) {
    if (!std::strcmp(argv[i], "--in") && i + 1 < argc) {
      fin = argv[++i];
    } else if (!std::strcmp(argv[i], "--out") && i + 1 < argc) {
      fout = argv[++i];
    } else if (!std::strcmp(argv[i], "--ewald") && i + 1 < argc) {
      fewald = argv[++i];
    } else if (!std::strcmp(argv[i], "--repeat") && i + 1 < argc) {
      repeat = std::atoi(argv[++i]);
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
  rtfmm::Bodies3 res;
  if (repeat <= 0) {
    res = fmm.solve();
  } else {
    // set-up, in solve()'s order (fmm.cpp:15-49)
    double t0 = omp_get_wtime();
    rtfmm::Tree tree;
    tree.build(fmm.bs, args.x, args.r, args.ncrit, rtfmm::Tree::TreeType::nonuniform);
    fmm.cs = tree.get_cells();
    fmm.traverser.traverse(tree, args.cycle, args.images);
    fmm.cs = fmm.traverser.get_cells();
    fmm.tree_depth_range = fmm.get_min_max_depth(fmm.cs);
    fmm.init_cell_matrix(fmm.cs);
    if (args.use_precompute) {
      fmm.kernel.precompute(args.P, args.r, args.images);
      fmm.kernel.precompute_m2l(args.P, args.r, fmm.cs, fmm.traverser.get_map(rtfmm::OperatorType::M2L),
                                args.images);
    }
    std::printf("[repeat_setup %.5f seconds]\n", omp_get_wtime() - t0);
    for (int k = 0; k < repeat; ++k) {
      fmm.init_cell_matrix(fmm.cs);
      for (auto& b : fmm.bs) {
        b.p = 0;
        b.f = rtfmm::vec3r(0, 0, 0);
      }
      const double ts = omp_get_wtime();
      fmm.P2M();
      fmm.M2M();
      fmm.M2L();
      fmm.P2L();
      fmm.L2L();
      fmm.L2P();
      fmm.M2P();
      fmm.P2P();
      std::printf("[repeat_pass %d %.6f seconds]\n", k, omp_get_wtime() - ts);
      std::fflush(stdout);
    }
    // post-processing (fmm.cpp:75-80)
    if (args.dipole_correction) rtfmm::dipole_correction(fmm.bs, args.cycle);
    if (args.divide_4pi) rtfmm::scale_bodies(fmm.bs);
    res = rtfmm::sort_bodies_by_idx(fmm.bs);
  }
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
