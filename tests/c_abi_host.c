/* A plain C99 caller of the C ABI (include/rtfmm_b200.h), as a maintainer's
 * binding would be: create a solver, set up a body set on the host (tree,
 * lists, operator tables: no GPU), read the plan's sizes and set-up times,
 * save the operator tables, and check the error paths.  Compiled and run by
 * tests/test_c_abi.py; prints one line "ok <ncell> <nleaf> <n_p2p>". */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "rtfmm_b200.h"

static double lcg(uint64_t* s) {
  *s = *s * 6364136223846793005ull + 1442695040888963407ull;
  return (double)(*s >> 11) / 9007199254740992.0;
}

int main(int argc, char** argv) {
  const char* ops_path = argc > 1 ? argv[1] : "ops.bin";
  const int64_t n = 2000;
  double* x = (double*)malloc(sizeof(double) * 3 * n);
  double* q = (double*)malloc(sizeof(double) * n);
  uint64_t s = 7;
  double mean = 0;
  for (int64_t i = 0; i < n; ++i) {
    for (int k = 0; k < 3; ++k) x[3 * i + k] = lcg(&s);
    q[i] = 2 * lcg(&s) - 1;
    mean += q[i] / n;
  }
  for (int64_t i = 0; i < n; ++i) q[i] -= mean;

  rtfmm_args a;
  rtfmm_b200_default_args(&a);
  a.P = 5;
  a.ncrit = 32;
  a.images = 2;
  a.cycle = 1.0;
  a.x[0] = a.x[1] = a.x[2] = 0.5;
  a.dipole_correction = 0;
  a.divide_4pi = 1;

  rtfmm_fmm* h = NULL;
  if (rtfmm_b200_create(&a, &h) != RTFMM_OK) {
    printf("create failed: %s\n", rtfmm_b200_last_error());
    return 1;
  }
  /* out of order: no pass has run */
  double phi0;
  if (rtfmm_b200_download(h, &phi0, NULL) != RTFMM_ESTATE) {
    printf("download before setup was not refused\n");
    return 1;
  }
  if (rtfmm_b200_setup(h, n, x, q) != RTFMM_OK) {
    printf("setup failed: %s\n", rtfmm_b200_last_error());
    return 1;
  }
  int64_t info[12];
  memset(info, 0, sizeof(info));
  rtfmm_b200_info(h, info, 12);
  double st[6];
  if (rtfmm_b200_setup_times(h, st, 6) != RTFMM_OK || !(st[4] > 0)) {
    printf("setup times missing\n");
    return 1;
  }
  if (rtfmm_b200_save_operators(h, ops_path) != RTFMM_OK) {
    printf("save failed: %s\n", rtfmm_b200_last_error());
    return 1;
  }
  /* a non-finite position is refused with a message */
  x[5] = 0.0 / 0.0;
  if (rtfmm_b200_setup(h, n, x, q) != RTFMM_EINVAL || strlen(rtfmm_b200_last_error()) == 0) {
    printf("non-finite input was not refused\n");
    return 1;
  }
  rtfmm_b200_destroy(h);
  free(x);
  free(q);
  printf("ok %lld %lld %lld\n", (long long)info[0], (long long)info[1], (long long)info[4]);
  return 0;
}
