// DFT implementation of the FFTW3 calls the reference makes (see fftw3.h in
// this directory).  Written for this repository; test infrastructure for
// building the reference, not part of the product.
//
// Each axis is a dense DFT applied as a small matrix product whose innermost
// loop runs over the contiguous trailing dimensions, so the compiler
// vectorises it; twiddle matrices are built once per plan in double.
#include "fftw3.h"

#include <cmath>
#include <cstring>
#include <vector>

struct fftw_plan_s {
  int rank, n[3], howmany, idist, odist, r2c;
  double *in, *out;
  // per dimension: cos / sin of 2 pi k j / n, row-major [k][j]
  std::vector<double> c[3], s[3];
};

static fftw_plan make(int rank, const int* n, int howmany, double* in, int idist, double* out, int odist, int r2c) {
  fftw_plan p = new fftw_plan_s();
  p->rank = rank;
  for (int k = 0; k < 3; ++k) p->n[k] = 1;
  // FFTW's dims: the last one is the contiguous (halved) one; store as n[0..2]
  for (int k = 0; k < rank; ++k) p->n[3 - rank + k] = n[k];
  p->howmany = howmany;
  p->idist = idist;
  p->odist = odist;
  p->r2c = r2c;
  p->in = in;
  p->out = out;
  for (int d = 0; d < 3; ++d) {
    const int m = p->n[d];
    p->c[d].resize((size_t)m * m);
    p->s[d].resize((size_t)m * m);
    for (int k = 0; k < m; ++k)
      for (int j = 0; j < m; ++j) {
        const long t = ((long)k * j) % m;
        p->c[d][(size_t)k * m + j] = std::cos(2.0 * M_PI * t / m);
        p->s[d][(size_t)k * m + j] = std::sin(2.0 * M_PI * t / m);
      }
  }
  return p;
}

// complex DFT along axis d (0 or 1) of a split re/im array shaped
// [n0][n1][h]; sign -1 forward, +1 inverse.  out may not alias in.
static void axis(const fftw_plan p, int d, int h, const double* ir, const double* ii, double* orr, double* oi,
                 int sign) {
  const int n0 = p->n[0], n1 = p->n[1];
  const int len = d == 0 ? n0 : n1;
  const int inner = d == 0 ? n1 * h : h;   // contiguous block per index
  const int outer = d == 0 ? 1 : n0;
  const double* C = p->c[d].data();
  const double* S = p->s[d].data();
  for (int o = 0; o < outer; ++o) {
    const size_t base = (size_t)o * len * inner;
    for (int k = 0; k < len; ++k) {
      double* yr = orr + base + (size_t)k * inner;
      double* yi = oi + base + (size_t)k * inner;
      std::memset(yr, 0, sizeof(double) * inner);
      std::memset(yi, 0, sizeof(double) * inner);
      for (int j = 0; j < len; ++j) {
        const double c = C[(size_t)k * len + j], s = sign * S[(size_t)k * len + j];
        const double* xr = ir + base + (size_t)j * inner;
        const double* xi = ii + base + (size_t)j * inner;
        for (int t = 0; t < inner; ++t) {
          yr[t] += xr[t] * c - xi[t] * s;
          yi[t] += xr[t] * s + xi[t] * c;
        }
      }
    }
  }
}

static void r2c_one(const fftw_plan p, const double* in, double* out) {
  const int n0 = p->n[0], n1 = p->n[1], n2 = p->n[2], h = n2 / 2 + 1;
  const size_t tot = (size_t)n0 * n1 * h;
  std::vector<double> ar(tot), ai(tot), br(tot), bi(tot);
  const double* C = p->c[2].data();
  const double* S = p->s[2].data();
  for (int r = 0; r < n0 * n1; ++r) {
    const double* x = in + (size_t)r * n2;
    for (int k = 0; k < h; ++k) {
      double re = 0, im = 0;
      for (int j = 0; j < n2; ++j) {
        re += x[j] * C[(size_t)k * n2 + j];
        im -= x[j] * S[(size_t)k * n2 + j];
      }
      ar[(size_t)r * h + k] = re;
      ai[(size_t)r * h + k] = im;
    }
  }
  const double *fr = ar.data(), *fi = ai.data();
  if (n1 > 1) {
    axis(p, 1, h, ar.data(), ai.data(), br.data(), bi.data(), -1);
    fr = br.data();
    fi = bi.data();
  }
  if (n0 > 1) {
    double* tr = (fr == ar.data()) ? br.data() : ar.data();
    double* ti = (fi == ai.data()) ? bi.data() : ai.data();
    axis(p, 0, h, fr, fi, tr, ti, -1);
    fr = tr;
    fi = ti;
  }
  for (size_t e = 0; e < tot; ++e) {
    out[2 * e] = fr[e];
    out[2 * e + 1] = fi[e];
  }
}

static void c2r_one(const fftw_plan p, const double* in, double* out) {
  const int n0 = p->n[0], n1 = p->n[1], n2 = p->n[2], h = n2 / 2 + 1;
  const size_t tot = (size_t)n0 * n1 * h;
  std::vector<double> ar(tot), ai(tot), br(tot), bi(tot);
  for (size_t e = 0; e < tot; ++e) {
    ar[e] = in[2 * e];
    ai[e] = in[2 * e + 1];
  }
  const double *fr = ar.data(), *fi = ai.data();
  if (n0 > 1) {
    axis(p, 0, h, ar.data(), ai.data(), br.data(), bi.data(), +1);
    fr = br.data();
    fi = bi.data();
  }
  if (n1 > 1) {
    double* tr = (fr == ar.data()) ? br.data() : ar.data();
    double* ti = (fi == ai.data()) ? bi.data() : ai.data();
    axis(p, 1, h, fr, fi, tr, ti, +1);
    fr = tr;
    fi = ti;
  }
  const double* C = p->c[2].data();
  const double* S = p->s[2].data();
  for (int r = 0; r < n0 * n1; ++r) {
    const double* xr = fr + (size_t)r * h;
    const double* xi = fi + (size_t)r * h;
    for (int j = 0; j < n2; ++j) {
      // Hermitian completion along the last axis: X[n2-k] = conj(X[k]);
      // the imaginary part of the k = 0 (and Nyquist) term is ignored
      double v = xr[0];
      for (int k = 1; k < h; ++k) {
        const double t = xr[k] * C[(size_t)k * n2 + j] - xi[k] * S[(size_t)k * n2 + j];
        v += ((n2 % 2 == 0) && (k == n2 / 2)) ? t : 2 * t;
      }
      out[(size_t)r * n2 + j] = v;
    }
  }
}

extern "C" {
fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double* in, fftw_complex* out, unsigned) {
  int n[3] = {n0, n1, n2};
  return make(3, n, 1, in, n0 * n1 * n2, (double*)out, n0 * n1 * (n2 / 2 + 1), 1);
}
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex* in, double* out, unsigned) {
  int n[3] = {n0, n1, n2};
  return make(3, n, 1, (double*)in, n0 * n1 * (n2 / 2 + 1), out, n0 * n1 * n2, 0);
}
fftw_plan fftw_plan_many_dft_r2c(int rank, const int* n, int howmany, double* in, const int*, int, int idist,
                                 fftw_complex* out, const int*, int, int odist, unsigned) {
  return make(rank, n, howmany, in, idist, (double*)out, odist, 1);
}
fftw_plan fftw_plan_many_dft_c2r(int rank, const int* n, int howmany, fftw_complex* in, const int*, int,
                                 int idist, double* out, const int*, int, int odist, unsigned) {
  return make(rank, n, howmany, (double*)in, idist, out, odist, 0);
}
void fftw_execute_dft_r2c(const fftw_plan p, double* in, fftw_complex* out) {
  for (int b = 0; b < p->howmany; ++b)
    r2c_one(p, in + (size_t)b * p->idist, (double*)out + 2 * (size_t)b * p->odist);
}
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex* in, double* out) {
  for (int b = 0; b < p->howmany; ++b)
    c2r_one(p, (double*)in + 2 * (size_t)b * p->idist, out + (size_t)b * p->odist);
}
void fftw_execute(const fftw_plan p) {
  if (p->r2c)
    fftw_execute_dft_r2c(p, p->in, (fftw_complex*)p->out);
  else
    fftw_execute_dft_c2r(p, (fftw_complex*)p->in, p->out);
}
void fftw_destroy_plan(fftw_plan p) { delete p; }
}
