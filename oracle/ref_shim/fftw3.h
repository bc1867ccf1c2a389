/*
 * Stand-in for the FFTW3 header, written for this repository.  FFTW3 is not
 * installed in this environment; the reference (3dpp/include/kernel.h:7)
 * includes <fftw3.h> and calls the eight entry points declared below.  The
 * declarations follow FFTW3's public API; fftw_shim.cpp implements them with
 * a separable O(n^2)-per-line discrete Fourier transform in double
 * precision, with FFTW's conventions: forward r2c uses exp(-2 pi i k n / N),
 * c2r is the unnormalised inverse, and the last dimension of a real array
 * holds n/2+1 complex values.
 */
#ifndef RTFMM_ORACLE_FFTW3_SHIM_H
#define RTFMM_ORACLE_FFTW3_SHIM_H
#ifdef __cplusplus
extern "C" {
#endif
typedef double fftw_complex[2];
typedef struct fftw_plan_s* fftw_plan;
#define FFTW_ESTIMATE (1U << 6)
fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double* in, fftw_complex* out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex* in, double* out, unsigned flags);
fftw_plan fftw_plan_many_dft_r2c(int rank, const int* n, int howmany, double* in, const int* inembed,
                                 int istride, int idist, fftw_complex* out, const int* onembed, int ostride,
                                 int odist, unsigned flags);
fftw_plan fftw_plan_many_dft_c2r(int rank, const int* n, int howmany, fftw_complex* in, const int* inembed,
                                 int istride, int idist, double* out, const int* onembed, int ostride,
                                 int odist, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_execute_dft_r2c(const fftw_plan p, double* in, fftw_complex* out);
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex* in, double* out);
void fftw_destroy_plan(fftw_plan p);
#ifdef __cplusplus
}
#endif
#endif
