/*
 * fftw3.h -- the subset of the FFTW3 API that pstuermer/BDG_LOBPCG calls,
 * backed by a project-written CPU FFT (fftw_shim.c).
 *
 * TEST INFRASTRUCTURE ONLY: it exists so that the reference's own C sources
 * (src/*.c) compile unmodified into the CPU oracle library under oracle/_ref.
 * Nothing in the product library includes it.
 *
 * Calls covered (src/matmul_ctx.c:135-171, src/fft_helpers_impl.inc:24-82,
 * tests/test_setup.c:192-286): plan_dft, plan_dft_r2c, plan_dft_c2r,
 * execute_dft{,_r2c,_c2r}, destroy_plan, init_threads, plan_with_nthreads.
 * Conventions are FFTW's: unnormalised transforms, FFTW_FORWARD = -1 is
 * X[k] = sum_j x[j] exp(-2 pi i jk/N), dims listed slowest first (the
 * reference passes them reversed so that x is fastest), r2c/c2r halve the
 * LAST listed dim to n/2+1.  Plans are created for a pair of arrays but may be
 * executed on any other arrays of the same shape (the new-array execute
 * interface).  Flags select nothing: there is one algorithm.
 */
#ifndef FFTW3_H
#define FFTW3_H

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct fftw_plan_s *fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_PRESERVE_INPUT (1U << 4)
#define FFTW_PATIENT (1U << 5)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_dft(int rank, const int *n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_r2c(int rank, const int *n, double *in, fftw_complex *out, unsigned flags);
fftw_plan fftw_plan_dft_c2r(int rank, const int *n, fftw_complex *in, double *out, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_execute_dft(const fftw_plan p, fftw_complex *in, fftw_complex *out);
void fftw_execute_dft_r2c(const fftw_plan p, double *in, fftw_complex *out);
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex *in, double *out);
void fftw_destroy_plan(fftw_plan p);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);
void fftw_cleanup_threads(void);
void fftw_cleanup(void);

#ifdef __cplusplus
}
#endif

#endif /* FFTW3_H */
