/*
 * fftw_shim.c -- project-written CPU FFT behind the FFTW3 subset of fftw3.h.
 *
 * TEST INFRASTRUCTURE ONLY (the oracle build of the reference library).
 *
 * One line transform serves every axis: a self-sorting mixed-radix Stockham
 * FFT (radix 4, 2, 3, 5 butterflies written out, any other prime factor as a
 * plain DFT), twiddles from one table e^{-2 pi i t/n} per line length.
 * Multi-dimensional transforms run the line transform along each axis:
 * the fastest axis on contiguous rows, the others on blocks of up to 16
 * adjacent lines gathered into a contiguous buffer.  r2c packs two real rows
 * into one complex row and splits the spectrum (X_a = (Z_k + conj Z_-k)/2,
 * X_b = (Z_k - conj Z_-k)/2i); c2r rebuilds the two Hermitian rows, sums them
 * as A + iB and takes real and imaginary parts of the inverse.  As in FFTW the
 * imaginary parts of the DC and Nyquist terms of a c2r input are ignored.
 * OpenMP threads split the lines (count set by fftw_plan_with_nthreads).
 */
#include "fftw3.h"

#include <complex.h>
#include <math.h>
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef double _Complex cplx;

#define MAXDIM 8
#define MAXFAC 40
#define LINE_BLOCK 16

typedef struct {
  int n;
  int nf;
  int fac[MAXFAC];
  int maxr;
  cplx *tw; /* e^{-2 pi i t / n}, t = 0..n-1 */
} line_plan;

enum { KIND_C2C = 0, KIND_R2C = 1, KIND_C2R = 2 };

struct fftw_plan_s {
  int kind, sign, rank;
  int n[MAXDIM];
  line_plan lp[MAXDIM];
  size_t total;  /* real-space points */
  size_t ktotal; /* complex points of the (half) spectrum */
  void *in, *out;
  int nthreads;
};

static int g_nthreads = 1;

static void line_plan_init(line_plan *lp, int n) {
  lp->n = n;
  lp->nf = 0;
  lp->maxr = 1;
  int r = n;
  while (r % 4 == 0) { lp->fac[lp->nf++] = 4; r /= 4; }
  while (r % 2 == 0) { lp->fac[lp->nf++] = 2; r /= 2; }
  while (r % 3 == 0) { lp->fac[lp->nf++] = 3; r /= 3; }
  while (r % 5 == 0) { lp->fac[lp->nf++] = 5; r /= 5; }
  for (int p = 7; r > 1; p += 2)
    while (r % p == 0) { lp->fac[lp->nf++] = p; r /= p; }
  for (int i = 0; i < lp->nf; i++)
    if (lp->fac[i] > lp->maxr) lp->maxr = lp->fac[i];
  lp->tw = (cplx *)malloc((size_t)(n > 0 ? n : 1) * sizeof(cplx));
  for (int t = 0; t < n; t++) {
    const double a = -2.0 * M_PI * (double)t / (double)n;
    lp->tw[t] = cos(a) + I * sin(a);
  }
}

static inline cplx twid(const line_plan *lp, int t, int sign) {
  return sign < 0 ? lp->tw[t] : conj(lp->tw[t]);
}

/* length-R DFT of v in place, X_k = sum_r v_r e^{sign 2 pi i rk/R} */
static void small_dft(const line_plan *lp, cplx *v, int R, int sign, cplx *tmp) {
  const double sg = (double)sign;
  switch (R) {
  case 2: {
    const cplx a = v[0], b = v[1];
    v[0] = a + b;
    v[1] = a - b;
    return;
  }
  case 3: {
    const double c = -0.5, s = 0.86602540378443864676;
    const cplx t1 = v[1] + v[2], t2 = v[0] + c * t1, t3 = (sg * s * I) * (v[1] - v[2]);
    v[0] = v[0] + t1;
    v[1] = t2 + t3;
    v[2] = t2 - t3;
    return;
  }
  case 4: {
    const cplx a = v[0] + v[2], b = v[0] - v[2], c = v[1] + v[3], d = (sg * I) * (v[1] - v[3]);
    v[0] = a + c;
    v[2] = a - c;
    v[1] = b + d;
    v[3] = b - d;
    return;
  }
  default: {
    const int step = lp->n / R;
    for (int k = 0; k < R; k++) {
      cplx acc = 0;
      for (int r = 0; r < R; r++) acc += v[r] * twid(lp, ((r * k) % R) * step, sign);
      tmp[k] = acc;
    }
    memcpy(v, tmp, (size_t)R * sizeof(cplx));
  }
  }
}

/* In-place line transform of x (length lp->n) using work w (length n). */
static void line_fft(const line_plan *lp, cplx *x, cplx *w, int sign) {
  const int n = lp->n;
  if (n <= 1) return;
  cplx *a = x, *b = w;
  cplx v[64], tmp[64];
  cplx *vv = lp->maxr > 64 ? (cplx *)malloc(2 * (size_t)lp->maxr * sizeof(cplx)) : v;
  cplx *tt = lp->maxr > 64 ? vv + lp->maxr : tmp;
  int Ns = 1;
  for (int s = 0; s < lp->nf; s++) {
    const int R = lp->fac[s], m = n / R, step = n / (Ns * R);
    for (int j = 0; j < m; j++) {
      const int k = j % Ns;
      for (int r = 0; r < R; r++) vv[r] = a[j + r * m];
      if (k)
        for (int r = 1; r < R; r++) vv[r] *= twid(lp, k * r * step, sign);
      small_dft(lp, vv, R, sign, tt);
      const int base = (j / Ns) * Ns * R + k;
      for (int r = 0; r < R; r++) b[base + r * Ns] = vv[r];
    }
    cplx *t = a;
    a = b;
    b = t;
    Ns *= R;
  }
  if (a != x) memcpy(x, a, (size_t)n * sizeof(cplx));
  if (vv != v) free(vv);
}

/* c2c along axis d of a complex array with extents ext[0..rank-1] (slowest
 * first), in place. */
static void axis_c2c(const struct fftw_plan_s *p, cplx *data, const int *ext, int d, int sign) {
  size_t outer = 1, inner = 1;
  for (int i = 0; i < d; i++) outer *= (size_t)ext[i];
  for (int i = d + 1; i < p->rank; i++) inner *= (size_t)ext[i];
  const int nd = ext[d];
  const line_plan *lp = &p->lp[d];
  if (nd <= 1) return;
  if (inner == 1) {
#pragma omp parallel num_threads(p->nthreads)
    {
      cplx *w = (cplx *)malloc((size_t)nd * sizeof(cplx));
#pragma omp for schedule(static)
      for (size_t o = 0; o < outer; o++) line_fft(lp, data + o * (size_t)nd, w, sign);
      free(w);
    }
    return;
  }
  const size_t nblk = (inner + LINE_BLOCK - 1) / LINE_BLOCK;
#pragma omp parallel num_threads(p->nthreads)
  {
    cplx *buf = (cplx *)malloc((size_t)LINE_BLOCK * nd * sizeof(cplx));
    cplx *w = (cplx *)malloc((size_t)nd * sizeof(cplx));
#pragma omp for schedule(static) collapse(2)
    for (size_t o = 0; o < outer; o++)
      for (size_t bk = 0; bk < nblk; bk++) {
        const size_t i0 = bk * LINE_BLOCK;
        const size_t nb = (inner - i0) < LINE_BLOCK ? (inner - i0) : LINE_BLOCK;
        cplx *base = data + o * (size_t)nd * inner + i0;
        for (int j = 0; j < nd; j++)
          for (size_t q = 0; q < nb; q++) buf[q * nd + j] = base[(size_t)j * inner + q];
        for (size_t q = 0; q < nb; q++) line_fft(lp, buf + q * nd, w, sign);
        for (int j = 0; j < nd; j++)
          for (size_t q = 0; q < nb; q++) base[(size_t)j * inner + q] = buf[q * nd + j];
      }
    free(w);
    free(buf);
  }
}

static fftw_plan plan_new(int kind, int rank, const int *n, void *in, void *out, int sign) {
  if (rank < 1 || rank > MAXDIM) {
    fprintf(stderr, "fftw_shim: rank %d unsupported\n", rank);
    return NULL;
  }
  struct fftw_plan_s *p = (struct fftw_plan_s *)calloc(1, sizeof *p);
  p->kind = kind;
  p->sign = sign;
  p->rank = rank;
  p->total = 1;
  for (int d = 0; d < rank; d++) {
    if (n[d] < 1) {
      free(p);
      return NULL;
    }
    p->n[d] = n[d];
    p->total *= (size_t)n[d];
  }
  p->ktotal = p->total;
  if (kind != KIND_C2C) p->ktotal = p->total / (size_t)n[rank - 1] * (size_t)(n[rank - 1] / 2 + 1);
  for (int d = 0; d < rank; d++) line_plan_init(&p->lp[d], n[d]);
  p->in = in;
  p->out = out;
  p->nthreads = g_nthreads > 0 ? g_nthreads : 1;
  return p;
}

fftw_plan fftw_plan_dft(int rank, const int *n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags) {
  (void)flags;
  return plan_new(KIND_C2C, rank, n, in, out, sign < 0 ? -1 : 1);
}

fftw_plan fftw_plan_dft_r2c(int rank, const int *n, double *in, fftw_complex *out, unsigned flags) {
  (void)flags;
  return plan_new(KIND_R2C, rank, n, in, out, -1);
}

fftw_plan fftw_plan_dft_c2r(int rank, const int *n, fftw_complex *in, double *out, unsigned flags) {
  (void)flags;
  return plan_new(KIND_C2R, rank, n, in, out, 1);
}

static void exec_c2c(const struct fftw_plan_s *p, const cplx *in, cplx *out) {
  if (in != out) memcpy(out, in, p->total * sizeof(cplx));
  for (int d = p->rank - 1; d >= 0; d--) axis_c2c(p, out, p->n, d, p->sign);
}

static void exec_r2c(const struct fftw_plan_s *p, const double *in, cplx *out) {
  const int N = p->n[p->rank - 1], H = N / 2 + 1;
  const size_t rows = p->total / (size_t)N, pairs = (rows + 1) / 2;
  const line_plan *lp = &p->lp[p->rank - 1];
#pragma omp parallel num_threads(p->nthreads)
  {
    cplx *z = (cplx *)malloc((size_t)N * sizeof(cplx));
    cplx *w = (cplx *)malloc((size_t)N * sizeof(cplx));
#pragma omp for schedule(static)
    for (size_t q = 0; q < pairs; q++) {
      const size_t ra = 2 * q, rb = 2 * q + 1;
      const double *a = in + ra * (size_t)N, *b = rb < rows ? in + rb * (size_t)N : NULL;
      for (int j = 0; j < N; j++) z[j] = a[j] + I * (b ? b[j] : 0.0);
      line_fft(lp, z, w, -1);
      cplx *oa = out + ra * (size_t)H, *ob = rb < rows ? out + rb * (size_t)H : NULL;
      for (int k = 0; k < H; k++) {
        const cplx zk = z[k], zm = conj(z[(N - k) % N]);
        oa[k] = 0.5 * (zk + zm);
        if (ob) ob[k] = -0.5 * I * (zk - zm);
      }
    }
    free(w);
    free(z);
  }
  int ext[MAXDIM];
  for (int d = 0; d < p->rank; d++) ext[d] = p->n[d];
  ext[p->rank - 1] = H;
  for (int d = p->rank - 2; d >= 0; d--) axis_c2c(p, out, ext, d, -1);
}

static void exec_c2r(const struct fftw_plan_s *p, const cplx *in, double *out) {
  const int N = p->n[p->rank - 1], H = N / 2 + 1;
  const size_t rows = p->total / (size_t)N, pairs = (rows + 1) / 2;
  const line_plan *lp = &p->lp[p->rank - 1];
  cplx *spec = (cplx *)malloc(p->ktotal * sizeof(cplx));
  memcpy(spec, in, p->ktotal * sizeof(cplx));
  int ext[MAXDIM];
  for (int d = 0; d < p->rank; d++) ext[d] = p->n[d];
  ext[p->rank - 1] = H;
  for (int d = p->rank - 2; d >= 0; d--) axis_c2c(p, spec, ext, d, 1);
#pragma omp parallel num_threads(p->nthreads)
  {
    cplx *z = (cplx *)malloc((size_t)N * sizeof(cplx));
    cplx *w = (cplx *)malloc((size_t)N * sizeof(cplx));
#pragma omp for schedule(static)
    for (size_t q = 0; q < pairs; q++) {
      const size_t ra = 2 * q, rb = 2 * q + 1;
      const cplx *A = spec + ra * (size_t)H, *Bv = rb < rows ? spec + rb * (size_t)H : NULL;
      for (int k = 0; k < N; k++) {
        cplx ak, bk = 0;
        if (k < H) {
          ak = A[k];
          if (Bv) bk = Bv[k];
          if (k == 0 || 2 * k == N) {
            ak = creal(ak);
            bk = creal(bk);
          }
        } else {
          ak = conj(A[N - k]);
          if (Bv) bk = conj(Bv[N - k]);
        }
        z[k] = ak + I * bk;
      }
      line_fft(lp, z, w, 1);
      double *oa = out + ra * (size_t)N, *ob = rb < rows ? out + rb * (size_t)N : NULL;
      for (int j = 0; j < N; j++) {
        oa[j] = creal(z[j]);
        if (ob) ob[j] = cimag(z[j]);
      }
    }
    free(w);
    free(z);
  }
  free(spec);
}

void fftw_execute_dft(const fftw_plan p, fftw_complex *in, fftw_complex *out) {
  if (!p) return;
  exec_c2c(p, (const cplx *)in, (cplx *)out);
}

void fftw_execute_dft_r2c(const fftw_plan p, double *in, fftw_complex *out) {
  if (!p) return;
  exec_r2c(p, in, (cplx *)out);
}

void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex *in, double *out) {
  if (!p) return;
  exec_c2r(p, (const cplx *)in, out);
}

void fftw_execute(const fftw_plan p) {
  if (!p) return;
  if (p->kind == KIND_C2C) exec_c2c(p, (const cplx *)p->in, (cplx *)p->out);
  else if (p->kind == KIND_R2C) exec_r2c(p, (const double *)p->in, (cplx *)p->out);
  else exec_c2r(p, (const cplx *)p->in, (double *)p->out);
}

void fftw_destroy_plan(fftw_plan p) {
  if (!p) return;
  for (int d = 0; d < p->rank; d++) free(p->lp[d].tw);
  free(p);
}

int fftw_init_threads(void) { return 1; }

void fftw_plan_with_nthreads(int nthreads) { g_nthreads = nthreads > 0 ? nthreads : 1; }

void fftw_cleanup_threads(void) {}

void fftw_cleanup(void) {}
