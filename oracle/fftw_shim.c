/*
 * fftw_shim.c -- restatement of the FFTW3 real-data 3-D DFT semantics that the
 * reference's CPU path relies on.
 *
 * TEST INFRASTRUCTURE ONLY (oracle).  Only tests/, the smoke check and the CPU
 * baseline leg of bench.py load code built from this file; the product never does.
 *
 * FFTW3 (the reference's third-party FFT; version unpinned, README.md:68) is not
 * available here.  What the reference needs from it is the mathematical DFT with
 * FFTW's array conventions (see fftw3.h).  This file computes exactly that with a
 * textbook mixed-radix decimation-in-time Cooley-Tukey recursion (radices 4, 2, 3,
 * 5 and a direct DFT for any other prime factor), applied axis by axis.  Twiddle
 * factors are taken from one table of cos/sin(2*pi*j/n) evaluated in double, so
 * results agree with FFTW to a few ulps times log(n).
 *
 * Threads: the per-line transforms of each axis are independent; when built with
 * OpenMP they are spread over CF_FFT_THREADS threads (environment variable;
 * default 1, which is what the reference's own, unthreaded FFTW plans do).
 */
#include "fftw3.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
  int n;
  int nfac;
  int fac[40];
  double *cs; /* cs[2j] = cos(2 pi j/n), cs[2j+1] = sin(2 pi j/n) */
} line_plan;

struct cf_fftw_plan_s {
  int kind; /* 0 = r2c, 1 = c2r */
  int n0, n1, n2;
  void *in;
  void *out;
  line_plan lp[3];
};

static void line_plan_init(line_plan *p, int n) {
  p->n = n;
  p->nfac = 0;
  int m = n;
  while (m % 4 == 0) { p->fac[p->nfac++] = 4; m /= 4; }
  while (m % 2 == 0) { p->fac[p->nfac++] = 2; m /= 2; }
  for (int f = 3; m > 1; f += 2) {
    while (m % f == 0) { p->fac[p->nfac++] = f; m /= f; }
  }
  p->cs = (double *)malloc(sizeof(double) * 2 * (size_t)(n > 0 ? n : 1));
  const double two_pi = 6.283185307179586476925286766559;
  for (int j = 0; j < n; ++j) {
    long double ang = (long double)two_pi * (long double)j / (long double)n;
    p->cs[2 * j] = (double)cosl(ang);
    p->cs[2 * j + 1] = (double)sinl(ang);
  }
}

static void line_plan_free(line_plan *p) { free(p->cs); p->cs = NULL; }

/* W^e with W = exp(sign * 2 pi i / n): writes (re, im). */
static inline void twiddle(const line_plan *p, long e, int sign, double *re, double *im) {
  long n = p->n;
  e %= n;
  if (e < 0) e += n;
  *re = p->cs[2 * e];
  *im = sign * p->cs[2 * e + 1];
}

/* out[0..n) = DFT_n(in[0], in[is], ...) with exponent sign; `tws` maps a
 * length-n root of unity to the table: W_n^j = W_N^(j*tws). */
static void dft_rec(const line_plan *p, int lvl, int n, const double *in, size_t is,
                    double *out, int sign, long tws) {
  if (n == 1) {
    out[0] = in[0];
    out[1] = in[1];
    return;
  }
  int r = p->fac[lvl];
  int m = n / r;
  for (int q = 0; q < r; ++q)
    dft_rec(p, lvl + 1, m, in + 2 * (size_t)q * is, is * (size_t)r, out + 2 * (size_t)q * m,
            sign, tws * r);
  double tre[r], tim[r];
  for (int k = 0; k < m; ++k) {
    for (int q = 0; q < r; ++q) {
      double xr = out[2 * ((size_t)q * m + k)], xi = out[2 * ((size_t)q * m + k) + 1];
      if (q == 0 || k == 0) {
        tre[q] = xr;
        tim[q] = xi;
      } else {
        double wr, wi;
        twiddle(p, (long)q * k * tws, sign, &wr, &wi);
        tre[q] = xr * wr - xi * wi;
        tim[q] = xr * wi + xi * wr;
      }
    }
    if (r == 2) {
      out[2 * k] = tre[0] + tre[1];
      out[2 * k + 1] = tim[0] + tim[1];
      out[2 * (m + k)] = tre[0] - tre[1];
      out[2 * (m + k) + 1] = tim[0] - tim[1];
    } else if (r == 4) {
      /* radix-4 butterfly; multiplication by (sign*i) is exact */
      double a0r = tre[0] + tre[2], a0i = tim[0] + tim[2];
      double a1r = tre[0] - tre[2], a1i = tim[0] - tim[2];
      double b0r = tre[1] + tre[3], b0i = tim[1] + tim[3];
      double b1r = tre[1] - tre[3], b1i = tim[1] - tim[3];
      /* (sign*i) * b1 */
      double jb1r = -sign * b1i, jb1i = sign * b1r;
      out[2 * k] = a0r + b0r;
      out[2 * k + 1] = a0i + b0i;
      out[2 * (m + k)] = a1r + jb1r;
      out[2 * (m + k) + 1] = a1i + jb1i;
      out[2 * (2 * m + k)] = a0r - b0r;
      out[2 * (2 * m + k) + 1] = a0i - b0i;
      out[2 * (3 * m + k)] = a1r - jb1r;
      out[2 * (3 * m + k) + 1] = a1i - jb1i;
    } else {
      long step = (long)p->n / r;
      for (int s = 0; s < r; ++s) {
        double yr = tre[0], yi = tim[0];
        for (int q = 1; q < r; ++q) {
          double wr, wi;
          twiddle(p, (long)((q * s) % r) * step, sign, &wr, &wi);
          yr += tre[q] * wr - tim[q] * wi;
          yi += tre[q] * wi + tim[q] * wr;
        }
        out[2 * ((size_t)s * m + k)] = yr;
        out[2 * ((size_t)s * m + k) + 1] = yi;
      }
    }
  }
}

static void line_dft(const line_plan *p, const double *in, double *out, int sign) {
  dft_rec(p, 0, p->n, in, 1, out, sign, 1);
}

static int nthreads(void) {
  const char *e = getenv("CF_FFT_THREADS");
  int n = e ? atoi(e) : 1;
  return n > 0 ? n : 1;
}

/* In-place complex transform of every line along axis `ax` of a complex
 * n0 x n1 x nh array. */
static void axis_pass(const line_plan *p, double *z, int n0, int n1, int nh, int ax, int sign) {
  long nlines;
  if (ax == 0) nlines = (long)n1 * nh;
  else nlines = (long)n0 * nh;
  int len = (ax == 0) ? n0 : n1;
  size_t stride = (ax == 0) ? (size_t)n1 * nh : (size_t)nh;
#pragma omp parallel num_threads(nthreads()) if (nthreads() > 1)
  {
    double *a = (double *)malloc(sizeof(double) * 4 * (size_t)len);
    double *b = a + 2 * (size_t)len;
#pragma omp for schedule(static)
    for (long l = 0; l < nlines; ++l) {
      size_t base;
      if (ax == 0) base = (size_t)l; /* (j,k) flattened */
      else base = (size_t)(l / nh) * (size_t)n1 * nh + (size_t)(l % nh);
      for (int i = 0; i < len; ++i) {
        a[2 * i] = z[2 * (base + i * stride)];
        a[2 * i + 1] = z[2 * (base + i * stride) + 1];
      }
      line_dft(p, a, b, sign);
      for (int i = 0; i < len; ++i) {
        z[2 * (base + i * stride)] = b[2 * i];
        z[2 * (base + i * stride) + 1] = b[2 * i + 1];
      }
    }
    free(a);
  }
}

static void exec_r2c(const struct cf_fftw_plan_s *pl, const double *in, double *out) {
  const int n0 = pl->n0, n1 = pl->n1, n2 = pl->n2, nh = n2 / 2 + 1;
  const long rows = (long)n0 * n1;
  double *z = (double *)malloc(sizeof(double) * 2 * (size_t)rows * nh);
#pragma omp parallel num_threads(nthreads()) if (nthreads() > 1)
  {
    double *a = (double *)malloc(sizeof(double) * 4 * (size_t)n2);
    double *b = a + 2 * (size_t)n2;
#pragma omp for schedule(static)
    for (long r = 0; r < rows; ++r) {
      for (int k = 0; k < n2; ++k) {
        a[2 * k] = in[(size_t)r * n2 + k];
        a[2 * k + 1] = 0.0;
      }
      line_dft(&pl->lp[2], a, b, -1);
      memcpy(z + 2 * (size_t)r * nh, b, sizeof(double) * 2 * nh);
    }
    free(a);
  }
  axis_pass(&pl->lp[1], z, n0, n1, nh, 1, -1);
  axis_pass(&pl->lp[0], z, n0, n1, nh, 0, -1);
  memcpy(out, z, sizeof(double) * 2 * (size_t)rows * nh);
  free(z);
}

static void exec_c2r(const struct cf_fftw_plan_s *pl, const double *in, double *out) {
  const int n0 = pl->n0, n1 = pl->n1, n2 = pl->n2, nh = n2 / 2 + 1;
  const long rows = (long)n0 * n1;
  const int inplace = ((const void *)in == (const void *)out);
  const size_t pitch = inplace ? (size_t)2 * nh : (size_t)n2;
  double *z = (double *)malloc(sizeof(double) * 2 * (size_t)rows * nh);
  memcpy(z, in, sizeof(double) * 2 * (size_t)rows * nh);
  axis_pass(&pl->lp[0], z, n0, n1, nh, 0, +1);
  axis_pass(&pl->lp[1], z, n0, n1, nh, 1, +1);
#pragma omp parallel num_threads(nthreads()) if (nthreads() > 1)
  {
    double *a = (double *)malloc(sizeof(double) * 4 * (size_t)n2);
    double *b = a + 2 * (size_t)n2;
#pragma omp for schedule(static)
    for (long r = 0; r < rows; ++r) {
      const double *zr = z + 2 * (size_t)r * nh;
      for (int k = 0; k < nh; ++k) {
        a[2 * k] = zr[2 * k];
        a[2 * k + 1] = zr[2 * k + 1];
      }
      for (int k = nh; k < n2; ++k) { /* Hermitian extension along the last axis */
        a[2 * k] = zr[2 * (n2 - k)];
        a[2 * k + 1] = -zr[2 * (n2 - k) + 1];
      }
      line_dft(&pl->lp[2], a, b, +1);
      for (int k = 0; k < n2; ++k) out[(size_t)r * pitch + k] = b[2 * k];
    }
    free(a);
  }
  free(z);
}

static fftw_plan make_plan(int kind, int n0, int n1, int n2, void *in, void *out) {
  struct cf_fftw_plan_s *p = (struct cf_fftw_plan_s *)calloc(1, sizeof(*p));
  p->kind = kind;
  p->n0 = n0;
  p->n1 = n1;
  p->n2 = n2;
  p->in = in;
  p->out = out;
  line_plan_init(&p->lp[0], n0);
  line_plan_init(&p->lp[1], n1);
  line_plan_init(&p->lp[2], n2);
  return p;
}

fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in, fftw_complex *out, unsigned flags) {
  (void)flags;
  return make_plan(0, n0, n1, n2, in, out);
}

fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in, double *out, unsigned flags) {
  (void)flags;
  return make_plan(1, n0, n1, n2, in, out);
}

void fftw_execute(const fftw_plan p) {
  if (p->kind == 0) exec_r2c(p, (const double *)p->in, (double *)p->out);
  else exec_c2r(p, (const double *)p->in, (double *)p->out);
}

void fftw_execute_dft_r2c(const fftw_plan p, double *in, fftw_complex *out) {
  exec_r2c(p, in, (double *)out);
}

void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex *in, double *out) {
  exec_c2r(p, (const double *)in, out);
}

void fftw_destroy_plan(fftw_plan p) {
  if (!p) return;
  for (int i = 0; i < 3; ++i) line_plan_free(&p->lp[i]);
  free(p);
}

void *fftw_malloc(size_t n) {
  void *ptr = NULL;
  if (posix_memalign(&ptr, 64, n ? n : 64) != 0) return NULL;
  return ptr;
}

void fftw_free(void *p) { free(p); }

fftw_complex *fftw_alloc_complex(size_t n) { return (fftw_complex *)fftw_malloc(n * sizeof(fftw_complex)); }

double *fftw_alloc_real(size_t n) { return (double *)fftw_malloc(n * sizeof(double)); }
