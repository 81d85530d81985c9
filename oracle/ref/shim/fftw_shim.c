/*
 * FFTW3-API shim (test infrastructure only): a mixed-radix complex FFT used to
 * implement FFTW's R2HC / HC2R real transforms in FFTW's halfcomplex layout.
 * The reference applies it to lengths (2n-1)^3 = 125, 343, 729, 1331, ...
 * (include/compute.hpp:340, src/H2_3D_Tree.cpp:591), all smooth numbers.
 *
 * Plans are small structs; twiddle tables are cached per length behind a
 * mutex, and scratch is allocated per execution so that plans created by
 * different OpenMP threads (include/compute.hpp:363-366) never share state.
 */
#include "fftw3.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  double re, im;
} cpx;

struct oracle_fftw_plan_s {
  int n;
  int kind;
  double *in;
  double *out;
  const cpx *tw; /* tw[k] = exp(-2 pi i k / n) */
};

#define MAX_TW 64
static struct {
  int n;
  cpx *tw;
} g_tw[MAX_TW];
static int g_ntw = 0;
static pthread_mutex_t g_tw_lock = PTHREAD_MUTEX_INITIALIZER;

static const cpx *twiddles(int n) {
  pthread_mutex_lock(&g_tw_lock);
  for (int i = 0; i < g_ntw; ++i) {
    if (g_tw[i].n == n) {
      const cpx *t = g_tw[i].tw;
      pthread_mutex_unlock(&g_tw_lock);
      return t;
    }
  }
  cpx *t = (cpx *)malloc(sizeof(cpx) * (size_t)n);
  for (int k = 0; k < n; ++k) {
    double a = -2.0 * M_PI * (double)k / (double)n;
    t[k].re = cos(a);
    t[k].im = sin(a);
  }
  if (g_ntw < MAX_TW) {
    g_tw[g_ntw].n = n;
    g_tw[g_ntw].tw = t;
    ++g_ntw;
  }
  pthread_mutex_unlock(&g_tw_lock);
  return t;
}

static int smallest_factor(int n) {
  for (int p = 2; p * p <= n; ++p)
    if (n % p == 0) return p;
  return n;
}

/* Recursive decimation-in-time FFT of length n over in[0], in[s], ...
 * writing out[0..n).  W_n^e = tw[(e * wstep) mod N]; inverse conjugates.
 * Scratch lives on the stack (radices are small for the lengths used). */
static void fft_rec(const cpx *in, int s, cpx *out, int n, const cpx *tw,
                    int N, int wstep, int inverse) {
  if (n == 1) {
    out[0] = in[0];
    return;
  }
  int p = smallest_factor(n);
  int m = n / p;
  for (int q = 0; q < p; ++q)
    fft_rec(in + (size_t)q * s, s * p, out + (size_t)q * m, m, tw, N,
            wstep * p, inverse);
  cpx t[p], r[p];
  const double sg = inverse ? -1.0 : 1.0;
  const long stepm = (long)m * wstep; /* W_p^1 = W_n^m */
  for (int k = 0; k < m; ++k) {
    long e = 0;
    const long ek = (long)k * wstep;
    for (int q = 0; q < p; ++q) {
      cpx w = tw[e];
      double wi = sg * w.im;
      cpx y = out[(size_t)q * m + k];
      t[q].re = y.re * w.re - y.im * wi;
      t[q].im = y.re * wi + y.im * w.re;
      e += ek;
      if (e >= N) e %= N;
    }
    for (int sidx = 0; sidx < p; ++sidx) {
      double ar = 0.0, ai = 0.0;
      long e2 = 0;
      const long es = (long)sidx * stepm % N;
      for (int q = 0; q < p; ++q) {
        cpx w = tw[e2];
        double wi = sg * w.im;
        ar += t[q].re * w.re - t[q].im * wi;
        ai += t[q].re * wi + t[q].im * w.re;
        e2 += es;
        if (e2 >= N) e2 -= N;
      }
      r[sidx].re = ar;
      r[sidx].im = ai;
    }
    for (int sidx = 0; sidx < p; ++sidx) out[(size_t)k + (size_t)sidx * m] = r[sidx];
  }
}

fftw_plan fftw_plan_r2r_1d(int n, double *in, double *out, fftw_r2r_kind kind,
                           unsigned flags) {
  (void)flags;
  fftw_plan p = (fftw_plan)malloc(sizeof(*p));
  p->n = n;
  p->kind = (int)kind;
  p->in = in;
  p->out = out;
  p->tw = twiddles(n);
  return p;
}

void fftw_execute(const fftw_plan p) {
  int n = p->n;
  cpx *a = (cpx *)malloc(sizeof(cpx) * (size_t)n);
  cpx *b = (cpx *)malloc(sizeof(cpx) * (size_t)n);
  if (p->kind == FFTW_R2HC) {
    for (int j = 0; j < n; ++j) {
      a[j].re = p->in[j];
      a[j].im = 0.0;
    }
    fft_rec(a, 1, b, n, p->tw, n, 1, 0);
    for (int k = 0; k <= n / 2; ++k) p->out[k] = b[k].re;
    for (int k = 1; k < (n + 1) / 2; ++k) p->out[n - k] = b[k].im;
  } else {
    a[0].re = p->in[0];
    a[0].im = 0.0;
    for (int k = 1; k < (n + 1) / 2; ++k) {
      a[k].re = p->in[k];
      a[k].im = p->in[n - k];
      a[n - k].re = p->in[k];
      a[n - k].im = -p->in[n - k];
    }
    if (n % 2 == 0) {
      a[n / 2].re = p->in[n / 2];
      a[n / 2].im = 0.0;
    }
    fft_rec(a, 1, b, n, p->tw, n, 1, 1);
    for (int j = 0; j < n; ++j) p->out[j] = b[j].re;
  }
  free(a);
  free(b);
}

void fftw_destroy_plan(fftw_plan p) { free(p); }

double *fftw_alloc_real(size_t n) {
  return (double *)malloc(sizeof(double) * (n ? n : 1));
}

void fftw_free(void *p) { free(p); }
