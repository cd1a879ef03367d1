/*
 * Mixed-radix complex FFT (double) for the CPU oracle.  TEST INFRASTRUCTURE:
 * only the oracle restatement and the reference-build shim use it.
 * See fft.h for conventions.
 */
#include "fft.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double _Complex cplx;

struct orc_fft_plan {
  long n;
  int sign;
  int nfac;
  long fac[2 * 64]; /* pairs (radix p, remaining length m) */
  cplx *tw;         /* tw[j] = exp(sign * 2 pi i j / n), j < n */
};

#define ORC_MAX_PLANS 256
static orc_fft_plan *g_plans[ORC_MAX_PLANS];
static int g_nplans = 0;

static void factorize(orc_fft_plan *p) {
  long n = p->n, m = n;
  int k = 0;
  while (m > 1) {
    long r;
    if (m % 4 == 0) r = 4;
    else if (m % 2 == 0) r = 2;
    else if (m % 3 == 0) r = 3;
    else if (m % 5 == 0) r = 5;
    else {
      r = 7;
      while (m % r != 0) r += 2;
    }
    m /= r;
    p->fac[2 * k] = r;
    p->fac[2 * k + 1] = m;
    k++;
  }
  p->nfac = k;
}

static orc_fft_plan *plan_new(long n, int sign) {
  orc_fft_plan *p = (orc_fft_plan *)calloc(1, sizeof(orc_fft_plan));
  p->n = n;
  p->sign = sign;
  p->tw = (cplx *)malloc(sizeof(cplx) * (size_t)(n > 0 ? n : 1));
  for (long j = 0; j < n; j++) {
    /* reduce the angle to keep twiddles accurate for large n */
    double ang = 2.0 * M_PI * (double)j / (double)n;
    p->tw[j] = cos(ang) + (double)sign * sin(ang) * I;
  }
  if (n == 1) {
    p->nfac = 1;
    p->fac[0] = 1;
    p->fac[1] = 1;
  } else {
    factorize(p);
  }
  return p;
}

const orc_fft_plan *orc_fft_plan_get(long n, int sign) {
  const orc_fft_plan *found = NULL;
#pragma omp critical(orc_fft_plan_cache)
  {
    for (int i = 0; i < g_nplans; i++)
      if (g_plans[i]->n == n && g_plans[i]->sign == sign) {
        found = g_plans[i];
        break;
      }
    if (!found) {
      orc_fft_plan *p = plan_new(n, sign);
      if (g_nplans < ORC_MAX_PLANS) g_plans[g_nplans++] = p;
      found = p;
    }
  }
  return found;
}

static void bfly2(cplx *out, long fs, const orc_fft_plan *P, long m) {
  const cplx *tw = P->tw;
  for (long k = 0; k < m; k++) {
    cplx t = out[k + m] * tw[k * fs];
    out[k + m] = out[k] - t;
    out[k] += t;
  }
}

static void bfly4(cplx *out, long fs, const orc_fft_plan *P, long m) {
  const cplx *tw = P->tw;
  const double sg = (double)P->sign;
  for (long k = 0; k < m; k++) {
    cplx s0 = out[k];
    cplx s1 = out[k + m] * tw[k * fs];
    cplx s2 = out[k + 2 * m] * tw[2 * k * fs];
    cplx s3 = out[k + 3 * m] * tw[3 * k * fs];
    cplx a0 = s0 + s2, a1 = s0 - s2, a2 = s1 + s3, a3 = s1 - s3;
    /* exp(sign*2 pi i/4) = sign*i */
    cplx ia3 = sg * I * a3;
    out[k] = a0 + a2;
    out[k + 2 * m] = a0 - a2;
    out[k + m] = a1 + ia3;
    out[k + 3 * m] = a1 - ia3;
  }
}

static void bfly3(cplx *out, long fs, const orc_fft_plan *P, long m) {
  const cplx *tw = P->tw;
  const double c = -0.5, s = (double)P->sign * 0.86602540378443864676;
  for (long k = 0; k < m; k++) {
    cplx s0 = out[k];
    cplx s1 = out[k + m] * tw[k * fs];
    cplx s2 = out[k + 2 * m] * tw[2 * k * fs];
    cplx t = s1 + s2, d = s1 - s2;
    cplx base = s0 + c * t;
    cplx rot = s * I * d;
    out[k] = s0 + t;
    out[k + m] = base + rot;
    out[k + 2 * m] = base - rot;
  }
}

static void bfly_generic(cplx *out, long fs, const orc_fft_plan *P, long m,
                         long p) {
  const cplx *tw = P->tw;
  const long n = P->n;
  cplx sbuf[64];
  cplx *s = p <= 64 ? sbuf : (cplx *)malloc(sizeof(cplx) * (size_t)p);
  for (long k = 0; k < m; k++) {
    for (long q = 0; q < p; q++) s[q] = out[k + q * m] * tw[(q * k * fs) % n];
    for (long q2 = 0; q2 < p; q2++) {
      cplx acc = 0;
      for (long q1 = 0; q1 < p; q1++)
        acc += s[q1] * tw[((q1 * q2) % p) * m * fs];
      out[k + q2 * m] = acc;
    }
  }
  if (s != sbuf) free(s);
}

static void work(cplx *out, const cplx *in, long fs, const long *fac,
                 const orc_fft_plan *P) {
  const long p = fac[0], m = fac[1];
  if (m == 1) {
    for (long k = 0; k < p; k++) out[k] = in[k * fs];
  } else {
    for (long k = 0; k < p; k++) work(out + k * m, in + k * fs, fs * p, fac + 2, P);
  }
  switch (p) {
    case 1: break;
    case 2: bfly2(out, fs, P, m); break;
    case 3: bfly3(out, fs, P, m); break;
    case 4: bfly4(out, fs, P, m); break;
    default: bfly_generic(out, fs, P, m, p); break;
  }
}

void orc_fft_exec(const orc_fft_plan *p, double *data, double *wk) {
  if (p->n <= 1) return;
  cplx *x = (cplx *)data, *w = (cplx *)wk;
  memcpy(w, x, sizeof(cplx) * (size_t)p->n);
  work(x, w, 1, p->fac, p);
}

void orc_fft_1d(double *data, long n, int sign) {
  const orc_fft_plan *p = orc_fft_plan_get(n, sign);
  double *w = (double *)malloc(sizeof(double) * 2 * (size_t)(n > 0 ? n : 1));
  orc_fft_exec(p, data, w);
  free(w);
}

/* Transform `nl` lines of length n; line l starts at base + l*lstride and
 * its elements are `estride` apart (in complex units).  Lines are processed
 * four at a time so strided gathers use whole cache lines. */
static void fft_lines(cplx *base, long nl, long lstride, long n, long estride,
                      int sign, int nthreads) {
  if (n <= 1) return;
  const orc_fft_plan *p = orc_fft_plan_get(n, sign);
  const long G = (estride == 1) ? 1 : 4;
  const long ngroups = (nl + G - 1) / G;
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1) if (nthreads > 1)
  {
    cplx *buf = (cplx *)malloc(sizeof(cplx) * (size_t)(n * G));
    cplx *wk = (cplx *)malloc(sizeof(cplx) * (size_t)n);
#pragma omp for schedule(static)
    for (long g = 0; g < ngroups; g++) {
      long l0 = g * G, gl = (l0 + G <= nl) ? G : nl - l0;
      if (estride == 1) {
        for (long t = 0; t < gl; t++)
          orc_fft_exec(p, (double *)(base + (l0 + t) * lstride), (double *)wk);
      } else {
        for (long e = 0; e < n; e++)
          for (long t = 0; t < gl; t++)
            buf[t * n + e] = base[(l0 + t) * lstride + e * estride];
        for (long t = 0; t < gl; t++)
          orc_fft_exec(p, (double *)(buf + t * n), (double *)wk);
        for (long e = 0; e < n; e++)
          for (long t = 0; t < gl; t++)
            base[(l0 + t) * lstride + e * estride] = buf[t * n + e];
      }
    }
    free(buf);
    free(wk);
  }
}

void orc_fft_3d(double *data, long n1, long n2, long n3, int sign,
                int nthreads) {
  cplx *x = (cplx *)data;
  /* along n3: n1*n2 contiguous lines */
  fft_lines(x, n1 * n2, n3, n3, 1, sign, nthreads);
  /* along n2: for each i1, n3 lines with stride n3; adjacent lines are
   * adjacent in memory so treat (i1, i3) as the line index */
  for (long i1 = 0; i1 < n1; i1++)
    fft_lines(x + i1 * n2 * n3, n3, 1, n2, n3, sign, nthreads);
  /* along n1: n2*n3 lines with element stride n2*n3 */
  fft_lines(x, n2 * n3, 1, n1, n2 * n3, sign, nthreads);
}

void orc_fft_3d_many(double *data, long K, long n1, long n2, long n3, int sign,
                     int nthreads) {
  for (long k = 0; k < K; k++)
    orc_fft_3d(data + 2 * k * n1 * n2 * n3, n1, n2, n3, sign, nthreads);
}
