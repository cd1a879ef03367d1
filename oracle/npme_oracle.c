/*
 * CPU restatement of npme's potential-evaluation path (FP64, C99 + OpenMP).
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle the GPU product is checked
 * against: tests/, the smoke check and bench.py's CPU-baseline leg call it;
 * the product never links or executes it.  Each function cites the reference
 * file:line (ElkingD/npme, paths relative to the project root) whose
 * algorithm it restates.  The restatement is pinned against the reference
 * itself, compiled from its own sources by oracle/ref/Makefile, in
 * tests/test_oracle_vs_reference.py and through the fixtures in tests/golden/.
 *
 * Layout conventions (same as the reference):
 *   coord[3n] xyz interleaved; real charges q[n]; complex charges as
 *   (re, im) pairs; V[n][4] = (V, dV/dx, dV/dy, dV/dz), complex V as
 *   (re, im) pairs per component.  Compact grids are (N1/2)(N2/2)(N3/2),
 *   row major, grid index p = m mod (N/2) for m in [-N/4, N/4).
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "fft.h"
#include "npme_oracle.h"

typedef double _Complex cplx;
#define ORC_PI 3.14159265358979323846

/* ------------------------------------------------------------------------ */
/* B-splines.  Cardinal B-spline of order n on (0, n) by the Cox-de Boor
 * recursion; the reference tabulates the same piecewise polynomials
 * explicitly (src/Bspline.cpp:16714, derivative :16766). */
double orc_bspline(int n, double w) {
  if (n < 1 || w < 0.0 || w >= (double)n) return 0.0;
  const int i0 = (int)floor(w);
  const double u = w - i0; /* w = i0 + u, 0 <= u < 1 */
  /* c[k] = B_j(u + k), k = 0..j-1, raised from j = 1 to j = n with
   * B_{j+1}(x) = [x B_j(x) + (j + 1 - x) B_j(x - 1)] / j */
  double c[64];
  c[0] = 1.0;
  for (int j = 1; j < n; j++) {
    for (int k = j; k >= 0; k--) {
      const double x = u + k;
      const double left = (k <= j - 1) ? c[k] : 0.0;
      const double right = (k >= 1) ? c[k - 1] : 0.0;
      c[k] = (x * left + ((double)(j + 1) - x) * right) / (double)j;
    }
  }
  return c[i0];
}

double orc_bspline_dB(int n, double w, double *dB) {
  /* dB_n/dw = B_{n-1}(w) - B_{n-1}(w - 1)  (src/Bspline.cpp:16771+) */
  *dB = orc_bspline(n - 1, w) - orc_bspline(n - 1, w - 1.0);
  return orc_bspline(n, w);
}

/* src/RecSumSupportFunctions.h:123-127 */
static long start_index(double w) {
  if (w < 0) return (long)(-w) + 1;
  return (long)(-w);
}
/* src/RecSumSupportFunctions.h:155-162: m -> array index on a length-M axis */
static long dft2array(long m, long M) { return m < 0 ? m + M : m; }
static long array2dft(long k, long M) { return k >= M / 2 ? k - M : k; }

/* ------------------------------------------------------------------------ */
/* Derivative-match coefficients. */

/* (1/r d/dr)^n r^alpha, src/FunctionDerivMatch.cpp:76-88 */
static void radial_deriv_ralpha(double *f, int N, double r, double alpha) {
  const double r2 = r * r;
  f[0] = pow(r, alpha);
  for (int n = 1; n <= N; n++) f[n] = f[n - 1] * (alpha - 2 * n + 2) / r2;
}

/* (1/r d/dr)^n exp(i k0 r)/r, src/FunctionDerivMatch.cpp:42-55 */
static void radial_deriv_helmholtz(cplx *f, int N, double r, cplx k0) {
  const double r2 = r * r;
  const cplx C = cexp(I * k0 * r), A = k0 * k0 / r2;
  f[0] = C / r;
  if (N >= 1) f[1] = -C / r / r2 + I * k0 * C / r2;
  for (int n = 2; n <= N; n++) f[n] = -(2.0 * n - 1.0) / r2 * f[n - 1] - A * f[n - 2];
}

/* C_np = Rdir^(2(p-n)) 2^n p!/(p-n)!, src/FunctionDerivMatch.cpp:226-236 */
static double calc_cnp(int n, int p, double Rdir) {
  if (n > p) return 0.0;
  double c = 1.0;
  for (int i = 0; i < p - n; i++) c *= Rdir * Rdir;
  for (int i = 0; i < n; i++) c *= 2.0;
  for (int i = p - n + 1; i <= p; i++) c *= (double)i;
  return c;
}

/* Back substitution for a[], then b[n] = 2(n+1) a[n+1],
 * src/FunctionDerivMatch.cpp:238-266 */
static void even_series(cplx *a, cplx *b, const cplx *f, int Nder, double Rdir) {
  for (int p = 0; p <= Nder; p++) {
    cplx s = f[Nder - p];
    for (int q = 0; q < p; q++) s -= calc_cnp(Nder - p, Nder - q, Rdir) * a[Nder - q];
    a[Nder - p] = s / calc_cnp(Nder - p, Nder - p, Rdir);
  }
  for (int i = 0; i <= Nder - 1; i++) b[i] = a[i + 1] * 2.0 * (i + 1);
  b[Nder] = 0;
}

int orc_dm_coeffs(int func, double alpha, double k0r, double k0i, int Nder,
                  double Rdir, double *a_out, double *b_out) {
  if (Nder < 2 || Nder > 30) return 1;
  cplx f[32], a[32], b[32];
  if (func == ORC_HELMHOLTZ) {
    radial_deriv_helmholtz(f, Nder, Rdir, k0r + I * k0i);
  } else {
    double fr[32];
    radial_deriv_ralpha(fr, Nder, Rdir, func == ORC_LAPLACE ? -1.0 : alpha);
    for (int i = 0; i <= Nder; i++) f[i] = fr[i];
  }
  even_series(a, b, f, Nder, Rdir);
  memcpy(a_out, a, sizeof(cplx) * (Nder + 1));
  memcpy(b_out, b, sizeof(cplx) * (Nder + 1));
  return 0;
}

/* beta with erfc(beta Rdir)/Rdir ~ tol by Newton iteration,
 * src/KernelFunctionLaplace.cpp:41-76 */
double orc_orig_beta(double Rdir, double tol) {
  const double C = log(sqrt(ORC_PI) * tol * Rdir);
  double x = 0.1;
  for (int n = 0; n < 1000; n++) {
    double F0 = x * x + log(x) + C, F1 = 2 * x + 1.0 / x;
    if (fabs(F0) < 1e-12) return x / Rdir;
    x -= F0 / F1;
  }
  return -1.0;
}

/* ------------------------------------------------------------------------ */
/* Kernels.  Each returns f0 and f1 = (1/r) df/dr for the requested part. */

typedef struct {
  int func, split, Nder;
  double Rdir, alpha, beta;
  cplx k0;
  cplx a[32], b[32];
} kern_t;

static void kern_init(kern_t *k, const orc_params *p) {
  memset(k, 0, sizeof(*k));
  k->func = p->func;
  k->split = p->split;
  k->Nder = p->nDeriv;
  k->Rdir = p->Rdir;
  k->alpha = p->alpha;
  k->k0 = p->k0r + I * p->k0i;
  if (p->split == ORC_SPLIT_DM)
    orc_dm_coeffs(p->func, p->alpha, p->k0r, p->k0i, p->nDeriv, p->Rdir,
                  (double *)k->a, (double *)k->b);
  else
    k->beta = orc_orig_beta(p->Rdir, p->tol);
}

/* Even-series Horner evaluation, src/FunctionDerivMatch.cpp:379-402 */
static cplx poly_f(const kern_t *k, double r2, cplx *f1) {
  const int N = k->Nder;
  cplx f0 = k->a[N - 1] + k->a[N] * r2;
  for (int i = N - 2; i >= 0; i--) f0 = f0 * r2 + k->a[i];
  cplx g = k->b[N - 2] + k->b[N - 1] * r2;
  for (int i = N - 3; i >= 0; i--) g = g * r2 + k->b[i];
  *f1 = g;
  return f0;
}

/* erf(x)/x and its (1/x d/dx), the reference's NPME_Berf_1
 * (src/MathFunctions.cpp) restated from the definition */
static double berf0(double x, double *b1) {
  if (x < 1e-3) {
    const double c = 2.0 / sqrt(ORC_PI);
    double x2 = x * x;
    *b1 = c * (-2.0 / 3.0 + x2 * (2.0 / 5.0 - x2 / 7.0));
    return c * (1.0 - x2 / 3.0 + x2 * x2 / 10.0);
  }
  double e = erf(x) / x;
  *b1 = (2.0 / sqrt(ORC_PI) * exp(-x * x) - e) / (x * x);
  return e;
}

/* Full kernel f (src/KernelFunctionLaplace.cpp, KernelFunctionRalpha.cpp,
 * KernelFunctionHelmholtz.cpp: NPME_Kfunc_*::Calc) */
static cplx kern_full(const kern_t *k, double r2, cplx *f1) {
  double r = sqrt(r2);
  if (k->func == ORC_LAPLACE) {
    double f0 = 1.0 / r;
    *f1 = -f0 / r2;
    return f0;
  } else if (k->func == ORC_RALPHA) {
    double f0 = pow(r2, k->alpha / 2);
    *f1 = k->alpha * f0 / r2;
    return f0;
  } else {
    cplx f0 = cexp(I * k->k0 * r) / r;
    *f1 = (I * k->k0 * f0 - f0 / r) / r;
    return f0;
  }
}

/* Smooth long-range part: DM polynomial inside Rdir, f outside
 * (src/KernelFunctionLaplace.cpp:394-436, KernelFunctionRalpha.cpp:342-384,
 * KernelFunctionHelmholtz.cpp:506-563); original Ewald beta*erf(beta r)/(beta r)
 * (src/KernelFunctionLaplace.cpp:1087-1118). */
static cplx kern_lr(const kern_t *k, double r2, cplx *f1) {
  if (k->split == ORC_SPLIT_ORIG) {
    double b1, b0 = berf0(sqrt(r2) * k->beta, &b1);
    *f1 = k->beta * k->beta * k->beta * b1;
    return k->beta * b0;
  }
  if (r2 > k->Rdir * k->Rdir) return kern_full(k, r2, f1);
  return poly_f(k, r2, f1);
}

/* Short-range part f - f_LR, zero beyond Rdir for DM
 * (src/PotentialLaplace.cpp:488-612, PotentialHelmholtz.cpp:353-418,
 * KernelFunctionRalpha.cpp:723-757); erfc(beta r)/r for the original split
 * (src/PotentialLaplace.cpp:614-719). */
static cplx kern_sr(const kern_t *k, double r2, cplx *f1) {
  if (k->split == ORC_SPLIT_ORIG) {
    double r = sqrt(r2), x = k->beta * r;
    double f0 = erfc(x) / r;
    *f1 = (-2.0 / sqrt(ORC_PI) * k->beta * exp(-x * x) - f0) / r2;
    return f0;
  }
  if (r2 > k->Rdir * k->Rdir) {
    *f1 = 0;
    return 0;
  }
  cplx g1, g0 = poly_f(k, r2, &g1);
  cplx e1, e0 = kern_full(k, r2, &e1);
  *f1 = e1 - g1;
  return e0 - g0;
}

/* ------------------------------------------------------------------------ */
/* Box: src/RecSumSupportFunctions.cpp:137-147 (CalcMinX_Compact), :182-201
 * (box dimension/centre), :276-296 (PME-corrected box). */
static double min_x_compact(double X0, double del, long order, long N) {
  const double a1 = 1.0 - 2.0 * (order + 1) / N;
  const double a2 = 1.0 - 4.0 * (order + 1) / N;
  double X = X0 / a1 - del / 2.0 * a2 / a1;
  return X0 > X ? X0 : X;
}

void orc_box(const orc_params *p, size_t n, const double *coord, double *box) {
  double mx[3] = {-1e12, -1e12, -1e12}, mn[3] = {1e12, 1e12, 1e12};
  for (size_t i = 0; i < n; i++)
    for (int d = 0; d < 3; d++) {
      double x = coord[3 * i + d];
      if (mx[d] < x) mx[d] = x;
      if (mn[d] > x) mn[d] = x;
    }
  for (int d = 0; d < 3; d++) {
    double X0 = mx[d] - mn[d], R0 = 0.5 * (mx[d] + mn[d]);
    double X = min_x_compact(X0, p->del[d], p->order, p->N[d]);
    box[d] = X;                       /* X, Y, Z */
    box[3 + d] = R0 + 0.5 * (X0 - X); /* R */
    box[6 + d] = 2 * (X + p->del[d]); /* L = 2 (X + del) */
  }
}

/* ------------------------------------------------------------------------ */
/* Fourier-extension window, src/RecSumGrid.cpp:1124-1231. */
static double hramp(double x, double a) {
  const double erf_max = 6.0;
  if (x < -1.0) return 0.0;
  if (x > 1.0) return 1.0;
  const double z = erf_max / a, xMax = z / sqrt(1.0 + z * z);
  if (x >= xMax) return 1.0;
  if (x <= -xMax) return 0.0;
  return 0.5 * (1.0 + erf(a * x / sqrt(1.0 - x * x)));
}

static double tsmooth(double x, double X, double Xmax, double a) {
  if (x < -X) {
    double del = (Xmax - X) * 0.5;
    return hramp((x + X + del) / del, a);
  } else if (x <= X) {
    return 1.0;
  } else {
    double del = (Xmax - X) * 0.5;
    return hramp((-x + X + del) / del, a);
  }
}

/* T1, T2 and the image coordinate x2, src/RecSumGrid.cpp:1181-1212 */
static void overlap_smooth(double *T1, double *T2, double *x2, long M,
                           const double *x1, double X, double Xmax, double a) {
  for (long i = 0; i < M; i++) {
    if (x1[i] > X) {
      T1[i] = tsmooth(x1[i], X, 2 * Xmax - X, a);
      x2[i] = x1[i] - 2 * Xmax;
      T2[i] = tsmooth(x2[i], X, 2 * Xmax - X, a);
    } else if (x1[i] > -X) {
      T1[i] = 1.0;
      x2[i] = 1.0;
      T2[i] = 0.0;
    } else {
      T1[i] = tsmooth(x1[i], X, 2 * Xmax - X, a);
      x2[i] = x1[i] + 2 * Xmax;
      T2[i] = tsmooth(x2[i], X, 2 * Xmax - X, a);
    }
  }
}

/* Compact Fourier transform of the smooth kernel on the (N/2+1)^3 octant:
 * sample with the 8-image Fourier extension (src/RecSumGrid.cpp:45-162,
 * 388-424), then the even-extension DFT along each axis
 * (src/RecSumGrid.cpp:470-582).  out: complex (N1/2+1)(N2/2+1)(N3/2+1). */
void orc_fhat_compact(const orc_params *p, const double *box, double *out) {
  kern_t k;
  kern_init(&k, p);
  long M[3];
  double *x1[3], *x2[3], *T1[3], *T2[3];
  for (int d = 0; d < 3; d++) {
    M[d] = p->N[d] / 2 + 1;
    double X = box[d], Xmax = box[d] + p->del[d], L = 2 * Xmax, h = L / p->N[d];
    x1[d] = malloc(sizeof(double) * M[d]);
    x2[d] = malloc(sizeof(double) * M[d]);
    T1[d] = malloc(sizeof(double) * M[d]);
    T2[d] = malloc(sizeof(double) * M[d]);
    for (long i = 0; i < M[d]; i++) x1[d][i] = i * h;
    overlap_smooth(T1[d], T2[d], x2[d], M[d], x1[d], X, Xmax, p->a[d]);
  }
  cplx *f = (cplx *)out;
  const long M1 = M[0], M2 = M[1], M3 = M[2];
#pragma omp parallel for schedule(static)
  for (long ij = 0; ij < M1 * M2; ij++) {
    long i1 = ij / M2, i2 = ij % M2;
    for (long i3 = 0; i3 < M3; i3++) {
      cplx s = 0;
      for (int c = 0; c < 8; c++) {
        int s1 = c >> 2, s2 = (c >> 1) & 1, s3 = c & 1;
        double xx = s1 ? x2[0][i1] : x1[0][i1];
        double yy = s2 ? x2[1][i2] : x1[1][i2];
        double zz = s3 ? x2[2][i3] : x1[2][i3];
        double t = (s1 ? T2[0][i1] : T1[0][i1]) * (s2 ? T2[1][i2] : T1[1][i2]) *
                   (s3 ? T2[2][i3] : T1[2][i3]);
        cplx f1, f0 = kern_lr(&k, xx * xx + yy * yy + zz * zz, &f1);
        s += t * f0;
      }
      f[(ij)*M3 + i3] = s;
    }
  }
  /* even-extension DFT along each axis, the same as NPME_Compact2FullGrid1D
   * + 1-D FFT + NPME_Full2CompactGrid1D */
  for (int d = 0; d < 3; d++) {
    const long N = p->N[d], Md = M[d];
    const long stride = d == 0 ? M2 * M3 : (d == 1 ? M3 : 1);
    const long nlines = M1 * M2 * M3 / Md;
#pragma omp parallel
    {
      cplx *xf = malloc(sizeof(cplx) * N), *wk = malloc(sizeof(cplx) * N);
      const orc_fft_plan *pl = orc_fft_plan_get(N, -1);
#pragma omp for schedule(static)
      for (long l = 0; l < nlines; l++) {
        long base;
        if (d == 0) base = l;
        else if (d == 1) base = (l / M3) * M2 * M3 + (l % M3);
        else base = l * M3;
        for (long i = 0; i < N / 2; i++) xf[i] = f[base + i * stride];
        for (long i = N / 2; i < N; i++) xf[i] = f[base + (N - i) * stride];
        orc_fft_exec(pl, (double *)xf, (double *)wk);
        f[base] = xf[0];
        f[base + (N / 2) * stride] = xf[N / 2];
        for (long i = 1; i < N / 2; i++) f[base + i * stride] = 0.5 * (xf[i] + xf[N - i]);
      }
      free(xf);
      free(wk);
    }
  }
  for (int d = 0; d < 3; d++) free(x1[d]), free(x2[d]), free(T1[d]), free(T2[d]);
}

/* |1 / sum_p B_n(p) exp(-2 pi i z p)|^2, src/RecSumV.cpp:565-581 */
void orc_lambda2(long N, int order, double *lam2) {
  for (long k = 0; k < N; k++) {
    double z = (double)array2dft(k, N) / (double)N;
    cplx den = 0;
    for (int p = 0; p <= order; p++) den += orc_bspline(order, p) * cexp(-2.0 * ORC_PI * I * z * p);
    cplx l = 1.0 / den;
    lam2[k] = creal(l * conj(l));
  }
}

/* ------------------------------------------------------------------------ */
/* Spread: Q[p] += conj(q) B1 B2 B3 on the compact grid,
 * src/RecSumQ.cpp:93-168 (NPME_RecSumQ_CalcQ1_Basic); real charges use q. */
void orc_spread(const orc_params *p, const double *box, size_t n,
                const double *coord, const double *q, int complex_q, double *Qout) {
  const long H1 = p->N[0] / 2, H2 = p->N[1] / 2, H3 = p->N[2] / 2;
  const int ord = p->order;
  cplx *Q = (cplx *)Qout;
  memset(Q, 0, sizeof(cplx) * H1 * H2 * H3);
  for (size_t i = 0; i < n; i++) {
    double w[3];
    long ms[3];
    double B[3][64];
    for (int d = 0; d < 3; d++) {
      w[d] = p->N[d] / box[6 + d] * (coord[3 * i + d] - box[3 + d]);
      ms[d] = start_index(w[d]);
      for (int t = 0; t < ord; t++) B[d][t] = orc_bspline(ord, w[d] + ms[d] + t);
    }
    cplx qi = complex_q ? conj(q[2 * i] + I * q[2 * i + 1]) : q[i];
    for (int t1 = 0; t1 < ord; t1++) {
      long p1 = dft2array(ms[0] + t1, H1);
      for (int t2 = 0; t2 < ord; t2++) {
        long p2 = dft2array(ms[1] + t2, H2);
        cplx c = qi * B[0][t1] * B[1][t2];
        for (int t3 = 0; t3 < ord; t3++) {
          long p3 = dft2array(ms[2] + t3, H3);
          Q[(p1 * H2 + p2) * H3 + p3] += c * B[2][t3];
        }
      }
    }
  }
}

/* theta from Q by 8 even/odd half-size transforms, src/RecSumV.cpp:766-840
 * with NPME_RecSumQ_CalcQfft (src/RecSumQ.cpp:466-522), the compact-F
 * multiply (src/RecSumV.cpp:639-707) and the twiddle accumulation
 * (src/RecSumV.cpp:709-761). */
void orc_theta(const orc_params *p, const double *fhat_in, const double *Qin,
               double *Tout, int nthreads) {
  const long N1 = p->N[0], N2 = p->N[1], N3 = p->N[2];
  const long M1 = N1 / 2, M2 = N2 / 2, M3 = N3 / 2;
  const long F2 = N2 / 2 + 1, F3 = N3 / 2 + 1;
  const cplx *F = (const cplx *)fhat_in, *Q = (const cplx *)Qin;
  cplx *T = (cplx *)Tout;
  cplx *X = malloc(sizeof(cplx) * M1 * M2 * M3);
  cplx *C[3];
  double *l2[3];
  for (int d = 0; d < 3; d++) {
    long N = p->N[d];
    C[d] = malloc(sizeof(cplx) * N / 2);
    l2[d] = malloc(sizeof(double) * N);
    for (long k = 0; k < N / 2; k++) C[d][k] = cexp(-2.0 * ORC_PI * I / N * array2dft(k, N / 2));
    orc_lambda2(N, p->order, l2[d]);
  }
  memset(T, 0, sizeof(cplx) * M1 * M2 * M3);
  for (int a1 = 0; a1 <= 1; a1++)
    for (int a2 = 0; a2 <= 1; a2++)
      for (int a3 = 0; a3 <= 1; a3++) {
        /* twiddle */
        for (long n1 = 0; n1 < M1; n1++)
          for (long n2 = 0; n2 < M2; n2++) {
            cplx c = 1.0;
            if (a1) c = C[0][n1];
            if (a2) c *= C[1][n2];
            long base = (n1 * M2 + n2) * M3;
            for (long n3 = 0; n3 < M3; n3++)
              X[base + n3] = Q[base + n3] * c * (a3 ? C[2][n3] : 1.0);
          }
        orc_fft_3d((double *)X, M1, M2, M3, -1, nthreads);
        /* C conj(X) F lambda^2 / (N1 N2 N3) with |m| folding of compact F */
        for (long n1 = 0; n1 < M1; n1++)
          for (long n2 = 0; n2 < M2; n2++) {
            long mt1 = 2 * array2dft(n1, M1) + a1, mt2 = 2 * array2dft(n2, M2) + a2;
            long f1 = labs(mt1), f2 = labs(mt2);
            double c = l2[0][dft2array(mt1, N1)] * l2[1][dft2array(mt2, N2)] /
                       ((double)N1 * N2 * N3);
            long base = (n1 * M2 + n2) * M3;
            for (long n3 = 0; n3 < M3; n3++) {
              long mt3 = 2 * array2dft(n3, M3) + a3;
              long f3 = labs(mt3);
              X[base + n3] = c * conj(X[base + n3]) * F[(f1 * F2 + f2) * F3 + f3] *
                             l2[2][dft2array(mt3, N3)];
            }
          }
        orc_fft_3d((double *)X, M1, M2, M3, -1, nthreads);
        for (long n1 = 0; n1 < M1; n1++)
          for (long n2 = 0; n2 < M2; n2++) {
            cplx c = 1.0;
            if (a1) c = C[0][n1];
            if (a2) c *= C[1][n2];
            long base = (n1 * M2 + n2) * M3;
            for (long n3 = 0; n3 < M3; n3++)
              T[base + n3] += X[base + n3] * c * (a3 ? C[2][n3] : 1.0);
          }
      }
  for (int d = 0; d < 3; d++) free(C[d]), free(l2[d]);
  free(X);
}

/* Interpolation V = sum theta B1 B2 B3 (+ gradient by dB), accumulated into
 * V; real kernels keep the real part.  src/RecSumV.cpp:44-149 (Basic) and
 * :395-398 (creal). */
void orc_interp(const orc_params *p, const double *box, size_t n,
                const double *coord, const double *Tin, int complex_out,
                double *Vout) {
  const long H1 = p->N[0] / 2, H2 = p->N[1] / 2, H3 = p->N[2] / 2;
  const int ord = p->order;
  const cplx *T = (const cplx *)Tin;
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < n; i++) {
    double w[3], C[3];
    long ms[3];
    double B[3][64], D[3][64];
    for (int d = 0; d < 3; d++) {
      C[d] = p->N[d] / box[6 + d];
      w[d] = C[d] * (coord[3 * i + d] - box[3 + d]);
      ms[d] = start_index(w[d]);
      for (int t = 0; t < ord; t++) B[d][t] = orc_bspline_dB(ord, w[d] + ms[d] + t, &D[d][t]);
    }
    cplx v[4] = {0, 0, 0, 0};
    for (int t1 = 0; t1 < ord; t1++) {
      long p1 = dft2array(ms[0] + t1, H1);
      for (int t2 = 0; t2 < ord; t2++) {
        long p2 = dft2array(ms[1] + t2, H2);
        double A1 = B[0][t1] * B[1][t2], A2 = D[0][t1] * B[1][t2], A3 = B[0][t1] * D[1][t2];
        cplx tb = 0, td = 0;
        for (int t3 = 0; t3 < ord; t3++) {
          long p3 = dft2array(ms[2] + t3, H3);
          cplx th = T[(p1 * H2 + p2) * H3 + p3];
          tb += th * B[2][t3];
          td += th * D[2][t3];
        }
        v[0] += A1 * tb;
        v[1] += A2 * tb;
        v[2] += A3 * tb;
        v[3] += A1 * td;
      }
    }
    v[1] *= C[0];
    v[2] *= C[1];
    v[3] *= C[2];
    if (complex_out) {
      cplx *Vc = (cplx *)Vout;
      for (int c = 0; c < 4; c++) Vc[4 * i + c] += v[c];
    } else {
      for (int c = 0; c < 4; c++) Vout[4 * i + c] += creal(v[c]);
    }
  }
}

/* ------------------------------------------------------------------------ */
/* Short-range direct sum over all pairs i != j with r_ij <= Rdir (DM: the
 * kernel vanishes beyond Rdir; src/PotentialLaplace.cpp:201-264 with the
 * pair kernels cited at kern_sr).  The pairs are found with a uniform cell
 * list of edge >= Rdir; V is overwritten. */
void orc_direct(const orc_params *p, size_t n, const double *coord,
                const double *q, int complex_q, double *Vout) {
  kern_t k;
  kern_init(&k, p);
  const double R = p->Rdir, R2 = R * R;
  double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
  for (size_t i = 0; i < n; i++)
    for (int d = 0; d < 3; d++) {
      if (coord[3 * i + d] < mn[d]) mn[d] = coord[3 * i + d];
      if (coord[3 * i + d] > mx[d]) mx[d] = coord[3 * i + d];
    }
  long nc[3];
  for (int d = 0; d < 3; d++) {
    nc[d] = (long)floor((mx[d] - mn[d]) / R) + 1;
    if (nc[d] < 1) nc[d] = 1;
  }
  const long ncell = nc[0] * nc[1] * nc[2];
  long *cnt = calloc(ncell + 1, sizeof(long)), *idx = malloc(sizeof(long) * (n ? n : 1));
  long *cell_of = malloc(sizeof(long) * (n ? n : 1));
  for (size_t i = 0; i < n; i++) {
    long c[3];
    for (int d = 0; d < 3; d++) {
      c[d] = (long)floor((coord[3 * i + d] - mn[d]) / R);
      if (c[d] >= nc[d]) c[d] = nc[d] - 1;
    }
    cell_of[i] = (c[0] * nc[1] + c[1]) * nc[2] + c[2];
    cnt[cell_of[i] + 1]++;
  }
  for (long c = 0; c < ncell; c++) cnt[c + 1] += cnt[c];
  long *fill = malloc(sizeof(long) * (ncell ? ncell : 1));
  memcpy(fill, cnt, sizeof(long) * ncell);
  for (size_t i = 0; i < n; i++) idx[fill[cell_of[i]]++] = (long)i;
  free(fill);
#pragma omp parallel for schedule(dynamic, 64)
  for (size_t i = 0; i < n; i++) {
    long c = cell_of[i];
    long c1 = c / (nc[1] * nc[2]), c2 = (c / nc[2]) % nc[1], c3 = c % nc[2];
    cplx v[4] = {0, 0, 0, 0};
    for (long d1 = c1 - 1; d1 <= c1 + 1; d1++) {
      if (d1 < 0 || d1 >= nc[0]) continue;
      for (long d2 = c2 - 1; d2 <= c2 + 1; d2++) {
        if (d2 < 0 || d2 >= nc[1]) continue;
        for (long d3 = c3 - 1; d3 <= c3 + 1; d3++) {
          if (d3 < 0 || d3 >= nc[2]) continue;
          long cc = (d1 * nc[1] + d2) * nc[2] + d3;
          for (long t = cnt[cc]; t < cnt[cc + 1]; t++) {
            long j = idx[t];
            if (j == (long)i) continue;
            double x = coord[3 * i] - coord[3 * j], y = coord[3 * i + 1] - coord[3 * j + 1],
                   z = coord[3 * i + 2] - coord[3 * j + 2];
            double r2 = x * x + y * y + z * z;
            if (r2 > R2) continue;
            cplx f1, f0 = kern_sr(&k, r2, &f1);
            cplx qj = complex_q ? q[2 * j] + I * q[2 * j + 1] : q[j];
            v[0] += f0 * qj;
            v[1] += x * f1 * qj;
            v[2] += y * f1 * qj;
            v[3] += z * f1 * qj;
          }
        }
      }
    }
    if (complex_q) {
      cplx *Vc = (cplx *)Vout;
      for (int m = 0; m < 4; m++) Vc[4 * i + m] = v[m];
    } else {
      for (int m = 0; m < 4; m++) Vout[4 * i + m] = creal(v[m]);
    }
  }
  free(cnt);
  free(idx);
  free(cell_of);
}

/* f_LR(0): a[0] for DM, 2 beta / sqrt(pi) for the original split
 * (src/Interface.cpp:1946-1952). */
static cplx fself(const kern_t *k) {
  cplx f1;
  if (k->split == ORC_SPLIT_ORIG) return kern_lr(k, 0.0, &f1);
  return k->a[0];
}

/* Exact O(N^2) sum with the full kernel, no self term
 * (src/PotentialLaplace.cpp:40-132, PotentialHelmholtz.cpp:41,
 * PotentialGenFunc.cpp:321).  Targets [t0, t1) only, so large systems can be
 * checked on a sample; V has (t1 - t0) rows. */
void orc_exact(const orc_params *p, size_t n, const double *coord,
               const double *q, int complex_q, size_t t0, size_t t1, double *Vout) {
  kern_t k;
  kern_init(&k, p);
#pragma omp parallel for schedule(dynamic, 16)
  for (size_t i = t0; i < t1; i++) {
    cplx v[4] = {0, 0, 0, 0};
    for (size_t j = 0; j < n; j++) {
      if (j == i) continue;
      double x = coord[3 * i] - coord[3 * j], y = coord[3 * i + 1] - coord[3 * j + 1],
             z = coord[3 * i + 2] - coord[3 * j + 2];
      cplx f1, f0 = kern_full(&k, x * x + y * y + z * z, &f1);
      cplx qj = complex_q ? q[2 * j] + I * q[2 * j + 1] : q[j];
      v[0] += f0 * qj;
      v[1] += x * f1 * qj;
      v[2] += y * f1 * qj;
      v[3] += z * f1 * qj;
    }
    if (complex_q) {
      cplx *Vc = (cplx *)Vout;
      for (int m = 0; m < 4; m++) Vc[4 * (i - t0) + m] = v[m];
    } else {
      for (int m = 0; m < 4; m++) Vout[4 * (i - t0) + m] = creal(v[m]);
    }
  }
}

/* CalcV: direct + self + reciprocal sum (src/Interface.cpp:2017-2100). */
int orc_calcv(const orc_params *p, size_t n, const double *coord, const double *q,
              int complex_q, double *V, int nthreads) {
  kern_t k;
  kern_init(&k, p);
  double box[9];
  orc_box(p, n, coord, box);
  const long H = (p->N[0] / 2) * (p->N[1] / 2) * (p->N[2] / 2);
  const long FS = (p->N[0] / 2 + 1) * (p->N[1] / 2 + 1) * (p->N[2] / 2 + 1);
  double *F = malloc(sizeof(cplx) * FS), *Q = malloc(sizeof(cplx) * H),
         *T = malloc(sizeof(cplx) * H);
  if (!F || !Q || !T) return 2;
  orc_direct(p, n, coord, q, complex_q, V);
  cplx fs = fself(&k);
  for (size_t i = 0; i < n; i++) {
    if (complex_q) {
      cplx *Vc = (cplx *)V;
      Vc[4 * i] -= fs * (q[2 * i] + I * q[2 * i + 1]);
    } else {
      V[4 * i] -= creal(fs) * q[i];
    }
  }
  orc_fhat_compact(p, box, F);
  orc_spread(p, box, n, coord, q, complex_q, Q);
  orc_theta(p, F, Q, T, nthreads);
  orc_interp(p, box, n, coord, T, complex_q, V);
  free(F);
  free(Q);
  free(T);
  return 0;
}
