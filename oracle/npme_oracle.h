/*
 * CPU oracle: FP64 restatement of npme's potential-evaluation path.
 * TEST INFRASTRUCTURE ONLY (see npme_oracle.c).
 */
#ifndef NPME_ORACLE_H
#define NPME_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_LAPLACE = 0, ORC_RALPHA = 1, ORC_HELMHOLTZ = 2 };
enum { ORC_SPLIT_DM = 0, ORC_SPLIT_ORIG = 1 };

typedef struct {
  int func;    /* ORC_LAPLACE, ORC_RALPHA, ORC_HELMHOLTZ */
  int split;   /* ORC_SPLIT_DM, ORC_SPLIT_ORIG */
  int nDeriv;  /* derivative-match order */
  int order;   /* B-spline order (BnOrder) */
  double alpha, k0r, k0i, Rdir, tol;
  long N[3];   /* full FFT box N1, N2, N3 */
  double a[3], del[3];
} orc_params;

double orc_bspline(int n, double w);
double orc_bspline_dB(int n, double w, double *dB);
int orc_dm_coeffs(int func, double alpha, double k0r, double k0i, int Nder,
                  double Rdir, double *a, double *b);
double orc_orig_beta(double Rdir, double tol);
/* box[9] = X, Y, Z, R[3], L[3] */
void orc_box(const orc_params *p, size_t n, const double *coord, double *box);
void orc_fhat_compact(const orc_params *p, const double *box, double *out);
void orc_lambda2(long N, int order, double *lam2);
void orc_spread(const orc_params *p, const double *box, size_t n,
                const double *coord, const double *q, int complex_q, double *Q);
void orc_theta(const orc_params *p, const double *fhat, const double *Q,
               double *T, int nthreads);
void orc_interp(const orc_params *p, const double *box, size_t n,
                const double *coord, const double *T, int complex_out,
                double *V);
void orc_direct(const orc_params *p, size_t n, const double *coord,
                const double *q, int complex_q, double *V);
void orc_exact(const orc_params *p, size_t n, const double *coord,
               const double *q, int complex_q, size_t t0, size_t t1, double *V);
int orc_calcv(const orc_params *p, size_t n, const double *coord,
              const double *q, int complex_q, double *V, int nthreads);

#ifdef __cplusplus
}
#endif

#endif
