// FFT box choice by measurement (npme_gpu_choose_grid).
//
// The reference fills in a missing FFT box in NPME_AddMissingKeywords
// (src/Interface.cpp:256-432) from its RSEM model, which predicts the RMS
// absolute potential error eps_V of the reciprocal sum from fitted
// polynomials (src/EstimateParm.cpp:210-420) and solves eps_V(N) = tol.
// On a GPU a few solves of the system itself cost less than the model's
// caveats (its fits cover given kernels, orders and derivative degrees), so
// this chooser measures: it samples up to kTargets points, computes their
// exact potentials once (FP64 O(n m)), then solves on successively finer
// boxes until the RMS absolute error of V over the sample is <= tol.  The
// next spacing comes from the measured error and the B-spline order P
// (reciprocal-sum error ~ h^P), damped so that a step refines by at most 2x
// and at least 10 %.  Boxes are uniform in spacing, FFT-friendly (2,3,5
// smooth multiples of 4) and PME-corrected per axis like the reference's.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "internal.h"

namespace {

constexpr size_t kTargets = 4096;
constexpr int kMaxTrials = 14;

long nice_fft(long n) {
  n = std::max(4L, n);
  for (;; n++) {
    if (n % 4) continue;
    long m = n;
    for (long f : {2L, 3L, 5L})
      while (m % f == 0) m /= f;
    if (m == 1) return n;
  }
}

// FFT box of spacing <= h for half extents X0 (iterated twice: the PME
// correction of the extent depends on N)
void box_for_spacing(const double *X0, const double *del, int order, double h, long *N) {
  for (int d = 0; d < 3; d++) {
    long n = nice_fft((long)std::ceil(2.0 * (X0[d] + del[d]) / h));
    for (int it = 0; it < 2; it++) {
      const double X = npme::compact_extent(X0[d], del[d], order, n);
      n = nice_fft((long)std::ceil(2.0 * (X + del[d]) / h));
    }
    n = std::max(n, nice_fft(4L * (order + 1)));  // order < N/4
    N[d] = n;
  }
}

// device bytes of the FFT arrays (grid, spectrum, kernel transform)
double fft_gb(const long *N, bool cplx, bool fp32) {
  const double s = fp32 ? 4 : 8;
  const double n3 = (double)N[0] * N[1] * N[2];
  const double oct = (double)(N[0] / 2 + 1) * (N[1] / 2 + 1) * (N[2] / 2 + 1);
  const double grid = cplx ? 2 * s * n3 : s * n3 + 2 * s * N[0] * N[1] * (N[2] / 2 + 1);
  return (grid + oct * s * (cplx ? 2 : 1)) / 1e9;
}

}  // namespace

extern "C" int npme_gpu_choose_grid(const npme_params *p, size_t n, const double *coord,
                                    const double *charge, double tol, double maxFFTmemGB,
                                    npme_params *out, double *err) {
  if (!p || !coord || !charge || !out || n < 2) return NPME_EINVAL;
  if (!(tol > 0) || !(maxFFTmemGB > 0)) return NPME_EINVAL;
  const bool cplx = p->funcType == NPME_FUNC_HELMHOLTZ;
  const bool fp32 = p->precision == NPME_PREC_FP32;
  const int order = p->BnOrder;
  const double del[3] = {p->del1 > 0 ? p->del1 : p->Rdir, p->del2 > 0 ? p->del2 : p->Rdir,
                         p->del3 > 0 ? p->del3 : p->Rdir};
  double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
  for (size_t i = 0; i < n; i++)
    for (int d = 0; d < 3; d++) {
      mn[d] = std::min(mn[d], coord[3 * i + d]);
      mx[d] = std::max(mx[d], coord[3 * i + d]);
    }
  const double X0[3] = {0.5 * (mx[0] - mn[0]), 0.5 * (mx[1] - mn[1]), 0.5 * (mx[2] - mn[2])};

  // sampled targets, evenly spread over the caller's index order
  const size_t m = std::min(n, kTargets);
  std::vector<unsigned int> tid(m);
  for (size_t k = 0; k < m; k++) tid[k] = (unsigned int)(((2 * k + 1) * n) / (2 * m));

  npme_params q = *p;
  double h = 0.5 * p->Rdir;  // coarse start
  long N[3];
  box_for_spacing(X0, del, order, h, N);
  q.N1 = N[0], q.N2 = N[1], q.N3 = N[2];
  npme_handle *hd = nullptr;
  int rc = npme_gpu_create(&q, &hd);
  if (rc) return rc;
  const int C = cplx ? 2 : 1;
  std::vector<double> Vex(4 * C * m), V(4 * C * n);
  rc = npme_gpu_setup(hd, n, coord);
  if (!rc) rc = npme_gpu_calcv_exact_subset(hd, Vex.data(), m, tid.data(), charge);
  double best_err = INFINITY;
  long best[3] = {N[0], N[1], N[2]};
  for (int trial = 0; !rc && trial < kMaxTrials; trial++) {
    rc = cplx ? npme_gpu_calcv_complex(hd, V.data(), n, charge, nullptr)
              : npme_gpu_calcv_real(hd, V.data(), n, charge, nullptr);
    if (rc) break;
    double e2 = 0;
    for (size_t k = 0; k < m; k++) {
      const double *a = &V[4 * C * tid[k]], *b = &Vex[4 * C * k];
      for (int c = 0; c < C; c++) e2 += (a[c] - b[c]) * (a[c] - b[c]);
    }
    const double e = std::sqrt(e2 / (double)m);
    if (e < best_err) best_err = e, best[0] = N[0], best[1] = N[1], best[2] = N[2];
    if (e <= tol) break;
    // next spacing from e ~ h^P, refining by 10 % to 2x per step
    double f = std::pow(0.9 * tol / e, 1.0 / order);
    f = std::min(0.9, std::max(0.5, f));
    long Nn[3];
    box_for_spacing(X0, del, order, h * f, Nn);
    if (fft_gb(Nn, cplx, fp32) > maxFFTmemGB || std::max({Nn[0], Nn[1], Nn[2]}) > 2048) break;
    h *= f;
    std::memcpy(N, Nn, sizeof N);
    q.N1 = N[0], q.N2 = N[1], q.N3 = N[2];
    rc = npme_gpu_set_params(hd, &q);
    if (!rc) rc = npme_gpu_setup(hd, n, coord);
  }
  npme_gpu_destroy(hd);
  if (rc) return rc;
  *out = *p;
  out->N1 = best[0], out->N2 = best[1], out->N3 = best[2];
  if (err) *err = best_err;
  return NPME_OK;
}
