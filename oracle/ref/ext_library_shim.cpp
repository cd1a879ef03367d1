// Project-written replacement for the reference's MKL wrapper translation
// unit (src/ExtLibrary.cpp).  TEST INFRASTRUCTURE ONLY: it exists so that the
// reference's own sources can be compiled here with g++ (Intel MKL and icpx
// are not installed) and used as the parity oracle and the timed CPU
// baseline.  It implements exactly the functions the reference links against
// (found with `nm --undefined-only` on the other 23 objects):
//
//   NPME_1D_FFT_NoNorm, NPME_3D_FFT_NoNorm    (src/ExtLibrary.h:253-262)
//   NPME_TransposeComplex                      (src/ExtLibrary.h:43)
//   NPME_SolveLinearSystem(Complex)            (src/ExtLibrary.h:49-65)
//   NPME_RandomNumberArray                     (src/ExtLibrary.h:33)
//   NPME_malloc / NPME_free                    (src/ExtLibrary.h:27-29)
//   mkl_set_num_threads                        (the MKL threading knob)
//
// The FFTs are the oracle's own mixed-radix FFT (oracle/fft.c): same sign and
// normalisation as MKL's DFTI_FORWARD without scaling.  They are slower than
// MKL, which makes the reciprocal-sum part of the CPU baseline slower than it
// would be with MKL.
#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "ExtLibrary.h"
#include "../fft.h"

static int g_mkl_threads = 1;

extern "C" void mkl_set_num_threads(int nt) { g_mkl_threads = nt > 0 ? nt : 1; }

namespace NPME_Library {

void *NPME_malloc(size_t size, size_t alignment) {
  void *p = nullptr;
  if (alignment < sizeof(void *)) alignment = sizeof(void *);
  size_t sz = (size + alignment - 1) / alignment * alignment;
  if (posix_memalign(&p, alignment, sz ? sz : alignment) != 0) return nullptr;
  return p;
}

void NPME_free(void *ptr) { free(ptr); }

// Not MKL's R250 stream: a 64-bit LCG mapped to [a, b).  Only the reference's
// input generator (app/makeRandomBox.cpp) uses it; the harness supplies its
// own inputs.
void NPME_RandomNumberArray(const size_t N, double *x, const double a,
                            const double b, const size_t seed) {
  unsigned long long s = 0x9E3779B97F4A7C15ULL ^ (unsigned long long)seed;
  for (size_t i = 0; i < N; i++) {
    s = s * 6364136223846793005ULL + 1442695040888963407ULL;
    double u = (double)(s >> 11) * (1.0 / 9007199254740992.0);
    x[i] = a + (b - a) * u;
  }
}

void NPME_TransposeComplex(const size_t M, const size_t N, _Complex double *A) {
  std::vector<_Complex double> tmp(A, A + M * N);
  for (size_t i = 0; i < M; i++)
    for (size_t j = 0; j < N; j++) A[j * M + i] = tmp[i * N + j];
}

template <class T>
static bool gauss_solve(size_t N, size_t M, T *A, T *X) {
  // A[N][N] * X[N][M] = B (B in X on entry).  Partial pivoting.
  for (size_t c = 0; c < N; c++) {
    size_t piv = c;
    double best = std::abs(A[c * N + c]);
    for (size_t r = c + 1; r < N; r++) {
      double v = std::abs(A[r * N + c]);
      if (v > best) best = v, piv = r;
    }
    if (best == 0.0) return false;
    if (piv != c) {
      for (size_t k = 0; k < N; k++) std::swap(A[c * N + k], A[piv * N + k]);
      for (size_t k = 0; k < M; k++) std::swap(X[c * M + k], X[piv * M + k]);
    }
    for (size_t r = c + 1; r < N; r++) {
      T f = A[r * N + c] / A[c * N + c];
      for (size_t k = c; k < N; k++) A[r * N + k] -= f * A[c * N + k];
      for (size_t k = 0; k < M; k++) X[r * M + k] -= f * X[c * M + k];
    }
  }
  for (size_t c = N; c-- > 0;) {
    for (size_t k = 0; k < M; k++) {
      T s = X[c * M + k];
      for (size_t j = c + 1; j < N; j++) s -= A[c * N + j] * X[j * M + k];
      X[c * M + k] = s / A[c * N + c];
    }
  }
  return true;
}

bool NPME_SolveLinearSystem(const size_t N, const size_t M, double *A, double *b,
                            double *x) {
  std::vector<std::complex<double>> Ac(A, A + N * N), Xc(b, b + N * M);
  if (!gauss_solve(N, M, Ac.data(), Xc.data())) return false;
  for (size_t i = 0; i < N * M; i++) x[i] = Xc[i].real();
  return true;
}

bool NPME_SolveLinearSystemComplex(const size_t N, const size_t M,
                                   _Complex double *A, _Complex double *b,
                                   _Complex double *x) {
  std::vector<std::complex<double>> Ac(N * N), Xc(N * M);
  memcpy(Ac.data(), A, sizeof(_Complex double) * N * N);
  memcpy(Xc.data(), b, sizeof(_Complex double) * N * M);
  if (!gauss_solve(N, M, Ac.data(), Xc.data())) return false;
  memcpy(x, Xc.data(), sizeof(_Complex double) * N * M);
  return true;
}

void NPME_1D_FFT_NoNorm(_Complex double *F, long int N1) {
  const orc_fft_plan *p = orc_fft_plan_get(N1, -1);
  std::vector<double> wk(2 * (size_t)N1);
  orc_fft_exec(p, (double *)F, wk.data());
}

void NPME_3D_FFT_NoNorm(_Complex double *F, long int N1, long int N2,
                        long int N3) {
  orc_fft_3d((double *)F, N1, N2, N3, -1, g_mkl_threads);
}

}  // namespace NPME_Library
