/*
 * Project-written per-lane stand-ins for the Intel SVML vector math
 * intrinsics the reference's AVX code calls (_mm256_exp_pd, _mm256_sincos_pd,
 * _mm256_pow_pd, _mm256_erf_pd, _mm256_erfc_pd).  GCC has no SVML, so the
 * timed AVX2 build of the reference force-includes this header; each lane is
 * evaluated with the C library.  TEST INFRASTRUCTURE ONLY (CPU baseline).
 */
#ifndef NPME_ORACLE_SVML_SHIM_H
#define NPME_ORACLE_SVML_SHIM_H
#ifdef __AVX__
#include <immintrin.h>
#include <math.h>

#define NPME_SHIM_LANEWISE1(name, fn)                        \
  static inline __m256d name(__m256d a) {                    \
    double t[4] __attribute__((aligned(32)));                \
    _mm256_store_pd(t, a);                                   \
    for (int i = 0; i < 4; i++) t[i] = fn(t[i]);             \
    return _mm256_load_pd(t);                                \
  }
NPME_SHIM_LANEWISE1(_mm256_exp_pd, exp)
NPME_SHIM_LANEWISE1(_mm256_erf_pd, erf)
NPME_SHIM_LANEWISE1(_mm256_erfc_pd, erfc)
#undef NPME_SHIM_LANEWISE1

static inline __m256d _mm256_pow_pd(__m256d a, __m256d b) {
  double x[4] __attribute__((aligned(32))), y[4] __attribute__((aligned(32)));
  _mm256_store_pd(x, a);
  _mm256_store_pd(y, b);
  for (int i = 0; i < 4; i++) x[i] = pow(x[i], y[i]);
  return _mm256_load_pd(x);
}

static inline __m256d _mm256_sincos_pd(__m256d *cos_out, __m256d a) {
  double x[4] __attribute__((aligned(32))), s[4] __attribute__((aligned(32))),
      c[4] __attribute__((aligned(32)));
  _mm256_store_pd(x, a);
  for (int i = 0; i < 4; i++) s[i] = sin(x[i]), c[i] = cos(x[i]);
  *cos_out = _mm256_load_pd(c);
  return _mm256_load_pd(s);
}
#endif
#endif
