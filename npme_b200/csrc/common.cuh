// Device-side building blocks shared by the npme_b200 kernels: B-spline
// weights, the short-range / full pair kernels and small vector helpers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

namespace npme {

constexpr int kMaxDeriv = 15;  // derivative-match order supported on device

template <typename T> struct Vec2;
template <> struct Vec2<float> { using type = float2; };
template <> struct Vec2<double> { using type = double2; };

// Pair-kernel constants, passed by value to the kernels.  Polynomial
// coefficients are stored in the scaled variable s = r^2 / Rdir^2:
//   f_LR(r) = sum_n ar[n] s^n,   (1/r) d f_LR / dr = sum_n br[n] s^n
// (the reference's a_n r^(2n) and b_n r^(2n), src/FunctionDerivMatch.cpp:379-402,
// with a_n Rdir^(2n) folded in, which keeps the coefficients O(1/Rdir)).
template <typename T>
struct PairCoef {
  int func;   // 0 Laplace, 1 Ralpha, 2 Helmholtz
  int split;  // 0 derivative match, 1 original Ewald
  int nder;
  T R2, invR2;
  T alpha, half_alpha;
  T beta, beta2, two_beta_rpi;  // original Ewald: beta, beta^2, 2 beta/sqrt(pi)
  T k0r, k0i;
  T ar[kMaxDeriv + 1], ai[kMaxDeriv + 1];
  T br[kMaxDeriv + 1], bi[kMaxDeriv + 1];
  // Packed (two pairs per instruction) evaluation of the real kernels
  // works in coordinates scaled by 1/Rdir, so r^2 is s itself.  With
  // alpha = -1 for 1/r it accumulates
  //   f0' = s^(alpha/2) - Rdir^(-alpha) f_LR  = Rdir^(-alpha) f0,
  //   t'  = Rdir^(2-alpha) d - alpha s^(alpha/2) / s = -Rdir^(2-alpha) f1,
  // so V = vscale sum q f0' and grad V = -gscale sum q t' x' with
  // vscale = Rdir^alpha, gscale = Rdir^(alpha-1).  Coefficient pairs:
  // nar2[n] = -Rdir^(-alpha) ar[n], br2[n] = Rdir^(2-alpha) br[n].
  typename Vec2<T>::type nar2[kMaxDeriv + 1], br2[kMaxDeriv + 1];
  double invR, vscale, gscale;
  // Helmholtz packed evaluation: (re, im) pairs of -ar/-ai and -br/-bi
  typename Vec2<T>::type nac2[kMaxDeriv + 1], nbc2[kMaxDeriv + 1];
};

template <typename T> struct Vec4;
template <> struct Vec4<float> { using type = float4; };
template <> struct Vec4<double> { using type = double4; };

__device__ __forceinline__ float rsqrt_t(float x) { return rsqrtf(x); }
__device__ __forceinline__ double rsqrt_t(double x) { return rsqrt(x); }
__device__ __forceinline__ float sqrt_t(float x) { return sqrtf(x); }
__device__ __forceinline__ double sqrt_t(double x) { return sqrt(x); }
__device__ __forceinline__ float exp_t(float x) { return expf(x); }
__device__ __forceinline__ double exp_t(double x) { return exp(x); }
__device__ __forceinline__ float pow_t(float x, float y) { return powf(x, y); }
__device__ __forceinline__ double pow_t(double x, double y) { return pow(x, y); }
// x^y for x > 0 as 2^(y log2 x): the r^alpha kernel's power; in FP64 about
// 5e-16 relative (log2 and exp2 each within an ulp, |y log2 x| < ~8 here),
// cheaper than pow's special-case handling
__device__ __forceinline__ float rpow_t(float x, float y) { return powf(x, y); }
__device__ __forceinline__ double rpow_t(double x, double y) { return exp2(y * log2(x)); }
__device__ __forceinline__ float erfc_t(float x) { return erfcf(x); }
__device__ __forceinline__ double erfc_t(double x) { return erfc(x); }
__device__ __forceinline__ void sincos_t(float x, float *s, float *c) { sincosf(x, s, c); }
__device__ __forceinline__ void sincos_t(double x, double *s, double *c) { sincos(x, s, c); }

// Cardinal B-spline weights of order P at the stencil points u + t,
// t = 0..P-1, with u = w + mStart in [0, 1] (the reference evaluates
// B_P(w + m) for m = mStart..mStart+P-1, src/RecSumQ.cpp:58-84).  Raised by
// B_{j+1}(x) = [x B_j(x) + (j + 1 - x) B_j(x - 1)] / j.  The derivative uses
// dB_P/dw (x) = B_{P-1}(x) - B_{P-1}(x - 1) (src/Bspline.cpp:16766).
template <typename T, int P, bool DERIV>
__device__ __forceinline__ void bspline_weights(T u, T (&w)[P], T (&dw)[P]) {
  T c[P];
  c[0] = T(1);
#pragma unroll
  for (int k = 1; k < P; k++) c[k] = T(0);
#pragma unroll
  for (int j = 1; j < P; j++) {
    if (DERIV && j == P - 1) {
#pragma unroll
      for (int t = 0; t < P; t++) {
        const T cur = (t <= P - 2) ? c[t] : T(0);
        const T prev = (t >= 1) ? c[t - 1] : T(0);
        dw[t] = cur - prev;
      }
    }
    const T inv = T(1) / T(j);
#pragma unroll
    for (int k = j; k >= 0; k--) {
      const T x = u + T(k);
      const T left = (k <= j - 1) ? c[k] : T(0);
      const T right = (k >= 1) ? c[k - 1] : T(0);
      c[k] = (x * left + (T(j + 1) - x) * right) * inv;
    }
  }
#pragma unroll
  for (int t = 0; t < P; t++) w[t] = c[t];
}

// Horner in s for the scaled derivative-match polynomial and its radial
// derivative.  Returns f_LR, writes (1/r) d f_LR/dr.  ND > 0 is the degree
// known at compile time (fully unrolled, coefficients read at fixed offsets
// of the parameter bank); ND == 0 reads the degree from k.nder.
template <typename T, int ND>
__device__ __forceinline__ T dm_poly_real(const PairCoef<T> &k, T s, T &f1) {
  const int N = ND > 0 ? ND : k.nder;
  T p = k.ar[N];
#pragma unroll
  for (int n = N - 1; n >= 0; n--) p = fma(p, s, k.ar[n]);
  T d = k.br[N - 1];
#pragma unroll
  for (int n = N - 2; n >= 0; n--) d = fma(d, s, k.br[n]);
  f1 = d;
  return p;
}

template <typename T, int ND>
__device__ __forceinline__ void dm_poly_cplx(const PairCoef<T> &k, T s, T &pr, T &pi,
                                             T &dr, T &di) {
  const int N = ND > 0 ? ND : k.nder;
  pr = k.ar[N];
  pi = k.ai[N];
#pragma unroll
  for (int n = N - 1; n >= 0; n--) {
    pr = fma(pr, s, k.ar[n]);
    pi = fma(pi, s, k.ai[n]);
  }
  dr = k.br[N - 1];
  di = k.bi[N - 1];
#pragma unroll
  for (int n = N - 2; n >= 0; n--) {
    dr = fma(dr, s, k.br[n]);
    di = fma(di, s, k.bi[n]);
  }
}

// Short-range pair kernel for real kernels: f0 = f - f_LR and
// f1 = (1/r) d(f - f_LR)/dr, zero beyond Rdir for the derivative match
// (src/PotentialLaplace.cpp:488-612, src/KernelFunctionRalpha.cpp:723-757);
// erfc(beta r)/r for the original split (src/PotentialLaplace.cpp:614-719).
// The caller has already checked r2 <= R2 and r2 > 0.
template <typename T, int FUNC, int SPLIT, int ND = 0>
__device__ __forceinline__ T pair_sr_real(const PairCoef<T> &k, T r2, T &f1) {
  if (SPLIT == 1) {
    const T rinv = rsqrt_t(r2);
    const T r = r2 * rinv;
    const T x = k.beta * r;
    const T f0 = erfc_t(x) * rinv;
    f1 = (-k.two_beta_rpi * exp_t(-x * x) - f0) * (rinv * rinv);
    return f0;
  }
  T g1;
  const T g0 = dm_poly_real<T, ND>(k, r2 * k.invR2, g1);
  if (FUNC == 0) {
    const T rinv = rsqrt_t(r2);
    f1 = -rinv * rinv * rinv - g1;
    return rinv - g0;
  } else {
    const T e0 = rpow_t(r2, k.half_alpha);
    f1 = k.alpha * e0 / r2 - g1;
    return e0 - g0;
  }
}

// Helmholtz short-range kernel exp(i k0 r)/r minus the DM polynomial
// (src/PotentialHelmholtz.cpp:353-418).
template <typename T, int ND = 0>
__device__ __forceinline__ void pair_sr_helmholtz(const PairCoef<T> &k, T r2, T &f0r,
                                                  T &f0i, T &f1r, T &f1i) {
  const T rinv = rsqrt_t(r2);
  const T r = r2 * rinv;
  T s, c;
  sincos_t(k.k0r * r, &s, &c);
  const T damp = (k.k0i != T(0)) ? exp_t(-k.k0i * r) * rinv : rinv;
  const T er = c * damp, ei = s * damp;  // exp(i k0 r)/r
  // f1_exact = (i k0 f0 - f0 / r) / r
  const T ikr = -k.k0i * er - k.k0r * ei;
  const T iki = k.k0r * er - k.k0i * ei;
  const T e1r = (ikr - er * rinv) * rinv, e1i = (iki - ei * rinv) * rinv;
  T pr, pi, dr, di;
  dm_poly_cplx<T, ND>(k, r2 * k.invR2, pr, pi, dr, di);
  f0r = er - pr;
  f0i = ei - pi;
  f1r = e1r - dr;
  f1i = e1i - di;
}

// Pair-kernel policy of the direct sums: the built-in kernels selected by
// (FUNC, SPLIT, ND), or a caller's functor type U (include/npme_user_kernel.cuh)
// with  template <typename T> __device__ static T sr(T r2, T &f1).
struct BuiltinPair {};

template <typename T, int FUNC, int SPLIT, int ND, class PK>
__device__ __forceinline__ T pair_sr(const PairCoef<T> &k, T r2, T &f1) {
  if constexpr (std::is_same<PK, BuiltinPair>::value)
    return pair_sr_real<T, FUNC, SPLIT, ND>(k, r2, f1);
  else
    return PK::template sr<T>(r2, f1);
}

// Complex kernels: the built-in Helmholtz kernel, or a caller's functor with
//   template <typename T> __device__ static void sr_c(T r2, T &f0r, T &f0i,
//                                                     T &f1r, T &f1i).
template <typename T, int ND, class PK>
__device__ __forceinline__ void pair_sr_cplx(const PairCoef<T> &k, T r2, T &f0r, T &f0i, T &f1r,
                                             T &f1i) {
  if constexpr (std::is_same<PK, BuiltinPair>::value)
    pair_sr_helmholtz<T, ND>(k, r2, f0r, f0i, f1r, f1i);
  else
    PK::template sr_c<T>(r2, f0r, f0i, f1r, f1i);
}

}  // namespace npme
