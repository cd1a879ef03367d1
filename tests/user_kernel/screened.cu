// Caller-defined kernels for the tests, instantiated through
// include/npme_user_kernel.cuh and exported as C functions that fill the
// launch table:
//   GaussScreened  f = exp(-a r^2) / r, split with erf(beta r):
//                  f_LR = f erf(beta r) (smooth: even in r), f_SR = f erfc(beta r)
//   CoulombErf     a = 0: 1/r with the original Ewald split
//   WaveErf        exp(i k r)/r (complex), real part split with erf
// (A plain Yukawa exp(-kappa r)/r split this way would leave f_LR with a
// term linear in r at the origin, which the grid does not resolve.)
#include <cmath>

#include "npme_user_kernel.cuh"

namespace {

constexpr double kBeta = 0.475;
constexpr double kTwoOverSqrtPi = 1.1283791670955126;

template <int A_MICRO>
struct GaussScreened {
  static constexpr double kA = A_MICRO * 1e-6;
  __host__ __device__ static void full(double r2, double &f0, double &f1) {
    const double r = sqrt(r2), e = exp(-kA * r2);
    f0 = e / r;
    f1 = -e * (2.0 * kA * r2 + 1.0) / (r2 * r);
  }
  __host__ __device__ static double lr(double r2) {
    if (r2 == 0.0) return kBeta * kTwoOverSqrtPi;
    const double r = sqrt(r2);
    return exp(-kA * r2) * erf(kBeta * r) / r;
  }
  template <typename T>
  __device__ static T sr(T r2, T &f1) {
    const T r = sqrt(r2), ri = T(1) / r;
    const T f0 = exp(-T(kA) * r2) * erfc(T(kBeta) * r) * ri;
    const T g = T(kTwoOverSqrtPi * kBeta) * exp(-T(kA + kBeta * kBeta) * r2) * ri;
    f1 = (-(T(2 * kA) * r + ri) * f0 - g) * ri;
    return f0;
  }
};

using Screened = GaussScreened<20000>;  // a = 0.02
using CoulombErf = GaussScreened<0>;

// Complex: exp(i k r) / r, k = 0.5, with the real part split by erf(beta r)
// and the imaginary part sin(k r)/r (smooth everywhere) left to f_LR.
struct WaveErf {
  static constexpr bool kComplex = true;
  static constexpr double kK = 0.5;
  __host__ __device__ static void full_c(double r2, double &f0r, double &f0i, double &f1r,
                                         double &f1i) {
    const double r = sqrt(r2), c = cos(kK * r), s = sin(kK * r);
    f0r = c / r, f0i = s / r;
    f1r = (-c - kK * r * s) / (r2 * r);
    f1i = (-s + kK * r * c) / (r2 * r);
  }
  __host__ __device__ static double2 lr_c(double r2) {
    if (r2 == 0.0) return make_double2(kBeta * kTwoOverSqrtPi, kK);
    const double r = sqrt(r2);
    return make_double2(cos(kK * r) * erf(kBeta * r) / r, sin(kK * r) / r);
  }
  template <typename T>
  __device__ static void sr_c(T r2, T &f0r, T &f0i, T &f1r, T &f1i) {
    const T r = sqrt(r2), ri = T(1) / r;
    const T c = cos(T(kK) * r), s = sin(T(kK) * r), ec = erfc(T(kBeta) * r);
    f0r = c * ec * ri;
    f0i = T(0);
    const T g = T(kTwoOverSqrtPi * kBeta) * exp(-T(kBeta * kBeta) * r2);
    f1r = (-T(kK) * s * ec - c * g - f0r) * ri * ri;
    f1i = T(0);
  }
};

}  // namespace

extern "C" void screened_ops(npme_user_ops *out) { *out = npme_user::ops<Screened>(); }
extern "C" void coulomb_erf_ops(npme_user_ops *out) { *out = npme_user::ops<CoulombErf>(); }
extern "C" void wave_erf_ops(npme_user_ops *out) { *out = npme_user::ops<WaveErf>(); }
extern "C" double user_kernel_beta() { return kBeta; }
