// Caller-defined kernels for npme_b200 (the GPU form of the reference's
// NPME_InterfaceReal_GenFunc with NPME_KfuncReal functors for f, f_LR and
// f_SR, src/Interface.h:302-304, src/KernelFunction.h:25-65).
//
// The reference calls virtual C++ functors on the host.  Here the kernel is
// device code, so the caller writes a functor type in CUDA and compiles this
// header with nvcc (-std=c++17 -gencode arch=compute_100a,code=sm_100a, -I to
// this directory and to npme_b200/csrc), linking -lnpme_gpu:
//
//   struct Yukawa {                      // f = exp(-kappa r) / r
//     // full kernel f and (1/r) df/dr at r^2 > 0 (exact sum, FP64)
//     __host__ __device__ static void full(double r2, double &f0, double &f1);
//     // smooth long-range part f_LR at r^2 >= 0 (kernel transform, FP64);
//     // pairs beyond Rdir are left to it, so f_LR should equal f there
//     __host__ __device__ static double lr(double r2);
//     // short-range part f - f_LR and its (1/r) d/dr for 0 < r^2 <= Rdir^2,
//     // in the bulk precision T (float or double)
//     template <typename T> __device__ static T sr(T r2, T &f1);
//   };
//
//   A complex kernel (the reference's NPME_KfuncComplex) declares
//     static constexpr bool kComplex = true;
//   and provides instead
//     __host__ __device__ static void full_c(double r2, double &f0r, double &f0i,
//                                            double &f1r, double &f1i);
//     __host__ __device__ static double2 lr_c(double r2);
//     template <typename T> __device__ static void sr_c(T r2, T &f0r, T &f0i,
//                                                       T &f1r, T &f1i);
//   (charges and V complex, as for Helmholtz).
//
//   npme_params p;  npme_gpu_default_params(&p);
//   p.funcType = NPME_FUNC_USER;  p.Rdir = ...;  p.N1 = ...;
//   npme_handle *h;  npme_gpu_create(&p, &h);
//   npme_user_ops ops = npme_user::ops<Yukawa>();
//   npme_gpu_set_user_kernel(h, &ops);
//   npme_gpu_setup(h, n, coord);   npme_gpu_calcv_real(h, V, n, q, coord);
//
// The spreading, FFTs, kernel multiply and interpolation are the library's;
// this header instantiates the three kernel-dependent launches: the direct
// sum (every pair once for real kernels, the one-sided warp-group body for
// complex ones, with the functor's sr / sr_c),
// the sampling of f_LR for the kernel transform and the exact sum.
#pragma once

#include <cuda_runtime.h>

#include <type_traits>

#include "npme_gpu.h"
#include "bodies.cuh"

namespace npme_user {

// Complex kernels declare  static constexpr bool kComplex = true  and
// provide full_c / lr_c / sr_c (see the header comment); real kernels need
// not declare kComplex.
template <class K, class = void>
struct is_complex : std::false_type {};
template <class K>
struct is_complex<K, std::void_t<decltype(K::kComplex)>>
    : std::integral_constant<bool, K::kComplex> {};

// The pair-kernel policy handed to the library's direct-sum bodies; both
// entries exist so that either body compiles, only K's kind is ever called.
template <class K>
struct Pair {
  template <typename T>
  __device__ static T sr(T r2, T &f1) {
    if constexpr (is_complex<K>::value) {
      f1 = T(0);
      return T(0);
    } else {
      return K::template sr<T>(r2, f1);
    }
  }
  template <typename T>
  __device__ static void sr_c(T r2, T &f0r, T &f0i, T &f1r, T &f1i) {
    if constexpr (is_complex<K>::value) {
      K::template sr_c<T>(r2, f0r, f0i, f1r, f1i);
    } else {
      f0r = f0i = f1r = f1i = T(0);
    }
  }
};

template <class K>
struct LR {
  __device__ double2 operator()(double r2) const {
    if constexpr (is_complex<K>::value) return K::lr_c(r2);
    else return make_double2(K::lr(r2), 0.0);
  }
};

template <class K>
__global__ void __launch_bounds__(32 * npme::kGroupWarps) groups_kernel(
    npme::PairCoef<float> k, const double4 *__restrict__ gpos, const double4 *__restrict__ spos,
    const float *__restrict__ qs, const double *__restrict__ qcaller,
    const int4 *__restrict__ groups, const double4 *__restrict__ gcen,
    const int2 *__restrict__ segs, const uint32_t *__restrict__ perm, long ngroups,
    float refine2, double fself, double fself_i, double *__restrict__ V) {
  __shared__ float4 sp[npme::kGroupWarps][32];
  __shared__ float4 slo[npme::kGroupWarps][32];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long g = (long)blockIdx.x * npme::kGroupWarps + wid;
  if (g >= ngroups) return;  // warp-uniform
  npme::direct_group_body<is_complex<K>::value, NPME_FUNC_USER, 0, 0, Pair<K>>(
      k, gpos, spos, qs, qcaller, groups[g], gcen[g], segs, perm, refine2, fself, fself_i, V,
      sp[wid], slo[wid], lane);
}

template <class K>
__global__ void __launch_bounds__(32 * npme::kGroupWarps) groups64_kernel(
    npme::PairCoef<double> k, const double4 *__restrict__ gpos,
    const double4 *__restrict__ spos, const double *__restrict__ qs,
    const double *__restrict__ qcaller, const int4 *__restrict__ groups,
    const double4 *__restrict__ gcen, const int2 *__restrict__ segs,
    const uint32_t *__restrict__ perm, long ngroups, double fself, double fself_i,
    double *__restrict__ V) {
  __shared__ double4 sp[npme::kGroupWarps][32];
  __shared__ double sqi[npme::kGroupWarps][32];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long g = (long)blockIdx.x * npme::kGroupWarps + wid;
  if (g >= ngroups) return;  // warp-uniform
  npme::direct_group_fp64<is_complex<K>::value, NPME_FUNC_USER, 0, 0, Pair<K>>(
      k, gpos, spos, qs, qcaller, groups[g], gcen[g], segs, perm, fself, fself_i, V, sp[wid],
      sqi[wid], lane);
}

// Real kernels: every pair once (the pair-once walk of the built-in kernels)
template <class K>
__global__ void __launch_bounds__(32 * npme::kGroupWarps) sym_kernel(
    npme::PairCoef<float> k, const double4 *__restrict__ gpos, const double4 *__restrict__ spos,
    const float *__restrict__ qs, const double *__restrict__ qcaller,
    const int4 *__restrict__ groups, const double4 *__restrict__ gcen,
    const int2 *__restrict__ segs, const uint32_t *__restrict__ perm, long ngroups,
    float refine2, double fself, double *__restrict__ V, float4 *__restrict__ vsrc) {
  __shared__ float4 th[npme::kGroupWarps][32];
  __shared__ float4 tl[npme::kGroupWarps][32];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long g = (long)blockIdx.x * npme::kGroupWarps + wid;
  if (g >= ngroups) return;  // warp-uniform
  npme::direct_group_sym_scalar<NPME_FUNC_USER, 0, 0, Pair<K>>(
      k, gpos, spos, qs, qcaller, groups[g], gcen[g], segs, perm, refine2, fself, V, vsrc,
      th[wid], tl[wid], lane);
}

template <class K>
__global__ void __launch_bounds__(32 * npme::kGroupWarps) sym64_kernel(
    npme::PairCoef<double> k, const double4 *__restrict__ gpos,
    const double4 *__restrict__ spos, const double *__restrict__ qs,
    const double *__restrict__ qcaller, const int4 *__restrict__ groups,
    const double4 *__restrict__ gcen, const int2 *__restrict__ segs,
    const uint32_t *__restrict__ perm, long ngroups, double fself, double *__restrict__ V,
    double *__restrict__ vsrc) {
  __shared__ double4 tsm[npme::kGroupWarps][32];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long g = (long)blockIdx.x * npme::kGroupWarps + wid;
  if (g >= ngroups) return;  // warp-uniform
  npme::direct_group_sym64<NPME_FUNC_USER, 0, 0, Pair<K>>(k, gpos, spos, qs, qcaller, groups[g],
                                                         gcen[g], segs, perm, fself, V, vsrc,
                                                         tsm[wid], lane);
}

template <class K>
__global__ void sample_kernel(int M1, int M2, int M3, const double *__restrict__ ax,
                              const double *__restrict__ ay, const double *__restrict__ az,
                              double2 *out) {
  const long total = (long)M1 * M2 * M3;
  const LR<K> lr{};
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x)
    out[idx] = npme::fhat_sample_body(lr, idx, M1, M2, M3, ax, ay, az);
}

constexpr int kExactTile = 128;

// Exact FP64 sum with the full kernel; output row t is target tidx[t] (every
// point when tidx is null).
template <class K>
__global__ void __launch_bounds__(kExactTile) exact_kernel(const double *__restrict__ coord,
                                                           const double *__restrict__ q, long n,
                                                           const unsigned int *__restrict__ tidx,
                                                           long nt, double *__restrict__ V) {
  __shared__ double4 sp[kExactTile];
  const long t = blockIdx.x * (long)kExactTile + threadIdx.x;
  const bool active = t < nt;
  const long i = active ? (tidx ? (long)tidx[t] : t) : -1;
  double xi = 0, yi = 0, zi = 0;
  if (active) xi = coord[3 * i], yi = coord[3 * i + 1], zi = coord[3 * i + 2];
  double a[4] = {0, 0, 0, 0};
  for (long j0 = 0; j0 < n; j0 += kExactTile) {
    __syncthreads();
    const long j = j0 + threadIdx.x;
    if (j < n) sp[threadIdx.x] = make_double4(coord[3 * j], coord[3 * j + 1], coord[3 * j + 2], q[j]);
    __syncthreads();
    const int cnt = (int)min((long)kExactTile, n - j0);
    for (int s = 0; s < cnt; s++) {
      if (j0 + s == i) continue;
      const double x = xi - sp[s].x, y = yi - sp[s].y, z = zi - sp[s].z;
      double f0, f1;
      K::full(x * x + y * y + z * z, f0, f1);
      a[0] += f0 * sp[s].w;
      a[1] += f1 * sp[s].w * x;
      a[2] += f1 * sp[s].w * y;
      a[3] += f1 * sp[s].w * z;
    }
  }
  if (active) reinterpret_cast<double4 *>(V)[t] = make_double4(a[0], a[1], a[2], a[3]);
}

// The same for complex kernels and charges (V rows of four complex values).
template <class K>
__global__ void __launch_bounds__(kExactTile) exact_kernel_c(const double *__restrict__ coord,
                                                             const double *__restrict__ q, long n,
                                                             const unsigned int *__restrict__ tidx,
                                                             long nt, double *__restrict__ V) {
  __shared__ double4 sp[kExactTile];
  __shared__ double2 sq[kExactTile];
  const long t = blockIdx.x * (long)kExactTile + threadIdx.x;
  const bool active = t < nt;
  const long i = active ? (tidx ? (long)tidx[t] : t) : -1;
  double xi = 0, yi = 0, zi = 0;
  if (active) xi = coord[3 * i], yi = coord[3 * i + 1], zi = coord[3 * i + 2];
  double a[4] = {0, 0, 0, 0}, ai[4] = {0, 0, 0, 0};
  for (long j0 = 0; j0 < n; j0 += kExactTile) {
    __syncthreads();
    const long j = j0 + threadIdx.x;
    if (j < n) {
      sp[threadIdx.x] = make_double4(coord[3 * j], coord[3 * j + 1], coord[3 * j + 2], 0.0);
      sq[threadIdx.x] = make_double2(q[2 * j], q[2 * j + 1]);
    }
    __syncthreads();
    const int cnt = (int)min((long)kExactTile, n - j0);
    for (int s = 0; s < cnt; s++) {
      if (j0 + s == i) continue;
      const double x = xi - sp[s].x, y = yi - sp[s].y, z = zi - sp[s].z;
      double f0r, f0i, f1r, f1i;
      K::full_c(x * x + y * y + z * z, f0r, f0i, f1r, f1i);
      const double qr = sq[s].x, qi = sq[s].y;
      a[0] += f0r * qr - f0i * qi;
      ai[0] += f0r * qi + f0i * qr;
      const double gr = f1r * qr - f1i * qi, gi = f1r * qi + f1i * qr;
      a[1] += gr * x, a[2] += gr * y, a[3] += gr * z;
      ai[1] += gi * x, ai[2] += gi * y, ai[3] += gi * z;
    }
  }
  if (active) {
    double2 *Vo = reinterpret_cast<double2 *>(V) + 4 * t;
    for (int m = 0; m < 4; m++) Vo[m] = make_double2(a[m], ai[m]);
  }
}

template <class K>
int direct(npme_handle *h, const void *args, void *stream) {
  const npme::DirectArgs &a = *static_cast<const npme::DirectArgs *>(args);
  cudaStream_t s = (cudaStream_t)stream;
  if (npme::pairs_once(h)) {  // real kernel: the half-shell walk, then the source-side sums
    const long blocks = (h->n_hgroups + npme::kGroupWarps - 1) / npme::kGroupWarps;
    if (blocks == 0) return NPME_OK;
    if (h->fp32)
      sym_kernel<K><<<(unsigned)blocks, 32 * npme::kGroupWarps, 0, s>>>(
          npme::make_pair_coef<float>(h), h->d_gpos, h->d_spos, (const float *)a.q, a.qcaller,
          h->d_hgroups, h->d_hcen, h->d_hsegs, h->d_cperm, h->n_hgroups, (float)h->refine2,
          a.fself_r, a.V, h->d_vsrc);
    else
      sym64_kernel<K><<<(unsigned)blocks, 32 * npme::kGroupWarps, 0, s>>>(
          npme::make_pair_coef<double>(h), h->d_gpos, h->d_spos, (const double *)a.q, a.qcaller,
          h->d_hgroups, h->d_hcen, h->d_hsegs, h->d_cperm, h->n_hgroups, a.fself_r, a.V,
          h->d_vsrc64);
    if (cudaPeekAtLastError() != cudaSuccess) return NPME_ECUDA;
    npme::launch_merge_source(h, a.V, s, 1.0, 1.0);
    return cudaPeekAtLastError() == cudaSuccess ? NPME_OK : NPME_ECUDA;
  }
  if (h->fp32) {
    const long blocks = (h->n_groups + npme::kGroupWarps - 1) / npme::kGroupWarps;
    if (blocks == 0) return NPME_OK;
    groups_kernel<K><<<(unsigned)blocks, 32 * npme::kGroupWarps, 0, s>>>(
        npme::make_pair_coef<float>(h), h->d_gpos, h->d_spos, (const float *)a.q, a.qcaller,
        h->d_groups, h->d_gcen, h->d_segs, h->d_cperm, h->n_groups, (float)h->refine2,
        a.fself_r, a.fself_i, a.V);
  } else {
    const long blocks = (h->n_groups + npme::kGroupWarps - 1) / npme::kGroupWarps;
    if (blocks == 0) return NPME_OK;
    groups64_kernel<K><<<(unsigned)blocks, 32 * npme::kGroupWarps, 0, s>>>(
        npme::make_pair_coef<double>(h), h->d_gpos, h->d_spos, (const double *)a.q, a.qcaller,
        h->d_groups, h->d_gcen, h->d_segs, h->d_cperm, h->n_groups, a.fself_r, a.fself_i, a.V);
  }
  return cudaPeekAtLastError() == cudaSuccess ? NPME_OK : NPME_ECUDA;
}

template <class K>
int sample_lr(npme_handle *, int M1, int M2, int M3, const double *ax, const double *ay,
              const double *az, void *out, void *stream) {
  sample_kernel<K><<<148 * 8, 256, 0, (cudaStream_t)stream>>>(M1, M2, M3, ax, ay, az,
                                                             (double2 *)out);
  return cudaPeekAtLastError() == cudaSuccess ? NPME_OK : NPME_ECUDA;
}

template <class K>
int exact(npme_handle *h, const double *d_q, double *d_V, void *stream,
          const unsigned int *d_tidx, long nt) {
  const long n = (long)h->n;
  if (!d_tidx) nt = n;
  const int blocks = (int)((nt + kExactTile - 1) / kExactTile);
  if (blocks == 0) return NPME_OK;
  if constexpr (is_complex<K>::value)
    exact_kernel_c<K><<<blocks, kExactTile, 0, (cudaStream_t)stream>>>(h->d_coord, d_q, n, d_tidx,
                                                                        nt, d_V);
  else
    exact_kernel<K><<<blocks, kExactTile, 0, (cudaStream_t)stream>>>(h->d_coord, d_q, n, d_tidx,
                                                                      nt, d_V);
  return cudaPeekAtLastError() == cudaSuccess ? NPME_OK : NPME_ECUDA;
}

// The launch table of functor K for npme_gpu_set_user_kernel.
template <class K>
npme_user_ops ops() {
  npme_user_ops o;
  if constexpr (is_complex<K>::value) {
    const double2 f = K::lr_c(0.0);
    o.fself = f.x, o.fself_i = f.y, o.complex_kernel = 1;
  } else {
    o.fself = K::lr(0.0), o.fself_i = 0.0, o.complex_kernel = 0;
  }
  o.direct = &direct<K>;
  o.sample_lr = &sample_lr<K>;
  o.exact = &exact<K>;
  return o;
}

}  // namespace npme_user
