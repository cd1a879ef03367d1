// Short-range direct sum over warp groups (every pair once for the built-in
// kernels, one-sided otherwise), the pair count and the exact
// O(N^2) sum.
//
// Direct sum (src/PotentialLaplace.cpp:201-264 and the pair kernels cited in
// common.cuh): V_i = sum_{j != i, r_ij <= Rdir} q_j f_SR(r_ij),
// dV_i/dx = sum q_j f1_SR(r_ij) (x_i - x_j).  Targets are grouped by 32 in
// z-sorted coarse columns and every group owns a list of source segments
// (built on the device at set-up, setup.cu); one warp walks one group in both
// precisions.  In the pair-once walk the target-side sums stay in registers
// and each output row is written once, while the source-side sums are added
// with float (FP32) or double (FP64) atomics into a per-source buffer that a
// merge kernel folds into V: results are reproducible only up to the order
// of those atomic additions.  The one-sided walk uses no atomics.
#include <cuda_runtime.h>

#include <cmath>

#include "bodies.cuh"
#include "internal.h"

namespace npme {

template <typename T>
PairCoef<T> make_pair_coef(const npme_handle *h) {
  PairCoef<T> k;
  memset(&k, 0, sizeof(k));
  const double R = h->p.Rdir, R2 = R * R;
  k.func = h->p.funcType;
  k.split = h->p.EwaldSplit;
  k.nder = h->p.nDeriv;
  k.R2 = (T)R2;
  k.invR2 = (T)(1.0 / R2);
  k.alpha = (T)h->p.alpha;
  k.half_alpha = (T)(0.5 * h->p.alpha);
  k.beta = (T)h->beta;
  k.beta2 = (T)(h->beta * h->beta);
  k.two_beta_rpi = (T)(2.0 * h->beta / std::sqrt(M_PI));
  k.k0r = (T)h->p.k0_r;
  k.k0i = (T)h->p.k0_i;
  double s = 1.0;  // R^(2n)
  for (int i = 0; i <= k.nder && i <= kMaxDeriv; i++) {
    k.ar[i] = (T)(h->a_r[i] * s);
    k.ai[i] = (T)(h->a_i[i] * s);
    k.br[i] = (T)(h->b_r[i] * s);
    k.bi[i] = (T)(h->b_i[i] * s);
    const double al = h->p.funcType == NPME_FUNC_RALPHA ? h->p.alpha : -1.0;
    k.nac2[i].x = (T)(-h->a_r[i] * s), k.nac2[i].y = (T)(-h->a_i[i] * s);
    k.nbc2[i].x = (T)(-h->b_r[i] * s), k.nbc2[i].y = (T)(-h->b_i[i] * s);
    k.nar2[i].x = k.nar2[i].y = (T)(-h->a_r[i] * s * std::pow(R, -al));
    k.br2[i].x = k.br2[i].y = (T)(h->b_r[i] * s * std::pow(R, 2.0 - al));
    s *= R2;
  }
  // the radial-derivative polynomials have degree nder - 1: their entry nder
  // is zero, as are all entries above nder (the zero-padded evaluation of
  // the packed bodies relies on it)
  if (k.nder >= 0 && k.nder <= kMaxDeriv) {
    k.br[k.nder] = k.bi[k.nder] = (T)0;
    k.br2[k.nder].x = k.br2[k.nder].y = (T)0;
    k.nbc2[k.nder].x = k.nbc2[k.nder].y = (T)0;
  }
  {
    const double al = h->p.funcType == NPME_FUNC_RALPHA ? h->p.alpha : -1.0;
    k.invR = 1.0 / R;
    k.vscale = std::pow(R, al);
    k.gscale = std::pow(R, al - 1.0);
  }
  return k;
}
template PairCoef<float> make_pair_coef<float>(const npme_handle *);
template PairCoef<double> make_pair_coef<double>(const npme_handle *);

// ---------------------------------------------------------------------------
// FP32 bulk direct sum over warp groups.
// One warp owns one group of <= 32 targets (one per lane) and walks the
// group's source segments in chunks of 32 that run across segment
// boundaries: every lane loads one source (FP64 position), the warp stages
// the chunk in shared memory as float coordinates relative to the group
// centre and every lane then sweeps the staged chunk for its target.  The next chunk's loads are issued before the
// sweep, so global latency hides behind the arithmetic.  Warps are
// independent: only __syncwarp, no block barrier.
//
// Coordinates: each FP64 offset from the group centre is split into a float
// head and the float residual (hi + lo).  The distance test and the pair
// arithmetic use the heads; for the rare close pairs (r^2 < refine2) the
// difference is recomputed as (t_hi - s_hi) + (t_lo - s_lo), which is exact
// to ~1e-15 because the heads of two close points subtract exactly.  Without
// this, a pair at r ~ 0.01 in a group of radius ~2 carries a ~1e-5 relative
// error that dominates the gradient.

template <bool CPLX, int FUNC, int SPLIT, int ND>
__global__ void __launch_bounds__(32 * kGroupWarps, kGroupMinBlocks) direct_groups_kernel(
    PairCoef<float> k, const double4 *__restrict__ gpos, const double4 *__restrict__ spos,
    const float *__restrict__ qs, const double *__restrict__ qcaller,
    const int4 *__restrict__ groups, const double4 *__restrict__ gcen,
    const int2 *__restrict__ segs, const uint32_t *__restrict__ perm, long ngroups,
    float refine2, double fself_r, double fself_i, double *__restrict__ V) {
  __shared__ float4 sp[kGroupWarps][32];   // (x_hi, y_hi, z_hi, q) / q.re
  __shared__ float4 slo[kGroupWarps][32];  // (x_lo, y_lo, z_lo, q.im)
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long g = (long)blockIdx.x * kGroupWarps + wid;
  if (g >= ngroups) return;  // warp-uniform; nothing below synchronises the block
  direct_group_body<CPLX, FUNC, SPLIT, ND>(k, gpos, spos, qs, qcaller, groups[g], gcen[g], segs,
                                           perm, refine2, fself_r, fself_i, V, sp[wid], slo[wid],
                                           lane);
}


template <bool CPLX, int FUNC, int SPLIT, int ND>
static void groups_launch_nd(npme_handle *h, const DirectArgs &a, cudaStream_t s) {
  const long blocks = (h->n_groups + kGroupWarps - 1) / kGroupWarps;
  if (blocks == 0) return;
  direct_groups_kernel<CPLX, FUNC, SPLIT, ND><<<(unsigned)blocks, 32 * kGroupWarps, 0, s>>>(
      make_pair_coef<float>(h), h->d_gpos, h->d_spos, (const float *)a.q, a.qcaller, h->d_groups,
      h->d_gcen, h->d_segs, h->d_cperm, h->n_groups, (float)h->refine2, a.fself_r, a.fself_i,
      a.V);
}

// After a pair-once launch: the source-side sums are merged into V now, or,
// when CalcV asked for it, left for the interpolation (which visits every
// point in brick order and folds its slot in, saving a pass over V).
static void merge_or_defer(npme_handle *h, const DirectArgs &a, cudaStream_t s, double vs,
                           double gs) {
  if (a.defer_merge) {
    h->merge_pending = true;
    h->merge_vs = vs, h->merge_gs = gs;
  } else {
    launch_merge_source(h, a.V, s, vs, gs);
    h->launches++;
  }
}

// FP32 real-DM direct sum with every pair evaluated once (direct_group_sym),
// then the source-side sums folded into V.
template <int FUNC, int ND>
__global__ void __launch_bounds__(32 * kGroupWarps, kGroupMinBlocks) direct_sym_kernel(
    PairCoef<float> k, const double4 *__restrict__ gpos, const double4 *__restrict__ spos,
    const float *__restrict__ qs, const double *__restrict__ qcaller,
    const int4 *__restrict__ groups, const double4 *__restrict__ gcen,
    const int2 *__restrict__ segs, const uint32_t *__restrict__ perm, long ngroups,
    float refine2, double fself_r, double *__restrict__ V, float4 *__restrict__ vsrc) {
  __shared__ float4 tsm[kGroupWarps][32];  // group targets (x, y, z, q), heads
  __shared__ float4 tlo[kGroupWarps][32];  // residuals of the target coordinates
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long g = (long)blockIdx.x * kGroupWarps + wid;
  if (g >= ngroups) return;  // warp-uniform; nothing below synchronises the block
  direct_group_sym<FUNC, ND>(k, gpos, spos, qs, qcaller, groups[g], gcen[g], segs, perm,
                             refine2, fself_r, V, vsrc, tsm[wid], tlo[wid], lane);
}

// V[caller(i)] += scale * vsrc[i] for every brick-order slot i, then
// vsrc[i] = 0 for the next call.
__global__ void merge_source_kernel(float4 *__restrict__ vsrc, const uint32_t *__restrict__ bperm,
                                    long n, double vs, double gs, double *__restrict__ V) {
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const float4 a = vsrc[s];
  vsrc[s] = make_float4(0.f, 0.f, 0.f, 0.f);
  double4 *o = reinterpret_cast<double4 *>(V) + bperm[s];
  double4 v = *o;
  v.x += vs * (double)a.x;
  v.y += gs * (double)a.y;
  v.z += gs * (double)a.z;
  v.w += gs * (double)a.w;
  *o = v;
}

// FP32 Helmholtz DM form (direct_group_sym_helm).
template <int ND>
__global__ void __launch_bounds__(32 * kGroupWarps) direct_sym_helm_kernel(
    PairCoef<float> k, const double4 *__restrict__ gpos, const double4 *__restrict__ spos,
    const float *__restrict__ qs, const double *__restrict__ qcaller,
    const int4 *__restrict__ groups, const double4 *__restrict__ gcen,
    const int2 *__restrict__ segs, const uint32_t *__restrict__ perm, long ngroups,
    float refine2, double fself_r, double fself_i, double *__restrict__ V,
    float4 *__restrict__ vsrc) {
  __shared__ float4 th[kGroupWarps][32];  // group targets: heads, Re q
  __shared__ float4 tl[kGroupWarps][32];  // residuals, Im q
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long g = (long)blockIdx.x * kGroupWarps + wid;
  if (g >= ngroups) return;  // warp-uniform
  direct_group_sym_helm<ND>(k, gpos, spos, qs, qcaller, groups[g], gcen[g], segs, perm, refine2,
                            fself_r, fself_i, V, vsrc, th[wid], tl[wid], lane);
}

// Complex V[caller(i)][0..3] += vsrc[2i], vsrc[2i + 1] (re, im pairs), then zero.
__global__ void merge_source_cplx_kernel(float4 *__restrict__ vsrc,
                                         const uint32_t *__restrict__ bperm, long n,
                                         double *__restrict__ V) {
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const float4 a = vsrc[2 * s], b = vsrc[2 * s + 1];
  vsrc[2 * s] = vsrc[2 * s + 1] = make_float4(0.f, 0.f, 0.f, 0.f);
  double4 *o = reinterpret_cast<double4 *>(V) + 2 * (long)bperm[s];
  double4 u = o[0], w = o[1];
  u.x += a.x, u.y += a.y, u.z += a.z, u.w += a.w;
  w.x += b.x, w.y += b.y, w.z += b.z, w.w += b.w;
  o[0] = u, o[1] = w;
}

template <int ND>
static void sym_helm_launch_nd(npme_handle *h, const DirectArgs &a, cudaStream_t s) {
  const long blocks = (h->n_hgroups + kGroupWarps - 1) / kGroupWarps;
  if (blocks == 0) return;
  direct_sym_helm_kernel<ND><<<(unsigned)blocks, 32 * kGroupWarps, 0, s>>>(
      make_pair_coef<float>(h), h->d_gpos, h->d_spos, (const float *)a.q, a.qcaller,
      h->d_hgroups, h->d_hcen, h->d_hsegs, h->d_cperm, h->n_hgroups, (float)h->refine2,
      a.fself_r, a.fself_i, a.V, h->d_vsrc);
  merge_or_defer(h, a, s, 1.0, 1.0);
}

template <int FUNC, int ND>
static void sym_launch_nd(npme_handle *h, const DirectArgs &a, cudaStream_t s) {
  const long blocks = (h->n_hgroups + kGroupWarps - 1) / kGroupWarps;
  if (blocks == 0) return;
  const PairCoef<float> k = make_pair_coef<float>(h);
  direct_sym_kernel<FUNC, ND><<<(unsigned)blocks, 32 * kGroupWarps, 0, s>>>(
      k, h->d_gpos, h->d_spos, (const float *)a.q, a.qcaller, h->d_hgroups, h->d_hcen,
      h->d_hsegs, h->d_cperm, h->n_hgroups, (float)h->refine2, a.fself_r, a.V, h->d_vsrc);
  merge_or_defer(h, a, s, k.vscale, k.gscale);
}

// FP32 form with the scalar pair kernel (original Ewald split).
template <int FUNC, int SPLIT, int ND>
__global__ void __launch_bounds__(32 * kGroupWarps) direct_sym_scalar_kernel(
    PairCoef<float> k, const double4 *__restrict__ gpos, const double4 *__restrict__ spos,
    const float *__restrict__ qs, const double *__restrict__ qcaller,
    const int4 *__restrict__ groups, const double4 *__restrict__ gcen,
    const int2 *__restrict__ segs, const uint32_t *__restrict__ perm, long ngroups,
    float refine2, double fself_r, double *__restrict__ V, float4 *__restrict__ vsrc) {
  __shared__ float4 th[kGroupWarps][32];  // group targets: heads, q
  __shared__ float4 tl[kGroupWarps][32];  // residuals
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long g = (long)blockIdx.x * kGroupWarps + wid;
  if (g >= ngroups) return;  // warp-uniform
  direct_group_sym_scalar<FUNC, SPLIT, ND>(k, gpos, spos, qs, qcaller, groups[g], gcen[g], segs,
                                           perm, refine2, fself_r, V, vsrc, th[wid], tl[wid],
                                           lane);
}

// FP64 form for the real built-in kernels (DM and original Ewald).
template <int FUNC, int SPLIT, int ND>
__global__ void __launch_bounds__(32 * kGroupWarps) direct_sym64_kernel(
    PairCoef<double> k, const double4 *__restrict__ gpos, const double4 *__restrict__ spos,
    const double *__restrict__ qs, const double *__restrict__ qcaller,
    const int4 *__restrict__ groups, const double4 *__restrict__ gcen,
    const int2 *__restrict__ segs, const uint32_t *__restrict__ perm, long ngroups,
    double fself_r, double *__restrict__ V, double *__restrict__ vsrc) {
  __shared__ double4 tsm[kGroupWarps][32];  // group targets (x, y, z, q)
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long g = (long)blockIdx.x * kGroupWarps + wid;
  if (g >= ngroups) return;  // warp-uniform
  direct_group_sym64<FUNC, SPLIT, ND>(k, gpos, spos, qs, qcaller, groups[g], gcen[g], segs, perm,
                                      fself_r, V, vsrc, tsm[wid], lane);
}

// V[caller(i)][m] += vsrc[i][m], then vsrc[i] = 0 for the next call.
__global__ void merge_source64_kernel(double4 *__restrict__ vsrc,
                                      const uint32_t *__restrict__ bperm, long n,
                                      double *__restrict__ V) {
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const double4 a = vsrc[s];
  vsrc[s] = make_double4(0, 0, 0, 0);
  double4 *o = reinterpret_cast<double4 *>(V) + bperm[s];
  double4 v = *o;
  v.x += a.x, v.y += a.y, v.z += a.z, v.w += a.w;
  *o = v;
}

template <int FUNC, int SPLIT, int ND>
static void sym64_launch_nd(npme_handle *h, const DirectArgs &a, cudaStream_t s) {
  const long blocks = (h->n_hgroups + kGroupWarps - 1) / kGroupWarps;
  if (blocks == 0) return;
  direct_sym64_kernel<FUNC, SPLIT, ND><<<(unsigned)blocks, 32 * kGroupWarps, 0, s>>>(
      make_pair_coef<double>(h), h->d_gpos, h->d_spos, (const double *)a.q, a.qcaller,
      h->d_hgroups, h->d_hcen, h->d_hsegs, h->d_cperm, h->n_hgroups, a.fself_r, a.V,
      h->d_vsrc64);
  merge_or_defer(h, a, s, 1.0, 1.0);
}

template <int FUNC, int SPLIT>
static void sym64_launch(npme_handle *h, const DirectArgs &a, cudaStream_t s) {
  switch (SPLIT == 1 ? 0 : h->p.nDeriv) {
    case 3: sym64_launch_nd<FUNC, SPLIT, 3>(h, a, s); break;
    case 6: sym64_launch_nd<FUNC, SPLIT, 6>(h, a, s); break;
    case 8: sym64_launch_nd<FUNC, SPLIT, 8>(h, a, s); break;
    default: sym64_launch_nd<FUNC, SPLIT, 0>(h, a, s); break;
  }
}

void launch_merge_source(npme_handle *h, double *V, cudaStream_t s, double vs, double gs) {
  const long n = (long)h->n;
  const unsigned blocks = (unsigned)((n + 255) / 256);
  if (!h->fp32)
    merge_source64_kernel<<<blocks, 256, 0, s>>>(reinterpret_cast<double4 *>(h->d_vsrc64),
                                                 h->d_bperm, n, V);
  else if (h->complex_kernel)
    merge_source_cplx_kernel<<<blocks, 256, 0, s>>>(h->d_vsrc, h->d_bperm, n, V);
  else
    merge_source_kernel<<<blocks, 256, 0, s>>>(h->d_vsrc, h->d_bperm, n, vs, gs, V);
}

// The pair-once form applies to the built-in kernels: in FP32 the DM kernels
// (1/r, r^alpha, Helmholtz; derivative orders 3, 6 and 8 compiled with the
// order fixed, the others by one instance at degree kMaxDeriv with
// zero-padded coefficients) and the original
// Ewald split, in FP64 the real kernels (any order, original Ewald
// included); FP64 Helmholtz and caller-defined complex kernels walk the full
// segments.
bool pairs_once(const npme_handle *h) {
  if (!h->use_sym || h->n_hgroups == 0) return false;
  if (h->user_kernel) return !h->complex_kernel;  // the functor's scalar pair kernel
  const int f = h->p.funcType;
  if (f == NPME_FUNC_HELMHOLTZ) return h->fp32;
  return f == NPME_FUNC_LAPLACE || f == NPME_FUNC_RALPHA;
}

static bool sym_launch(npme_handle *h, const DirectArgs &a, cudaStream_t s) {
  if (!pairs_once(h)) return false;
  const int f = h->p.funcType, nd = h->p.nDeriv;
  if (f == NPME_FUNC_HELMHOLTZ) {
    if (nd == 3) sym_helm_launch_nd<3>(h, a, s);
    else if (nd == 6) sym_helm_launch_nd<6>(h, a, s);
    else if (nd == 8) sym_helm_launch_nd<8>(h, a, s);
    else sym_helm_launch_nd<0>(h, a, s);
    return true;
  }
  if (h->fp32 && h->p.EwaldSplit == NPME_SPLIT_LAPLACE_ORIG) {
    const long blocks = (h->n_hgroups + kGroupWarps - 1) / kGroupWarps;
    if (blocks > 0) {
      direct_sym_scalar_kernel<0, 1, 0><<<(unsigned)blocks, 32 * kGroupWarps, 0, s>>>(
          make_pair_coef<float>(h), h->d_gpos, h->d_spos, (const float *)a.q, a.qcaller,
          h->d_hgroups, h->d_hcen, h->d_hsegs, h->d_cperm, h->n_hgroups, (float)h->refine2,
          a.fself_r, a.V, h->d_vsrc);
      merge_or_defer(h, a, s, 1.0, 1.0);
    }
    return true;
  }
  if (!h->fp32) {
    if (h->p.EwaldSplit == NPME_SPLIT_LAPLACE_ORIG) sym64_launch<0, 1>(h, a, s);
    else if (f == NPME_FUNC_RALPHA) sym64_launch<1, 0>(h, a, s);
    else sym64_launch<0, 0>(h, a, s);
    return true;
  }
  if (f == NPME_FUNC_LAPLACE) {
    if (nd == 3) sym_launch_nd<0, 3>(h, a, s);
    else if (nd == 6) sym_launch_nd<0, 6>(h, a, s);
    else if (nd == 8) sym_launch_nd<0, 8>(h, a, s);
    else sym_launch_nd<0, 0>(h, a, s);
  } else {
    if (nd == 3) sym_launch_nd<1, 3>(h, a, s);
    else if (nd == 6) sym_launch_nd<1, 6>(h, a, s);
    else if (nd == 8) sym_launch_nd<1, 8>(h, a, s);
    else sym_launch_nd<1, 0>(h, a, s);
  }
  return true;
}

template <bool CPLX, int FUNC, int SPLIT, int ND>
__global__ void __launch_bounds__(32 * kGroupWarps) direct_groups64_kernel(
    PairCoef<double> k, const double4 *__restrict__ gpos, const double4 *__restrict__ spos,
    const double *__restrict__ qs, const double *__restrict__ qcaller,
    const int4 *__restrict__ groups, const double4 *__restrict__ gcen,
    const int2 *__restrict__ segs, const uint32_t *__restrict__ perm, long ngroups,
    double fself_r, double fself_i, double *__restrict__ V) {
  __shared__ double4 sp[kGroupWarps][32];
  __shared__ double sqi[kGroupWarps][32];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long g = (long)blockIdx.x * kGroupWarps + wid;
  if (g >= ngroups) return;  // warp-uniform
  direct_group_fp64<CPLX, FUNC, SPLIT, ND>(k, gpos, spos, qs, qcaller, groups[g], gcen[g], segs,
                                           perm, fself_r, fself_i, V, sp[wid], sqi[wid], lane);
}

template <bool CPLX, int FUNC, int SPLIT, int ND>
static void groups64_launch_nd(npme_handle *h, const DirectArgs &a, cudaStream_t s) {
  const long blocks = (h->n_groups + kGroupWarps - 1) / kGroupWarps;
  if (blocks == 0) return;
  direct_groups64_kernel<CPLX, FUNC, SPLIT, ND><<<(unsigned)blocks, 32 * kGroupWarps, 0, s>>>(
      make_pair_coef<double>(h), h->d_gpos, h->d_spos, (const double *)a.q, a.qcaller,
      h->d_groups, h->d_gcen, h->d_segs, h->d_cperm, h->n_groups, a.fself_r, a.fself_i, a.V);
}

template <bool CPLX, int FUNC, int SPLIT>
static void groups_launch(npme_handle *h, const DirectArgs &a, cudaStream_t s) {
  if (!h->fp32) {
    switch (SPLIT == 1 ? 0 : h->p.nDeriv) {
      case 3: groups64_launch_nd<CPLX, FUNC, SPLIT, 3>(h, a, s); break;
      case 6: groups64_launch_nd<CPLX, FUNC, SPLIT, 6>(h, a, s); break;
      case 8: groups64_launch_nd<CPLX, FUNC, SPLIT, 8>(h, a, s); break;
      default: groups64_launch_nd<CPLX, FUNC, SPLIT, 0>(h, a, s); break;
    }
    return;
  }
  switch (SPLIT == 1 ? 0 : h->p.nDeriv) {
    case 3: groups_launch_nd<CPLX, FUNC, SPLIT, 3>(h, a, s); break;
    case 6: groups_launch_nd<CPLX, FUNC, SPLIT, 6>(h, a, s); break;
    case 8: groups_launch_nd<CPLX, FUNC, SPLIT, 8>(h, a, s); break;
    default: groups_launch_nd<CPLX, FUNC, SPLIT, 0>(h, a, s); break;
  }
}

int launch_direct_args(npme_handle *h, const DirectArgs &a, cudaStream_t s) {
  int rc = NPME_OK;
  if (h->user_kernel) {
    rc = h->uops.direct(h, &a, s);
  } else if (!sym_launch(h, a, s)) {  // both precisions walk warp groups
    const int f = h->p.funcType, sp = h->p.EwaldSplit;
    if (f == NPME_FUNC_HELMHOLTZ) groups_launch<true, 2, 0>(h, a, s);
    else if (sp == NPME_SPLIT_LAPLACE_ORIG) groups_launch<false, 0, 1>(h, a, s);
    else if (f == NPME_FUNC_RALPHA) groups_launch<false, 1, 0>(h, a, s);
    else groups_launch<false, 0, 0>(h, a, s);
  }
  h->launches++;
  return rc;
}

int launch_direct(npme_handle *h, const double *d_q, double *d_V, cudaStream_t s) {
  DirectArgs a{h->d_qc, d_q, h->fself_r, h->fself_i, d_V};
  a.defer_merge = true;  // CalcV: the interpolation folds the source-side sums in
  return launch_direct_args(h, a, s);
}

// Ordered pairs with 0 < r <= Rdir (FP64 distances) over the one-sided group
// walk, every target of a group against every source of its segments: the
// work count of the roofline report (set-up only, not on the CalcV path).
__global__ void __launch_bounds__(32 * kGroupWarps) count_pairs_kernel(
    const double4 *__restrict__ gpos, const double4 *__restrict__ spos,
    const int4 *__restrict__ groups, const int2 *__restrict__ segs, long ngroups, double R2,
    unsigned long long *__restrict__ count) {
  __shared__ double4 sp[kGroupWarps][32];
  const unsigned FULL = 0xffffffffu;
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long g = (long)blockIdx.x * kGroupWarps + wid;
  if (g >= ngroups) return;  // warp-uniform
  const int4 G = groups[g];
  const double4 t = lane < G.y ? gpos[G.x + lane] : make_double4(1e150, 1e150, 1e150, 0.0);
  unsigned long long mine = 0;
  SrcCursor cur{G.z, lane};
  cur.normalize(segs, G.w);
  while (__any_sync(FULL, cur.seg < G.w)) {
    const bool v = cur.seg < G.w;
    const int cnt = __popc(__ballot_sync(FULL, v));  // valid lanes form a prefix
    __syncwarp();
    if (v) sp[wid][lane] = spos[(long)segs[cur.seg].x + cur.off];
    __syncwarp();
    for (int s = 0; s < cnt; s++) {
      const double4 q = sp[wid][s];
      const double x = t.x - q.x, y = t.y - q.y, z = t.z - q.z;
      const double r2 = x * x + y * y + z * z;
      mine += (r2 <= R2 && r2 > 0.0) ? 1ull : 0ull;
    }
    cur.off += 32;
    cur.normalize(segs, G.w);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(FULL, mine, o);
  if (lane == 0) atomicAdd(count, mine);
}

void launch_count_pairs(npme_handle *h, unsigned long long *d_count, cudaStream_t s) {
  const long blocks = (h->n_groups + kGroupWarps - 1) / kGroupWarps;
  if (blocks == 0) return;
  count_pairs_kernel<<<(unsigned)blocks, 32 * kGroupWarps, 0, s>>>(
      h->d_gpos, h->d_spos, h->d_groups, h->d_segs, h->n_groups, h->p.Rdir * h->p.Rdir, d_count);
}

// ---------------------------------------------------------------------------
// Exact sum (src/PotentialLaplace.cpp:40-132, src/PotentialHelmholtz.cpp:41,
// src/PotentialGenFunc.cpp:321): all pairs j != i with the full kernel, FP64,
// no self term.  Sources are tiled through shared memory.

constexpr int kExactBS = 128;

template <int FUNC>
__global__ void __launch_bounds__(kExactBS) exact_kernel(const double *__restrict__ coord,
                                                          const double *__restrict__ q, long n,
                                                          double alpha, double k0r, double k0i,
                                                          const uint32_t *__restrict__ tidx,
                                                          long nt, double *__restrict__ V) {
  constexpr bool CPLX = FUNC == 2;
  __shared__ double4 sp[kExactBS];
  __shared__ double2 sq[kExactBS];
  // output row t holds target tidx[t] (every point when tidx is null)
  const long t = blockIdx.x * (long)kExactBS + threadIdx.x;
  const bool active = t < nt;
  const long i = active ? (tidx ? (long)tidx[t] : t) : -1;
  double xi = 0, yi = 0, zi = 0;
  if (active) xi = coord[3 * i], yi = coord[3 * i + 1], zi = coord[3 * i + 2];
  double a[4] = {0, 0, 0, 0}, ai[4] = {0, 0, 0, 0};
  for (long j0 = 0; j0 < n; j0 += kExactBS) {
    __syncthreads();
    const long j = j0 + threadIdx.x;
    if (j < n) {
      sp[threadIdx.x] = make_double4(coord[3 * j], coord[3 * j + 1], coord[3 * j + 2], 0.0);
      sq[threadIdx.x] = CPLX ? make_double2(q[2 * j], q[2 * j + 1]) : make_double2(q[j], 0.0);
    }
    __syncthreads();
    const int cnt = (int)min((long)kExactBS, n - j0);
    for (int s = 0; s < cnt; s++) {
      if (j0 + s == i) continue;
      const double x = xi - sp[s].x, y = yi - sp[s].y, z = zi - sp[s].z;
      const double r2 = x * x + y * y + z * z;
      if (FUNC == 0) {
        const double rinv = rsqrt(r2);
        const double f0 = rinv, f1 = -rinv * rinv * rinv;
        const double qj = sq[s].x;
        a[0] += f0 * qj;
        a[1] += f1 * qj * x;
        a[2] += f1 * qj * y;
        a[3] += f1 * qj * z;
      } else if (FUNC == 1) {
        const double f0 = pow(r2, 0.5 * alpha), f1 = alpha * f0 / r2;
        const double qj = sq[s].x;
        a[0] += f0 * qj;
        a[1] += f1 * qj * x;
        a[2] += f1 * qj * y;
        a[3] += f1 * qj * z;
      } else {
        const double r = sqrt(r2);
        double sn, cs;
        sincos(k0r * r, &sn, &cs);
        const double d = exp(-k0i * r) / r;
        const double er = cs * d, ei = sn * d;
        const double ikr = -k0i * er - k0r * ei, iki = k0r * er - k0i * ei;
        const double f1r = (ikr - er / r) / r, f1i = (iki - ei / r) / r;
        const double qr = sq[s].x, qi = sq[s].y;
        a[0] += er * qr - ei * qi;
        ai[0] += er * qi + ei * qr;
        const double gr = f1r * qr - f1i * qi, gi = f1r * qi + f1i * qr;
        a[1] += gr * x, a[2] += gr * y, a[3] += gr * z;
        ai[1] += gi * x, ai[2] += gi * y, ai[3] += gi * z;
      }
    }
  }
  if (active) {
    if (CPLX) {
      double2 *Vo = reinterpret_cast<double2 *>(V) + 4 * t;
      for (int m = 0; m < 4; m++) Vo[m] = make_double2(a[m], ai[m]);
    } else {
      reinterpret_cast<double4 *>(V)[t] = make_double4(a[0], a[1], a[2], a[3]);
    }
  }
}

int launch_exact(npme_handle *h, const double *d_q, double *d_V, cudaStream_t s,
                 const uint32_t *d_tidx, long nt) {
  const long n = (long)h->n;
  if (!d_tidx) nt = n;
  const int blocks = (int)((nt + kExactBS - 1) / kExactBS);
  if (blocks == 0) return NPME_OK;
  if (h->user_kernel) {
    h->launches++;
    return h->uops.exact(h, d_q, d_V, s, d_tidx, nt);
  }
  const int f = h->p.funcType;
  if (f == 0)
    exact_kernel<0><<<blocks, kExactBS, 0, s>>>(h->d_coord, d_q, n, h->p.alpha, h->p.k0_r,
                                                 h->p.k0_i, d_tidx, nt, d_V);
  else if (f == 1)
    exact_kernel<1><<<blocks, kExactBS, 0, s>>>(h->d_coord, d_q, n, h->p.alpha, h->p.k0_r,
                                                 h->p.k0_i, d_tidx, nt, d_V);
  else
    exact_kernel<2><<<blocks, kExactBS, 0, s>>>(h->d_coord, d_q, n, h->p.alpha, h->p.k0_r,
                                                 h->p.k0_i, d_tidx, nt, d_V);
  h->launches++;
  return NPME_OK;
}

}  // namespace npme
