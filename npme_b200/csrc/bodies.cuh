// Device bodies of the per-call kernels, shared by the single-system kernels
// (recsum.cu, direct.cu) and the multi-system batch kernels (batch.cu).  Each
// body processes one unit of work (one point, one brick, one spectrum
// element, one warp group) of one system; the kernels only map threads to
// (system, unit).
#pragma once

#include "internal.h"

namespace npme {

#ifndef NPME_GROUP_MIN_BLOCKS
#define NPME_GROUP_MIN_BLOCKS 1
#endif
constexpr int kGroupMinBlocks = NPME_GROUP_MIN_BLOCKS;  // resident CTAs asked of ptxas
#ifndef NPME_DIRECT_UNROLL
#define NPME_DIRECT_UNROLL 8
#endif
constexpr int kDirectUnroll = NPME_DIRECT_UNROLL;  // pair-loop unroll factor

// Charges into brick order (spread/interp) and the direct sum's source
// order (dperm: source slot -> caller index).
template <typename T, bool CPLX>
__device__ __forceinline__ void gather_body(const double *__restrict__ q,
                                            const BrickPoint<T> *__restrict__ bp,
                                            const uint32_t *__restrict__ dperm,
                                            T *__restrict__ qb, T *__restrict__ qc, long i) {
  const uint32_t ob = bp[i].orig, oc = dperm[i];
  if (CPLX) {
    qb[2 * i] = (T)q[2 * (long)ob];
    qb[2 * i + 1] = (T)q[2 * (long)ob + 1];
    qc[2 * i] = (T)q[2 * (long)oc];
    qc[2 * i + 1] = (T)q[2 * (long)oc + 1];
  } else {
    qb[i] = (T)q[ob];
    qc[i] = (T)q[oc];
  }
}

// Unroll of the outer stencil axis: complete up to order 12; orders 14 and
// 16 (up to 16^3 = 4,096 stencil points) keep it as a loop, so the unrolled
// inner P^2 block stays a size the instruction cache holds.
template <int P>
constexpr int kStencilUnroll = P <= 12 ? P : 1;

// Points of a brick are stored in rounds over the shared-memory banks of
// their stencil origins in the brick's tile (set-up, setup.cu): round r holds
// the r-th point of every bank that has more than r points, in bank order.
// Virtual warp vw of a brick with nb points takes the 32 consecutive points
// at positions 32 vw + lane (contiguous record loads).  Two lanes share a
// bank only where a warp's run of 32 spans rounds; but the bank counts of a
// brick are Poisson-like (uniform points over 512 stencil origins, 16 per
// bank), so a brick's fullest bank usually holds more points than the brick
// has warps, and no assignment of one point per lane avoids conflicts: at
// 1M points (244 per brick) a stencil step costs 2.08 shared wavefronts per
// warp on average, against 1.71 for the best possible assignment and 1 for
// none.
__device__ __forceinline__ int brick_point(int nb, int vw, int lane) {
  const int p = vw * 32 + lane;
  return p < nb ? p : -1;
}

// Spread of one brick by the whole CTA (src/RecSumQ.cpp:184-314): the
// brick's points accumulate their p^3 stencils into the shared tile of
// (kBrick + P - 1)^3 grid points, which is then added to the global grid.
template <typename T, int P, bool CPLX>
__device__ __forceinline__ void spread_brick_body(int brick, const int *__restrict__ brick_start,
                                                  const BrickPoint<T> *__restrict__ bp,
                                                  const T *__restrict__ q, T *__restrict__ grid,
                                                  int nb2, int nb3, long N1, long N2, long N3,
                                                  T *tile) {
  constexpr int TL = kBrick + P - 1;
  constexpr int TV = TL * TL * TL;
  constexpr int C = CPLX ? 2 : 1;
  const int b3 = brick % nb3, b2 = (brick / nb3) % nb2, b1 = brick / (nb3 * nb2);
  for (int t = threadIdx.x; t < TV * C; t += blockDim.x) tile[t] = T(0);
  __syncthreads();
  const int beg = brick_start[brick], nbp = brick_start[brick + 1] - beg;
  const int nvw = (nbp + 31) >> 5, lane = threadIdx.x & 31;
  for (int vw = threadIdx.x >> 5; vw < nvw; vw += blockDim.x >> 5) {
    const int pi = brick_point(nbp, vw, lane);
    if (pi < 0) continue;
    const int i = beg + pi;
    const BrickPoint<T> pt = bp[i];
    T w1[P], w2[P], w3[P], dummy[P];
    bspline_weights<T, P, false>(pt.u[0], w1, dummy);
    bspline_weights<T, P, false>(pt.u[1], w2, dummy);
    bspline_weights<T, P, false>(pt.u[2], w3, dummy);
    const int l1 = (int)(pt.g0 >> 20) - b1 * kBrick;
    const int l2 = (int)((pt.g0 >> 10) & 1023u) - b2 * kBrick;
    const int l3 = (int)(pt.g0 & 1023u) - b3 * kBrick;
    const T qr = q[C * (long)i], qi = CPLX ? q[2 * (long)i + 1] : T(0);
#pragma unroll(kStencilUnroll<P>)
    for (int t1 = 0; t1 < P; t1++) {
#pragma unroll
      for (int t2 = 0; t2 < P; t2++) {
        const T c12 = w1[t1] * w2[t2];
        T *row = tile + C * (((l1 + t1) * TL + (l2 + t2)) * TL + l3);
#pragma unroll
        for (int t3 = 0; t3 < P; t3++) {
          const T c = c12 * w3[t3];
          atomicAdd(row + C * t3, c * qr);
          if (CPLX) atomicAdd(row + C * t3 + 1, c * qi);
        }
      }
    }
  }
  __syncthreads();
  const long g1 = (long)b1 * kBrick, g2 = (long)b2 * kBrick, g3 = (long)b3 * kBrick;
  for (int t = threadIdx.x; t < TV; t += blockDim.x) {
    const int i3 = t % TL, i2 = (t / TL) % TL, i1 = t / (TL * TL);
    if (g1 + i1 >= N1) continue;
    if (g2 + i2 >= N2 || g3 + i3 >= N3) continue;  // beyond the box: always zero
    const long gi = ((g1 + i1) * N2 + (g2 + i2)) * N3 + (g3 + i3);
#pragma unroll
    for (int c = 0; c < C; c++) {
      const T v = tile[C * t + c];
      if (v != T(0)) atomicAdd(grid + C * gi + c, v);
    }
  }
}

// FP32 spreading with two native 32-bit integer shared atomics per
// contribution instead of one floating-point shared atomic (which the
// hardware does not have and executes as a compare-and-swap loop; a probe
// ran 3.5x faster with integer atomics).  Each contribution v = c q is
// scaled by S = 2^k so that |v S| <= 2^B, B = min(21, 30 - ceil(log2
// n_brick)): the high words round(v S) of all contributions to a tile point
// cannot exceed 2^30 in sum, and the low words round((v S - hi) 2^B) carry
// B more bits.  The integer sums are exact and independent of the order of
// the atomics; each tile value hi + lo 2^-L is rounded once, to float, when
// it is added to the grid.  Same points, weights and tile as
// spread_brick_body.
template <int P, bool CPLX>
__device__ __forceinline__ void spread_brick_fixed(int brick, const int *__restrict__ brick_start,
                                                   const BrickPoint<float> *__restrict__ bp,
                                                   const float *__restrict__ q,
                                                   float *__restrict__ grid, int nb2, int nb3,
                                                   long N1, long N2, long N3, int *tile) {
  constexpr int TL = kBrick + P - 1;
  constexpr int TV = TL * TL * TL;
  constexpr int C = CPLX ? 2 : 1;
  __shared__ float s_max[32];
  int *thi = tile, *tlo = tile + TV * C;
  const int b3 = brick % nb3, b2 = (brick / nb3) % nb2, b1 = brick / (nb3 * nb2);
  for (int t = threadIdx.x; t < 2 * TV * C; t += blockDim.x) tile[t] = 0;
  const int beg = brick_start[brick], nbp = brick_start[brick + 1] - beg;
  float m = 0.f;
  for (int i = threadIdx.x; i < nbp * C; i += blockDim.x) m = fmaxf(m, fabsf(q[C * (long)beg + i]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  if (lane == 0) s_max[threadIdx.x >> 5] = m;
  __syncthreads();
  m = s_max[0];
  for (int w = 1; w < nw; w++) m = fmaxf(m, s_max[w]);
  if (m == 0.f) return;  // nothing to spread (the whole CTA returns)
  const int lnb = 32 - __clz(max(nbp - 1, 1));  // ceil(log2(nbp)), nbp >= 2
  // bits per contribution: sums of nbp of them stay below 2^30, and single
  // words below 2^22 so that a float converts to int by the add-magic trick
  const int B = min(21, 30 - lnb);
  const int k = max(-120, min(120, B - (ilogbf(m) + 1)));
  const int L = B;
  const float S = ldexpf(1.f, k), SL = ldexpf(1.f, L);
  const int nvw = (nbp + 31) >> 5;
  for (int vw = threadIdx.x >> 5; vw < nvw; vw += nw) {
    const int pi = brick_point(nbp, vw, lane);
    if (pi < 0) continue;
    const int i = beg + pi;
    const BrickPoint<float> pt = bp[i];
    float w1[P], w2[P], w3[P], dummy[P];
    bspline_weights<float, P, false>(pt.u[0], w1, dummy);
    bspline_weights<float, P, false>(pt.u[1], w2, dummy);
    bspline_weights<float, P, false>(pt.u[2], w3, dummy);
    const int l1 = (int)(pt.g0 >> 20) - b1 * kBrick;
    const int l2 = (int)((pt.g0 >> 10) & 1023u) - b2 * kBrick;
    const int l3 = (int)(pt.g0 & 1023u) - b3 * kBrick;
    const float qr = q[C * (long)i] * S, qi = CPLX ? q[2 * (long)i + 1] * S : 0.f;
#pragma unroll(kStencilUnroll<P>)
    for (int t1 = 0; t1 < P; t1++) {
#pragma unroll
      for (int t2 = 0; t2 < P; t2++) {
        const float c12 = w1[t1] * w2[t2];
        const int row = C * (((l1 + t1) * TL + (l2 + t2)) * TL + l3);
#pragma unroll
        for (int t3 = 0; t3 < P; t3++) {
          const float c = c12 * w3[t3];
#pragma unroll
          for (int part = 0; part < C; part++) {
            // |v| <= 2^21: adding 1.5 * 2^23 rounds v to an integer held in
            // the low mantissa bits (no conversion instruction needed)
            constexpr float kMagic = 12582912.f;
            const float v = c * (part ? qi : qr);
            const float vm = v + kMagic;
            const float r = v - (vm - kMagic);  // exact remainder, |r| <= 1/2
            atomicAdd(thi + row + C * t3 + part, __float_as_int(vm) - 0x4B400000);
            atomicAdd(tlo + row + C * t3 + part,
                      __float_as_int(fmaf(r, SL, kMagic)) - 0x4B400000);
          }
        }
      }
    }
  }
  __syncthreads();
  const float invS = ldexpf(1.f, -k), invSL = ldexpf(1.f, -L);
  const long g1 = (long)b1 * kBrick, g2 = (long)b2 * kBrick, g3 = (long)b3 * kBrick;
  for (int t = threadIdx.x; t < TV; t += blockDim.x) {
    const int i3 = t % TL, i2 = (t / TL) % TL, i1 = t / (TL * TL);
    if (g1 + i1 >= N1) continue;
    if (g2 + i2 >= N2 || g3 + i3 >= N3) continue;  // beyond the box: always zero
    const long gi = ((g1 + i1) * N2 + (g2 + i2)) * N3 + (g3 + i3);
#pragma unroll
    for (int c = 0; c < C; c++) {
      const int hv = thi[C * t + c], lv = tlo[C * t + c];
      if (hv != 0 || lv != 0) {
        const double v = ((double)hv + (double)lv * (double)invSL) * (double)invS;
        atomicAdd(grid + C * gi + c, (float)v);
      }
    }
  }
}

// X(k) *= G(|k1|, |k2|, k3) on the R2C half spectrum (src/RecSumV.cpp:639-707),
// one spectrum row (k1, k2) = (r / N2, r % N2) per warp: one division per
// row, and the lanes stride the row's contiguous k3 run (coalesced X and G
// rows; the compact G octant stays in L2).
template <typename T>
__device__ __forceinline__ void multiply_real_row(typename Vec2<T>::type *__restrict__ X,
                                                  const T *__restrict__ G, int r, int N1, int N2,
                                                  int N3h, int M2, int M3, int lane) {
  const int k1 = r / N2, k2 = r - k1 * N2;
  const int f1 = k1 <= N1 / 2 ? k1 : N1 - k1;
  const int f2 = k2 <= N2 / 2 ? k2 : N2 - k2;
  const T *__restrict__ g = G + ((long)f1 * M2 + f2) * M3;
  typename Vec2<T>::type *__restrict__ x = X + (long)r * N3h;
  for (int k3 = lane; k3 < N3h; k3 += 32) {
    const T gv = __ldg(g + k3);
    typename Vec2<T>::type v = x[k3];
    v.x *= gv;
    v.y *= gv;
    x[k3] = v;
  }
}

// X(k) *= G(|k1|, |k2|, |k3|) on the full complex spectrum, one row per warp.
template <typename T>
__device__ __forceinline__ void multiply_cplx_row(typename Vec2<T>::type *__restrict__ X,
                                                  const typename Vec2<T>::type *__restrict__ G,
                                                  int r, int N1, int N2, int N3, int M2, int M3,
                                                  int lane) {
  const int k1 = r / N2, k2 = r - k1 * N2;
  const int f1 = k1 <= N1 / 2 ? k1 : N1 - k1;
  const int f2 = k2 <= N2 / 2 ? k2 : N2 - k2;
  const typename Vec2<T>::type *__restrict__ g = G + ((long)f1 * M2 + f2) * M3;
  typename Vec2<T>::type *__restrict__ x = X + (long)r * N3;
  for (int k3 = lane; k3 < N3; k3 += 32) {
    const int f3 = k3 <= N3 / 2 ? k3 : N3 - k3;
    const typename Vec2<T>::type gv = g[f3];
    const typename Vec2<T>::type v = x[k3];
    typename Vec2<T>::type o;
    o.x = v.x * gv.x - v.y * gv.y;
    o.y = v.x * gv.y + v.y * gv.x;
    x[k3] = o;
  }
}

// One element of the windowed eight-image sum that samples f_LR on the
// compact octant for the kernel transform (src/RecSumGrid.cpp:45-282): per
// axis the two image coordinates x1, x2 and window values T1, T2 are stored
// as ax[0..M) = x1, ax[M..2M) = x2, ax[2M..3M) = T1, ax[3M..4M) = T2.  LR is
// a functor double2 operator()(double r2) returning f_LR (re, im).
template <class LR>
__device__ __forceinline__ double2 fhat_sample_body(const LR &lr, long idx, int M1, int M2,
                                                    int M3, const double *__restrict__ ax,
                                                    const double *__restrict__ ay,
                                                    const double *__restrict__ az) {
  const int i3 = idx % M3, i2 = (idx / M3) % M2, i1 = idx / ((long)M2 * M3);
  double sr = 0, si = 0;
#pragma unroll
  for (int c = 0; c < 8; c++) {
    const int s1 = c >> 2, s2 = (c >> 1) & 1, s3 = c & 1;
    const double x = ax[s1 * M1 + i1], y = ay[s2 * M2 + i2], z = az[s3 * M3 + i3];
    const double t = ax[(2 + s1) * M1 + i1] * ay[(2 + s2) * M2 + i2] * az[(2 + s3) * M3 + i3];
    if (t == 0.0) continue;
    const double2 f = lr(x * x + y * y + z * z);
    sr += t * f.x;
    si += t * f.y;
  }
  return make_double2(sr, si);
}

// Interpolation of one brick by the whole CTA (src/RecSumV.cpp:201-306):
// the brick's theta tile of (kBrick + P - 1)^3 grid points is read into
// shared memory once, then every point gathers its p^3 stencil from the
// tile: V += sum theta B1 B2 B3, grad += (N/L) sum theta dB ..., added into
// the caller-order output.  With vsrc (CalcV after a pair-once direct sum)
// the point's source-side direct-sum slot (same brick-order position) is
// added in the same read-modify-write of V (potential scaled by vs,
// gradient by gs) and cleared for the next call.
template <typename T, int P, bool CPLX>
__device__ __forceinline__ void interp_brick_body(int brick, const int *__restrict__ brick_start,
                                                  const BrickPoint<T> *__restrict__ bp,
                                                  const T *__restrict__ theta,
                                                  double *__restrict__ V, int nb2, int nb3,
                                                  long N1, long N2, long N3, T c1, T c2, T c3,
                                                  T *tile, void *vsrc = nullptr, double vs = 1.0,
                                                  double gs = 1.0) {
  constexpr int TL = kBrick + P - 1;
  constexpr int TV = TL * TL * TL;
  constexpr int C = CPLX ? 2 : 1;
  const int b3 = brick % nb3, b2 = (brick / nb3) % nb2, b1 = brick / (nb3 * nb2);
  const long g1 = (long)b1 * kBrick, g2 = (long)b2 * kBrick, g3 = (long)b3 * kBrick;
  for (int t = threadIdx.x; t < TV; t += blockDim.x) {
    const int i3 = t % TL, i2 = (t / TL) % TL, i1 = t / (TL * TL);
    T vr = T(0), vi = T(0);
    if (g1 + i1 < N1 && g2 + i2 < N2 && g3 + i3 < N3) {
      const long gi = ((g1 + i1) * N2 + (g2 + i2)) * N3 + (g3 + i3);
      vr = theta[C * gi];
      if (CPLX) vi = theta[C * gi + 1];
    }
    tile[C * t] = vr;
    if (CPLX) tile[C * t + 1] = vi;
  }
  __syncthreads();
  const int beg = brick_start[brick], nbp = brick_start[brick + 1] - beg;
  const int nvw = (nbp + 31) >> 5, lane = threadIdx.x & 31;
  for (int vw = threadIdx.x >> 5; vw < nvw; vw += blockDim.x >> 5) {
    const int pi = brick_point(nbp, vw, lane);
    if (pi < 0) continue;
    const BrickPoint<T> pt = bp[beg + pi];
    T w1[P], w2[P], w3[P], d1[P], d2[P], d3[P];
    bspline_weights<T, P, true>(pt.u[0], w1, d1);
    bspline_weights<T, P, true>(pt.u[1], w2, d2);
    bspline_weights<T, P, true>(pt.u[2], w3, d3);
    const int l1 = (int)(pt.g0 >> 20) - b1 * kBrick;
    const int l2 = (int)((pt.g0 >> 10) & 1023u) - b2 * kBrick;
    const int l3 = (int)(pt.g0 & 1023u) - b3 * kBrick;
    T v[4] = {0, 0, 0, 0}, vi[4] = {0, 0, 0, 0};
#pragma unroll(kStencilUnroll<P>)
    for (int t1 = 0; t1 < P; t1++) {
#pragma unroll
      for (int t2 = 0; t2 < P; t2++) {
        const T *row = tile + C * (((l1 + t1) * TL + (l2 + t2)) * TL + l3);
        T tb = 0, td = 0, tbi = 0, tdi = 0;
#pragma unroll
        for (int t3 = 0; t3 < P; t3++) {
          const T th = row[C * t3];
          tb = fma(th, w3[t3], tb);
          td = fma(th, d3[t3], td);
          if (CPLX) {
            const T thi = row[C * t3 + 1];
            tbi = fma(thi, w3[t3], tbi);
            tdi = fma(thi, d3[t3], tdi);
          }
        }
        const T A1 = w1[t1] * w2[t2], A2 = d1[t1] * w2[t2], A3 = w1[t1] * d2[t2];
        v[0] = fma(A1, tb, v[0]);
        v[1] = fma(A2, tb, v[1]);
        v[2] = fma(A3, tb, v[2]);
        v[3] = fma(A1, td, v[3]);
        if (CPLX) {
          vi[0] = fma(A1, tbi, vi[0]);
          vi[1] = fma(A2, tbi, vi[1]);
          vi[2] = fma(A3, tbi, vi[2]);
          vi[3] = fma(A1, tdi, vi[3]);
        }
      }
    }
    const T sc[4] = {T(1), c1, c2, c3};
    const long o = pt.orig, slot = beg + pi;
    if (CPLX) {
      // source-side slot (FP32 complex): (V re, V im, x re, x im), (y .., z ..)
      double d[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      if (vsrc) {
        float4 *vp = reinterpret_cast<float4 *>(vsrc) + 2 * slot;
        const float4 a = vp[0], b = vp[1];
        vp[0] = vp[1] = make_float4(0.f, 0.f, 0.f, 0.f);
        d[0] = a.x, d[1] = a.y, d[2] = a.z, d[3] = a.w;
        d[4] = b.x, d[5] = b.y, d[6] = b.z, d[7] = b.w;
      }
      double2 *Vo = reinterpret_cast<double2 *>(V) + 4 * o;
#pragma unroll
      for (int m = 0; m < 4; m++) {
        double2 a = Vo[m];
        a.x += (double)(v[m] * sc[m]) + d[2 * m];
        a.y += (double)(vi[m] * sc[m]) + d[2 * m + 1];
        Vo[m] = a;
      }
    } else {
      double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
      if (vsrc) {
        if (sizeof(T) == 4) {  // FP32: float4 per slot, scaled frame
          float4 *vp = reinterpret_cast<float4 *>(vsrc) + slot;
          const float4 a = *vp;
          *vp = make_float4(0.f, 0.f, 0.f, 0.f);
          s0 = vs * (double)a.x, s1 = gs * (double)a.y, s2 = gs * (double)a.z,
          s3 = gs * (double)a.w;
        } else {  // FP64: [4] doubles per slot
          double4 *vp = reinterpret_cast<double4 *>(vsrc) + slot;
          const double4 a = *vp;
          *vp = make_double4(0, 0, 0, 0);
          s0 = vs * a.x, s1 = gs * a.y, s2 = gs * a.z, s3 = gs * a.w;
        }
      }
      double4 *Vo = reinterpret_cast<double4 *>(V) + o;
      double4 a = *Vo;
      a.x += (double)v[0] + s0;
      a.y += (double)(v[1] * c1) + s1;
      a.z += (double)(v[2] * c2) + s2;
      a.w += (double)(v[3] * c3) + s3;
      *Vo = a;
    }
  }
}

// kPackedBlock consecutive source-pair steps of the packed direct sum: the
// differences and distances of all steps first, then the refinement of close
// pairs (rare, a divergent branch), then the pair kernel of all steps without
// branches, so that the scheduler can interleave the independent polynomial
// chains of the block.  Pairs outside the cutoff (and the target itself) get
// r^2 = Rdir^2 and charge 0.  The whole pair phase is skipped when no lane
// of the warp has a hit in the block.
#ifndef NPME_PACKED_BLOCK
#define NPME_PACKED_BLOCK 2
#endif
constexpr int kPackedBlock = NPME_PACKED_BLOCK;

// Real DM pair kernel in the scaled frame (coordinates in units of Rdir,
// s = r^2): f0 = Rdir^(-alpha)... scaled f_SR and t = -(scaled f1) for two
// squared distances at once.  1/r: f0 = 1/r - P(s), t = 1/r^3 + D(s);
// r^alpha: f0 = s^(alpha/2) - P(s), t = -alpha s^(alpha/2) / s + D(s), with
// P, D the DM polynomials (src/KernelFunctionLaplace.cpp:394-436,
// src/KernelFunctionRalpha.cpp:342-384).
// ND > 0: the derivative-match order as a compile-time constant (the
// polynomials fully unrolled); ND = 0: any order up to kMaxDeriv, evaluated
// as the polynomials of degree kMaxDeriv whose coefficients above the order
// are zero (make_pair_coef), so Horner's leading steps give exactly 0 and
// the result is bit for bit that of the exact degree, at the cost of the
// extra steps but with every coefficient at a fixed offset of the parameter
// bank (a loop over a run-time degree indexes it dynamically and is ~2x
// slower still).
template <int ND>
constexpr int dm_degree() {
  return ND > 0 ? ND : kMaxDeriv;
}

template <int FUNC, int ND>
__device__ __forceinline__ void dm_eval2(const PairCoef<float> &k, float2 sv, float2 &f0,
                                         float2 &t) {
  constexpr int nd = dm_degree<ND>();
  float2 np = k.nar2[nd];  // -Rdir^(-alpha) f_LR polynomial
#pragma unroll
  for (int n = nd - 1; n >= 0; n--) np = __ffma2_rn(np, sv, k.nar2[n]);
  float2 d = k.br2[nd - 1];  // Rdir^(2-alpha) (1/r) d f_LR / dr polynomial
#pragma unroll
  for (int n = nd - 2; n >= 0; n--) d = __ffma2_rn(d, sv, k.br2[n]);
  if (FUNC == 0) {
    const float2 ri = make_float2(rsqrtf(sv.x), rsqrtf(sv.y));
    f0 = __fadd2_rn(ri, np);                    // Rdir (1/r - f_LR)
    t = __ffma2_rn(__fmul2_rn(ri, ri), ri, d);  // -Rdir^3 f1
  } else {
    // s^(alpha/2) = 2^((alpha/2) log2 s) on the special-function unit;
    // 1/s = rsqrt(s)^2
    const float2 e0 = make_float2(exp2f(k.half_alpha * __log2f(sv.x)),
                                  exp2f(k.half_alpha * __log2f(sv.y)));
    const float2 ri = make_float2(rsqrtf(sv.x), rsqrtf(sv.y));
    f0 = __fadd2_rn(e0, np);
    t = __ffma2_rn(__fmul2_rn(e0, make_float2(-k.alpha, -k.alpha)), __fmul2_rn(ri, ri), d);
  }
}

// The same pair kernel for one squared distance.
template <int FUNC, int ND>
__device__ __forceinline__ void dm_eval1(const PairCoef<float> &k, float sv, float &f0,
                                         float &t) {
  constexpr int nd = dm_degree<ND>();
  float np = k.nar2[nd].x;
#pragma unroll
  for (int n = nd - 1; n >= 0; n--) np = fmaf(np, sv, k.nar2[n].x);
  float d = k.br2[nd - 1].x;
#pragma unroll
  for (int n = nd - 2; n >= 0; n--) d = fmaf(d, sv, k.br2[n].x);
  const float ri = rsqrtf(sv);
  if (FUNC == 0) {
    f0 = ri + np;
    t = fmaf(ri * ri, ri, d);
  } else {
    const float e0 = exp2f(k.half_alpha * __log2f(sv));
    f0 = e0 + np;
    t = fmaf(e0 * -k.alpha, ri * ri, d);
  }
}

template <int FUNC, int ND, bool REFINE>
__device__ __forceinline__ void packed_block(
    const PairCoef<float> &k, const float4 *sp, const float4 *slo, int s0, float2 tx2,
    float2 ty2, float2 tz2, float2 tl2x, float2 tl2y, float2 tl2z, float R2, float refine2,
    float2 &P0, float2 &N1, float2 &N2, float2 &N3) {
  constexpr int U = kPackedBlock;
  // rr: r^2 of the pairs inside the cutoff, R2 for the others (and for the
  // target itself); qm: their charges, 0 for the others.  A pair is inside
  // iff 0 < r^2 <= R2, i.e. iff bits(r^2) - 1 < bits(R2) as unsigned
  // integers (r^2 >= 0).
  float2 x[U], y[U], z[U], rr[U], qm[U];
  float rmin = 3.0e38f;
  bool any = false;
  const unsigned rb = __float_as_uint(R2);
#pragma unroll
  for (int u = 0; u < U; u++) {
    const float4 A = sp[s0 + u], B = sp[16 + s0 + u];
    x[u] = __fadd2_rn(tx2, make_float2(A.x, A.y));
    y[u] = __fadd2_rn(ty2, make_float2(A.z, A.w));
    z[u] = __fadd2_rn(tz2, make_float2(B.x, B.y));
    const float2 r2 = __ffma2_rn(x[u], x[u], __ffma2_rn(y[u], y[u], __fmul2_rn(z[u], z[u])));
    const bool h0 = __float_as_uint(r2.x) - 1u < rb, h1 = __float_as_uint(r2.y) - 1u < rb;
    rr[u] = make_float2(h0 ? r2.x : R2, h1 ? r2.y : R2);
    qm[u] = make_float2(h0 ? B.z : 0.f, h1 ? B.w : 0.f);
    if (REFINE) rmin = fminf(rmin, fminf(rr[u].x, rr[u].y));
    any |= h0 | h1;
  }
  if (!__any_sync(0xffffffffu, any)) return;
  if (REFINE && rmin < refine2) {  // close pair: exact difference from head + residual
#pragma unroll
    for (int u = 0; u < U; u++) {
      if (fminf(rr[u].x, rr[u].y) < refine2) {
        const float4 LA = slo[s0 + u], LB = slo[16 + s0 + u];
        x[u] = __fadd2_rn(x[u], __fadd2_rn(tl2x, make_float2(LA.x, LA.y)));
        y[u] = __fadd2_rn(y[u], __fadd2_rn(tl2y, make_float2(LA.z, LA.w)));
        z[u] = __fadd2_rn(z[u], __fadd2_rn(tl2z, make_float2(LB.x, LB.y)));
        const float2 rn = __ffma2_rn(x[u], x[u], __ffma2_rn(y[u], y[u], __fmul2_rn(z[u], z[u])));
        // the hit decision stays that of the unrefined distance
        rr[u].x = rr[u].x < R2 ? rn.x : rr[u].x;
        rr[u].y = rr[u].y < R2 ? rn.y : rr[u].y;
      }
    }
  }
#pragma unroll
  for (int u = 0; u < U; u++) {
    float2 f0, t;  // t = -f1
    dm_eval2<FUNC, ND>(k, rr[u], f0, t);
    const float2 gq = __fmul2_rn(t, qm[u]);
    P0 = __ffma2_rn(f0, qm[u], P0);
    N1 = __ffma2_rn(gq, x[u], N1);
    N2 = __ffma2_rn(gq, y[u], N2);
    N3 = __ffma2_rn(gq, z[u], N3);
  }
}

// Position of a lane in the virtual concatenation of a group's source
// segments (segment index and offset in it), so that a staged chunk of 32
// sources runs across segment boundaries.
struct SrcCursor {
  int seg, off;
  __device__ __forceinline__ void normalize(const int2 *__restrict__ segs, int end) {
    while (seg < end) {
      const int c = segs[seg].y;
      if (off < c) break;
      off -= c;
      seg++;
    }
  }
};

// Real derivative-match kernels (1/r, r^alpha) of the FP32 direct sum with
// packed arithmetic: every lane evaluates its target against two sources per
// step with sm_100's two-wide FP32 instructions (__fadd2_rn / __fmul2_rn /
// __ffma2_rn), which halves the issued arithmetic of the distance test and
// of the polynomial.  The staged chunk is laid out in source pairs:
//   sp[p]      = (-x_2p, -x_2p+1, -y_2p, -y_2p+1)
//   sp[16 + p] = (-z_2p, -z_2p+1,  q_2p,  q_2p+1)
// (coordinates negated so that t + (-s) gives t - s exactly), slo the same
// for the low parts of the rounded differences.  Slots past the chunk hold a
// far source with charge 0.  Same arithmetic per pair as the scalar body
// (difference, r^2, hit test, refinement below refine2, polynomial in
// s = r^2/Rdir^2), except that a refined step refines both of its pairs.
template <int FUNC, int ND>
__device__ __forceinline__ void direct_group_packed(
    const PairCoef<float> &k, const double4 *__restrict__ gpos, const double4 *__restrict__ spos,
    const float *__restrict__ qs, const double *__restrict__ qcaller, const int4 G,
    const double4 c, const int2 *__restrict__ segs, const uint32_t *__restrict__ perm,
    float refine2, double fself_r, double *__restrict__ V, float4 *sp, float4 *slo, int lane) {
  const int ti = G.x + lane;
  const bool active = lane < G.y;
  // idle lanes sit far outside the cutoff
  float tx = 1e18f, ty = 1e18f, tz = 1e18f, tlx = 0.f, tly = 0.f, tlz = 0.f;
  const double ir = k.invR;  // coordinates in units of Rdir
  if (active) {
    const double4 p = gpos[ti];
    const double dx = (p.x - c.x) * ir, dy = (p.y - c.y) * ir, dz = (p.z - c.z) * ir;
    tx = (float)dx, ty = (float)dy, tz = (float)dz;
    tlx = (float)(dx - (double)tx), tly = (float)(dy - (double)ty), tlz = (float)(dz - (double)tz);
  }
  const float2 tx2 = make_float2(tx, tx), ty2 = make_float2(ty, ty), tz2 = make_float2(tz, tz);
  const float2 tl2x = make_float2(tlx, tlx), tl2y = make_float2(tly, tly),
               tl2z = make_float2(tlz, tlz);
  const float R2 = 1.f;
  refine2 = (float)((double)refine2 * ir * ir);
  double acc[4] = {0, 0, 0, 0};
  float *sa = reinterpret_cast<float *>(sp), *la = reinterpret_cast<float *>(slo);
  const int slot = (lane >> 1) * 4 + (lane & 1);

  // A pair closer than sqrt(refine2) needs its source within the group's
  // half-diagonal (c.w) plus sqrt(refine2) of the centre; chunks with no
  // such source skip the refinement bookkeeping.
  const double rfs = sqrt((double)refine2) + c.w * ir;
  const double near2 = rfs * rfs;
  bool near = false;
  // register prefetch of the next chunk: lane l holds source l of the chunk
  SrcCursor cur{G.z, lane};
  cur.normalize(segs, G.w);
  bool pv = cur.seg < G.w;
  double px = 0, py = 0, pz = 0;
  float pq = 0.f;
  if (pv) {
    const long j = (long)segs[cur.seg].x + cur.off;
    const double4 p = spos[j];
    px = p.x, py = p.y, pz = p.z, pq = qs[j];
  }
  while (__any_sync(0xffffffffu, pv)) {
    const int pcnt = __popc(__ballot_sync(0xffffffffu, pv));  // valid lanes form a prefix
    __syncwarp();
    {
      float hx = 1e18f, hy = 1e18f, hz = 1e18f, q = 0.f, lx = 0.f, ly = 0.f, lz = 0.f;
      near = false;
      if (pv) {
        const double dx = (px - c.x) * ir, dy = (py - c.y) * ir, dz = (pz - c.z) * ir;
        hx = (float)dx, hy = (float)dy, hz = (float)dz;
        lx = (float)(dx - (double)hx), ly = (float)(dy - (double)hy), lz = (float)(dz - (double)hz);
        q = pq;
        near = dx * dx + dy * dy + dz * dz < near2;
      }
      sa[slot] = -hx;
      sa[slot + 2] = -hy;
      sa[64 + slot] = -hz;
      sa[64 + slot + 2] = q;
      la[slot] = -lx;
      la[slot + 2] = -ly;
      la[64 + slot] = -lz;
    }
    __syncwarp();
    cur.off += 32;
    cur.normalize(segs, G.w);
    pv = cur.seg < G.w;
    if (pv) {
      const long j = (long)segs[cur.seg].x + cur.off;
      const double4 p = spos[j];
      px = p.x, py = p.y, pz = p.z, pq = qs[j];
    }
    const int npair = (pcnt + 1) >> 1;
    float2 P0 = make_float2(0.f, 0.f), N1 = P0, N2 = P0, N3 = P0;  // N*: minus the gradient
    // blocks of kPackedBlock steps; slots past the chunk hold far sources, so
    // the step count is rounded up to whole blocks
    if (__any_sync(0xffffffffu, near)) {
      for (int s0 = 0; s0 < npair; s0 += kPackedBlock)
        packed_block<FUNC, ND, true>(k, sp, slo, s0, tx2, ty2, tz2, tl2x, tl2y, tl2z, R2, refine2,
                                     P0, N1, N2, N3);
    } else {
      for (int s0 = 0; s0 < npair; s0 += kPackedBlock)
        packed_block<FUNC, ND, false>(k, sp, slo, s0, tx2, ty2, tz2, tl2x, tl2y, tl2z, R2,
                                      refine2, P0, N1, N2, N3);
    }
    acc[0] += (double)P0.x + (double)P0.y;
    acc[1] -= (double)N1.x + (double)N1.y;
    acc[2] -= (double)N2.x + (double)N2.y;
    acc[3] -= (double)N3.x + (double)N3.y;
  }
  if (active) {
    const long o = perm[ti];
    const double vs = k.vscale, gs = k.gscale;
    // V -= f_LR(0) q (src/Interface.cpp:2061-2062)
    reinterpret_cast<double4 *>(V)[o] =
        make_double4(vs * acc[0] - fself_r * qcaller[o], gs * acc[1], gs * acc[2], gs * acc[3]);
  }
}

// One block of steps of the Newton's-third-law sweep (below):
// lane l holds the source pair (a, b) of a 64-source chunk in registers and
// meets target (l + k) mod 32 of the group at step k, read from the group's
// target tile in shared memory.  Every pair is evaluated once and gives both
// sides: the target-side sums (aV, aX, aY, aZ) travel with their target,
// one lane down per step (__shfl_sync from lane + 1), and the source-side
// sums (SV, SX, SY, SZ, packed for a and b) stay in the lane.  Source
// coordinates are held negated (sx2 = -x_s) as in the staged layout of the
// one-sided body; misses get r^2 = 1 (Rdir^2) and charge 0 on both sides.
#ifndef NPME_SYM_BLOCK
#define NPME_SYM_BLOCK 0
#endif
// steps per block of the pair-once sweep (measured: 2 for 1/r, 4 for r^alpha)
template <int FUNC>
constexpr int sym_block_steps() {
  return NPME_SYM_BLOCK > 0 ? NPME_SYM_BLOCK : (FUNC == 1 ? 4 : 2);
}

template <int FUNC, int ND, bool REFINE>
__device__ __forceinline__ void sym_block(
    const PairCoef<float> &k, const float4 *tsm, const float4 *tlo, int lane, int k0,
    float2 sx2, float2 sy2, float2 sz2, float2 q2, float2 lx2, float2 ly2, float2 lz2,
    float refine2, float &aV, float &aX, float &aY, float &aZ, float2 &SV, float2 &SX,
    float2 &SY, float2 &SZ) {
  constexpr int U = sym_block_steps<FUNC>();
  const unsigned FULL = 0xffffffffu;
  const unsigned rb = __float_as_uint(1.f);
  float2 x[U], y[U], z[U], rr[U], qm[U], qt[U];
  int tt[U];
  float rmin = 3.0e38f;
  bool any = false;
#pragma unroll
  for (int u = 0; u < U; u++) {
    tt[u] = (lane + k0 + u) & 31;
    const float4 T = tsm[tt[u]];
    x[u] = __fadd2_rn(make_float2(T.x, T.x), sx2);
    y[u] = __fadd2_rn(make_float2(T.y, T.y), sy2);
    z[u] = __fadd2_rn(make_float2(T.z, T.z), sz2);
    const float2 r2 = __ffma2_rn(x[u], x[u], __ffma2_rn(y[u], y[u], __fmul2_rn(z[u], z[u])));
    const bool h0 = __float_as_uint(r2.x) - 1u < rb, h1 = __float_as_uint(r2.y) - 1u < rb;
    rr[u] = make_float2(h0 ? r2.x : 1.f, h1 ? r2.y : 1.f);
    qm[u] = make_float2(h0 ? q2.x : 0.f, h1 ? q2.y : 0.f);
    qt[u] = make_float2(h0 ? T.w : 0.f, h1 ? T.w : 0.f);
    if (REFINE) rmin = fminf(rmin, fminf(rr[u].x, rr[u].y));
    any |= h0 | h1;
  }
  if (!__any_sync(FULL, any)) {  // no pair of the block inside the cutoff
    const int src = (lane + U) & 31;
    aV = __shfl_sync(FULL, aV, src);
    aX = __shfl_sync(FULL, aX, src);
    aY = __shfl_sync(FULL, aY, src);
    aZ = __shfl_sync(FULL, aZ, src);
    return;
  }
  if (REFINE && rmin < refine2) {  // close pair: exact difference from head + residual
#pragma unroll
    for (int u = 0; u < U; u++) {
      if (fminf(rr[u].x, rr[u].y) < refine2) {
        const float4 L = tlo[tt[u]];
        x[u] = __fadd2_rn(x[u], __fadd2_rn(make_float2(L.x, L.x), lx2));
        y[u] = __fadd2_rn(y[u], __fadd2_rn(make_float2(L.y, L.y), ly2));
        z[u] = __fadd2_rn(z[u], __fadd2_rn(make_float2(L.z, L.z), lz2));
        const float2 rn = __ffma2_rn(x[u], x[u], __ffma2_rn(y[u], y[u], __fmul2_rn(z[u], z[u])));
        // the hit decision stays that of the unrefined distance
        rr[u].x = rr[u].x < 1.f ? rn.x : rr[u].x;
        rr[u].y = rr[u].y < 1.f ? rn.y : rr[u].y;
      }
    }
  }
  const int src = (lane + 1) & 31;
#pragma unroll
  for (int u = 0; u < U; u++) {
    float2 f0, t;  // t = -f1
    dm_eval2<FUNC, ND>(k, rr[u], f0, t);
    const float2 gq = __fmul2_rn(t, qm[u]), gs = __fmul2_rn(t, qt[u]);
    aV = fmaf(f0.x, qm[u].x, fmaf(f0.y, qm[u].y, aV));
    aX = fmaf(gq.x, x[u].x, fmaf(gq.y, x[u].y, aX));
    aY = fmaf(gq.x, y[u].x, fmaf(gq.y, y[u].y, aY));
    aZ = fmaf(gq.x, z[u].x, fmaf(gq.y, z[u].y, aZ));
    SV = __ffma2_rn(f0, qt[u], SV);
    SX = __ffma2_rn(gs, x[u], SX);
    SY = __ffma2_rn(gs, y[u], SY);
    SZ = __ffma2_rn(gs, z[u], SZ);
    aV = __shfl_sync(FULL, aV, src);
    aX = __shfl_sync(FULL, aX, src);
    aY = __shfl_sync(FULL, aY, src);
    aZ = __shfl_sync(FULL, aZ, src);
  }
}

// Real derivative-match kernels (1/r, r^alpha) of the FP32 direct sum with
// every unordered pair evaluated once (Newton's third law, as the
// reference's own cell-pair loops do: src/PotentialLaplace.cpp:145-197,
// :3447-3610).  The group walks its half-shell source segments: sources
// whose point lies in a later coarse column, or later in the group's own
// column, than the group's targets (set-up, setup.cu); the pairs inside the
// group are the first phase, from both sides with target-side sums only.
// Target-side sums accumulate per chunk in FP32 and across chunks in FP64,
// as in the one-sided body; the source-side sums of a chunk are added to
// vsrc (FP32, scaled frame; slot = the source's brick-order position, from
// spos[j].w) with one vector atomic per source, and folded into V by the
// interpolation (CalcV) or by merge_source_kernel.
template <int FUNC, int ND>
__device__ __forceinline__ void direct_group_sym(
    const PairCoef<float> &k, const double4 *__restrict__ gpos, const double4 *__restrict__ spos,
    const float *__restrict__ qs, const double *__restrict__ qcaller, const int4 G,
    const double4 c, const int2 *__restrict__ segs, const uint32_t *__restrict__ perm,
    float refine2, double fself_r, double *__restrict__ V, float4 *__restrict__ vsrc,
    float4 *tsm, float4 *tlo, int lane) {
  const unsigned FULL = 0xffffffffu;
  const int ti = G.x + lane;
  const bool active = lane < G.y;
  // idle lanes sit far outside the cutoff with charge 0
  float tx = 1e18f, ty = 1e18f, tz = 1e18f, tlx = 0.f, tly = 0.f, tlz = 0.f, tq = 0.f;
  const double ir = k.invR;  // coordinates in units of Rdir
  long o = 0;
  if (active) {
    const double4 p = gpos[ti];
    o = perm[ti];
    const double dx = (p.x - c.x) * ir, dy = (p.y - c.y) * ir, dz = (p.z - c.z) * ir;
    tx = (float)dx, ty = (float)dy, tz = (float)dz;
    tlx = (float)(dx - (double)tx), tly = (float)(dy - (double)ty), tlz = (float)(dz - (double)tz);
    tq = (float)qcaller[o];
  }
  tsm[lane] = make_float4(tx, ty, tz, tq);
  tlo[lane] = make_float4(tlx, tly, tlz, 0.f);
  __syncwarp();
  refine2 = (float)((double)refine2 * ir * ir);
  const unsigned rb = __float_as_uint(1.f);
  double acc[4] = {0, 0, 0, 0};

  // pairs inside the group, from both sides; the differences are always
  // refined (head difference + residual difference)
  {
    float aV = 0.f, aX = 0.f, aY = 0.f, aZ = 0.f;
    for (int s = 0; s < G.y; s++) {
      const float4 S = tsm[s], L = tlo[s];
      const float x = (tx - S.x) + (tlx - L.x), y = (ty - S.y) + (tly - L.y),
                  z = (tz - S.z) + (tlz - L.z);
      const float r2 = fmaf(x, x, fmaf(y, y, z * z));
      const bool hit = __float_as_uint(r2) - 1u < rb;  // 0 < r^2 <= 1, not the target itself
      float f0, t;
      dm_eval1<FUNC, ND>(k, hit ? r2 : 1.f, f0, t);
      const float q = hit ? S.w : 0.f, g = t * q;
      aV = fmaf(f0, q, aV);
      aX = fmaf(g, x, aX);
      aY = fmaf(g, y, aY);
      aZ = fmaf(g, z, aZ);
    }
    acc[0] += (double)aV;
    acc[1] -= (double)aX;
    acc[2] -= (double)aY;
    acc[3] -= (double)aZ;
  }

  // half-shell segments in chunks of 64 sources: lane l holds positions l
  // and l + 32 of the chunk (register prefetch of the next chunk)
  const double rfs = sqrt((double)refine2) + c.w * ir;
  const double near2 = rfs * rfs;
  SrcCursor ca{G.z, lane};
  ca.normalize(segs, G.w);
  SrcCursor cb{ca.seg, ca.off + 32};
  cb.normalize(segs, G.w);
  bool va = ca.seg < G.w, vb = cb.seg < G.w;
  long ja = -1, jb = -1;
  double4 pa = make_double4(0, 0, 0, 0), pb = pa;
  float qa = 0.f, qb = 0.f;
  if (va) ja = (long)segs[ca.seg].x + ca.off, pa = spos[ja], qa = qs[ja];
  if (vb) jb = (long)segs[cb.seg].x + cb.off, pb = spos[jb], qb = qs[jb];
  while (__any_sync(FULL, va)) {
    // this chunk's sources, relative to the group centre; empty slots far
    // away (on the other side from idle targets) with charge 0
    float hxa = -1e18f, hya = -1e18f, hza = -1e18f, lxa = 0.f, lya = 0.f, lza = 0.f;
    float hxb = -1e18f, hyb = -1e18f, hzb = -1e18f, lxb = 0.f, lyb = 0.f, lzb = 0.f;
    bool near = false;
    // source-side slots: the sources' brick-order positions
    const long ka = va ? (long)pa.w : -1, kb = vb ? (long)pb.w : -1;
    float q0 = 0.f, q1 = 0.f;
    if (va) {
      const double dx = (pa.x - c.x) * ir, dy = (pa.y - c.y) * ir, dz = (pa.z - c.z) * ir;
      hxa = (float)dx, hya = (float)dy, hza = (float)dz;
      lxa = (float)(dx - (double)hxa), lya = (float)(dy - (double)hya), lza = (float)(dz - (double)hza);
      q0 = qa;
      near = dx * dx + dy * dy + dz * dz < near2;
    }
    if (vb) {
      const double dx = (pb.x - c.x) * ir, dy = (pb.y - c.y) * ir, dz = (pb.z - c.z) * ir;
      hxb = (float)dx, hyb = (float)dy, hzb = (float)dz;
      lxb = (float)(dx - (double)hxb), lyb = (float)(dy - (double)hyb), lzb = (float)(dz - (double)hzb);
      q1 = qb;
      near = near || dx * dx + dy * dy + dz * dz < near2;
    }
    const float2 sx2 = make_float2(-hxa, -hxb), sy2 = make_float2(-hya, -hyb),
                 sz2 = make_float2(-hza, -hzb), q2 = make_float2(q0, q1);
    const float2 lx2 = make_float2(-lxa, -lxb), ly2 = make_float2(-lya, -lyb),
                 lz2 = make_float2(-lza, -lzb);
    // prefetch the next chunk
    ca.off += 64;
    ca.normalize(segs, G.w);
    cb.off += 64;
    cb.normalize(segs, G.w);
    va = ca.seg < G.w, vb = cb.seg < G.w;
    if (va) ja = (long)segs[ca.seg].x + ca.off, pa = spos[ja], qa = qs[ja];
    if (vb) jb = (long)segs[cb.seg].x + cb.off, pb = spos[jb], qb = qs[jb];

    float aV = 0.f, aX = 0.f, aY = 0.f, aZ = 0.f;
    float2 SV = make_float2(0.f, 0.f), SX = SV, SY = SV, SZ = SV;
    if (__any_sync(FULL, near)) {
      for (int k0 = 0; k0 < 32; k0 += sym_block_steps<FUNC>())
        sym_block<FUNC, ND, true>(k, tsm, tlo, lane, k0, sx2, sy2, sz2, q2, lx2, ly2, lz2,
                                  refine2, aV, aX, aY, aZ, SV, SX, SY, SZ);
    } else {
      for (int k0 = 0; k0 < 32; k0 += sym_block_steps<FUNC>())
        sym_block<FUNC, ND, false>(k, tsm, tlo, lane, k0, sx2, sy2, sz2, q2, lx2, ly2, lz2,
                                   refine2, aV, aX, aY, aZ, SV, SX, SY, SZ);
    }
    // after 32 steps every target's sums are back in its own lane
    acc[0] += (double)aV;
    acc[1] -= (double)aX;
    acc[2] -= (double)aY;
    acc[3] -= (double)aZ;
    if (ka >= 0) atomicAdd(vsrc + ka, make_float4(SV.x, SX.x, SY.x, SZ.x));
    if (kb >= 0) atomicAdd(vsrc + kb, make_float4(SV.y, SX.y, SY.y, SZ.y));
  }
  if (active) {
    const double vs = k.vscale, gs = k.gscale;
    // V -= f_LR(0) q (src/Interface.cpp:2061-2062)
    reinterpret_cast<double4 *>(V)[o] =
        make_double4(vs * acc[0] - fself_r * qcaller[o], gs * acc[1], gs * acc[2], gs * acc[3]);
  }
}

// sin and cos of x on the special-function unit after a Cody-Waite
// reduction to [-pi, pi] (2 pi split as 6.28125 + 1.9353071795864769e-3, the
// first part exact in 8 bits so n * 6.28125 is exact for |n| < 2^16).
__device__ __forceinline__ float2 sincos_sfu(float x) {
  const float n = rintf(x * 0.15915494309189535f);
  float y = fmaf(-n, 6.28125f, x);
  y = fmaf(-n, 1.9353071795864769e-3f, y);
  return make_float2(__cosf(y), __sinf(y));
}

// Helmholtz DM pair kernel at squared distance rr (FP32, complex as float2):
// F0 = exp(i k0 r)/r - f_LR (the DM polynomial in s = rr / Rdir^2, held
// negated in nac2) and F1 = (1/r) dF0/dr, with sin / cos on the
// special-function unit (src/KernelFunctionHelmholtz.cpp:506-563).
template <int ND>
__device__ __forceinline__ void helm_eval(const PairCoef<float> &k, float rr, float2 &F0,
                                          float2 &F1) {
  const float2 ik = make_float2(-k.k0i, k.k0r);  // i k0
  const float ri = rsqrtf(rr), r = rr * ri;
  const float2 cs = sincos_sfu(k.k0r * r);
  const float damp = k.k0i != 0.f ? __expf(-k.k0i * r) * ri : ri;
  const float2 E = __fmul2_rn(cs, make_float2(damp, damp));  // exp(i k0 r) / r
  // E1 = (i k0 E - E / r) / r, the radial derivative over r
  const float2 IK = __ffma2_rn(make_float2(ik.x, ik.x), E,
                               __fmul2_rn(make_float2(-ik.y, ik.y), make_float2(E.y, E.x)));
  const float ri2 = ri * ri;
  const float2 E1 = __ffma2_rn(E, make_float2(-ri2, -ri2), __fmul2_rn(IK, make_float2(ri, ri)));
  const float sv = rr * k.invR2;
  const float2 s2 = make_float2(sv, sv);
  constexpr int nd = dm_degree<ND>();  // ND = 0: zero-padded to kMaxDeriv
  float2 P = k.nac2[nd];
#pragma unroll
  for (int n = nd - 1; n >= 0; n--) P = __ffma2_rn(P, s2, k.nac2[n]);
  float2 D = k.nbc2[nd - 1];
#pragma unroll
  for (int n = nd - 2; n >= 0; n--) D = __ffma2_rn(D, s2, k.nbc2[n]);
  F0 = __fadd2_rn(E, P);
  F1 = __fadd2_rn(E1, D);
}

// Helmholtz DM kernel exp(i k0 r)/r of the FP32 direct sum with packed
// complex arithmetic: one source per lane per step, the (re, im) parts of
// exp(i k0 r)/r, of the DM polynomials and of the charge products in
// FP32x2 instructions, sin / cos on the special-function unit.  Same staged
// chunk as the scalar body (sp: x, y, z, Re q; slo: low parts, Im q); pairs
// outside the cutoff get r^2 = Rdir^2 and charge 0, the rare close pairs
// are refined as in the scalar body.
template <int ND>
__device__ __forceinline__ void helmholtz_steps(const PairCoef<float> &k, const float4 *sp,
                                                const float4 *slo, int cnt, float tx, float ty,
                                                float tz, float tlx, float tly, float tlz,
                                                float refine2, float2 &Pv, float2 &Gx,
                                                float2 &Gy, float2 &Gz) {
  const float R2 = k.R2;
  const unsigned rb = __float_as_uint(R2);
#pragma unroll 4
  for (int s = 0; s < cnt; s++) {
    const float4 src = sp[s];
    float x = tx - src.x, y = ty - src.y, z = tz - src.z;
    float r2 = fmaf(x, x, fmaf(y, y, z * z));
    const bool hit = __float_as_uint(r2) - 1u < rb;  // 0 < r2 <= R2
    if (hit && r2 < refine2) {  // close pair: exact difference from head + residual
      const float4 lo = slo[s];
      x += tlx - lo.x;
      y += tly - lo.y;
      z += tlz - lo.z;
      r2 = fmaf(x, x, fmaf(y, y, z * z));
    }
    const float rr = hit ? r2 : R2;
    const float4 lo = slo[s];
    const float2 q = hit ? make_float2(src.w, lo.w) : make_float2(0.f, 0.f);
    float2 F0, F1;
    helm_eval<ND>(k, rr, F0, F1);
    const float2 qs = make_float2(q.y, q.x);
    // V += F0 q, G = F1 q (complex products)
    Pv = __ffma2_rn(make_float2(F0.x, F0.x), q, Pv);
    Pv = __ffma2_rn(make_float2(-F0.y, F0.y), qs, Pv);
    const float2 G = __ffma2_rn(make_float2(-F1.y, F1.y), qs,
                                __fmul2_rn(make_float2(F1.x, F1.x), q));
    Gx = __ffma2_rn(G, make_float2(x, x), Gx);
    Gy = __ffma2_rn(G, make_float2(y, y), Gy);
    Gz = __ffma2_rn(G, make_float2(z, z), Gz);
  }
}

// complex a * b + c and a * b on float2 (re, im)
__device__ __forceinline__ float2 cfma(float2 a, float2 b, float2 c) {
  c = __ffma2_rn(make_float2(a.x, a.x), b, c);
  return __ffma2_rn(make_float2(-a.y, a.y), make_float2(b.y, b.x), c);
}
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return __ffma2_rn(make_float2(-a.y, a.y), make_float2(b.y, b.x),
                    __fmul2_rn(make_float2(a.x, a.x), b));
}

// Helmholtz DM kernel of the FP32 direct sum with every unordered pair
// evaluated once (the complex counterpart of direct_group_sym): the group's
// targets sit in shared memory (th = heads and Re q, tl = residuals and Im
// q), each lane holds two sources of a 64-source chunk of the half-shell
// segments, target (l + k) mod 32 meets lane l at step k and its complex sums
// (V, dV/dx, dV/dy, dV/dz) rotate one lane down per step; the source-side
// sums of a chunk go to vsrc as two float4 per source (V re, V im, x re,
// x im; y re, y im, z re, z im) with vector atomics.  Coordinates are
// unscaled offsets from the group centre, close pairs refined as in the
// one-sided body; pairs inside the group are a first, one-sided pass.
template <int ND>
__device__ __forceinline__ void direct_group_sym_helm(
    const PairCoef<float> &k, const double4 *__restrict__ gpos, const double4 *__restrict__ spos,
    const float *__restrict__ qs, const double *__restrict__ qcaller, const int4 G,
    const double4 c, const int2 *__restrict__ segs, const uint32_t *__restrict__ perm,
    float refine2, double fself_r, double fself_i, double *__restrict__ V,
    float4 *__restrict__ vsrc, float4 *th, float4 *tl, int lane) {
  const unsigned FULL = 0xffffffffu;
  const int ti = G.x + lane;
  const bool active = lane < G.y;
  float tx = 1e18f, ty = 1e18f, tz = 1e18f, tlx = 0.f, tly = 0.f, tlz = 0.f;
  float2 tq = make_float2(0.f, 0.f);
  long o = 0;
  if (active) {
    const double4 p = gpos[ti];
    o = perm[ti];
    const double dx = p.x - c.x, dy = p.y - c.y, dz = p.z - c.z;
    tx = (float)dx, ty = (float)dy, tz = (float)dz;
    tlx = (float)(dx - (double)tx), tly = (float)(dy - (double)ty), tlz = (float)(dz - (double)tz);
    tq = make_float2((float)qcaller[2 * o], (float)qcaller[2 * o + 1]);
  }
  th[lane] = make_float4(tx, ty, tz, tq.x);
  tl[lane] = make_float4(tlx, tly, tlz, tq.y);
  __syncwarp();
  const float R2 = k.R2;
  const unsigned rb = __float_as_uint(R2);
  double acc[4] = {0, 0, 0, 0}, acci[4] = {0, 0, 0, 0};

  // pairs inside the group, target side only, differences always refined
  {
    float2 Pv = make_float2(0.f, 0.f), Gx = Pv, Gy = Pv, Gz = Pv;
    for (int s = 0; s < G.y; s++) {
      const float4 S = th[s], L = tl[s];
      const float x = (tx - S.x) + (tlx - L.x), y = (ty - S.y) + (tly - L.y),
                  z = (tz - S.z) + (tlz - L.z);
      const float r2 = fmaf(x, x, fmaf(y, y, z * z));
      if (__float_as_uint(r2) - 1u < rb) {  // 0 < r^2 <= R2
        float2 F0, F1;
        helm_eval<ND>(k, r2, F0, F1);
        const float2 q = make_float2(S.w, L.w), g = cmul(F1, q);
        Pv = cfma(F0, q, Pv);
        Gx = __ffma2_rn(g, make_float2(x, x), Gx);
        Gy = __ffma2_rn(g, make_float2(y, y), Gy);
        Gz = __ffma2_rn(g, make_float2(z, z), Gz);
      }
    }
    acc[0] += Pv.x, acci[0] += Pv.y, acc[1] += Gx.x, acci[1] += Gx.y;
    acc[2] += Gy.x, acci[2] += Gy.y, acc[3] += Gz.x, acci[3] += Gz.y;
  }

  SrcCursor ca{G.z, lane};
  ca.normalize(segs, G.w);
  SrcCursor cb{ca.seg, ca.off + 32};
  cb.normalize(segs, G.w);
  bool va = ca.seg < G.w, vb = cb.seg < G.w;
  long ja = -1, jb = -1;
  double4 pa = make_double4(0, 0, 0, 0), pb = pa;
  float2 qa = make_float2(0.f, 0.f), qb = qa;
  if (va) ja = (long)segs[ca.seg].x + ca.off, pa = spos[ja], qa = make_float2(qs[2 * ja], qs[2 * ja + 1]);
  if (vb) jb = (long)segs[cb.seg].x + cb.off, pb = spos[jb], qb = make_float2(qs[2 * jb], qs[2 * jb + 1]);
  while (__any_sync(FULL, va)) {
    // this chunk's two sources of the lane; empty slots far away on the
    // other side from idle targets, with charge 0
    float sx[2] = {-1e18f, -1e18f}, sy[2] = {-1e18f, -1e18f}, sz[2] = {-1e18f, -1e18f};
    float lx[2] = {0.f, 0.f}, ly[2] = {0.f, 0.f}, lz[2] = {0.f, 0.f};
    float2 sq[2] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
    const long kidx[2] = {va ? (long)pa.w : -1, vb ? (long)pb.w : -1};  // brick positions
    if (va) {
      const double dx = pa.x - c.x, dy = pa.y - c.y, dz = pa.z - c.z;
      sx[0] = (float)dx, sy[0] = (float)dy, sz[0] = (float)dz;
      lx[0] = (float)(dx - (double)sx[0]), ly[0] = (float)(dy - (double)sy[0]);
      lz[0] = (float)(dz - (double)sz[0]);
      sq[0] = qa;
    }
    if (vb) {
      const double dx = pb.x - c.x, dy = pb.y - c.y, dz = pb.z - c.z;
      sx[1] = (float)dx, sy[1] = (float)dy, sz[1] = (float)dz;
      lx[1] = (float)(dx - (double)sx[1]), ly[1] = (float)(dy - (double)sy[1]);
      lz[1] = (float)(dz - (double)sz[1]);
      sq[1] = qb;
    }
    ca.off += 64;
    ca.normalize(segs, G.w);
    cb.off += 64;
    cb.normalize(segs, G.w);
    va = ca.seg < G.w, vb = cb.seg < G.w;
    if (va) ja = (long)segs[ca.seg].x + ca.off, pa = spos[ja], qa = make_float2(qs[2 * ja], qs[2 * ja + 1]);
    if (vb) jb = (long)segs[cb.seg].x + cb.off, pb = spos[jb], qb = make_float2(qs[2 * jb], qs[2 * jb + 1]);

    float2 Pv = make_float2(0.f, 0.f), Gx = Pv, Gy = Pv, Gz = Pv;  // target side, rotating
    float2 SV[2], SX[2], SY[2], SZ[2];                              // source side
#pragma unroll
    for (int u = 0; u < 2; u++) SV[u] = SX[u] = SY[u] = SZ[u] = make_float2(0.f, 0.f);
    const int src = (lane + 1) & 31;
    for (int kk = 0; kk < 32; kk++) {
      const int tt = (lane + kk) & 31;
      const float4 T = th[tt], L = tl[tt];
      float x[2], y[2], z[2], rr[2];
      bool hit[2];
#pragma unroll
      for (int u = 0; u < 2; u++) {
        x[u] = T.x - sx[u], y[u] = T.y - sy[u], z[u] = T.z - sz[u];
        float r2 = fmaf(x[u], x[u], fmaf(y[u], y[u], z[u] * z[u]));
        hit[u] = __float_as_uint(r2) - 1u < rb;
        if (hit[u] && r2 < refine2) {  // close pair: exact difference from head + residual
          x[u] += L.x - lx[u];
          y[u] += L.y - ly[u];
          z[u] += L.z - lz[u];
          r2 = fmaf(x[u], x[u], fmaf(y[u], y[u], z[u] * z[u]));
        }
        rr[u] = hit[u] ? r2 : R2;
      }
      if (__any_sync(FULL, hit[0] | hit[1])) {
        const float2 qt = make_float2(T.w, L.w);
#pragma unroll
        for (int u = 0; u < 2; u++) {
          float2 F0, F1;
          helm_eval<ND>(k, rr[u], F0, F1);
          const float2 qm = hit[u] ? sq[u] : make_float2(0.f, 0.f);
          const float2 qn = hit[u] ? qt : make_float2(0.f, 0.f);
          const float2 g = cmul(F1, qm), gs = cmul(F1, qn);
          Pv = cfma(F0, qm, Pv);
          Gx = __ffma2_rn(g, make_float2(x[u], x[u]), Gx);
          Gy = __ffma2_rn(g, make_float2(y[u], y[u]), Gy);
          Gz = __ffma2_rn(g, make_float2(z[u], z[u]), Gz);
          SV[u] = cfma(F0, qn, SV[u]);
          SX[u] = __ffma2_rn(gs, make_float2(-x[u], -x[u]), SX[u]);
          SY[u] = __ffma2_rn(gs, make_float2(-y[u], -y[u]), SY[u]);
          SZ[u] = __ffma2_rn(gs, make_float2(-z[u], -z[u]), SZ[u]);
        }
      }
      Pv.x = __shfl_sync(FULL, Pv.x, src), Pv.y = __shfl_sync(FULL, Pv.y, src);
      Gx.x = __shfl_sync(FULL, Gx.x, src), Gx.y = __shfl_sync(FULL, Gx.y, src);
      Gy.x = __shfl_sync(FULL, Gy.x, src), Gy.y = __shfl_sync(FULL, Gy.y, src);
      Gz.x = __shfl_sync(FULL, Gz.x, src), Gz.y = __shfl_sync(FULL, Gz.y, src);
    }
    acc[0] += Pv.x, acci[0] += Pv.y, acc[1] += Gx.x, acci[1] += Gx.y;
    acc[2] += Gy.x, acci[2] += Gy.y, acc[3] += Gz.x, acci[3] += Gz.y;
#pragma unroll
    for (int u = 0; u < 2; u++) {
      if (kidx[u] >= 0) {
        atomicAdd(vsrc + 2 * kidx[u], make_float4(SV[u].x, SV[u].y, SX[u].x, SX[u].y));
        atomicAdd(vsrc + 2 * kidx[u] + 1, make_float4(SY[u].x, SY[u].y, SZ[u].x, SZ[u].y));
      }
    }
  }
  if (active) {
    const double qr = qcaller[2 * o], qi = qcaller[2 * o + 1];
    acc[0] -= fself_r * qr - fself_i * qi;  // src/Interface.cpp:2909-2910
    acci[0] -= fself_r * qi + fself_i * qr;
    double2 *Vo = reinterpret_cast<double2 *>(V) + 4 * o;
#pragma unroll
    for (int m = 0; m < 4; m++) Vo[m] = make_double2(acc[m], acci[m]);
  }
}

// FP32 direct sum of one warp group (see direct.cu for the scheme): targets
// gpos[G.x, G.x + G.y) in group order, sources spos / qs (charges gathered
// into source order) over the segments [G.z, G.w); qcaller holds the
// caller-order charges for the self term.  sp and slo are this warp's
// 32-entry shared staging arrays.
template <bool CPLX, int FUNC, int SPLIT, int ND, class PK = BuiltinPair>
__device__ __forceinline__ void direct_group_body(
    const PairCoef<float> &k, const double4 *__restrict__ gpos, const double4 *__restrict__ spos,
    const float *__restrict__ qs, const double *__restrict__ qcaller, const int4 G,
    const double4 c, const int2 *__restrict__ segs, const uint32_t *__restrict__ perm,
    float refine2, double fself_r, double fself_i, double *__restrict__ V, float4 *sp,
    float4 *slo, int lane) {
#if !defined(NPME_SCALAR_DIRECT)
  if constexpr (!CPLX && SPLIT == 0 && std::is_same<PK, BuiltinPair>::value) {
    direct_group_packed<FUNC, ND>(k, gpos, spos, qs, qcaller, G, c, segs, perm, refine2, fself_r,
                                  V, sp, slo, lane);
    return;
  }
#endif
  const int ti = G.x + lane;
  const bool active = lane < G.y;
  // idle lanes sit far outside the cutoff
  float tx = 1e18f, ty = 1e18f, tz = 1e18f, tlx = 0.f, tly = 0.f, tlz = 0.f;
  if (active) {
    const double4 p = gpos[ti];
    const double dx = p.x - c.x, dy = p.y - c.y, dz = p.z - c.z;
    tx = (float)dx, ty = (float)dy, tz = (float)dz;
    tlx = (float)(dx - (double)tx), tly = (float)(dy - (double)ty), tlz = (float)(dz - (double)tz);
  }
  const float R2 = k.R2;
  double acc[4] = {0, 0, 0, 0}, acci[4] = {0, 0, 0, 0};

  // register prefetch of the next chunk: lane l holds source l of the chunk
  SrcCursor cur{G.z, lane};
  cur.normalize(segs, G.w);
  bool pv = cur.seg < G.w;
  double px = 0, py = 0, pz = 0;
  float pq = 0.f, pqi = 0.f;
#define NPME_PREFETCH                                          \
  if (pv) {                                                    \
    const long j_ = (long)segs[cur.seg].x + cur.off;           \
    const double4 p_ = spos[j_];                               \
    px = p_.x, py = p_.y, pz = p_.z;                           \
    if (CPLX) {                                                \
      pq = qs[2 * j_];                                         \
      pqi = qs[2 * j_ + 1];                                    \
    } else {                                                   \
      pq = qs[j_];                                             \
    }                                                          \
  }
  NPME_PREFETCH
  while (__any_sync(0xffffffffu, pv)) {
    const int cnt = __popc(__ballot_sync(0xffffffffu, pv));  // valid lanes form a prefix
    __syncwarp();
    if (pv) {
      const double dx = px - c.x, dy = py - c.y, dz = pz - c.z;
      const float hx = (float)dx, hy = (float)dy, hz = (float)dz;
      sp[lane] = make_float4(hx, hy, hz, pq);
      slo[lane] = make_float4((float)(dx - (double)hx), (float)(dy - (double)hy),
                              (float)(dz - (double)hz), pqi);
    }
    __syncwarp();
    cur.off += 32;
    cur.normalize(segs, G.w);
    pv = cur.seg < G.w;
    NPME_PREFETCH
    float p0 = 0, p1 = 0, p2 = 0, p3 = 0, p0i = 0, p1i = 0, p2i = 0, p3i = 0;
#if !defined(NPME_SCALAR_DIRECT)
    if constexpr (CPLX && SPLIT == 0 && std::is_same<PK, BuiltinPair>::value) {
      float2 Pv = make_float2(0.f, 0.f), Gx = Pv, Gy = Pv, Gz = Pv;
      helmholtz_steps<ND>(k, sp, slo, cnt, tx, ty, tz, tlx, tly, tlz, refine2, Pv, Gx, Gy, Gz);
      p0 = Pv.x, p0i = Pv.y, p1 = Gx.x, p1i = Gx.y, p2 = Gy.x, p2i = Gy.y, p3 = Gz.x, p3i = Gz.y;
    } else
#endif
#pragma unroll kDirectUnroll
    for (int s = 0; s < cnt; s++) {
      const float4 src = sp[s];
      float x = tx - src.x, y = ty - src.y, z = tz - src.z;
      float r2 = fmaf(x, x, fmaf(y, y, z * z));
      if (r2 <= R2 && r2 > 0.f) {
        if (r2 < refine2) {  // close pair: exact difference from head + residual
          const float4 lo = slo[s];
          x += tlx - lo.x;
          y += tly - lo.y;
          z += tlz - lo.z;
          r2 = fmaf(x, x, fmaf(y, y, z * z));
        }
        if (!CPLX) {
          float f1;
          const float f0 = pair_sr<float, FUNC, SPLIT, ND, PK>(k, r2, f1);
          const float gq = f1 * src.w;
          p0 = fmaf(f0, src.w, p0);
          p1 = fmaf(gq, x, p1);
          p2 = fmaf(gq, y, p2);
          p3 = fmaf(gq, z, p3);
        } else {
          float f0r, f0i, f1r, f1i;
          pair_sr_cplx<float, ND, PK>(k, r2, f0r, f0i, f1r, f1i);
          const float qr = src.w, qi = slo[s].w;
          p0 = fmaf(f0r, qr, fmaf(-f0i, qi, p0));
          p0i = fmaf(f0r, qi, fmaf(f0i, qr, p0i));
          const float gr = f1r * qr - f1i * qi, gi = f1r * qi + f1i * qr;
          p1 = fmaf(gr, x, p1);
          p2 = fmaf(gr, y, p2);
          p3 = fmaf(gr, z, p3);
          p1i = fmaf(gi, x, p1i);
          p2i = fmaf(gi, y, p2i);
          p3i = fmaf(gi, z, p3i);
        }
      }
    }
    acc[0] += p0, acc[1] += p1, acc[2] += p2, acc[3] += p3;
    if (CPLX) acci[0] += p0i, acci[1] += p1i, acci[2] += p2i, acci[3] += p3i;
  }
#undef NPME_PREFETCH
  if (active) {
    const long o = perm[ti];
    if (CPLX) {
      const double qr = qcaller[2 * o], qi = qcaller[2 * o + 1];
      acc[0] -= fself_r * qr - fself_i * qi;  // src/Interface.cpp:2909-2910
      acci[0] -= fself_r * qi + fself_i * qr;
      double2 *Vo = reinterpret_cast<double2 *>(V) + 4 * o;
#pragma unroll
      for (int m = 0; m < 4; m++) Vo[m] = make_double2(acc[m], acci[m]);
    } else {
      acc[0] -= fself_r * qcaller[o];  // src/Interface.cpp:2061-2062
      reinterpret_cast<double4 *>(V)[o] = make_double4(acc[0], acc[1], acc[2], acc[3]);
    }
  }
}

// FP64 direct sum of one warp group (the plain precision): the same groups
// and source segments as the FP32 body, every difference and pair kernel in
// double, no head/residual split needed.  sp holds 32 (x, y, z, Re q)
// entries relative to the group centre, sqi the imaginary parts.
template <bool CPLX, int FUNC, int SPLIT, int ND, class PK = BuiltinPair>
__device__ __forceinline__ void direct_group_fp64(
    const PairCoef<double> &k, const double4 *__restrict__ gpos,
    const double4 *__restrict__ spos, const double *__restrict__ qs,
    const double *__restrict__ qcaller, const int4 G, const double4 c,
    const int2 *__restrict__ segs, const uint32_t *__restrict__ perm, double fself_r,
    double fself_i, double *__restrict__ V, double4 *sp, double *sqi, int lane) {
  const int ti = G.x + lane;
  const bool active = lane < G.y;
  double tx = 1e150, ty = 1e150, tz = 1e150;  // idle lanes sit far outside the cutoff
  if (active) {
    const double4 p = gpos[ti];
    tx = p.x - c.x, ty = p.y - c.y, tz = p.z - c.z;
  }
  const double R2 = k.R2;
  double acc[4] = {0, 0, 0, 0}, acci[4] = {0, 0, 0, 0};
  SrcCursor cur{G.z, lane};
  cur.normalize(segs, G.w);
  bool pv = cur.seg < G.w;
  double4 pp = make_double4(0, 0, 0, 0);
  double pqi = 0;
#define NPME_PREFETCH64                                     \
  if (pv) {                                                 \
    const long j_ = (long)segs[cur.seg].x + cur.off;        \
    const double4 p_ = spos[j_];                            \
    pp = make_double4(p_.x - c.x, p_.y - c.y, p_.z - c.z,   \
                      CPLX ? qs[2 * j_] : qs[j_]);          \
    if (CPLX) pqi = qs[2 * j_ + 1];                         \
  }
  NPME_PREFETCH64
  while (__any_sync(0xffffffffu, pv)) {
    const int cnt = __popc(__ballot_sync(0xffffffffu, pv));  // valid lanes form a prefix
    __syncwarp();
    if (pv) {
      sp[lane] = pp;
      if (CPLX) sqi[lane] = pqi;
    }
    __syncwarp();
    cur.off += 32;
    cur.normalize(segs, G.w);
    pv = cur.seg < G.w;
    NPME_PREFETCH64
#pragma unroll 4
    for (int s = 0; s < cnt; s++) {
      const double4 src = sp[s];
      const double x = tx - src.x, y = ty - src.y, z = tz - src.z;
      const double r2 = fma(x, x, fma(y, y, z * z));
      if (r2 <= R2 && r2 > 0.0) {
        if (!CPLX) {
          double f1;
          const double f0 = pair_sr<double, FUNC, SPLIT, ND, PK>(k, r2, f1);
          const double gq = f1 * src.w;
          acc[0] = fma(f0, src.w, acc[0]);
          acc[1] = fma(gq, x, acc[1]);
          acc[2] = fma(gq, y, acc[2]);
          acc[3] = fma(gq, z, acc[3]);
        } else {
          double f0r, f0i, f1r, f1i;
          pair_sr_cplx<double, ND, PK>(k, r2, f0r, f0i, f1r, f1i);
          const double qr = src.w, qi = sqi[s];
          acc[0] = fma(f0r, qr, fma(-f0i, qi, acc[0]));
          acci[0] = fma(f0r, qi, fma(f0i, qr, acci[0]));
          const double gr = f1r * qr - f1i * qi, gi = f1r * qi + f1i * qr;
          acc[1] = fma(gr, x, acc[1]);
          acc[2] = fma(gr, y, acc[2]);
          acc[3] = fma(gr, z, acc[3]);
          acci[1] = fma(gi, x, acci[1]);
          acci[2] = fma(gi, y, acci[2]);
          acci[3] = fma(gi, z, acci[3]);
        }
      }
    }
  }
#undef NPME_PREFETCH64
  if (active) {
    const long o = perm[ti];
    if (CPLX) {
      const double qr = qcaller[2 * o], qi = qcaller[2 * o + 1];
      acc[0] -= fself_r * qr - fself_i * qi;  // src/Interface.cpp:2909-2910
      acci[0] -= fself_r * qi + fself_i * qr;
      double2 *Vo = reinterpret_cast<double2 *>(V) + 4 * o;
#pragma unroll
      for (int m = 0; m < 4; m++) Vo[m] = make_double2(acc[m], acci[m]);
    } else {
      acc[0] -= fself_r * qcaller[o];  // src/Interface.cpp:2061-2062
      reinterpret_cast<double4 *>(V)[o] = make_double4(acc[0], acc[1], acc[2], acc[3]);
    }
  }
}

// FP32 direct sum of one warp group with every unordered pair evaluated once,
// for the real kernels without a packed body (the original Ewald split and
// caller-defined kernels): the pair-once walk of direct_group_sym with the
// scalar pair kernel (pair_sr) of the one-sided body.  Coordinates are
// unscaled FP32 offsets from the group centre (heads in th with the target
// charge, residuals in tl), close pairs refined from the residuals; the
// source-side sums go to vsrc as the gradient itself (merge scale 1).
template <int FUNC, int SPLIT, int ND, class PK = BuiltinPair>
__device__ __forceinline__ void direct_group_sym_scalar(
    const PairCoef<float> &k, const double4 *__restrict__ gpos, const double4 *__restrict__ spos,
    const float *__restrict__ qs, const double *__restrict__ qcaller, const int4 G,
    const double4 c, const int2 *__restrict__ segs, const uint32_t *__restrict__ perm,
    float refine2, double fself_r, double *__restrict__ V, float4 *__restrict__ vsrc,
    float4 *th, float4 *tl, int lane) {
  const unsigned FULL = 0xffffffffu;
  const int ti = G.x + lane;
  const bool active = lane < G.y;
  float tx = 1e18f, ty = 1e18f, tz = 1e18f, tlx = 0.f, tly = 0.f, tlz = 0.f, tq = 0.f;
  long o = 0;
  if (active) {
    const double4 p = gpos[ti];
    o = perm[ti];
    const double dx = p.x - c.x, dy = p.y - c.y, dz = p.z - c.z;
    tx = (float)dx, ty = (float)dy, tz = (float)dz;
    tlx = (float)(dx - (double)tx), tly = (float)(dy - (double)ty), tlz = (float)(dz - (double)tz);
    tq = (float)qcaller[o];
  }
  th[lane] = make_float4(tx, ty, tz, tq);
  tl[lane] = make_float4(tlx, tly, tlz, 0.f);
  __syncwarp();
  const float R2 = k.R2;
  double acc[4] = {0, 0, 0, 0};
  {  // pairs inside the group, target side only, differences always refined
    float aV = 0.f, aX = 0.f, aY = 0.f, aZ = 0.f;
    for (int s = 0; s < G.y; s++) {
      const float4 S = th[s], L = tl[s];
      const float x = (tx - S.x) + (tlx - L.x), y = (ty - S.y) + (tly - L.y),
                  z = (tz - S.z) + (tlz - L.z);
      const float r2 = fmaf(x, x, fmaf(y, y, z * z));
      if (r2 <= R2 && r2 > 0.f) {
        float f1;
        const float f0 = pair_sr<float, FUNC, SPLIT, ND, PK>(k, r2, f1);
        const float g = f1 * S.w;
        aV = fmaf(f0, S.w, aV);
        aX = fmaf(g, x, aX);
        aY = fmaf(g, y, aY);
        aZ = fmaf(g, z, aZ);
      }
    }
    acc[0] += aV, acc[1] += aX, acc[2] += aY, acc[3] += aZ;
  }
  SrcCursor ca{G.z, lane};
  ca.normalize(segs, G.w);
  SrcCursor cb{ca.seg, ca.off + 32};
  cb.normalize(segs, G.w);
  bool va = ca.seg < G.w, vb = cb.seg < G.w;
  long ja = -1, jb = -1;
  double4 pa = make_double4(0, 0, 0, 0), pb = pa;
  float qa = 0.f, qb = 0.f;
  if (va) ja = (long)segs[ca.seg].x + ca.off, pa = spos[ja], qa = qs[ja];
  if (vb) jb = (long)segs[cb.seg].x + cb.off, pb = spos[jb], qb = qs[jb];
  while (__any_sync(FULL, va)) {
    // the lane's two sources; empty slots far away on the other side from
    // idle targets, with charge 0
    float sx[2] = {-1e18f, -1e18f}, sy[2] = {-1e18f, -1e18f}, sz[2] = {-1e18f, -1e18f};
    float lx[2] = {0.f, 0.f}, ly[2] = {0.f, 0.f}, lz[2] = {0.f, 0.f}, sq[2] = {0.f, 0.f};
    const long kidx[2] = {va ? (long)pa.w : -1, vb ? (long)pb.w : -1};  // brick positions
    if (va) {
      const double dx = pa.x - c.x, dy = pa.y - c.y, dz = pa.z - c.z;
      sx[0] = (float)dx, sy[0] = (float)dy, sz[0] = (float)dz;
      lx[0] = (float)(dx - (double)sx[0]), ly[0] = (float)(dy - (double)sy[0]);
      lz[0] = (float)(dz - (double)sz[0]);
      sq[0] = qa;
    }
    if (vb) {
      const double dx = pb.x - c.x, dy = pb.y - c.y, dz = pb.z - c.z;
      sx[1] = (float)dx, sy[1] = (float)dy, sz[1] = (float)dz;
      lx[1] = (float)(dx - (double)sx[1]), ly[1] = (float)(dy - (double)sy[1]);
      lz[1] = (float)(dz - (double)sz[1]);
      sq[1] = qb;
    }
    ca.off += 64;
    ca.normalize(segs, G.w);
    cb.off += 64;
    cb.normalize(segs, G.w);
    va = ca.seg < G.w, vb = cb.seg < G.w;
    if (va) ja = (long)segs[ca.seg].x + ca.off, pa = spos[ja], qa = qs[ja];
    if (vb) jb = (long)segs[cb.seg].x + cb.off, pb = spos[jb], qb = qs[jb];

    float aV = 0.f, aX = 0.f, aY = 0.f, aZ = 0.f;  // target side, rotating
    float S[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};  // source side
    const int src = (lane + 1) & 31;
    for (int kk = 0; kk < 32; kk++) {
      const int tt = (lane + kk) & 31;
      const float4 T = th[tt];
#pragma unroll
      for (int u = 0; u < 2; u++) {
        float x = T.x - sx[u], y = T.y - sy[u], z = T.z - sz[u];
        float r2 = fmaf(x, x, fmaf(y, y, z * z));
        if (r2 <= R2 && r2 > 0.f) {
          if (r2 < refine2) {  // close pair: exact difference from head + residual
            const float4 L = tl[tt];
            x += L.x - lx[u];
            y += L.y - ly[u];
            z += L.z - lz[u];
            r2 = fmaf(x, x, fmaf(y, y, z * z));
          }
          float f1;
          const float f0 = pair_sr<float, FUNC, SPLIT, ND, PK>(k, r2, f1);
          const float g = f1 * sq[u], gs = f1 * T.w;
          aV = fmaf(f0, sq[u], aV);
          aX = fmaf(g, x, aX);
          aY = fmaf(g, y, aY);
          aZ = fmaf(g, z, aZ);
          S[u][0] = fmaf(f0, T.w, S[u][0]);
          S[u][1] = fmaf(-gs, x, S[u][1]);
          S[u][2] = fmaf(-gs, y, S[u][2]);
          S[u][3] = fmaf(-gs, z, S[u][3]);
        }
      }
      aV = __shfl_sync(FULL, aV, src);
      aX = __shfl_sync(FULL, aX, src);
      aY = __shfl_sync(FULL, aY, src);
      aZ = __shfl_sync(FULL, aZ, src);
    }
    acc[0] += aV, acc[1] += aX, acc[2] += aY, acc[3] += aZ;
#pragma unroll
    for (int u = 0; u < 2; u++)
      if (kidx[u] >= 0) atomicAdd(vsrc + kidx[u], make_float4(S[u][0], S[u][1], S[u][2], S[u][3]));
  }
  if (active) {
    acc[0] -= fself_r * qcaller[o];  // src/Interface.cpp:2061-2062
    reinterpret_cast<double4 *>(V)[o] = make_double4(acc[0], acc[1], acc[2], acc[3]);
  }
}

// FP64 direct sum of one warp group with every unordered pair evaluated once
// (the FP64 counterpart of direct_group_sym, for the real kernels): the
// group's targets (x, y, z, q) sit in shared memory, each lane holds two
// sources of a 64-source chunk of the half-shell segments, target (l + k)
// mod 32 meets lane l at step k and its sums rotate one lane down per step;
// the source-side sums of a chunk go to vsrc ([n][4] doubles, slot = the
// source's brick-order position) with one FP64 atomic per component.  Pairs inside the group are a first,
// one-sided pass.  Same pair arithmetic as direct_group_fp64.
template <int FUNC, int SPLIT, int ND, class PK = BuiltinPair>
__device__ __forceinline__ void direct_group_sym64(
    const PairCoef<double> &k, const double4 *__restrict__ gpos,
    const double4 *__restrict__ spos, const double *__restrict__ qs,
    const double *__restrict__ qcaller, const int4 G, const double4 c,
    const int2 *__restrict__ segs, const uint32_t *__restrict__ perm, double fself_r,
    double *__restrict__ V, double *__restrict__ vsrc, double4 *tsm, int lane) {
  const unsigned FULL = 0xffffffffu;
  const int ti = G.x + lane;
  const bool active = lane < G.y;
  double tx = 1e150, ty = 1e150, tz = 1e150, tq = 0.0;  // idle lanes: far away, no charge
  long o = 0;
  if (active) {
    const double4 p = gpos[ti];
    o = perm[ti];
    tx = p.x - c.x, ty = p.y - c.y, tz = p.z - c.z;
    tq = qcaller[o];
  }
  tsm[lane] = make_double4(tx, ty, tz, tq);
  __syncwarp();
  const double R2 = k.R2;
  double acc[4] = {0, 0, 0, 0};
  // pairs inside the group, target side only (each is met from both ends)
  for (int s = 0; s < G.y; s++) {
    const double4 S = tsm[s];
    const double x = tx - S.x, y = ty - S.y, z = tz - S.z;
    const double r2 = fma(x, x, fma(y, y, z * z));
    if (r2 <= R2 && r2 > 0.0) {
      double f1;
      const double f0 = pair_sr<double, FUNC, SPLIT, ND, PK>(k, r2, f1);
      const double gq = f1 * S.w;
      acc[0] = fma(f0, S.w, acc[0]);
      acc[1] = fma(gq, x, acc[1]);
      acc[2] = fma(gq, y, acc[2]);
      acc[3] = fma(gq, z, acc[3]);
    }
  }
  // half-shell segments in chunks of 64 sources (register prefetch)
  SrcCursor ca{G.z, lane};
  ca.normalize(segs, G.w);
  SrcCursor cb{ca.seg, ca.off + 32};
  cb.normalize(segs, G.w);
  bool va = ca.seg < G.w, vb = cb.seg < G.w;
  long ja = -1, jb = -1, sla = -1, slb = -1;  // sla, slb: source-side slots (brick positions)
  double4 pa = make_double4(0, 0, 0, 0), pb = pa;
  if (va) ja = (long)segs[ca.seg].x + ca.off, pa = spos[ja], sla = (long)pa.w, pa.w = qs[ja];
  if (vb) jb = (long)segs[cb.seg].x + cb.off, pb = spos[jb], slb = (long)pb.w, pb.w = qs[jb];
  while (__any_sync(FULL, va)) {
    // empty slots far away on the other side from idle targets, no charge
    double4 A = make_double4(-1e150, -1e150, -1e150, 0.0), B = A;
    if (va) A = make_double4(pa.x - c.x, pa.y - c.y, pa.z - c.z, pa.w);
    if (vb) B = make_double4(pb.x - c.x, pb.y - c.y, pb.z - c.z, pb.w);
    const long ka = va ? sla : -1, kb = vb ? slb : -1;
    ca.off += 64;
    ca.normalize(segs, G.w);
    cb.off += 64;
    cb.normalize(segs, G.w);
    va = ca.seg < G.w, vb = cb.seg < G.w;
    if (va) ja = (long)segs[ca.seg].x + ca.off, pa = spos[ja], sla = (long)pa.w, pa.w = qs[ja];
    if (vb) jb = (long)segs[cb.seg].x + cb.off, pb = spos[jb], slb = (long)pb.w, pb.w = qs[jb];

    double aV = 0, aX = 0, aY = 0, aZ = 0;           // target side, rotating
    double sa[4] = {0, 0, 0, 0}, sb[4] = {0, 0, 0, 0};  // source side
    const int src = (lane + 1) & 31;
#pragma unroll 2
    for (int kk = 0; kk < 32; kk++) {
      const double4 T = tsm[(lane + kk) & 31];
      {
        const double x = T.x - A.x, y = T.y - A.y, z = T.z - A.z;
        const double r2 = fma(x, x, fma(y, y, z * z));
        if (r2 <= R2 && r2 > 0.0) {
          double f1;
          const double f0 = pair_sr<double, FUNC, SPLIT, ND, PK>(k, r2, f1);
          const double gq = f1 * A.w, gs = f1 * T.w;
          aV = fma(f0, A.w, aV);
          aX = fma(gq, x, aX);
          aY = fma(gq, y, aY);
          aZ = fma(gq, z, aZ);
          sa[0] = fma(f0, T.w, sa[0]);
          sa[1] = fma(-gs, x, sa[1]);
          sa[2] = fma(-gs, y, sa[2]);
          sa[3] = fma(-gs, z, sa[3]);
        }
      }
      {
        const double x = T.x - B.x, y = T.y - B.y, z = T.z - B.z;
        const double r2 = fma(x, x, fma(y, y, z * z));
        if (r2 <= R2 && r2 > 0.0) {
          double f1;
          const double f0 = pair_sr<double, FUNC, SPLIT, ND, PK>(k, r2, f1);
          const double gq = f1 * B.w, gs = f1 * T.w;
          aV = fma(f0, B.w, aV);
          aX = fma(gq, x, aX);
          aY = fma(gq, y, aY);
          aZ = fma(gq, z, aZ);
          sb[0] = fma(f0, T.w, sb[0]);
          sb[1] = fma(-gs, x, sb[1]);
          sb[2] = fma(-gs, y, sb[2]);
          sb[3] = fma(-gs, z, sb[3]);
        }
      }
      aV = __shfl_sync(FULL, aV, src);
      aX = __shfl_sync(FULL, aX, src);
      aY = __shfl_sync(FULL, aY, src);
      aZ = __shfl_sync(FULL, aZ, src);
    }
    acc[0] += aV;
    acc[1] += aX;
    acc[2] += aY;
    acc[3] += aZ;
    if (ka >= 0)
#pragma unroll
      for (int m = 0; m < 4; m++) atomicAdd(vsrc + 4 * ka + m, sa[m]);
    if (kb >= 0)
#pragma unroll
      for (int m = 0; m < 4; m++) atomicAdd(vsrc + 4 * kb + m, sb[m]);
  }
  if (active) {
    acc[0] -= fself_r * qcaller[o];  // src/Interface.cpp:2061-2062
    reinterpret_cast<double4 *>(V)[o] = make_double4(acc[0], acc[1], acc[2], acc[3]);
  }
}

}  // namespace npme
