// Per-geometry set-up on the device: everything CalcV needs that depends on
// the point positions, built from the caller's coordinates in HBM.
//
//  * bounding box and coordinate check (one reduction, read back by the host,
//    which derives the PME box, src/RecSumSupportFunctions.cpp:182-201,
//    276-296);
//  * brick order of the spreading and interpolation (src/RecSumQ.cpp:527-895,
//    NPME_RecSumQ_CreateBlock): each point's stencil origin and fractional
//    offset (src/RecSumSupportFunctions.h:123-151), points sorted by brick
//    and, inside a brick, by the shared-memory bank of their stencil origin;
//  * the direct sum's warp groups (the reference's cells and cluster pairs,
//    src/PartitionEmbeddedBox.cpp:47-205, src/PartitionBox.cpp:789-923):
//    targets sorted by (xy column, quantised z, index) and cut into runs of
//    32, sources sorted by (fine xy column, quantised z, index); for every group the z
//    ranges of the fine columns that can hold a point within Rdir of the
//    group's bounding box, and the half-shell part of them for the
//    every-pair-once walk; groups ordered by their work, heaviest first.
//
// Sorting is done with stable radix sorts (values = point indices in
// increasing order), so every order is (key, index) lexicographic and the
// result does not depend on timing.  Work per point or per group is a
// thread or a warp; the host reads back four small records (box, group
// count, segment counts) and sizes the buffers from them.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include "internal.h"

namespace npme {
namespace {

constexpr int kSourceSplit = 2;  // fine source columns per coarse column edge
constexpr long kHostBoxPoints = 1L << 15;  // below: bounding box on the host
// direct-sum groups of about one wave (148 SMs, about 4 resident CTAs each)
constexpr long kOneWaveGroups = 148 * 4 * kGroupWarps;

// Order-preserving 64-bit key of a double (total order of the finite values).
__device__ __forceinline__ unsigned long long dkey(double x) {
  const unsigned long long u = (unsigned long long)__double_as_longlong(x);
  return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}
inline double dkey_inv(unsigned long long k) {
  const unsigned long long u = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  double x;
  std::memcpy(&x, &u, sizeof(x));
  return x;
}

// Results the host reads back.
struct SetupStats {
  unsigned long long mn[3], mx[3];  // dkey of the per-axis minimum / maximum
  unsigned int nonfinite;
  unsigned int pad;
  long long bad;                    // lowest index whose stencil leaves the octant
  unsigned long long cand, hcand;   // staged (target, source) candidates, both walks
};

__global__ void init_stats_kernel(SetupStats *st, long long n) {
  for (int d = 0; d < 3; d++) st->mn[d] = ~0ull, st->mx[d] = 0ull;
  st->nonfinite = 0;
  st->bad = n;
  st->cand = st->hcand = 0;
}

__global__ void bbox_kernel(const double *__restrict__ coord, long n, SetupStats *st) {
  unsigned long long lo[3] = {~0ull, ~0ull, ~0ull}, hi[3] = {0ull, 0ull, 0ull};
  unsigned bad = 0;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const double x = coord[3 * i + d];
      if (!isfinite(x)) {
        bad = 1;
        continue;
      }
      const unsigned long long k = dkey(x);
      lo[d] = min(lo[d], k);
      hi[d] = max(hi[d], k);
    }
  }
  const unsigned FULL = 0xffffffffu;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int d = 0; d < 3; d++) {
      lo[d] = min(lo[d], __shfl_xor_sync(FULL, lo[d], o));
      hi[d] = max(hi[d], __shfl_xor_sync(FULL, hi[d], o));
    }
    bad |= __shfl_xor_sync(FULL, bad, o);
  }
  if ((threadIdx.x & 31) == 0) {
    for (int d = 0; d < 3; d++) {
      atomicMin(&st->mn[d], lo[d]);
      atomicMax(&st->mx[d], hi[d]);
    }
    if (bad) atomicOr(&st->nonfinite, 1u);
  }
}

// Geometry the binning kernel needs (host-computed from the box).
struct BinGeom {
  double N[3], L[3], R[3];
  long Nl[3], H[3], nb[3];
  int P, TL, nkeys;
  // direct-sum columns
  double mn[2], edge[2], sedge[2];
  int nc[2], ns[2];
  // quantised z: floor((z - zmin) * zscale) in [0, 2^zbits)
  double zmin, zscale;
  int zbits;
};

// z quantised to zbits bits (a quantum of at most 1/1024 of the column edge),
// non-decreasing in z.  The direct sum's two point orders sort by (column,
// quantised z, index); the source segments are searched with the same
// quantisation, widened to whole quanta, so a segment is a superset of the
// sources within reach (the pair test rejects the few extra) and no pair is
// lost.
__device__ __forceinline__ unsigned zquant(double z, double zmin, double zscale, int zbits) {
  const double t = __dmul_rn(__dsub_rn(z, zmin), zscale);
  if (!(t > 0.0)) return 0u;
  const double mx = (double)((1u << zbits) - 1u);
  return (unsigned)floor(fmin(t, mx));
}

// start index of the B-spline stencil (src/RecSumSupportFunctions.h:123-127)
__device__ __forceinline__ long stencil_start(double w) {
  return w < 0 ? (long)(-w) + 1 : (long)(-w);
}

// Per point: the spread/interpolation record, its brick-and-bank sort key,
// its (coarse column, quantised z) and (fine column, quantised z) sort keys;
// per brick and column the point counts.  Arithmetic as the host restatement of the reference
// (explicit round-to-nearest operations, no contraction), so that every
// point lands in the same brick, bank and column on any machine.
template <typename T>
__device__ __forceinline__ void bin_point(const double *__restrict__ coord, long i, BinGeom g,
                           BrickPoint<T> *__restrict__ pts, unsigned *__restrict__ bkey,
                           unsigned long long *__restrict__ ckey,
                           unsigned long long *__restrict__ skey, unsigned *__restrict__ iota,
                           int *__restrict__ bcount, int *__restrict__ ccount,
                           int *__restrict__ scount, SetupStats *st) {
  const double x[3] = {coord[3 * i], coord[3 * i + 1], coord[3 * i + 2]};
  long o[3];
  T u[3];
  bool out = false;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const double w = __dmul_rn(__ddiv_rn(g.N[d], g.L[d]), __dsub_rn(x[d], g.R[d]));
    const long ms = stencil_start(w);
    o[d] = ms + g.Nl[d] / 4;
    if (o[d] < 0 || o[d] + g.P - 1 > g.H[d] - 1) out = true;
    u[d] = (T)__dadd_rn(w, (double)ms);
  }
  if (out) {
    atomicMin(&st->bad, (long long)i);
    o[0] = o[1] = o[2] = 0;  // any in-range brick: the set-up fails anyway
  }
  const long b1 = o[0] / kBrick, b2 = o[1] / kBrick, b3 = o[2] / kBrick;
  const long bid = (b1 * g.nb[1] + b2) * g.nb[2] + b3;
  const long l1 = o[0] - b1 * kBrick, l2 = o[1] - b2 * kBrick, l3 = o[2] - b3 * kBrick;
  const unsigned key = (unsigned)(((l1 * g.TL + l2) * g.TL + l3) % g.nkeys);
  BrickPoint<T> bp;
  bp.u[0] = u[0], bp.u[1] = u[1], bp.u[2] = u[2];
  bp.g0 = ((uint32_t)o[0] << 20) | ((uint32_t)o[1] << 10) | (uint32_t)o[2];
  bp.orig = (uint32_t)i;
  pts[i] = bp;
  bkey[i] = ((unsigned)bid << 5) | key;
  if (!out) atomicAdd(&bcount[bid], 1);
  int cs[2], ss[2];
#pragma unroll
  for (int d = 0; d < 2; d++) {
    const double v = __dsub_rn(x[d], g.mn[d]);
    cs[d] = min(g.nc[d] - 1, max(0, (int)__ddiv_rn(v, g.edge[d])));
    const double r = __dsub_rn(v, __dmul_rn((double)cs[d], g.edge[d]));
    ss[d] = cs[d] * kSourceSplit +
            min(kSourceSplit - 1, max(0, (int)__ddiv_rn(r, g.sedge[d])));
  }
  const unsigned cc = (unsigned)(cs[0] * g.nc[1] + cs[1]);
  const unsigned sc = (unsigned)(ss[0] * g.ns[1] + ss[1]);
  const unsigned long long zq = zquant(x[2], g.zmin, g.zscale, g.zbits);
  ckey[i] = ((unsigned long long)cc << g.zbits) | zq;
  skey[i] = ((unsigned long long)sc << g.zbits) | zq;
  atomicAdd(&ccount[cc], 1);
  atomicAdd(&scount[sc], 1);
  iota[i] = (unsigned)i;
}

template <typename T>
__global__ void bin_kernel(const double *__restrict__ coord, long n, BinGeom g,
                           BrickPoint<T> *__restrict__ pts, unsigned *__restrict__ bkey,
                           unsigned long long *__restrict__ ckey,
                           unsigned long long *__restrict__ skey, unsigned *__restrict__ iota,
                           int *__restrict__ bcount, int *__restrict__ ccount,
                           int *__restrict__ scount, SetupStats *st) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) bin_point<T>(coord, i, g, pts, bkey, ckey, skey, iota, bcount, ccount, scount, st);
}

template <typename T>
__global__ void gather_bpts_kernel(const BrickPoint<T> *__restrict__ pts,
                                   const unsigned *__restrict__ perm, long n,
                                   BrickPoint<T> *__restrict__ out) {
  const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) out[k] = pts[perm[k]];
}

// Round-robin key (brick, rank inside its bank, bank), the rank in rbits
// bits: sorting by it puts the r-th point of every bank of a brick into
// round r.  The rank is the distance to the first equal key of the sorted
// (brick, bank) keys, found by binary search.
template <typename K>
__global__ void round_key_kernel(const unsigned *__restrict__ key, long n, int rbits,
                                 K *__restrict__ rkey) {
  const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const unsigned kk = key[k];
  long lo = 0, hi = k;  // first position with key == kk in [0, k]
  while (lo < hi) {
    const long m = (lo + hi) >> 1;
    if (key[m] < kk) lo = m + 1;
    else hi = m;
  }
  rkey[k] = ((K)(kk >> 5) << (rbits + 5)) | ((K)(k - lo) << 5) | (K)(kk & 31u);
}

__global__ void gather_u32_kernel(const unsigned *__restrict__ src,
                                  const unsigned *__restrict__ perm, long n,
                                  unsigned *__restrict__ out) {
  const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) out[k] = src[perm[k]];
}

// flag[b] = 1 for non-empty bricks (flag[nb] = 0)
__global__ void nonempty_flags_kernel(const int *__restrict__ count, long nb,
                                      int *__restrict__ flag) {
  const long b = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (b <= nb) flag[b] = b < nb && count[b] > 0;
}

__global__ void brick_list_kernel(const int *__restrict__ count, const int *__restrict__ pos,
                                  long nb, int *__restrict__ list) {
  const long b = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (b < nb && count[b] > 0) list[pos[b]] = (int)b;
}

// zq[k] = quantised z of source k (from its sorted key); cpos[cperm[k]] = k
// (position of a point in the group order)
__global__ void source_z_kernel(const unsigned long long *__restrict__ skey,
                                const unsigned *__restrict__ cperm, long n, int zbits,
                                unsigned *__restrict__ zq, unsigned *__restrict__ cpos) {
  const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  zq[k] = (unsigned)(skey[k] & ((1ull << zbits) - 1ull));
  cpos[cperm[k]] = (unsigned)k;
}

// inverse of the brick order: bpos[caller index] = brick-order position
__global__ void brick_position_kernel(const uint32_t *__restrict__ bperm, long n,
                                      unsigned *__restrict__ bpos) {
  const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) bpos[bperm[k]] = (unsigned)k;
}

// FP64 positions in the target (group) and source orders; a source's w holds
// its brick-order position, the slot of its source-side sums
__global__ void gather_positions_kernel(const double *__restrict__ coord,
                                        const uint32_t *__restrict__ gorder,
                                        const uint32_t *__restrict__ sorder,
                                        const unsigned *__restrict__ bpos, long n,
                                        double4 *__restrict__ gpos, double4 *__restrict__ spos) {
  const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const double *x = coord + 3 * (long)gorder[k];
  gpos[k] = make_double4(x[0], x[1], x[2], 0.0);
  const unsigned j = sorder[k];
  const double *y = coord + 3 * (long)j;
  spos[k] = make_double4(y[0], y[1], y[2], (double)bpos[j]);
}

// groups per coarse column: ceil(count / 32) (entry ncol = 0)
__global__ void groups_per_column_kernel(const int *__restrict__ ccount, long ncol,
                                         int *__restrict__ gcount) {
  const long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c <= ncol) gcount[c] = c < ncol ? (ccount[c] + 31) / 32 : 0;
}

// group g of column c: points [p0, p1) of the group order
__global__ void group_records_kernel(const int *__restrict__ cstart, const int *__restrict__ goff,
                                     long ncol, int4 *__restrict__ grec) {
  const long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncol) return;
  const int p_end = cstart[c + 1];
  int g = goff[c];
  for (int p0 = cstart[c]; p0 < p_end; p0 += 32, g++)
    grec[g] = make_int4(p0, min(p0 + 32, p_end), (int)c, 0);
}

struct GroupGeom {
  double R, R2;
  double mn[2], sedge[2];
  int ns[2], nc1;
  double zmin, zscale;  // the z quantisation of the sort keys
  int zbits;
};

// Bounding box of every group (warp per group): lo/hi corners, and the
// frame origin (centre) with the half diagonal in w.
__global__ void group_box_kernel(const double4 *__restrict__ gpos, const int4 *__restrict__ grec,
                                 const int *__restrict__ ngroups, double4 *__restrict__ blo,
                                 double4 *__restrict__ bhi, double4 *__restrict__ cen) {
  const long g = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (g >= *ngroups) return;  // warp-uniform (launched for an upper bound)
  const int4 G = grec[g];
  double l[3] = {1e300, 1e300, 1e300}, h[3] = {-1e300, -1e300, -1e300};
  if (G.x + lane < G.y) {
    const double4 p = gpos[G.x + lane];
    l[0] = h[0] = p.x, l[1] = h[1] = p.y, l[2] = h[2] = p.z;
  }
  const unsigned FULL = 0xffffffffu;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
#pragma unroll
    for (int d = 0; d < 3; d++) {
      l[d] = fmin(l[d], __shfl_xor_sync(FULL, l[d], o));
      h[d] = fmax(h[d], __shfl_xor_sync(FULL, h[d], o));
    }
  if (lane == 0) {
    blo[g] = make_double4(l[0], l[1], l[2], 0.0);
    bhi[g] = make_double4(h[0], h[1], h[2], 0.0);
    const double dx = __dsub_rn(h[0], l[0]), dy = __dsub_rn(h[1], l[1]),
                 dz = __dsub_rn(h[2], l[2]);
    cen[g] = make_double4(
        __dmul_rn(0.5, __dadd_rn(l[0], h[0])), __dmul_rn(0.5, __dadd_rn(l[1], h[1])),
        __dmul_rn(0.5, __dadd_rn(l[2], h[2])),
        __dmul_rn(0.5, __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)),
                                            __dmul_rn(dz, dz)))));
  }
}

// first index in [a, b) with v[index] >= x (lower) or > x (upper)
template <typename V>
__device__ __forceinline__ int lower_idx(const V *__restrict__ v, int a, int b, V x) {
  while (a < b) {
    const int m = (a + b) >> 1;
    if (v[m] < x) a = m + 1;
    else b = m;
  }
  return a;
}
__device__ __forceinline__ int upper_idx(const unsigned *__restrict__ v, int a, int b, unsigned x) {
  while (a < b) {
    const int m = (a + b) >> 1;
    if (v[m] <= x) a = m + 1;
    else b = m;
  }
  return a;
}

// Source segments of every group (warp per group; lanes over the fine
// columns of the group's window in (s0, s1) order, so that a group's
// segments come in the same order as a sequential sweep).  A fine column
// contributes the z range of its sources within Rdir of the group's box:
// |dz| <= sqrt(Rdir^2 - d_xy^2), d_xy the xy distance from the box to the
// column; the half shell keeps the fine columns of later coarse columns and,
// in the group's own coarse column, the sources after the group in the
// group order.  FILL = false counts (segments, work, candidates); FILL =
// true writes the segments at the offsets of the count pass.
template <bool FILL>
__global__ void group_segments_kernel(GroupGeom gg, const int4 *__restrict__ grec,
                                      const int *__restrict__ ngroups,
                                      const double4 *__restrict__ blo,
                                      const double4 *__restrict__ bhi,
                                      const int *__restrict__ sstart, const unsigned *__restrict__ zq,
                                      const unsigned *__restrict__ fcpos, int *__restrict__ nseg,
                                      int *__restrict__ nhseg, unsigned *__restrict__ work,
                                      unsigned *__restrict__ hwork,
                                      const int *__restrict__ segoff,
                                      const int *__restrict__ hsegoff, int2 *__restrict__ segs,
                                      int2 *__restrict__ hsegs, int4 *__restrict__ groups,
                                      int4 *__restrict__ hgroups, SetupStats *st) {
  const long g = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (g >= *ngroups) return;  // warp-uniform (launched for an upper bound)
  const unsigned FULL = 0xffffffffu;
  const int4 G = grec[g];
  const int p0 = G.x, p1 = G.y, c = G.z;
  const double4 L = blo[g], Hh = bhi[g];
  const double bl[2] = {L.x, L.y}, bh[2] = {Hh.x, Hh.y};
  int lo[2], hi[2];
#pragma unroll
  for (int d = 0; d < 2; d++) {
    // one column of margin on each side: the distance test below decides
    lo[d] = max(0, (int)floor((bl[d] - gg.R - gg.mn[d]) / gg.sedge[d]) - 1);
    hi[d] = min(gg.ns[d] - 1, (int)floor((bh[d] + gg.R - gg.mn[d]) / gg.sedge[d]) + 1);
  }
  const int w1 = hi[1] - lo[1] + 1;
  const int nwin = (hi[0] - lo[0] + 1) * w1;
  int ns_ = 0, nh_ = 0;
  unsigned long long wk = 0, hwk = 0, cand = 0, hcand = 0;
  const int base = FILL ? segoff[g] : 0, hbase = FILL ? hsegoff[g] : 0;
  for (int t0 = 0; t0 < nwin; t0 += 32) {
    const int t = t0 + lane;
    bool has = false, hhas = false;
    int a = 0, b = 0, a2 = 0;
    if (t < nwin) {
      const int s0 = lo[0] + t / w1, s1 = lo[1] + t % w1;
      const long sc = (long)s0 * gg.ns[1] + s1;
      const int zb = sstart[sc], ze = sstart[sc + 1];
      if (ze > zb) {
        const double l0 = __dadd_rn(gg.mn[0], __dmul_rn((double)s0, gg.sedge[0]));
        const double h0 = __dadd_rn(l0, gg.sedge[0]);
        const double l1 = __dadd_rn(gg.mn[1], __dmul_rn((double)s1, gg.sedge[1]));
        const double h1 = __dadd_rn(l1, gg.sedge[1]);
        const double dx = fmax(0.0, fmax(__dsub_rn(l0, bh[0]), __dsub_rn(bl[0], h0)));
        const double dy = fmax(0.0, fmax(__dsub_rn(l1, bh[1]), __dsub_rn(bl[1], h1)));
        const double d2 = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
        if (d2 <= gg.R2) {
          const double hz = __dsqrt_rn(__dsub_rn(gg.R2, d2));
          const double zlo = __dsub_rn(L.z, hz), zhi = __dadd_rn(Hh.z, hz);
          // whole quanta: every source with zlo <= z <= zhi is inside [a, b)
          a = lower_idx(zq, zb, ze, zquant(zlo, gg.zmin, gg.zscale, gg.zbits));
          b = upper_idx(zq, a, ze, zquant(zhi, gg.zmin, gg.zscale, gg.zbits));
          has = b > a;
          const long cc = (long)(s0 / kSourceSplit) * gg.nc1 + s1 / kSourceSplit;
          if (has && cc >= c) {
            a2 = cc == c ? lower_idx(fcpos, a, b, (unsigned)p1) : a;
            hhas = b > a2;
          }
        }
      }
    }
    const unsigned m = __ballot_sync(FULL, has), hm = __ballot_sync(FULL, hhas);
    const unsigned below = (1u << lane) - 1u;
    if (FILL) {
      if (has) segs[base + ns_ + __popc(m & below)] = make_int2(a, b - a);
      if (hhas) hsegs[hbase + nh_ + __popc(hm & below)] = make_int2(a2, b - a2);
    }
    ns_ += __popc(m);
    nh_ += __popc(hm);
    if (has) wk += (unsigned long long)(b - a);
    if (hhas) hwk += (unsigned long long)(b - a2);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    wk += __shfl_xor_sync(FULL, wk, o);
    hwk += __shfl_xor_sync(FULL, hwk, o);
  }
  if (lane == 0) {
    if (FILL) {
      groups[g] = make_int4(p0, p1 - p0, base, base + ns_);
      hgroups[g] = make_int4(p0, p1 - p0, hbase, hbase + nh_);
    } else {
      nseg[g] = ns_;
      nhseg[g] = nh_;
      // sources staged by the group (at most n: its segments are disjoint)
      work[g] = (unsigned)min(wk, 0xffffffffull);
      hwork[g] = (unsigned)min(hwk, 0xffffffffull);
      cand = wk * (unsigned long long)(p1 - p0);
      hcand = hwk * (unsigned long long)(p1 - p0);
      atomicAdd(&st->cand, cand);
      atomicAdd(&st->hcand, hcand);
    }
  }
}

// final group records and frame origins in work order (the first ngroups
// entries of the order; the slots past ngroups have no work and sort last)
__global__ void order_groups_kernel(const int4 *__restrict__ gin, const double4 *__restrict__ cin,
                                    const unsigned *__restrict__ ord,
                                    const int *__restrict__ ngroups, long bound,
                                    int4 *__restrict__ gout, double4 *__restrict__ cout) {
  const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= bound || k >= *ngroups) return;
  gout[k] = gin[ord[k]];
  cout[k] = cin[ord[k]];
}

// The counts the host needs after set-up, gathered for one copy.
struct SetupCounts {
  long long bad;
  unsigned long long cand, hcand;
  int ngroups, nnonempty, nsegs, nhsegs;
};
__global__ void collect_counts_kernel(const SetupStats *__restrict__ st,
                                      const int *__restrict__ ngroups,
                                      const int *__restrict__ nnonempty,
                                      const int *__restrict__ nsegs,
                                      const int *__restrict__ nhsegs,
                                      SetupCounts *__restrict__ out) {
  out->bad = st->bad;
  out->cand = st->cand;
  out->hcand = st->hcand;
  out->ngroups = *ngroups;
  out->nnonempty = *nnonempty;
  out->nsegs = *nsegs;
  out->nhsegs = *nhsegs;
}

__global__ void iota_kernel(unsigned *__restrict__ v, long n) {
  const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) v[k] = (unsigned)k;
}

int bits_for(unsigned long long v) {  // bits to hold values < v
  int b = 1;
  while (b < 64 && (1ull << b) < v) b++;
  return b;
}

inline unsigned blocks_for(long n, int t = 256) { return (unsigned)((n + t - 1) / t); }

// Scratch buffers of the set-up (handle-owned, reused by the next set-up).
enum Scratch {
  kPts, kBKey, kBKeyOut, kIota, kBPerm, kCKey, kSKey, kKeyOut,
  kBCount, kCStart, kSStart, kFlag, kPos, kZs, kCPos, kFCPos, kGCount, kGOff,
  kGRec, kBLo, kBHi, kCen, kNSeg, kSegOff, kHSegOff, kUGroups, kUHGroups,
  kWorkOut, kOrd, kStats, kCub, kRKey, kRKeyOut, kBPos, kCounts, kScratchCount
};
static_assert(kScratchCount <= kSetupScratch, "raise kSetupScratch");

#define SCK(call)                                                                         \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return record_error(h, NPME_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

template <typename P>
int scratch(npme_handle *h, Scratch i, size_t bytes, P **out) {
  const int rc = handle_buffer(h, &h->d_su[i], bytes);
  *out = (P *)h->d_su[i];
  return rc;
}

// CUB temporary storage of at least `bytes`
int cub_tmp(npme_handle *h, size_t bytes, void **out) {
  return scratch(h, kCub, std::max<size_t>(bytes, 256), out);
}

// stable radix sort of (key, value) pairs on bits [0, end_bit), ascending
// or descending
template <typename K>
int sort_pairs(npme_handle *h, const K *kin, K *kout, const unsigned *vin, unsigned *vout,
               long n, int end_bit, cudaStream_t s, bool descending = false) {
  size_t tb = 0;
  if (descending)
    SCK(cub::DeviceRadixSort::SortPairsDescending(nullptr, tb, kin, kout, vin, vout, (int)n, 0,
                                                   end_bit, s));
  else
    SCK(cub::DeviceRadixSort::SortPairs(nullptr, tb, kin, kout, vin, vout, (int)n, 0, end_bit,
                                        s));
  void *tmp;
  int rc;
  if ((rc = cub_tmp(h, tb, &tmp))) return rc;
  if (descending)
    SCK(cub::DeviceRadixSort::SortPairsDescending(tmp, tb, kin, kout, vin, vout, (int)n, 0,
                                                   end_bit, s));
  else
    SCK(cub::DeviceRadixSort::SortPairs(tmp, tb, kin, kout, vin, vout, (int)n, 0, end_bit, s));
  return NPME_OK;
}

int exclusive_sum(npme_handle *h, const int *in, int *out, long n, cudaStream_t s) {
  size_t tb = 0;
  SCK(cub::DeviceScan::ExclusiveSum(nullptr, tb, in, out, (int)n, s));
  void *tmp;
  int rc;
  if ((rc = cub_tmp(h, tb, &tmp))) return rc;
  SCK(cub::DeviceScan::ExclusiveSum(tmp, tb, in, out, (int)n, s));
  return NPME_OK;
}

template <typename T>
int bin_points(npme_handle *h) {
  const long n = (long)h->n;
  cudaStream_t s = h->stream;
  const GridGeom &gr = h->grid;
  const double *R = h->box + 3, *L = h->box + 6;
  int rc;
  SetupStats *st = (SetupStats *)h->d_su[kStats];
  BinGeom g;
  for (int d = 0; d < 3; d++) {
    g.N[d] = (double)gr.N[d], g.L[d] = L[d], g.R[d] = R[d];
    g.Nl[d] = gr.N[d], g.H[d] = gr.H[d], g.nb[d] = gr.nb[d];
  }
  g.P = gr.order;
  g.TL = kBrick + gr.order - 1;
  g.nkeys = 32 / ((int)(sizeof(T) / 4) * (h->complex_kernel ? 2 : 1));
  // direct-sum columns: edge e ~ (32 / density)^(1/3) over the bounding box
  // (degenerate axes are given a nominal thickness of Rdir / 4)
  const double Rd = h->p.Rdir;
  double vol = 1.0;
  for (int d = 0; d < 3; d++) vol *= std::max(h->bmax[d] - h->bmin[d], 0.25 * Rd);
  double e = std::cbrt(32.0 * vol / (double)n);
  e = std::max(e, 1e-3 * Rd);
  for (int d = 0; d < 2; d++) {
    const double ext = h->bmax[d] - h->bmin[d];
    g.nc[d] = std::max(1, std::min((int)std::ceil(ext / e), 1 << 14));
    g.edge[d] = std::max(ext / g.nc[d], 1e-12);
    g.ns[d] = g.nc[d] * kSourceSplit;
    g.sedge[d] = g.edge[d] / kSourceSplit;
    g.mn[d] = h->bmin[d];
  }
  {
    const double H = h->bmax[2] - h->bmin[2];
    g.zbits = std::max(8, std::min(20, (int)std::ceil(std::log2(std::max(1.0, 1024.0 * H / e)))));
    g.zmin = h->bmin[2];
    g.zscale = (double)((1u << g.zbits) - 1u) / std::max(H, 1e-300);
  }
  // heads of offsets up to ~the group half-diagonal carry ~6e-8 e absolute
  // error; below r = e/4 the relative error would exceed ~1e-6, so refine
  h->refine2 = (0.25 * e) * (0.25 * e);
  const long nbt = gr.nb[0] * gr.nb[1] * gr.nb[2];
  const long ncol = (long)g.nc[0] * g.nc[1], nscol = (long)g.ns[0] * g.ns[1];
  h->n_bricks = nbt;

  BrickPoint<T> *pts;
  unsigned *bkey, *bkey_out, *iota, *bperm;
  unsigned long long *ckey, *skey, *key_out;
  int *bcount, *ccount, *scount, *cstart, *sstart, *flag, *pos;
  if ((rc = scratch(h, kPts, sizeof(BrickPoint<T>) * n, &pts)) ||
      (rc = scratch(h, kBKey, sizeof(unsigned) * n, &bkey)) ||
      (rc = scratch(h, kBKeyOut, sizeof(unsigned) * n, &bkey_out)) ||
      (rc = scratch(h, kIota, sizeof(unsigned) * n, &iota)) ||
      (rc = scratch(h, kBPerm, sizeof(unsigned) * n, &bperm)) ||
      (rc = scratch(h, kCKey, sizeof(unsigned long long) * n, &ckey)) ||
      (rc = scratch(h, kSKey, sizeof(unsigned long long) * n, &skey)) ||
      (rc = scratch(h, kKeyOut, sizeof(unsigned long long) * n, &key_out)) ||
      (rc = scratch(h, kBCount, sizeof(int) * (nbt + ncol + nscol + 3), &bcount)) ||
      (rc = scratch(h, kCStart, sizeof(int) * (ncol + 1), &cstart)) ||
      (rc = scratch(h, kSStart, sizeof(int) * (nscol + 1), &sstart)) ||
      (rc = scratch(h, kFlag, sizeof(int) * (nbt + 1), &flag)) ||
      (rc = scratch(h, kPos, sizeof(int) * (nbt + 1), &pos)))
    return rc;
  const int C = h->complex_kernel ? 2 : 1;
  if ((rc = handle_buffer(h, &h->d_bpts, sizeof(BrickPoint<T>) * n)) ||
      (rc = handle_buffer(h, (void **)&h->d_brick_start, sizeof(int) * (nbt + 1))) ||
      (rc = handle_buffer(h, (void **)&h->d_cperm, sizeof(uint32_t) * n)) ||
      (rc = handle_buffer(h, (void **)&h->d_sperm, sizeof(uint32_t) * n)) ||
      (rc = handle_buffer(h, (void **)&h->d_gpos, sizeof(double4) * n)) ||
      (rc = handle_buffer(h, (void **)&h->d_spos, sizeof(double4) * n)) ||
      (rc = handle_buffer(h, &h->d_qb, sizeof(T) * C * n)) ||
      (rc = handle_buffer(h, &h->d_qc, sizeof(T) * C * n)) ||
      (rc = handle_buffer(h, (void **)&h->d_q_in, sizeof(double) * C * n)) ||
      (rc = handle_buffer(h, (void **)&h->d_V, sizeof(double) * 4 * C * n)))
    return rc;

  // brick, coarse-column and fine-column counts in one block, one clear
  ccount = bcount + nbt + 1;
  scount = ccount + ncol + 1;
  SCK(cudaMemsetAsync(bcount, 0, sizeof(int) * (nbt + ncol + nscol + 3), s));
  bin_kernel<T><<<blocks_for(n), 256, 0, s>>>(h->d_coord, n, g, pts, bkey, ckey, skey, iota,
                                              bcount, ccount, scount, st);
  SCK(cudaGetLastError());

  // --- brick order: by brick, inside a brick in rounds over the banks ---
  // (brick, bank, index) first; (brick, rank inside the bank, bank) below
  if ((rc = sort_pairs(h, bkey, bkey_out, iota, bperm, n, 5 + bits_for(nbt), s)) ||
      (rc = handle_buffer(h, (void **)&h->d_bperm, sizeof(uint32_t) * n)))
    return rc;
  if ((rc = exclusive_sum(h, bcount, h->d_brick_start, nbt + 1, s))) return rc;
  nonempty_flags_kernel<<<blocks_for(nbt + 1), 256, 0, s>>>(bcount, nbt, flag);
  if ((rc = exclusive_sum(h, flag, pos, nbt + 1, s))) return rc;

  // --- direct-sum orders: (column, quantised z, index) for targets and
  // sources, one radix sort each ---
  if ((rc = sort_pairs(h, ckey, key_out, iota, h->d_cperm, n, bits_for(ncol) + g.zbits, s)) ||
      (rc = sort_pairs(h, skey, key_out, iota, h->d_sperm, n, bits_for(nscol) + g.zbits, s)))
    return rc;
  if ((rc = exclusive_sum(h, ccount, cstart, ncol + 1, s))) return rc;
  if ((rc = exclusive_sum(h, scount, sstart, nscol + 1, s))) return rc;
  unsigned *zs;  // quantised z of the sources, in source order
  unsigned *cpos, *fcpos;
  int *gcount, *goff;
  if ((rc = scratch(h, kZs, sizeof(unsigned) * n, &zs)) ||
      (rc = scratch(h, kCPos, sizeof(unsigned) * n, &cpos)) ||
      (rc = scratch(h, kFCPos, sizeof(unsigned) * n, &fcpos)) ||
      (rc = scratch(h, kGCount, sizeof(int) * (ncol + 1), &gcount)) ||
      (rc = scratch(h, kGOff, sizeof(int) * (ncol + 1), &goff)))
    return rc;
  source_z_kernel<<<blocks_for(n), 256, 0, s>>>(key_out, h->d_cperm, n, g.zbits, zs, cpos);
  gather_u32_kernel<<<blocks_for(n), 256, 0, s>>>(cpos, h->d_sperm, n, fcpos);
  groups_per_column_kernel<<<blocks_for(ncol + 1), 256, 0, s>>>(ccount, ncol, gcount);
  if ((rc = exclusive_sum(h, gcount, goff, ncol + 1, s))) return rc;
  SCK(cudaGetLastError());

  // No read-back here: the group and segment arrays are sized from upper
  // bounds and the kernels read the actual counts on the device; the host
  // reads every count once, when the set-up has completed (finish_setup).
  //   groups   <= n / 32 + non-empty columns <= n / 32 + min(n, ncol)
  //   segments <= groups x the fine columns of a group's window (a group lies
  //               in one coarse column, so its window spans at most
  //               (edge + 2 Rdir) / sedge + 4 fine columns per axis)
  //   non-empty bricks <= min(n, nbt)
  const long ngb = n / 32 + std::min(n, ncol) + 1;
  long wmax = 1;
  for (int d = 0; d < 2; d++)
    wmax *= std::min<long>(g.ns[d], (long)std::floor((g.edge[d] + 2.0 * Rd) / g.sedge[d]) + 4);
  const long nsb = ngb * wmax;
  if (nsb >= (1L << 31))  // int offsets in the group records
    return record_error(h, NPME_EINVAL, "too many direct-sum source segments (2^31)");
  if ((rc = handle_buffer(h, (void **)&h->d_brick_list,
                          sizeof(int) * std::max<long>(1, std::min(n, nbt)))))
    return rc;
  brick_list_kernel<<<blocks_for(nbt), 256, 0, s>>>(bcount, pos, nbt, h->d_brick_list);

  // brick order in rounds over the banks: the rank inside a bank is below n
  {
    const int rbits = bits_for((unsigned long long)n);
    const int kbits = bits_for(nbt) + rbits + 5;
    unsigned *bperm2 = h->d_bperm;
    if (kbits <= 32) {
      unsigned *rkey, *rkey_out;
      if ((rc = scratch(h, kRKey, sizeof(unsigned) * n, &rkey)) ||
          (rc = scratch(h, kRKeyOut, sizeof(unsigned) * n, &rkey_out)))
        return rc;
      round_key_kernel<unsigned><<<blocks_for(n), 256, 0, s>>>(bkey_out, n, rbits, rkey);
      if ((rc = sort_pairs(h, rkey, rkey_out, bperm, bperm2, n, kbits, s))) return rc;
    } else {
      unsigned long long *rkey, *rkey_out;
      if ((rc = scratch(h, kRKey, sizeof(unsigned long long) * n, &rkey)) ||
          (rc = scratch(h, kRKeyOut, sizeof(unsigned long long) * n, &rkey_out)))
        return rc;
      round_key_kernel<unsigned long long>
          <<<blocks_for(n), 256, 0, s>>>(bkey_out, n, rbits, rkey);
      if ((rc = sort_pairs(h, rkey, rkey_out, bperm, bperm2, n, kbits, s))) return rc;
    }
    gather_bpts_kernel<T><<<blocks_for(n), 256, 0, s>>>(pts, bperm2, n,
                                                        (BrickPoint<T> *)h->d_bpts);
  }
  unsigned *bpos;
  if ((rc = scratch(h, kBPos, sizeof(unsigned) * n, &bpos))) return rc;
  brick_position_kernel<<<blocks_for(n), 256, 0, s>>>(h->d_bperm, n, bpos);
  gather_positions_kernel<<<blocks_for(n), 256, 0, s>>>(h->d_coord, h->d_cperm, h->d_sperm, bpos,
                                                        n, h->d_gpos, h->d_spos);

  // --- warp groups and their source segments ---
  const int *ngp = goff + ncol;  // the actual group count, on the device
  int4 *grec;
  double4 *blo, *bhi, *cen;
  int *nseg, *nhseg, *segoff, *hsegoff;
  unsigned *work, *hwork, *work_out, *ord;
  int4 *ug, *uh;
  if ((rc = scratch(h, kGRec, sizeof(int4) * ngb, &grec)) ||
      (rc = scratch(h, kBLo, sizeof(double4) * ngb, &blo)) ||
      (rc = scratch(h, kBHi, sizeof(double4) * ngb, &bhi)) ||
      (rc = scratch(h, kCen, sizeof(double4) * ngb, &cen)) ||
      (rc = scratch(h, kNSeg, sizeof(int) * 4 * (ngb + 1), &nseg)) ||
      (rc = scratch(h, kSegOff, sizeof(int) * (ngb + 1), &segoff)) ||
      (rc = scratch(h, kHSegOff, sizeof(int) * (ngb + 1), &hsegoff)) ||

      (rc = scratch(h, kWorkOut, sizeof(unsigned) * ngb, &work_out)) ||
      (rc = scratch(h, kOrd, sizeof(unsigned) * ngb, &ord)) ||
      (rc = scratch(h, kUGroups, sizeof(int4) * ngb, &ug)) ||
      (rc = scratch(h, kUHGroups, sizeof(int4) * ngb, &uh)) ||
      (rc = handle_buffer(h, (void **)&h->d_segs, sizeof(int2) * nsb)) ||
      (rc = handle_buffer(h, (void **)&h->d_hsegs, sizeof(int2) * nsb)) ||
      (rc = handle_buffer(h, (void **)&h->d_groups, sizeof(int4) * ngb)) ||
      (rc = handle_buffer(h, (void **)&h->d_gcen, sizeof(double4) * ngb)) ||
      (rc = handle_buffer(h, (void **)&h->d_hgroups, sizeof(int4) * ngb)) ||
      (rc = handle_buffer(h, (void **)&h->d_hcen, sizeof(double4) * ngb)))
    return rc;
  // Heaviest groups first, so that the last wave of a direct-sum launch holds
  // the light ones; when every group fits in one wave (4 groups per CTA,
  // about 4 CTAs per SM) the order does not matter and the lists are
  // written in column order directly.
  const bool order_by_work = ngb > kOneWaveGroups;
  if (!order_by_work) cen = h->d_gcen, ug = h->d_groups, uh = h->d_hgroups;
  group_records_kernel<<<blocks_for(ncol), 256, 0, s>>>(cstart, goff, ncol, grec);
  group_box_kernel<<<blocks_for(32 * ngb), 256, 0, s>>>(h->d_gpos, grec, ngp, blo, bhi, cen);
  GroupGeom gg;
  gg.R = Rd, gg.R2 = Rd * Rd;
  for (int d = 0; d < 2; d++) gg.mn[d] = g.mn[d], gg.sedge[d] = g.sedge[d], gg.ns[d] = g.ns[d];
  gg.nc1 = g.nc[1];
  gg.zmin = g.zmin, gg.zscale = g.zscale, gg.zbits = g.zbits;
  // segment counts and work of both lists in one block, one clear (slots
  // past the actual groups: no segments, no work, so they sort last)
  nhseg = nseg + (ngb + 1);
  work = (unsigned *)(nhseg + (ngb + 1));
  hwork = work + (ngb + 1);
  SCK(cudaMemsetAsync(nseg, 0, sizeof(int) * 4 * (ngb + 1), s));
  group_segments_kernel<false><<<blocks_for(32 * ngb), 256, 0, s>>>(
      gg, grec, ngp, blo, bhi, sstart, zs, fcpos, nseg, nhseg, work, hwork, nullptr, nullptr,
      nullptr, nullptr, nullptr, nullptr, st);
  if ((rc = exclusive_sum(h, nseg, segoff, ngb + 1, s))) return rc;
  if ((rc = exclusive_sum(h, nhseg, hsegoff, ngb + 1, s))) return rc;
  group_segments_kernel<true><<<blocks_for(32 * ngb), 256, 0, s>>>(
      gg, grec, ngp, blo, bhi, sstart, zs, fcpos, nullptr, nullptr, nullptr, nullptr, segoff,
      hsegoff, h->d_segs, h->d_hsegs, ug, uh, st);
  if (order_by_work) {  // each list by its own work; ties keep the column order
    iota_kernel<<<blocks_for(ngb), 256, 0, s>>>(iota, ngb);
    const int wbits = bits_for((unsigned long long)n + 1);
    if ((rc = sort_pairs(h, work, work_out, iota, ord, ngb, wbits, s, true))) return rc;
    order_groups_kernel<<<blocks_for(ngb), 256, 0, s>>>(ug, cen, ord, ngp, ngb, h->d_groups,
                                                        h->d_gcen);
    if ((rc = sort_pairs(h, hwork, work_out, iota, ord, ngb, wbits, s, true))) return rc;
    order_groups_kernel<<<blocks_for(ngb), 256, 0, s>>>(uh, cen, ord, ngp, ngb, h->d_hgroups,
                                                        h->d_hcen);
  } else {
    SCK(cudaMemcpyAsync(h->d_hcen, h->d_gcen, sizeof(double4) * ngb, cudaMemcpyDeviceToDevice, s));
  }
  // the counts, for the host to read when the set-up has completed
  SetupCounts *dc;
  if ((rc = scratch(h, kCounts, sizeof(SetupCounts), &dc))) return rc;
  collect_counts_kernel<<<1, 1, 0, s>>>(st, ngp, pos + nbt, segoff + ngb, hsegoff + ngb, dc);
  SCK(cudaMemcpyAsync(h->h_counts, dc, sizeof(SetupCounts), cudaMemcpyDeviceToHost, s));
  SCK(cudaGetLastError());
  h->d_dperm = h->d_sperm;  // direct-sum charges are gathered into the source order

  // source-side sums of the pair-once walk start (and are kept) at zero
  if (h->fp32) {
    const size_t nv = (size_t)C * n;  // float4 per source (two if complex)
    if ((rc = handle_buffer(h, (void **)&h->d_vsrc, sizeof(float4) * nv))) return rc;
    SCK(cudaMemsetAsync(h->d_vsrc, 0, sizeof(float4) * nv, s));
  } else {
    if ((rc = handle_buffer(h, (void **)&h->d_vsrc64, sizeof(double) * 4 * n))) return rc;
    SCK(cudaMemsetAsync(h->d_vsrc64, 0, sizeof(double) * 4 * n, s));
  }

  // --- grids ---
  const long *N = gr.N;
  const size_t Ntot = (size_t)N[0] * N[1] * N[2];
  const size_t Mtot = (size_t)(N[0] / 2 + 1) * (N[1] / 2 + 1) * (N[2] / 2 + 1);
  if (h->complex_kernel) {
    if ((rc = handle_buffer(h, &h->d_grid, sizeof(T) * 2 * Ntot)) ||
        (rc = handle_buffer(h, &h->d_G, sizeof(T) * 2 * Mtot)))
      return rc;
  } else {
    if ((rc = handle_buffer(h, &h->d_grid, sizeof(T) * Ntot)) ||
        (rc = handle_buffer(h, &h->d_kgrid, sizeof(T) * 2 * (size_t)N[0] * N[1] * (N[2] / 2 + 1))) ||
        (rc = handle_buffer(h, &h->d_G, sizeof(T) * Mtot)))
      return rc;
  }
  return NPME_OK;
}

}  // namespace

int device_bbox(npme_handle *h, const double *coord, double mn[3], double mx[3]) {
  const long n = (long)h->n;
  cudaStream_t s = h->stream;
  int rc;
  if ((rc = handle_buffer(h, (void **)&h->d_coord, sizeof(double) * 3 * n))) return rc;
  SetupStats *st;
  if ((rc = scratch(h, kStats, sizeof(SetupStats), &st))) return rc;
  if (!h->h_counts) SCK(cudaHostAlloc(&h->h_counts, sizeof(SetupCounts), cudaHostAllocDefault));
  SCK(cudaMemcpyAsync(h->d_coord, coord, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s));
  init_stats_kernel<<<1, 1, 0, s>>>(st, n);
  if (n < kHostBoxPoints) {
    // small systems: one host pass costs less than a device reduction and
    // the wait for it
    for (int d = 0; d < 3; d++) mn[d] = 1e300, mx[d] = -1e300;
    for (long i = 0; i < n; i++)
      for (int d = 0; d < 3; d++) {
        const double x = coord[3 * i + d];
        if (!std::isfinite(x)) return record_error(h, NPME_EINVAL, "non-finite coordinate");
        mn[d] = std::min(mn[d], x);
        mx[d] = std::max(mx[d], x);
      }
    SCK(cudaGetLastError());
    return NPME_OK;
  }
  const unsigned blocks = (unsigned)std::min<long>(blocks_for(n), 148 * 8);
  bbox_kernel<<<blocks, 256, 0, s>>>(h->d_coord, n, st);
  SCK(cudaGetLastError());
  SetupStats hs;
  SCK(cudaMemcpyAsync(&hs, st, sizeof(hs), cudaMemcpyDeviceToHost, s));
  SCK(cudaStreamSynchronize(s));
  if (hs.nonfinite) return record_error(h, NPME_EINVAL, "non-finite coordinate");
  for (int d = 0; d < 3; d++) mn[d] = dkey_inv(hs.mn[d]), mx[d] = dkey_inv(hs.mx[d]);
  return NPME_OK;
}

int finish_setup(npme_handle *h) {
  const SetupCounts &c = *static_cast<const SetupCounts *>(h->h_counts);
  const long n = (long)h->n;
  if (c.bad < n) {
    // the axis of the first offending point, from its coordinates
    double x[3];
    SCK(cudaMemcpy(x, h->d_coord + 3 * c.bad, sizeof(x), cudaMemcpyDeviceToHost));
    const GridGeom &gr = h->grid;
    const double *R = h->box + 3, *L = h->box + 6;
    int axis = 0;
    for (int d = 0; d < 3; d++) {
      const double w = (double)gr.N[d] / L[d] * (x[d] - R[d]);
      const long ms = w < 0 ? (long)(-w) + 1 : (long)(-w);
      const long o = ms + gr.N[d] / 4;
      if (o < 0 || o + gr.order - 1 > gr.H[d] - 1) {
        axis = d;
        break;
      }
    }
    return record_error(h, NPME_EINVAL,
                        "point " + std::to_string(c.bad) + " has a B-spline stencil outside "
                        "the charge octant (axis " + std::to_string(axis) + ")");
  }
  h->n_nonempty = c.nnonempty;
  h->n_groups = h->n_hgroups = c.ngroups;
  h->n_segs = c.nsegs;
  h->n_hsegs = c.nhsegs;
  h->cand_per_point = (double)c.cand / (double)n;
  h->hcand_per_point = (double)c.hcand / (double)n;
  return NPME_OK;
}

int device_bin(npme_handle *h) {
  return h->fp32 ? bin_points<float>(h) : bin_points<double>(h);
}

}  // namespace npme
