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
// Any number of systems are set up in one pass (a batch: the serving queue
// sets up the requests it admits together; npme_gpu_setup is a batch of
// one), so the kernel launches of a set-up are shared by all its systems.
// Sorting is done with stable radix sorts (values = point indices in
// increasing order) on keys that start with the system's index, so every
// order is (system, key, index) lexicographic and the result does not
// depend on timing or on the other systems of the batch.  Work per point or
// per group is a thread or a warp.  Buffers are sized from upper bounds and
// the host reads the counts once, when the set-up has completed.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "internal.h"

namespace npme {
namespace {

constexpr int kSourceSplit = 2;  // fine source columns per coarse column edge
constexpr long kHostBoxPoints = 1L << 15;  // below: bounding box on the host

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

// The bounding box of one system's coordinates, read back by the host.
struct SetupStats {
  unsigned long long mn[3], mx[3];  // dkey of the per-axis minimum / maximum
  unsigned int nonfinite;
};

__global__ void init_stats_kernel(SetupStats *st) {
  for (int d = 0; d < 3; d++) st->mn[d] = ~0ull, st->mx[d] = 0ull;
  st->nonfinite = 0;
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

struct GroupGeom {
  double R, R2;
  double mn[2], sedge[2];
  int ns[2], nc1;
  double zmin, zscale;  // the z quantisation of the sort keys
  int zbits;
};

// One system of a set-up batch: its geometry and sizes, where its elements
// start in the batch's concatenated scratch arrays, and its handle's output
// buffers.  Index spaces of the batch: points (p_off), brick slots (b_off,
// nbt + 1 per system: the bricks and an empty end slot), coarse and fine
// column slots (c_off, s_off: columns and an end slot), group slots (g_off,
// ngb per system: an upper bound of its groups).  Every sort key of the
// batch starts with the system's index, so a system's elements stay
// contiguous and in their own order through every sort.
struct SysDesc {
  BinGeom g;
  GroupGeom gg;
  long n, nbt, ncol, nscol, ngb;
  long p_off, b_off, c_off, s_off, g_off;
  const double *coord;
  void *bpts;        // BrickPoint<T>[n]
  int *brick_start;  // [nbt + 1]
  int *brick_list;   // [min(n, nbt)]
  uint32_t *cperm, *sperm, *bperm;
  double4 *gpos, *spos;
  int2 *segs, *hsegs;
  int4 *groups, *hgroups;
  double4 *gcen, *hcen;
};

// Per system, accumulated on the device.
struct SysStats {
  long long bad;                   // lowest index whose stencil leaves the octant
  unsigned long long cand, hcand;  // staged (target, source) candidates, both walks
};

// The counts the host reads once the set-up has completed.
struct SetupCounts {
  long long bad;
  unsigned long long cand, hcand;
  int ngroups, nnonempty, nsegs, nhsegs;
};

constexpr int kZField = 20;  // bits of the quantised-z field of the column keys

// The system owning element x of an index space with starts off[0..R).
__device__ __forceinline__ int owner(const long *__restrict__ off, int R, long x) {
  int lo = 0, hi = R - 1;
  while (lo < hi) {
    const int m = (lo + hi + 1) >> 1;
    if (off[m] <= x) lo = m;
    else hi = m - 1;
  }
  return lo;
}

__global__ void init_sys_stats_kernel(const SysDesc *__restrict__ d, int R, SysStats *st) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= R) return;
  st[r].bad = d[r].n;
  st[r].cand = st[r].hcand = 0;
}

// Per point: the spread/interpolation record, its brick-and-bank sort key,
// its (coarse column, quantised z) and (fine column, quantised z) sort keys;
// per brick and column the point counts.  Arithmetic as the host restatement
// of the reference (explicit round-to-nearest operations, no contraction),
// so that every point lands in the same brick, bank and column on any
// machine.
template <typename T>
__global__ void bin_kernel(const SysDesc *__restrict__ d, const long *__restrict__ poff, int R,
                           long P, int bbits, int cbits, int sbits,
                           BrickPoint<T> *__restrict__ pts, unsigned long long *__restrict__ bkey,
                           unsigned long long *__restrict__ ckey,
                           unsigned long long *__restrict__ skey, unsigned *__restrict__ iota,
                           int *__restrict__ bcount, int *__restrict__ ccount,
                           int *__restrict__ scount, SysStats *st) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  const int r = owner(poff, R, p);
  const SysDesc &D = d[r];
  const BinGeom &g = D.g;
  const long i = p - D.p_off;
  const double x[3] = {D.coord[3 * i], D.coord[3 * i + 1], D.coord[3 * i + 2]};
  long o[3];
  T u[3];
  bool out = false;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const double w = __dmul_rn(__ddiv_rn(g.N[a], g.L[a]), __dsub_rn(x[a], g.R[a]));
    const long ms = stencil_start(w);
    o[a] = ms + g.Nl[a] / 4;
    if (o[a] < 0 || o[a] + g.P - 1 > g.H[a] - 1) out = true;
    u[a] = (T)__dadd_rn(w, (double)ms);
  }
  if (out) {
    atomicMin(&st[r].bad, (long long)i);
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
  pts[p] = bp;
  bkey[p] = ((unsigned long long)r << (bbits + 5)) | ((unsigned long long)bid << 5) | key;
  // every point is counted in the brick its key names (a point outside the
  // octant in brick 0), so that the brick starts index the sorted keys
  atomicAdd(&bcount[D.b_off + bid], 1);
  int cs[2], ss[2];
#pragma unroll
  for (int a = 0; a < 2; a++) {
    const double v = __dsub_rn(x[a], g.mn[a]);
    cs[a] = min(g.nc[a] - 1, max(0, (int)__ddiv_rn(v, g.edge[a])));
    const double rr = __dsub_rn(v, __dmul_rn((double)cs[a], g.edge[a]));
    ss[a] = cs[a] * kSourceSplit + min(kSourceSplit - 1, max(0, (int)__ddiv_rn(rr, g.sedge[a])));
  }
  const unsigned long long cc = (unsigned long long)(cs[0] * g.nc[1] + cs[1]);
  const unsigned long long sc = (unsigned long long)(ss[0] * g.ns[1] + ss[1]);
  const unsigned long long zq = zquant(x[2], g.zmin, g.zscale, g.zbits);
  ckey[p] = ((unsigned long long)r << (cbits + kZField)) | (cc << kZField) | zq;
  skey[p] = ((unsigned long long)r << (sbits + kZField)) | (sc << kZField) | zq;
  atomicAdd(&ccount[D.c_off + (long)cc], 1);
  atomicAdd(&scount[D.s_off + (long)sc], 1);
  iota[p] = (unsigned)p;
}

// Brick order inside each brick in rounds over the banks: round r holds the
// r-th point (in index order) of every bank with more than r points, banks
// ascending, i.e. the order of a stable sort by (system, brick, rank inside
// the bank, bank).  Input: the point indices sorted by (system, brick, bank)
// and those keys; one warp per brick slot, lane b owns bank b (keys carry the
// bank in their low 5 bits).
__global__ void round_place_kernel(const unsigned long long *__restrict__ key,
                                   const unsigned *__restrict__ in, const int *__restrict__ bstart,
                                   const int *__restrict__ bcount, long B,
                                   unsigned *__restrict__ out) {
  const long b = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (b >= B) return;  // warp-uniform
  const int c = bcount[b];
  if (c == 0) return;
  const long s = bstart[b], e = s + c;
  // first position in [s, e) whose bank is >= v (banks ascend in the brick)
  auto first = [&](unsigned v) {
    long lo = s, hi = e;
    while (lo < hi) {
      const long m = (lo + hi) >> 1;
      if ((unsigned)(key[m] & 31ull) < v) lo = m + 1;
      else hi = m;
    }
    return lo;
  };
  const long lo = first((unsigned)lane), hi = first((unsigned)lane + 1u);
  const int cnt = (int)(hi - lo);
  int rounds = cnt;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) rounds = max(rounds, __shfl_xor_sync(0xffffffffu, rounds, o));
  const unsigned below = (1u << lane) - 1u;
  long base = s;
  for (int r = 0; r < rounds; r++) {
    const unsigned m = __ballot_sync(0xffffffffu, cnt > r);
    if (cnt > r) out[base + __popc(m & below)] = in[lo + r];
    base += __popc(m);
  }
}

// Final brick order of every system: its records, the brick-order
// permutation, and each point's brick-order position (the slot of its
// source-side direct-sum sums).
template <typename T>
__global__ void place_bricks_kernel(const SysDesc *__restrict__ d, const long *__restrict__ poff,
                                    int R, long P, const unsigned *__restrict__ order,
                                    const BrickPoint<T> *__restrict__ pts,
                                    unsigned *__restrict__ bpos) {
  const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= P) return;
  const int r = owner(poff, R, k);
  const SysDesc &D = d[r];
  const long p = order[k], kl = k - D.p_off;
  reinterpret_cast<BrickPoint<T> *>(D.bpts)[kl] = pts[p];
  D.bperm[kl] = (uint32_t)(p - D.p_off);
  bpos[p] = (unsigned)kl;
}

// flag[b] = 1 for non-empty brick slots (end slots are empty)
__global__ void nonempty_flags_kernel(const int *__restrict__ count, long nb,
                                      int *__restrict__ flag) {
  const long b = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (b < nb) flag[b] = count[b] > 0;
}

// Every system's brick starts (local positions) and non-empty brick list.
__global__ void bricks_kernel(const SysDesc *__restrict__ d, const long *__restrict__ boff, int R,
                              long B, const int *__restrict__ count, const int *__restrict__ start,
                              const int *__restrict__ pos) {
  const long slot = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (slot >= B) return;
  const int r = owner(boff, R, slot);
  const SysDesc &D = d[r];
  const long b = slot - D.b_off;  // 0 .. nbt (end slot)
  D.brick_start[b] = start[slot] - start[D.b_off];
  if (b < D.nbt && count[slot] > 0) D.brick_list[pos[slot] - pos[D.b_off]] = (int)b;
}

// The direct sum's two orders of every system: local permutations, FP64
// positions (a source's w holds its brick-order position), the sources'
// quantised z, and each point's position in the target (group) order.
__global__ void place_orders_kernel(const SysDesc *__restrict__ d, const long *__restrict__ poff,
                                    int R, long P, const unsigned *__restrict__ corder,
                                    const unsigned *__restrict__ sorder,
                                    const unsigned long long *__restrict__ skey,
                                    const unsigned *__restrict__ bpos, unsigned *__restrict__ zq,
                                    unsigned *__restrict__ cpos) {
  const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= P) return;
  const int r = owner(poff, R, k);
  const SysDesc &D = d[r];
  const long kl = k - D.p_off;
  const long pc = corder[k], ic = pc - D.p_off;
  D.cperm[kl] = (uint32_t)ic;
  cpos[pc] = (unsigned)k;
  const double *x = D.coord + 3 * ic;
  D.gpos[kl] = make_double4(x[0], x[1], x[2], 0.0);
  const long ps = sorder[k], is = ps - D.p_off;
  D.sperm[kl] = (uint32_t)is;
  zq[k] = (unsigned)(skey[k] & ((1ull << kZField) - 1ull));
  const double *y = D.coord + 3 * is;
  D.spos[kl] = make_double4(y[0], y[1], y[2], (double)bpos[ps]);
}

__global__ void gather_u32_kernel(const unsigned *__restrict__ src,
                                  const unsigned *__restrict__ perm, long n,
                                  unsigned *__restrict__ out) {
  const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) out[k] = src[perm[k]];
}

// groups per coarse column slot: ceil(count / 32) (end slots: 0)
__global__ void groups_per_column_kernel(const int *__restrict__ ccount, long ncol,
                                         int *__restrict__ gcount) {
  const long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c < ncol) gcount[c] = (ccount[c] + 31) / 32;
}

// The groups of every column: points [p0, p1) of the batch's target order
// (runs of 32 in the column), the column and the system.
__global__ void group_records_kernel(const SysDesc *__restrict__ d, const long *__restrict__ coff,
                                     int R, long C, const int *__restrict__ cstart,
                                     const int *__restrict__ goff, int4 *__restrict__ grec) {
  const long slot = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (slot >= C) return;
  const int r = owner(coff, R, slot);
  const SysDesc &D = d[r];
  const long c = slot - D.c_off;
  if (c >= D.ncol) return;  // end slot
  const int p_end = cstart[slot + 1];
  long gs = D.g_off + (goff[slot] - goff[D.c_off]);
  for (int p0 = cstart[slot]; p0 < p_end; p0 += 32, gs++)
    grec[gs] = make_int4(p0, min(p0 + 32, p_end), (int)c, r);
}

// the number of groups of system D (on the device)
__device__ __forceinline__ long sys_groups(const SysDesc &D, const int *__restrict__ goff) {
  return goff[D.c_off + D.ncol] - goff[D.c_off];
}

// Bounding box of every group (warp per group slot): lo/hi corners, and the
// frame origin (centre) with the half diagonal in w.
__global__ void group_box_kernel(const SysDesc *__restrict__ d, const long *__restrict__ goffs,
                                 int R, long G, const int *__restrict__ goff,
                                 const int4 *__restrict__ grec, double4 *__restrict__ blo,
                                 double4 *__restrict__ bhi, double4 *__restrict__ cen) {
  const long slot = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (slot >= G) return;  // warp-uniform
  const int r = owner(goffs, R, slot);
  const SysDesc &D = d[r];
  if (slot - D.g_off >= sys_groups(D, goff)) return;  // a spare slot of the bound
  const int4 Gr = grec[slot];
  double l[3] = {1e300, 1e300, 1e300}, h[3] = {-1e300, -1e300, -1e300};
  if (Gr.x + lane < Gr.y) {
    const double4 p = D.gpos[Gr.x + lane - D.p_off];
    l[0] = h[0] = p.x, l[1] = h[1] = p.y, l[2] = h[2] = p.z;
  }
  const unsigned FULL = 0xffffffffu;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
#pragma unroll
    for (int a = 0; a < 3; a++) {
      l[a] = fmin(l[a], __shfl_xor_sync(FULL, l[a], o));
      h[a] = fmax(h[a], __shfl_xor_sync(FULL, h[a], o));
    }
  if (lane == 0) {
    blo[slot] = make_double4(l[0], l[1], l[2], 0.0);
    bhi[slot] = make_double4(h[0], h[1], h[2], 0.0);
    const double dx = __dsub_rn(h[0], l[0]), dy = __dsub_rn(h[1], l[1]),
                 dz = __dsub_rn(h[2], l[2]);
    cen[slot] = make_double4(
        __dmul_rn(0.5, __dadd_rn(l[0], h[0])), __dmul_rn(0.5, __dadd_rn(l[1], h[1])),
        __dmul_rn(0.5, __dadd_rn(l[2], h[2])),
        __dmul_rn(0.5, __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)),
                                            __dmul_rn(dz, dz)))));
  }
}

// first index in [a, b) with v[index] >= x (lower) or > x (upper)
__device__ __forceinline__ int lower_idx(const unsigned *__restrict__ v, int a, int b, unsigned x) {
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

// Source segments of every group (warp per group slot; lanes over the fine
// columns of the group's window in (s0, s1) order, so that a group's
// segments come in the same order as a sequential sweep).  A fine column
// contributes the z range of its sources within Rdir of the group's box:
// |dz| <= sqrt(Rdir^2 - d_xy^2), d_xy the xy distance from the box to the
// column; the half shell keeps the fine columns of later coarse columns and,
// in the group's own coarse column, the sources after the group in the
// group order.  Positions are the batch's (cstart, sstart, fcpos); the
// written segments and group records are the system's own (local).  FILL =
// false counts (segments, work, candidates); FILL = true writes the
// segments at the offsets of the count pass.
template <bool FILL>
__global__ void group_segments_kernel(const SysDesc *__restrict__ d, const long *__restrict__ goffs,
                                      int R, long G, const int *__restrict__ goff,
                                      const int4 *__restrict__ grec,
                                      const double4 *__restrict__ blo,
                                      const double4 *__restrict__ bhi,
                                      const int *__restrict__ sstart,
                                      const unsigned *__restrict__ zq,
                                      const unsigned *__restrict__ fcpos, int *__restrict__ nseg,
                                      int *__restrict__ nhseg, unsigned *__restrict__ work,
                                      unsigned *__restrict__ hwork,
                                      const int *__restrict__ segoff,
                                      const int *__restrict__ hsegoff, int4 *__restrict__ ug,
                                      int4 *__restrict__ uh, SysStats *st) {
  const long slot = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (slot >= G) return;  // warp-uniform
  const int r = owner(goffs, R, slot);
  const SysDesc &D = d[r];
  if (slot - D.g_off >= sys_groups(D, goff)) return;  // a spare slot of the bound
  const GroupGeom &gg = D.gg;
  const unsigned FULL = 0xffffffffu;
  const int4 Gr = grec[slot];
  const int p0 = Gr.x, p1 = Gr.y, c = Gr.z;
  const double4 L = blo[slot], Hh = bhi[slot];
  const double bl[2] = {L.x, L.y}, bh[2] = {Hh.x, Hh.y};
  int lo[2], hi[2];
#pragma unroll
  for (int a = 0; a < 2; a++) {
    // one column of margin on each side: the distance test below decides
    lo[a] = max(0, (int)floor((bl[a] - gg.R - gg.mn[a]) / gg.sedge[a]) - 1);
    hi[a] = min(gg.ns[a] - 1, (int)floor((bh[a] + gg.R - gg.mn[a]) / gg.sedge[a]) + 1);
  }
  const int w1 = hi[1] - lo[1] + 1;
  const int nwin = (hi[0] - lo[0] + 1) * w1;
  int ns_ = 0, nh_ = 0;
  unsigned long long wk = 0, hwk = 0;
  const int base = FILL ? segoff[slot] - segoff[D.g_off] : 0;
  const int hbase = FILL ? hsegoff[slot] - hsegoff[D.g_off] : 0;
  const int pl = (int)D.p_off;  // batch position -> system position
  for (int t0 = 0; t0 < nwin; t0 += 32) {
    const int t = t0 + lane;
    bool has = false, hhas = false;
    int a = 0, b = 0, a2 = 0;
    if (t < nwin) {
      const int s0 = lo[0] + t / w1, s1 = lo[1] + t % w1;
      const long sc = D.s_off + (long)s0 * gg.ns[1] + s1;
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
      if (has) D.segs[base + ns_ + __popc(m & below)] = make_int2(a - pl, b - a);
      if (hhas) D.hsegs[hbase + nh_ + __popc(hm & below)] = make_int2(a2 - pl, b - a2);
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
      ug[slot] = make_int4(p0 - pl, p1 - p0, base, base + ns_);
      uh[slot] = make_int4(p0 - pl, p1 - p0, hbase, hbase + nh_);
    } else {
      nseg[slot] = ns_;
      nhseg[slot] = nh_;
      // sources staged by the group (at most n: its segments are disjoint)
      work[slot] = (unsigned)min(wk, 0xffffffffull);
      hwork[slot] = (unsigned)min(hwk, 0xffffffffull);
      atomicAdd(&st[r].cand, wk * (unsigned long long)(p1 - p0));
      atomicAdd(&st[r].hcand, hwk * (unsigned long long)(p1 - p0));
    }
  }
}

// Sort key of a group slot: the system, then the work, heaviest first; spare
// slots of a system's bound last.
__global__ void work_key_kernel(const SysDesc *__restrict__ d, const long *__restrict__ goffs,
                                int R, long G, const int *__restrict__ goff,
                                const unsigned *__restrict__ work, int wbits,
                                unsigned long long *__restrict__ key, unsigned *__restrict__ iota) {
  const long slot = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (slot >= G) return;
  const int r = owner(goffs, R, slot);
  const SysDesc &D = d[r];
  const unsigned long long mask = (1ull << wbits) - 1ull;
  const bool real = slot - D.g_off < sys_groups(D, goff);
  const unsigned long long w = real ? mask - min((unsigned long long)work[slot], mask) : mask;
  key[slot] = ((unsigned long long)r << wbits) | w;
  iota[slot] = (unsigned)slot;
}

// A system's final group records and frame origins, in work order.
__global__ void order_groups_kernel(const SysDesc *__restrict__ d, const long *__restrict__ goffs,
                                    int R, long G, const int *__restrict__ goff,
                                    const unsigned *__restrict__ ord,
                                    const int4 *__restrict__ gin, const double4 *__restrict__ cin,
                                    bool half) {
  const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= G) return;
  const int r = owner(goffs, R, k);
  const SysDesc &D = d[r];
  const long dest = k - D.g_off;
  if (dest >= sys_groups(D, goff)) return;
  const long s = ord[k];
  (half ? D.hgroups : D.groups)[dest] = gin[s];
  (half ? D.hcen : D.gcen)[dest] = cin[s];
}

__global__ void collect_counts_kernel(const SysDesc *__restrict__ d, int R,
                                      const SysStats *__restrict__ st,
                                      const int *__restrict__ goff, const int *__restrict__ pos,
                                      const int *__restrict__ segoff,
                                      const int *__restrict__ hsegoff,
                                      SetupCounts *__restrict__ out) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= R) return;
  const SysDesc &D = d[r];
  out[r].bad = st[r].bad;
  out[r].cand = st[r].cand;
  out[r].hcand = st[r].hcand;
  out[r].ngroups = (int)sys_groups(D, goff);
  out[r].nnonempty = pos[D.b_off + D.nbt] - pos[D.b_off];
  out[r].nsegs = segoff[D.g_off + D.ngb] - segoff[D.g_off];
  out[r].nhsegs = hsegoff[D.g_off + D.ngb] - hsegoff[D.g_off];
}

int bits_for(unsigned long long v) {  // bits to hold values < v
  int b = 1;
  while (b < 64 && (1ull << b) < v) b++;
  return b;
}

inline unsigned blocks_for(long n, int t = 256) { return (unsigned)((n + t - 1) / t); }

// Scratch buffers of the set-up, kept by the handle that owns a batch (the
// first) and reused by its next set-up.
enum Scratch {
  kPts, kBKey, kBKeyOut, kIota, kBPerm, kCKey, kSKey, kKeyOut, kCOrder, kSOrder, kBOrder,
  kCounts3, kBStart, kFlag, kPos, kCStart, kSStart, kZs, kCPos, kFCPos, kGCount, kGOff,
  kGRec, kBLo, kBHi, kCen, kGroupCounters, kSegOff, kHSegOff, kUGroups, kUHGroups,
  kWKey, kWKeyOut, kOrd, kGIota, kStats, kSysStats, kDesc, kOffs, kCub, kBPos, kCountsDev,
  kScratchCount
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
  const int rc = handle_buffer(h, &h->d_su[i], std::max<size_t>(bytes, 16));
  *out = (P *)h->d_su[i];
  return rc;
}

// CUB temporary storage of at least `bytes`
int cub_tmp(npme_handle *h, size_t bytes, void **out) {
  return scratch(h, kCub, std::max<size_t>(bytes, 256), out);
}

// stable radix sort of (key, value) pairs on bits [0, end_bit), ascending
template <typename K>
int sort_pairs(npme_handle *h, const K *kin, K *kout, const unsigned *vin, unsigned *vout,
               long n, int end_bit, cudaStream_t s) {
  size_t tb = 0;
  SCK(cub::DeviceRadixSort::SortPairs(nullptr, tb, kin, kout, vin, vout, (int)n, 0, end_bit, s));
  void *tmp;
  int rc;
  if ((rc = cub_tmp(h, tb, &tmp))) return rc;
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

// Host side of one system: its binning geometry (and the handle's refine2),
// its sizes and its output buffers.
template <typename T>
int describe(npme_handle *h, SysDesc &D) {
  const long n = (long)h->n;
  const GridGeom &gr = h->grid;
  const double *R = h->box + 3, *L = h->box + 6;
  int rc;
  BinGeom &g = D.g;
  for (int a = 0; a < 3; a++) {
    g.N[a] = (double)gr.N[a], g.L[a] = L[a], g.R[a] = R[a];
    g.Nl[a] = gr.N[a], g.H[a] = gr.H[a], g.nb[a] = gr.nb[a];
  }
  g.P = gr.order;
  g.TL = kBrick + gr.order - 1;
  g.nkeys = 32 / ((int)(sizeof(T) / 4) * (h->complex_kernel ? 2 : 1));
  // direct-sum columns: edge e ~ (32 / density)^(1/3) over the bounding box
  // (degenerate axes are given a nominal thickness of Rdir / 4)
  const double Rd = h->p.Rdir;
  double vol = 1.0;
  for (int a = 0; a < 3; a++) vol *= std::max(h->bmax[a] - h->bmin[a], 0.25 * Rd);
  double e = std::cbrt(32.0 * vol / (double)n);
  e = std::max(e, 1e-3 * Rd);
  for (int a = 0; a < 2; a++) {
    const double ext = h->bmax[a] - h->bmin[a];
    g.nc[a] = std::max(1, std::min((int)std::ceil(ext / e), 1 << 14));
    g.edge[a] = std::max(ext / g.nc[a], 1e-12);
    g.ns[a] = g.nc[a] * kSourceSplit;
    g.sedge[a] = g.edge[a] / kSourceSplit;
    g.mn[a] = h->bmin[a];
  }
  {
    const double H = h->bmax[2] - h->bmin[2];
    g.zbits = std::max(8, std::min(kZField,
                                   (int)std::ceil(std::log2(std::max(1.0, 1024.0 * H / e)))));
    g.zmin = h->bmin[2];
    g.zscale = (double)((1u << g.zbits) - 1u) / std::max(H, 1e-300);
  }
  GroupGeom &gg = D.gg;
  gg.R = Rd, gg.R2 = Rd * Rd;
  for (int a = 0; a < 2; a++) gg.mn[a] = g.mn[a], gg.sedge[a] = g.sedge[a], gg.ns[a] = g.ns[a];
  gg.nc1 = g.nc[1];
  gg.zmin = g.zmin, gg.zscale = g.zscale, gg.zbits = g.zbits;
  // heads of offsets up to ~the group half-diagonal carry ~6e-8 e absolute
  // error; below r = e/4 the relative error would exceed ~1e-6, so refine
  h->refine2 = (0.25 * e) * (0.25 * e);
  D.n = n;
  D.nbt = gr.nb[0] * gr.nb[1] * gr.nb[2];
  D.ncol = (long)g.nc[0] * g.nc[1];
  D.nscol = (long)g.ns[0] * g.ns[1];
  h->n_bricks = D.nbt;
  // Upper bounds (the kernels read the actual counts on the device; the
  // host reads them once the set-up has completed):
  //   groups   <= n / 32 + non-empty columns <= n / 32 + min(n, ncol)
  //   segments <= groups x the fine columns of a group's window (a group lies
  //               in one coarse column, so its window spans at most
  //               (edge + 2 Rdir) / sedge + 4 fine columns per axis)
  //   non-empty bricks <= min(n, nbt)
  D.ngb = n / 32 + std::min(n, D.ncol) + 1;
  long wmax = 1;
  for (int a = 0; a < 2; a++)
    wmax *= std::min<long>(g.ns[a], (long)std::floor((g.edge[a] + 2.0 * Rd) / g.sedge[a]) + 4);
  const long nsb = D.ngb * wmax;
  if (nsb >= (1L << 31))  // int offsets in the group records
    return record_error(h, NPME_EINVAL, "too many direct-sum source segments (2^31)");
  const int C = h->complex_kernel ? 2 : 1;
  if ((rc = handle_buffer(h, &h->d_bpts, sizeof(BrickPoint<T>) * n)) ||
      (rc = handle_buffer(h, (void **)&h->d_brick_start, sizeof(int) * (D.nbt + 1))) ||
      (rc = handle_buffer(h, (void **)&h->d_brick_list,
                          sizeof(int) * std::max<long>(1, std::min(n, D.nbt)))) ||
      (rc = handle_buffer(h, (void **)&h->d_cperm, sizeof(uint32_t) * n)) ||
      (rc = handle_buffer(h, (void **)&h->d_sperm, sizeof(uint32_t) * n)) ||
      (rc = handle_buffer(h, (void **)&h->d_bperm, sizeof(uint32_t) * n)) ||
      (rc = handle_buffer(h, (void **)&h->d_gpos, sizeof(double4) * n)) ||
      (rc = handle_buffer(h, (void **)&h->d_spos, sizeof(double4) * n)) ||
      (rc = handle_buffer(h, (void **)&h->d_segs, sizeof(int2) * nsb)) ||
      (rc = handle_buffer(h, (void **)&h->d_hsegs, sizeof(int2) * nsb)) ||
      (rc = handle_buffer(h, (void **)&h->d_groups, sizeof(int4) * D.ngb)) ||
      (rc = handle_buffer(h, (void **)&h->d_gcen, sizeof(double4) * D.ngb)) ||
      (rc = handle_buffer(h, (void **)&h->d_hgroups, sizeof(int4) * D.ngb)) ||
      (rc = handle_buffer(h, (void **)&h->d_hcen, sizeof(double4) * D.ngb)) ||
      (rc = handle_buffer(h, &h->d_qb, sizeof(T) * C * n)) ||
      (rc = handle_buffer(h, &h->d_qc, sizeof(T) * C * n)) ||
      (rc = handle_buffer(h, (void **)&h->d_q_in, sizeof(double) * C * n)) ||
      (rc = handle_buffer(h, (void **)&h->d_V, sizeof(double) * 4 * C * n)))
    return rc;
  // source-side sums of the pair-once walk start (and are kept) at zero
  if (h->fp32) {
    if ((rc = handle_buffer(h, (void **)&h->d_vsrc, sizeof(float4) * C * n))) return rc;
    cudaMemsetAsync(h->d_vsrc, 0, sizeof(float4) * C * n, h->stream);
  } else {
    if ((rc = handle_buffer(h, (void **)&h->d_vsrc64, sizeof(double) * 4 * n))) return rc;
    cudaMemsetAsync(h->d_vsrc64, 0, sizeof(double) * 4 * n, h->stream);
  }
  // grids
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
  D.coord = h->d_coord;
  D.bpts = h->d_bpts;
  D.brick_start = h->d_brick_start;
  D.brick_list = h->d_brick_list;
  D.cperm = h->d_cperm, D.sperm = h->d_sperm, D.bperm = h->d_bperm;
  D.gpos = h->d_gpos, D.spos = h->d_spos;
  D.segs = h->d_segs, D.hsegs = h->d_hsegs;
  D.groups = h->d_groups, D.hgroups = h->d_hgroups;
  D.gcen = h->d_gcen, D.hcen = h->d_hcen;
  h->d_dperm = h->d_sperm;  // direct-sum charges are gathered into the source order
  return NPME_OK;
}

// Brick order, direct-sum orders, warp groups and segment lists of R systems
// of one precision in one pass on stream s (h0 = hs[0] owns the scratch).
// Enqueued without waiting; the counts arrive in h0->h_counts with the
// caller's synchronisation.
template <typename T>
int geometry_batch(npme_handle **hs, int R, cudaStream_t s) {
  npme_handle *h = hs[0];
  int rc;
  std::vector<SysDesc> ds(R);
  long P = 0, B = 0, C = 0, S = 0, G = 0, nmax = 1, nbtmax = 1, ncolmax = 1, nscolmax = 1;
  for (int r = 0; r < R; r++) {
    if ((rc = describe<T>(hs[r], ds[r]))) {
      if (hs[r] != h) h->err = hs[r]->err;
      return rc;
    }
    SysDesc &D = ds[r];
    D.p_off = P, D.b_off = B, D.c_off = C, D.s_off = S, D.g_off = G;
    P += D.n, B += D.nbt + 1, C += D.ncol + 1, S += D.nscol + 1, G += D.ngb;
    nmax = std::max(nmax, D.n), nbtmax = std::max(nbtmax, D.nbt);
    ncolmax = std::max(ncolmax, D.ncol), nscolmax = std::max(nscolmax, D.nscol);
    // the system's coordinates and buffers (on its own stream) come first
    if (hs[r]->stream != s) {
      SCK(cudaEventRecord(hs[r]->ev_fork, hs[r]->stream));
      SCK(cudaStreamWaitEvent(s, hs[r]->ev_fork, 0));
    }
  }
  if (P >= (1L << 31) || B >= (1L << 31) || G >= (1L << 31))
    return record_error(h, NPME_EINVAL, "set-up batch too large for 32-bit indices");
  const int rbits = bits_for((unsigned long long)R);
  const int bbits = bits_for(nbtmax), cbits = bits_for(ncolmax), sbits = bits_for(nscolmax);
  const int wbits = bits_for((unsigned long long)nmax + 1) + 1;
  if (rbits + bbits + 5 > 64 || rbits + sbits + kZField > 64)
    return record_error(h, NPME_EINVAL, "set-up batch keys exceed 64 bits");

  // descriptors and the index-space starts (points, bricks, columns, fine
  // columns, groups), R each
  SysDesc *dd;
  long *offs;
  if ((rc = scratch(h, kDesc, sizeof(SysDesc) * R, &dd)) ||
      (rc = scratch(h, kOffs, sizeof(long) * 5 * R, &offs)))
    return rc;
  // staged in pinned memory: a copy from pageable memory would first wait
  // for everything enqueued on s
  static_assert(sizeof(SysDesc) % sizeof(long) == 0, "descriptor alignment");
  if ((rc = pinned_block(h, &h->h_desc, &h->desc_cap, (sizeof(SysDesc) + sizeof(long) * 5) * R)))
    return rc;
  SysDesc *hd = static_cast<SysDesc *>(h->h_desc);
  long *ho = reinterpret_cast<long *>(hd + R);
  for (int r = 0; r < R; r++) {
    hd[r] = ds[r];
    ho[r] = ds[r].p_off, ho[R + r] = ds[r].b_off, ho[2 * R + r] = ds[r].c_off;
    ho[3 * R + r] = ds[r].s_off, ho[4 * R + r] = ds[r].g_off;
  }
  SCK(cudaMemcpyAsync(dd, hd, sizeof(SysDesc) * R, cudaMemcpyHostToDevice, s));
  SCK(cudaMemcpyAsync(offs, ho, sizeof(long) * 5 * R, cudaMemcpyHostToDevice, s));
  const long *poff = offs, *boff = offs + R, *coff = offs + 2 * R, *goffs = offs + 4 * R;

  BrickPoint<T> *pts;
  unsigned long long *bkey, *bkey_out, *ckey, *skey, *key_out;
  unsigned *iota, *border, *corder, *sorder, *border2, *bpos, *zs, *cpos, *fcpos;
  int *counts, *bstart, *flag, *pos, *cstart, *sstart, *gcount, *goff;
  SysStats *st;
  if ((rc = scratch(h, kPts, sizeof(BrickPoint<T>) * P, &pts)) ||
      (rc = scratch(h, kBKey, sizeof(unsigned long long) * P, &bkey)) ||
      (rc = scratch(h, kBKeyOut, sizeof(unsigned long long) * P, &bkey_out)) ||
      (rc = scratch(h, kCKey, sizeof(unsigned long long) * P, &ckey)) ||
      (rc = scratch(h, kSKey, sizeof(unsigned long long) * P, &skey)) ||
      (rc = scratch(h, kKeyOut, sizeof(unsigned long long) * P, &key_out)) ||
      (rc = scratch(h, kIota, sizeof(unsigned) * P, &iota)) ||
      (rc = scratch(h, kBPerm, sizeof(unsigned) * P, &border)) ||
      (rc = scratch(h, kBOrder, sizeof(unsigned) * P, &border2)) ||
      (rc = scratch(h, kCOrder, sizeof(unsigned) * P, &corder)) ||
      (rc = scratch(h, kSOrder, sizeof(unsigned) * P, &sorder)) ||
      (rc = scratch(h, kBPos, sizeof(unsigned) * P, &bpos)) ||
      (rc = scratch(h, kZs, sizeof(unsigned) * P, &zs)) ||
      (rc = scratch(h, kCPos, sizeof(unsigned) * P, &cpos)) ||
      (rc = scratch(h, kFCPos, sizeof(unsigned) * P, &fcpos)) ||
      (rc = scratch(h, kCounts3, sizeof(int) * (B + C + S), &counts)) ||
      (rc = scratch(h, kBStart, sizeof(int) * B, &bstart)) ||
      (rc = scratch(h, kFlag, sizeof(int) * B, &flag)) ||
      (rc = scratch(h, kPos, sizeof(int) * B, &pos)) ||
      (rc = scratch(h, kCStart, sizeof(int) * C, &cstart)) ||
      (rc = scratch(h, kSStart, sizeof(int) * S, &sstart)) ||
      (rc = scratch(h, kGCount, sizeof(int) * C, &gcount)) ||
      (rc = scratch(h, kGOff, sizeof(int) * C, &goff)) ||
      (rc = scratch(h, kSysStats, sizeof(SysStats) * R, &st)))
    return rc;
  int *bcount = counts, *ccount = counts + B, *scount = counts + B + C;

  // --- binning: records, keys and counts of every point ---
  SCK(cudaMemsetAsync(counts, 0, sizeof(int) * (B + C + S), s));
  init_sys_stats_kernel<<<blocks_for(R, 64), 64, 0, s>>>(dd, R, st);
  bin_kernel<T><<<blocks_for(P), 256, 0, s>>>(dd, poff, R, P, bbits, cbits, sbits, pts, bkey,
                                              ckey, skey, iota, bcount, ccount, scount, st);
  SCK(cudaGetLastError());

  // --- brick order: by (system, brick), inside a brick in rounds over the
  // banks: a sort by (system, brick, bank, index), then each brick's banks
  // interleaved in rounds ---
  if ((rc = sort_pairs(h, bkey, bkey_out, iota, border, P, rbits + bbits + 5, s))) return rc;
  if ((rc = exclusive_sum(h, bcount, bstart, B, s))) return rc;
  round_place_kernel<<<blocks_for(32 * B), 256, 0, s>>>(bkey_out, border, bstart, bcount, B,
                                                       border2);
  place_bricks_kernel<T><<<blocks_for(P), 256, 0, s>>>(dd, poff, R, P, border2, pts, bpos);
  nonempty_flags_kernel<<<blocks_for(B), 256, 0, s>>>(bcount, B, flag);
  if ((rc = exclusive_sum(h, flag, pos, B, s))) return rc;
  bricks_kernel<<<blocks_for(B), 256, 0, s>>>(dd, boff, R, B, bcount, bstart, pos);

  // --- direct-sum orders: (system, column, quantised z, index) for targets
  // and sources, one radix sort each ---
  if ((rc = sort_pairs(h, ckey, key_out, iota, corder, P, rbits + cbits + kZField, s)) ||
      (rc = sort_pairs(h, skey, key_out, iota, sorder, P, rbits + sbits + kZField, s)))
    return rc;
  place_orders_kernel<<<blocks_for(P), 256, 0, s>>>(dd, poff, R, P, corder, sorder, key_out, bpos,
                                                    zs, cpos);
  gather_u32_kernel<<<blocks_for(P), 256, 0, s>>>(cpos, sorder, P, fcpos);
  if ((rc = exclusive_sum(h, ccount, cstart, C, s))) return rc;
  if ((rc = exclusive_sum(h, scount, sstart, S, s))) return rc;
  groups_per_column_kernel<<<blocks_for(C), 256, 0, s>>>(ccount, C, gcount);
  if ((rc = exclusive_sum(h, gcount, goff, C, s))) return rc;
  SCK(cudaGetLastError());

  // --- warp groups and their source segments ---
  int4 *grec, *ug, *uh;
  double4 *blo, *bhi, *cen;
  int *nseg, *segoff, *hsegoff;
  unsigned long long *wkey, *wkey_out;
  unsigned *ord, *giota;
  if ((rc = scratch(h, kGRec, sizeof(int4) * G, &grec)) ||
      (rc = scratch(h, kBLo, sizeof(double4) * G, &blo)) ||
      (rc = scratch(h, kBHi, sizeof(double4) * G, &bhi)) ||
      (rc = scratch(h, kCen, sizeof(double4) * G, &cen)) ||
      (rc = scratch(h, kGroupCounters, sizeof(int) * 4 * (G + 1), &nseg)) ||
      (rc = scratch(h, kSegOff, sizeof(int) * (G + 1), &segoff)) ||
      (rc = scratch(h, kHSegOff, sizeof(int) * (G + 1), &hsegoff)) ||
      (rc = scratch(h, kUGroups, sizeof(int4) * G, &ug)) ||
      (rc = scratch(h, kUHGroups, sizeof(int4) * G, &uh)) ||
      (rc = scratch(h, kWKey, sizeof(unsigned long long) * G, &wkey)) ||
      (rc = scratch(h, kWKeyOut, sizeof(unsigned long long) * G, &wkey_out)) ||
      (rc = scratch(h, kOrd, sizeof(unsigned) * G, &ord)) ||
      (rc = scratch(h, kGIota, sizeof(unsigned) * G, &giota)))
    return rc;
  // segment counts and work of both lists in one block, one clear (spare
  // slots of the bounds: no segments, no work)
  int *nhseg = nseg + (G + 1);
  unsigned *work = (unsigned *)(nhseg + (G + 1)), *hwork = work + (G + 1);
  SCK(cudaMemsetAsync(nseg, 0, sizeof(int) * 4 * (G + 1), s));
  group_records_kernel<<<blocks_for(C), 256, 0, s>>>(dd, coff, R, C, cstart, goff, grec);
  group_box_kernel<<<blocks_for(32 * G), 256, 0, s>>>(dd, goffs, R, G, goff, grec, blo, bhi, cen);
  group_segments_kernel<false><<<blocks_for(32 * G), 256, 0, s>>>(
      dd, goffs, R, G, goff, grec, blo, bhi, sstart, zs, fcpos, nseg, nhseg, work, hwork, nullptr,
      nullptr, nullptr, nullptr, st);
  if ((rc = exclusive_sum(h, nseg, segoff, G + 1, s))) return rc;
  if ((rc = exclusive_sum(h, nhseg, hsegoff, G + 1, s))) return rc;
  group_segments_kernel<true><<<blocks_for(32 * G), 256, 0, s>>>(
      dd, goffs, R, G, goff, grec, blo, bhi, sstart, zs, fcpos, nullptr, nullptr, nullptr,
      nullptr, segoff, hsegoff, ug, uh, st);
  // heaviest groups first, so that the last wave of a direct-sum launch
  // holds the light ones (each list by its own work; ties keep the column
  // order)
  for (int half = 0; half < 2; half++) {
    work_key_kernel<<<blocks_for(G), 256, 0, s>>>(dd, goffs, R, G, goff, half ? hwork : work,
                                                  wbits, wkey, giota);
    if ((rc = sort_pairs(h, wkey, wkey_out, giota, ord, G, rbits + wbits, s))) return rc;
    order_groups_kernel<<<blocks_for(G), 256, 0, s>>>(dd, goffs, R, G, goff, ord,
                                                      half ? uh : ug, cen, half != 0);
  }
  // the counts, for the host to read when the set-up has completed
  SetupCounts *dc;
  if ((rc = scratch(h, kCountsDev, sizeof(SetupCounts) * R, &dc))) return rc;
  if ((rc = pinned_block(h, &h->h_counts, &h->counts_cap, sizeof(SetupCounts) * R))) return rc;
  collect_counts_kernel<<<blocks_for(R, 64), 64, 0, s>>>(dd, R, st, goff, pos, segoff, hsegoff,
                                                         dc);
  SCK(cudaMemcpyAsync(h->h_counts, dc, sizeof(SetupCounts) * R, cudaMemcpyDeviceToHost, s));
  SCK(cudaGetLastError());
  return NPME_OK;
}

}  // namespace

int device_bbox(npme_handle *h, const double *coord, double mn[3], double mx[3]) {
  const long n = (long)h->n;
  cudaStream_t s = h->stream;
  int rc;
  if ((rc = handle_buffer(h, (void **)&h->d_coord, sizeof(double) * 3 * n))) return rc;
  SCK(cudaMemcpyAsync(h->d_coord, coord, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s));
  if (n < kHostBoxPoints) {
    // small systems: one host pass costs less than a device reduction and
    // the wait for it
    for (int a = 0; a < 3; a++) mn[a] = 1e300, mx[a] = -1e300;
    for (long i = 0; i < n; i++)
      for (int a = 0; a < 3; a++) {
        const double x = coord[3 * i + a];
        if (!std::isfinite(x)) return record_error(h, NPME_EINVAL, "non-finite coordinate");
        mn[a] = std::min(mn[a], x);
        mx[a] = std::max(mx[a], x);
      }
    SCK(cudaGetLastError());
    return NPME_OK;
  }
  SetupStats *st;
  if ((rc = scratch(h, kStats, sizeof(SetupStats), &st))) return rc;
  init_stats_kernel<<<1, 1, 0, s>>>(st);
  const unsigned blocks = (unsigned)std::min<long>(blocks_for(n), 148 * 8);
  bbox_kernel<<<blocks, 256, 0, s>>>(h->d_coord, n, st);
  SCK(cudaGetLastError());
  SetupStats hs;
  SCK(cudaMemcpyAsync(&hs, st, sizeof(hs), cudaMemcpyDeviceToHost, s));
  SCK(cudaStreamSynchronize(s));
  if (hs.nonfinite) return record_error(h, NPME_EINVAL, "non-finite coordinate");
  for (int a = 0; a < 3; a++) mn[a] = dkey_inv(hs.mn[a]), mx[a] = dkey_inv(hs.mx[a]);
  return NPME_OK;
}

int setup_geometry(npme_handle **hs, int R, cudaStream_t s) {
  return hs[0]->fp32 ? geometry_batch<float>(hs, R, s) : geometry_batch<double>(hs, R, s);
}

int finish_setup(npme_handle *h, const npme_handle *owner, int r) {
  const SetupCounts &c = static_cast<const SetupCounts *>(owner->h_counts)[r];
  const long n = (long)h->n;
  if (c.bad < n) {
    // the axis of the first offending point, from its coordinates
    double x[3];
    SCK(cudaMemcpy(x, h->d_coord + 3 * c.bad, sizeof(x), cudaMemcpyDeviceToHost));
    const GridGeom &gr = h->grid;
    const double *R = h->box + 3, *L = h->box + 6;
    int axis = 0;
    for (int a = 0; a < 3; a++) {
      const double w = (double)gr.N[a] / L[a] * (x[a] - R[a]);
      const long ms = w < 0 ? (long)(-w) + 1 : (long)(-w);
      const long o = ms + gr.N[a] / 4;
      if (o < 0 || o + gr.order - 1 > gr.H[a] - 1) {
        axis = a;
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

}  // namespace npme
