// Batched CalcV: many set-up systems (different sizes, kernels, B-spline
// orders and FFT boxes) in one pass, one launch per stage and launch class.
//
// A launch class groups the systems a single kernel instantiation can serve:
//   gather, multiply        -> real / complex charges
//   spread, interpolation   -> (B-spline order, real / complex)
//   direct sum              -> identical pair-kernel coefficients (kernel,
//                              split, Rdir, nDeriv, alpha, k0); the
//                              coefficients stay in the parameter bank, as in
//                              the single-system launch
// Each class launch gets a device array of per-system descriptors and the
// prefix sums of its work units (points, bricks, spectrum elements, warp
// groups); a thread finds its system by binary search over the prefix.  The
// FFTs run per system with each handle's cuFFT plans.  FP32-bulk handles use
// the batch kernels; FP64 handles run their ordinary single-system path in
// the same stream order.  Results equal the single-system path's: the same
// bodies (bodies.cuh) run on the same data.
#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "bodies.cuh"
#include "internal.h"

namespace npme {

struct BatchSys {
  const double *q;  // caller charges (device)
  double *V;        // caller output (device)
  const BrickPoint<float> *bpts;
  const uint32_t *cperm;  // targets: group order -> caller index
  const uint32_t *dperm;  // direct-sum sources: source order -> caller index
  float *qb, *qc;
  const int *brick_list, *brick_start;
  int nb2, nb3;
  float *grid;    // real N1 N2 N3 (real kernels) or complex (Helmholtz)
  float2 *kgrid;  // R2C half spectrum (real kernels)
  const float *G;
  long N1, N2, N3;
  float c1, c2, c3;
  const double4 *gpos, *spos;
  const int4 *groups;
  const double4 *gcen;
  const int2 *segs;
  // pair-once walk: half-shell groups and segments, source-side sums
  const int4 *hgroups;
  const double4 *hcen;
  const int2 *hsegs;
  float4 *vsrc;            // source-side sums, slot = brick-order position
  const uint32_t *bperm;   // brick-order position -> caller index
  float refine2;
  double fself_r, fself_i;
  // pair-once systems: the interpolation adds the source-side sums into V
  // (potential times vs, gradient times gs) and clears them
  int fold;
  double vs, gs;
};

__device__ __forceinline__ int find_sys(const long long *__restrict__ off, int count,
                                        long long u) {
  int lo = 0, hi = count - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= u) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

template <bool CPLX>
__global__ void batch_gather_kernel(const BatchSys *__restrict__ sys,
                                    const long long *__restrict__ off, int count) {
  const long long total = off[count];
  for (long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x; u < total;
       u += (long long)gridDim.x * blockDim.x) {
    const int s = find_sys(off, count, u);
    const BatchSys &S = sys[s];
    gather_body<float, CPLX>(S.q, S.bpts, S.dperm, S.qb, S.qc, (long)(u - off[s]));
  }
}

template <int P, bool CPLX>
__global__ void __launch_bounds__(256) batch_spread_kernel(const BatchSys *__restrict__ sys,
                                                           const long long *__restrict__ off,
                                                           int count) {
  extern __shared__ unsigned char smem_raw[];
  const long long u = blockIdx.x;
  const int s = find_sys(off, count, u);
  const BatchSys &S = sys[s];
  spread_brick_fixed<P, CPLX>(S.brick_list[u - off[s]], S.brick_start, S.bpts, S.qb, S.grid,
                              S.nb2, S.nb3, S.N1, S.N2, S.N3, reinterpret_cast<int *>(smem_raw));
}

// one warp per spectrum row of one system (units: rows)
template <bool CPLX>
__global__ void batch_multiply_kernel(const BatchSys *__restrict__ sys,
                                      const long long *__restrict__ off, int count) {
  const long long total = off[count];
  const int lane = threadIdx.x & 31;
  for (long long u = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; u < total;
       u += (gridDim.x * (long long)blockDim.x) >> 5) {
    const int s = find_sys(off, count, u);
    const BatchSys &S = sys[s];
    const int M2 = (int)(S.N2 / 2 + 1), M3 = (int)(S.N3 / 2 + 1);
    const int r = (int)(u - off[s]);
    if (CPLX)
      multiply_cplx_row<float>(reinterpret_cast<float2 *>(S.grid),
                               reinterpret_cast<const float2 *>(S.G), r, (int)S.N1, (int)S.N2,
                               (int)S.N3, M2, M3, lane);
    else
      multiply_real_row<float>(S.kgrid, S.G, r, (int)S.N1, (int)S.N2, (int)(S.N3 / 2 + 1), M2,
                               M3, lane);
  }
}

template <int P, bool CPLX>
__global__ void __launch_bounds__(256) batch_interp_kernel(const BatchSys *__restrict__ sys,
                                                           const long long *__restrict__ off,
                                                           int count) {
  extern __shared__ unsigned char smem_raw[];
  const long long u = blockIdx.x;
  const int s = find_sys(off, count, u);
  const BatchSys &S = sys[s];
  interp_brick_body<float, P, CPLX>(S.brick_list[u - off[s]], S.brick_start, S.bpts, S.grid, S.V,
                                    S.nb2, S.nb3, S.N1, S.N2, S.N3, S.c1, S.c2, S.c3,
                                    reinterpret_cast<float *>(smem_raw),
                                    S.fold ? (void *)S.vsrc : nullptr, S.vs, S.gs);
}

template <bool CPLX, int FUNC, int SPLIT, int ND>
__global__ void __launch_bounds__(32 * kGroupWarps, kGroupMinBlocks) batch_direct_kernel(
    PairCoef<float> k, const BatchSys *__restrict__ sys, const long long *__restrict__ off,
    int count) {
  __shared__ float4 sp[kGroupWarps][32];
  __shared__ float4 slo[kGroupWarps][32];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long u = (long long)blockIdx.x * kGroupWarps + wid;
  if (u >= off[count]) return;  // warp-uniform
  const int s = find_sys(off, count, u);
  const BatchSys &S = sys[s];
  const long g = (long)(u - off[s]);
  direct_group_body<CPLX, FUNC, SPLIT, ND>(k, S.gpos, S.spos, S.qc, S.q, S.groups[g], S.gcen[g],
                                           S.segs, S.cperm, S.refine2, S.fself_r, S.fself_i, S.V,
                                           sp[wid], slo[wid], lane);
}

// Pair-once direct sums of a batch (direct_group_sym and its complex and
// scalar forms): KIND 0 the packed real DM body, 1 Helmholtz DM, 2 the scalar
// body of the original Ewald split.
template <int KIND, int FUNC, int ND>
__global__ void __launch_bounds__(32 * kGroupWarps) batch_sym_kernel(
    PairCoef<float> k, const BatchSys *__restrict__ sys, const long long *__restrict__ off,
    int count) {
  __shared__ float4 ta[kGroupWarps][32];
  __shared__ float4 tb[kGroupWarps][32];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long u = (long long)blockIdx.x * kGroupWarps + wid;
  if (u >= off[count]) return;  // warp-uniform
  const int s = find_sys(off, count, u);
  const BatchSys &S = sys[s];
  const long g = (long)(u - off[s]);
  if constexpr (KIND == 0)
    direct_group_sym<FUNC, ND>(k, S.gpos, S.spos, S.qc, S.q, S.hgroups[g], S.hcen[g], S.hsegs,
                               S.cperm, S.refine2, S.fself_r, S.V, S.vsrc, ta[wid], tb[wid],
                               lane);
  else if constexpr (KIND == 1)
    direct_group_sym_helm<ND>(k, S.gpos, S.spos, S.qc, S.q, S.hgroups[g], S.hcen[g], S.hsegs,
                              S.cperm, S.refine2, S.fself_r, S.fself_i, S.V, S.vsrc, ta[wid],
                              tb[wid], lane);
  else
    direct_group_sym_scalar<0, 1, 0>(k, S.gpos, S.spos, S.qc, S.q, S.hgroups[g], S.hcen[g],
                                     S.hsegs, S.cperm, S.refine2, S.fself_r, S.V, S.vsrc,
                                     ta[wid], tb[wid], lane);
}

}  // namespace npme

using npme::BatchSys;

struct npme_batch {
  int device = 0;
  cudaStream_t stream2 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_done = nullptr;
  bool pending = false;  // ev_done recorded: buffers and members may be in use
  unsigned char *h_pinned = nullptr;  // host image of the descriptor block
  size_t h_cap = 0;
  unsigned char *d_block = nullptr;
  size_t d_cap = 0;
  std::string err;
  int launches = 0;
};

namespace {

int bfail(npme_batch *b, int code, const std::string &m) {
  if (b) b->err = m;
  return code;
}

// One launch class: the systems it serves and the prefix of its work units.
struct Class {
  std::vector<int> members;  // indices into the batch's FP32 handle list
  std::vector<long long> off;   // prefix of the class's work units
  size_t desc_at = 0, off_at = 0;  // byte offsets in the descriptor block
};

size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

}  // namespace

extern "C" {

int npme_gpu_batch_create(int device, npme_batch **out) {
  if (!out) return NPME_EINVAL;
  *out = nullptr;
  npme_batch *b = new (std::nothrow) npme_batch;
  if (!b) return NPME_ENOMEM;
  b->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream2, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_done, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    delete b;
    return NPME_ECUDA;
  }
  *out = b;
  return NPME_OK;
}

int npme_gpu_batch_destroy(npme_batch *b) {
  if (!b) return NPME_OK;
  cudaSetDevice(b->device);
  if (b->pending) cudaEventSynchronize(b->ev_done);
  if (b->stream2) cudaStreamSynchronize(b->stream2);
  if (b->stream2) cudaStreamDestroy(b->stream2);
  if (b->ev_fork) cudaEventDestroy(b->ev_fork);
  if (b->ev_join) cudaEventDestroy(b->ev_join);
  if (b->ev_done) cudaEventDestroy(b->ev_done);
  if (b->h_pinned) cudaFreeHost(b->h_pinned);
  if (b->d_block) cudaFree(b->d_block);
  delete b;
  return NPME_OK;
}

int npme_gpu_batch_sync(npme_batch *b) {
  if (!b) return NPME_EINVAL;
  if (cudaSetDevice(b->device) != cudaSuccess) return bfail(b, NPME_ECUDA, "cudaSetDevice");
  cudaError_t e = cudaSuccess;
  if (b->pending) e = cudaEventSynchronize(b->ev_done);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream2);
  b->pending = false;
  if (e != cudaSuccess) return bfail(b, NPME_ECUDA, cudaGetErrorString(e));
  return NPME_OK;
}

int npme_gpu_batch_last_error(const npme_batch *b, char *buf, size_t len) {
  if (!b || !buf || len == 0) return NPME_EINVAL;
  strncpy(buf, b->err.c_str(), len - 1);
  buf[len - 1] = 0;
  return NPME_OK;
}

int npme_gpu_calcv_batch(npme_batch *b, npme_handle *const *hs, int count,
                         double *const *d_V, const double *const *d_q, void *stream) {
  using namespace npme;
  if (!b) return NPME_EINVAL;
  if (count < 0 || (count > 0 && (!hs || !d_V || !d_q)))
    return bfail(b, NPME_EINVAL, "bad batch arguments");
  if (count == 0) return NPME_OK;
  for (int i = 0; i < count; i++) {
    if (!hs[i] || !hs[i]->ready) return bfail(b, NPME_ESTATE, "batch member not set up");
    if (hs[i]->device != b->device) return bfail(b, NPME_EINVAL, "batch member on another device");
    if (!d_V[i] || !d_q[i]) return bfail(b, NPME_EINVAL, "null buffer in batch");
  }
  if (cudaSetDevice(b->device) != cudaSuccess) return bfail(b, NPME_ECUDA, "cudaSetDevice");
  cudaStream_t s = (cudaStream_t)stream;
  b->launches = 0;

  // FP64 (plain) and caller-defined-kernel members take their ordinary path
  // in stream order
  std::vector<int> f32;
  for (int i = 0; i < count; i++) {
    if (hs[i]->fp32 && !hs[i]->user_kernel) {
      f32.push_back(i);
    } else {
      const int rc = npme_gpu_calcv_device(hs[i], d_V[i], d_q[i], stream);
      if (rc) return bfail(b, rc, "batch member: " + hs[i]->err);
      b->launches += hs[i]->launches;
    }
  }
  const int m = (int)f32.size();
  if (m == 0) {
    // the members' own CalcVs are on `stream`: npme_gpu_batch_sync waits for them
    if (cudaEventRecord(b->ev_done, s) != cudaSuccess)
      return bfail(b, NPME_ECUDA, "batch: event record failed");
    b->pending = true;
    return NPME_OK;
  }

  // descriptors
  std::vector<BatchSys> desc(m);
  for (int k = 0; k < m; k++) {
    const npme_handle *h = hs[f32[k]];
    BatchSys &S = desc[k];
    memset(&S, 0, sizeof(S));
    S.q = d_q[f32[k]];
    S.V = d_V[f32[k]];
    S.bpts = (const BrickPoint<float> *)h->d_bpts;
    S.cperm = h->d_cperm;
    S.dperm = h->d_dperm;
    S.qb = (float *)h->d_qb;
    S.qc = (float *)h->d_qc;
    S.brick_list = h->d_brick_list;
    S.brick_start = h->d_brick_start;
    S.nb2 = (int)h->grid.nb[1];
    S.nb3 = (int)h->grid.nb[2];
    S.grid = (float *)h->d_grid;
    S.kgrid = (float2 *)h->d_kgrid;
    S.G = (const float *)h->d_G;
    S.N1 = h->grid.N[0], S.N2 = h->grid.N[1], S.N3 = h->grid.N[2];
    S.c1 = (float)(h->grid.N[0] / h->box[6]);
    S.c2 = (float)(h->grid.N[1] / h->box[7]);
    S.c3 = (float)(h->grid.N[2] / h->box[8]);
    S.gpos = h->d_gpos;
    S.spos = h->d_spos;
    S.groups = h->d_groups;
    S.gcen = h->d_gcen;
    S.segs = h->d_segs;
    S.hgroups = h->d_hgroups;
    S.hcen = h->d_hcen;
    S.hsegs = h->d_hsegs;
    S.vsrc = h->d_vsrc;
    S.bperm = h->d_bperm;
    S.refine2 = (float)h->refine2;
    S.fself_r = h->fself_r;
    S.fself_i = h->fself_i;
    S.fold = pairs_once(h) ? 1 : 0;
    const bool scaled =
        h->p.funcType != NPME_FUNC_HELMHOLTZ && h->p.EwaldSplit != NPME_SPLIT_LAPLACE_ORIG;
    const PairCoef<float> pc = make_pair_coef<float>(h);
    S.vs = scaled ? pc.vscale : 1.0;
    S.gs = scaled ? pc.gscale : 1.0;
  }

  // launch classes
  std::map<int, Class> gath, mult;                           // key: complex
  std::map<std::pair<int, int>, Class> spr;                  // (order, complex)
  typedef std::tuple<int, int, int, int, double, double, double, double, double> DKey;
  std::map<DKey, Class> dir;  // direct sums
  for (int k = 0; k < m; k++) {
    const npme_handle *h = hs[f32[k]];
    const int cx = h->complex_kernel ? 1 : 0;
    gath[cx].members.push_back(k);
    mult[cx].members.push_back(k);
    spr[{h->grid.order, cx}].members.push_back(k);
    const DKey key(pairs_once(h) ? 1 : 0, h->p.funcType, h->p.EwaldSplit, h->p.nDeriv,
                   h->p.Rdir, h->p.alpha, h->p.k0_r, h->p.k0_i, h->beta);
    dir[key].members.push_back(k);
  }
  auto units_gather = [&](int k) { return (long long)hs[f32[k]]->n; };
  auto units_spread = [&](int k) { return (long long)hs[f32[k]]->n_nonempty; };
  auto units_mult = [&](int k) {  // spectrum rows
    const long *N = hs[f32[k]]->grid.N;
    return (long long)N[0] * N[1];
  };
  auto units_dir = [&](int k) {
    const npme_handle *h = hs[f32[k]];
    return (long long)(pairs_once(h) ? h->n_hgroups : h->n_groups);
  };

  // descriptor block layout: for every class, its descriptors then offsets
  size_t bytes = 0;
  std::vector<Class *> all;
  auto lay = [&](Class &c, auto units) {
    c.off.assign(c.members.size() + 1, 0);
    for (size_t t = 0; t < c.members.size(); t++) c.off[t + 1] = c.off[t] + units(c.members[t]);
    c.desc_at = bytes;
    bytes = align16(bytes + sizeof(BatchSys) * c.members.size());
    c.off_at = bytes;
    bytes = align16(bytes + sizeof(long long) * c.off.size());
    all.push_back(&c);
  };
  for (auto &kv : gath) lay(kv.second, units_gather);
  for (auto &kv : mult) lay(kv.second, units_mult);
  for (auto &kv : spr) lay(kv.second, units_spread);  // spread and interpolation: bricks
  for (auto &kv : dir) lay(kv.second, units_dir);

  // the pinned staging buffer is reused: wait for the previous batch's copy
  if (b->pending) {
    cudaEventSynchronize(b->ev_done);
    b->pending = false;
  }
  if (bytes > b->h_cap) {
    if (b->h_pinned) cudaFreeHost(b->h_pinned);
    b->h_pinned = nullptr;
    b->h_cap = 0;
    // at least 1 MiB: a serving loop then never grows it (cudaMallocHost /
    // cudaFreeHost are slow and take driver locks other threads wait for)
    const size_t cap = std::max<size_t>(bytes * 2, size_t(1) << 20);
    if (cudaMallocHost((void **)&b->h_pinned, cap) != cudaSuccess)
      return bfail(b, NPME_ENOMEM, "pinned descriptor buffer");
    b->h_cap = cap;
  }
  if (bytes > b->d_cap) {
    if (b->d_block) cudaFree(b->d_block);
    b->d_block = nullptr;
    b->d_cap = 0;
    // the same floor: cudaFree waits for the whole device
    const size_t cap = std::max<size_t>(bytes * 2, size_t(1) << 20);
    if (cudaMalloc((void **)&b->d_block, cap) != cudaSuccess)
      return bfail(b, NPME_ENOMEM, "device descriptor buffer");
    b->d_cap = cap;
  }
  for (Class *c : all) {
    BatchSys *dd = (BatchSys *)(b->h_pinned + c->desc_at);
    for (size_t t = 0; t < c->members.size(); t++) dd[t] = desc[c->members[t]];
    memcpy(b->h_pinned + c->off_at, c->off.data(), sizeof(long long) * c->off.size());
  }
  cudaMemcpyAsync(b->d_block, b->h_pinned, bytes, cudaMemcpyHostToDevice, s);
  auto D = [&](const Class &c) { return (const BatchSys *)(b->d_block + c.desc_at); };
  auto O = [&](const Class &c) { return (const long long *)(b->d_block + c.off_at); };
  auto grid_of = [](long long units, int threads, int cap) {
    return (unsigned)std::max<long long>(1, std::min<long long>((units + threads - 1) / threads, cap));
  };

  // 1. gather
  for (auto &kv : gath) {
    Class &c = kv.second;
    const unsigned g = grid_of(c.off.back(), 256, 148 * 16);
    if (kv.first) batch_gather_kernel<true><<<g, 256, 0, s>>>(D(c), O(c), (int)c.members.size());
    else batch_gather_kernel<false><<<g, 256, 0, s>>>(D(c), O(c), (int)c.members.size());
    b->launches++;
  }
  // 2. direct sums on the second stream, overlapped with the reciprocal sums
  cudaEventRecord(b->ev_fork, s);
  cudaStreamWaitEvent(b->stream2, b->ev_fork, 0);
  for (auto &kv : dir) {
    Class &c = kv.second;
    const npme_handle *h0 = hs[f32[c.members[0]]];
    const PairCoef<float> k = make_pair_coef<float>(h0);
    const long long ng = c.off.back();
    if (ng == 0) continue;
    const unsigned g = (unsigned)((ng + kGroupWarps - 1) / kGroupWarps);
    const int cnt = (int)c.members.size();
    const int f = h0->p.funcType, sp = h0->p.EwaldSplit, nd = sp == 1 ? 0 : h0->p.nDeriv;
    if (std::get<0>(kv.first)) {  // pair-once walk, then the source-side sums
#define NPME_BSYM(KD, FN, ND) \
  batch_sym_kernel<KD, FN, ND><<<g, 32 * kGroupWarps, 0, b->stream2>>>(k, D(c), O(c), cnt)
#define NPME_BSYM_ND(KD, FN)                \
  switch (nd) {                             \
    case 3: NPME_BSYM(KD, FN, 3); break;    \
    case 6: NPME_BSYM(KD, FN, 6); break;    \
    case 8: NPME_BSYM(KD, FN, 8); break;    \
    default: NPME_BSYM(KD, FN, 0); break;   \
  }
      if (f == NPME_FUNC_HELMHOLTZ) { NPME_BSYM_ND(1, 2); }
      else if (sp == NPME_SPLIT_LAPLACE_ORIG) { NPME_BSYM(2, 0, 0); }
      else if (f == NPME_FUNC_RALPHA) { NPME_BSYM_ND(0, 1); }
      else { NPME_BSYM_ND(0, 0); }
#undef NPME_BSYM_ND
#undef NPME_BSYM
      // the source-side sums are folded into V by the interpolation below
      b->launches++;
      continue;
    }
#define NPME_BD(CX, FN, SL, ND) \
  batch_direct_kernel<CX, FN, SL, ND><<<g, 32 * kGroupWarps, 0, b->stream2>>>(k, D(c), O(c), cnt)
#define NPME_BD_ND(CX, FN, SL)               \
  switch (nd) {                              \
    case 3: NPME_BD(CX, FN, SL, 3); break;   \
    case 6: NPME_BD(CX, FN, SL, 6); break;   \
    case 8: NPME_BD(CX, FN, SL, 8); break;   \
    default: NPME_BD(CX, FN, SL, 0); break;  \
  }
    if (f == NPME_FUNC_HELMHOLTZ) { NPME_BD_ND(true, 2, 0); }
    else if (sp == NPME_SPLIT_LAPLACE_ORIG) { NPME_BD(false, 0, 1, 0); }
    else if (f == NPME_FUNC_RALPHA) { NPME_BD_ND(false, 1, 0); }
    else { NPME_BD_ND(false, 0, 0); }
#undef NPME_BD_ND
#undef NPME_BD
    b->launches++;
  }
  cudaEventRecord(b->ev_join, b->stream2);
  // 3. spread (grids zeroed first)
  for (int k = 0; k < m; k++) {
    grid_clear(hs[f32[k]], s);
  }
  for (auto &kv : spr) {
    Class &c = kv.second;
    const long long nb = c.off.back();
    if (nb == 0) continue;
    const int P = kv.first.first;
    const bool cx = kv.first.second;
    const int cnt = (int)c.members.size();
#define NPME_BS(PP, CX)                                                                    \
  {                                                                                        \
    constexpr int TL = kBrick + PP - 1;                                                    \
    const size_t smem = 2 * sizeof(int) * TL * TL * TL * (CX ? 2 : 1);                     \
    auto kern = batch_spread_kernel<PP, CX>;                                               \
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);   \
    kern<<<(unsigned)nb, 256, smem, s>>>(D(c), O(c), cnt);                                 \
  }
#define NPME_BS_P(CX)                    \
  switch (P) {                           \
    case 4: NPME_BS(4, CX); break;       \
    case 6: NPME_BS(6, CX); break;       \
    case 8: NPME_BS(8, CX); break;       \
    case 10: NPME_BS(10, CX); break;     \
    case 12: NPME_BS(12, CX); break;     \
    case 14: NPME_BS(14, CX); break;     \
    case 16: NPME_BS(16, CX); break;     \
  }
    if (cx) { NPME_BS_P(true); } else { NPME_BS_P(false); }
#undef NPME_BS_P
#undef NPME_BS
    b->launches++;
  }
  {  // launch errors are checked before cuFFT runs
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return bfail(b, NPME_ECUDA, std::string("batch: ") + cudaGetErrorString(e));
  }
  // 4. forward transforms
  for (int k = 0; k < m; k++) {
    npme_handle *h = hs[f32[k]];
    if (fft_forward(h, s)) return bfail(b, NPME_ECUDA, "batch: " + h->err);
  }
  // 5. kernel multiply
  for (auto &kv : mult) {
    Class &c = kv.second;
    const unsigned g = grid_of(c.off.back(), 8, 148 * 16);  // 8 rows (warps) per CTA
    if (kv.first) batch_multiply_kernel<true><<<g, 256, 0, s>>>(D(c), O(c), (int)c.members.size());
    else batch_multiply_kernel<false><<<g, 256, 0, s>>>(D(c), O(c), (int)c.members.size());
    b->launches++;
  }
  {  // launch errors are checked before cuFFT runs
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return bfail(b, NPME_ECUDA, std::string("batch: ") + cudaGetErrorString(e));
  }
  // 6. inverse transforms
  for (int k = 0; k < m; k++) {
    npme_handle *h = hs[f32[k]];
    if (fft_inverse(h, s)) return bfail(b, NPME_ECUDA, "batch: " + h->err);
  }
  // 7. interpolation after the direct sums
  cudaStreamWaitEvent(s, b->ev_join, 0);
  for (auto &kv : spr) {
    Class &c = kv.second;
    const int P = kv.first.first;
    const bool cx = kv.first.second;
    const long long nb = c.off.back();
    if (nb == 0) continue;
    const int cnt = (int)c.members.size();
#define NPME_BI(PP, CX)                                                                    \
  {                                                                                        \
    constexpr int TL = kBrick + PP - 1;                                                    \
    const size_t smem = sizeof(float) * TL * TL * TL * (CX ? 2 : 1);                       \
    auto kern = batch_interp_kernel<PP, CX>;                                               \
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);   \
    kern<<<(unsigned)nb, 256, smem, s>>>(D(c), O(c), cnt);                                 \
  }
#define NPME_BI_P(CX)                   \
  switch (P) {                          \
    case 4: NPME_BI(4, CX); break;      \
    case 6: NPME_BI(6, CX); break;      \
    case 8: NPME_BI(8, CX); break;      \
    case 10: NPME_BI(10, CX); break;    \
    case 12: NPME_BI(12, CX); break;    \
    case 14: NPME_BI(14, CX); break;    \
    case 16: NPME_BI(16, CX); break;    \
  }
    if (cx) { NPME_BI_P(true); } else { NPME_BI_P(false); }
#undef NPME_BI_P
#undef NPME_BI
    b->launches++;
  }
  cudaEventRecord(b->ev_done, s);
  b->pending = true;
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return bfail(b, NPME_ECUDA, std::string("batch: ") + cudaGetErrorString(e));
  return NPME_OK;
}

}  // extern "C"
