// C ABI of npme_b200 (include/npme_gpu.h): parameter handling, set-up
// (derivative-match coefficients, box, point binning, buffers, FFT plans,
// kernel transform) and the CalcV orchestration on CUDA streams.
#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "internal.h"


namespace {

std::mutex g_err_mu;
std::string g_err;

void set_global_err(const std::string &s) {
  std::lock_guard<std::mutex> lk(g_err_mu);
  g_err = s;
}

int fail(npme_handle *h, int code, const std::string &msg) {
  if (h) h->err = msg;
  else set_global_err(msg);
  return code;
}

#define CK(call)                                                                  \
  do {                                                                            \
    cudaError_t e_ = (call);                                                      \
    if (e_ != cudaSuccess)                                                        \
      return fail(h, NPME_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define CKFFT(call)                                                              \
  do {                                                                           \
    cufftResult r_ = (call);                                                     \
    if (r_ != CUFFT_SUCCESS)                                                     \
      return fail(h, NPME_ECUDA, std::string(#call) + ": cufft error " + std::to_string((int)r_)); \
  } while (0)

// --- derivative-match coefficients (FP64, host) ---------------------------
// (1/r d/dr)^n f at Rdir: r^alpha (src/FunctionDerivMatch.cpp:76-88) and
// exp(i k0 r)/r (src/FunctionDerivMatch.cpp:42-55); a_n by back substitution
// and b_n = 2 (n+1) a_{n+1} (src/FunctionDerivMatch.cpp:226-266).
using cd = std::complex<double>;

double calc_cnp(int n, int p, double R) {
  if (n > p) return 0.0;
  double c = 1.0;
  for (int i = 0; i < p - n; i++) c *= R * R;
  for (int i = 0; i < n; i++) c *= 2.0;
  for (int i = p - n + 1; i <= p; i++) c *= (double)i;
  return c;
}

void dm_coefficients(const npme_params &p, cd *a, cd *b) {
  const int N = p.nDeriv;
  const double R = p.Rdir, r2 = R * R;
  cd f[32];
  if (p.funcType == NPME_FUNC_HELMHOLTZ) {
    const cd k0(p.k0_r, p.k0_i), I(0, 1);
    const cd C = std::exp(I * k0 * R), A = k0 * k0 / r2;
    f[0] = C / R;
    if (N >= 1) f[1] = -C / R / r2 + I * k0 * C / r2;
    for (int n = 2; n <= N; n++) f[n] = -(2.0 * n - 1.0) / r2 * f[n - 1] - A * f[n - 2];
  } else {
    const double alpha = p.funcType == NPME_FUNC_LAPLACE ? -1.0 : p.alpha;
    f[0] = std::pow(R, alpha);
    for (int n = 1; n <= N; n++) f[n] = f[n - 1] * (alpha - 2 * n + 2) / r2;
  }
  for (int q = 0; q <= N; q++) {
    cd s = f[N - q];
    for (int t = 0; t < q; t++) s -= calc_cnp(N - q, N - t, R) * a[N - t];
    a[N - q] = s / calc_cnp(N - q, N - q, R);
  }
  for (int i = 0; i <= N - 1; i++) b[i] = a[i + 1] * 2.0 * (double)(i + 1);
  b[N] = 0;
}

// beta with erfc(beta Rdir)/Rdir ~ tol (src/KernelFunctionLaplace.cpp:41-76)
double orig_beta(double R, double tol) {
  const double C = std::log(std::sqrt(M_PI) * tol * R);
  double x = 0.1;
  for (int n = 0; n < 1000; n++) {
    const double F0 = x * x + std::log(x) + C, F1 = 2 * x + 1.0 / x;
    if (std::fabs(F0) < 1e-12) return x / R;
    x -= F0 / F1;
  }
  return -1.0;
}

// src/RecSumSupportFunctions.cpp:137-147
double min_x_compact(double X0, double del, long order, long N) {
  const double a1 = 1.0 - 2.0 * (order + 1) / N;
  const double a2 = 1.0 - 4.0 * (order + 1) / N;
  const double X = X0 / a1 - del / 2.0 * a2 / a1;
  return X0 > X ? X0 : X;
}


// Device memory of all handles comes from one stream-ordered pool per device
// (cudaMallocFromPoolAsync / cudaFreeAsync on the handle's stream).  Unlike
// cudaMalloc / cudaFree, neither synchronises the device, so a handle that
// grows its buffers during set-up does not stall the CalcV of other handles
// running meanwhile; freed blocks stay in the pool for the next handle.  The
// pool returns its memory to the device when the last handle of the device
// is destroyed.
std::mutex g_pool_mu;
std::map<int, std::pair<cudaMemPool_t, int>> g_pools;  // device -> (pool, live handles)

// The device's pool, created on first use; *count gets its live users.
// Caller holds g_pool_mu.
static int pool_get(int device, cudaMemPool_t *out, std::string &err) {
  auto it = g_pools.find(device);
  if (it == g_pools.end()) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool;
    cudaError_t e = cudaMemPoolCreate(&pool, &props);
    if (e != cudaSuccess) {
      err = std::string("cudaMemPoolCreate: ") + cudaGetErrorString(e);
      return NPME_ECUDA;
    }
    unsigned long long keep = ~0ull;  // keep freed blocks for reuse
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    it = g_pools.emplace(device, std::make_pair(pool, 0)).first;
  }
  it->second.second++;
  *out = it->second.first;
  return NPME_OK;
}

int pool_acquire(npme_handle *h) {
  std::lock_guard<std::mutex> lk(g_pool_mu);
  std::string err;
  const int rc = pool_get(h->device, &h->pool, err);
  return rc ? fail(h, rc, err) : NPME_OK;
}

// One live user less; the last one returns the pool's memory to the device.
static void pool_put(int device) {
  std::lock_guard<std::mutex> lk(g_pool_mu);
  auto it = g_pools.find(device);
  if (it != g_pools.end() && --it->second.second == 0) cudaMemPoolTrimTo(it->second.first, 0);
}

void pool_release(npme_handle *h) {
  if (!h->pool) return;
  pool_put(h->device);
  h->pool = nullptr;
}

// Frees every device buffer of the handle (stream-ordered; the caller has
// synchronised the handle's streams).
void release(npme_handle *h) {
  h->pf = h->pi = h->px = nullptr;  // shared plans stay in the process-wide cache
  h->d_dperm = nullptr;
  // every device buffer was obtained through dalloc, which records the
  // address of the pointer field it fills
  for (auto &kv : h->caps) {
    void **field = (void **)kv.first;
    if (*field) cudaFreeAsync(*field, h->stream);
    *field = nullptr;
  }
  if (!h->caps.empty()) cudaStreamSynchronize(h->stream);
  h->caps.clear();
  h->n_groups = h->n_segs = 0;
  h->n_hgroups = h->n_hsegs = 0;
  h->dev_bytes = 0;
  h->ready = false;
}

// Device buffer of at least `bytes`: reused when the handle already holds a
// large enough one (set-up of a new geometry on the same handle allocates
// only what grew), otherwise freed and allocated again from the pool, in
// the order of the handle's stream.  A buffer that grows takes half again
// its old capacity at least, so a handle serving systems of varying sizes
// settles after a few growths instead of reallocating (and the pool
// reserving more memory) on every larger system.
template <typename P>
int dalloc(npme_handle *h, P **ptr, size_t bytes) {
  if (bytes == 0) bytes = 16;
  size_t &cap = h->caps[(void *)ptr];
  if (*ptr && cap >= bytes) return NPME_OK;
  size_t want = bytes;
  if (*ptr) {
    want = std::max(bytes, cap + cap / 2);
    cudaFreeAsync(*ptr, h->stream);
    h->dev_bytes -= cap;
    *ptr = nullptr;
    cap = 0;
  }
  cudaError_t e = cudaMallocFromPoolAsync((void **)ptr, want, h->pool, h->stream);
  if (e != cudaSuccess && want > bytes) {  // no room for the headroom: exact size
    cudaGetLastError();
    want = bytes;
    e = cudaMallocFromPoolAsync((void **)ptr, want, h->pool, h->stream);
  }
  bytes = want;
  if (e != cudaSuccess) {
    *ptr = nullptr;
    cudaGetLastError();
    return fail(h, NPME_ENOMEM, "device allocation of " + std::to_string(bytes) +
                                    " bytes failed: " + cudaGetErrorString(e));
  }
  cap = bytes;
  h->dev_bytes += bytes;
  return NPME_OK;
}

}  // namespace

namespace {
std::mutex g_pinned_mu;
std::multimap<size_t, void *> g_pinned;  // capacity -> idle pinned block
size_t g_pinned_bytes = 0;               // bytes held by idle blocks
constexpr size_t kPinnedKeep = 256ull << 20;  // above: idle blocks are freed
}  // namespace

int npme::pinned_block(npme_handle *h, void **block, size_t *cap, size_t bytes) {
  if (*block && *cap >= bytes) return NPME_OK;
  pinned_return(block, cap);
  // power-of-two capacities (at least 4 KiB), so blocks are reused across sizes
  size_t want = 4096;
  while (want < bytes) want <<= 1;
  {
    std::lock_guard<std::mutex> lk(g_pinned_mu);
    auto it = g_pinned.lower_bound(want);
    if (it != g_pinned.end() && it->first <= 4 * want) {
      *block = it->second, *cap = it->first;
      g_pinned_bytes -= it->first;
      g_pinned.erase(it);
      return NPME_OK;
    }
  }
  cudaError_t e = cudaHostAlloc(block, want, cudaHostAllocDefault);
  if (e != cudaSuccess) {
    *block = nullptr, *cap = 0;
    cudaGetLastError();
    return fail(h, NPME_ENOMEM, std::string("pinned host allocation: ") + cudaGetErrorString(e));
  }
  *cap = want;
  return NPME_OK;
}

void npme::pinned_return(void **block, size_t *cap) {
  if (!*block) return;
  bool keep;
  {
    std::lock_guard<std::mutex> lk(g_pinned_mu);
    keep = g_pinned_bytes + *cap <= kPinnedKeep;
    if (keep) g_pinned.emplace(*cap, *block), g_pinned_bytes += *cap;
  }
  if (!keep) cudaFreeHost(*block);
  *block = nullptr, *cap = 0;
}

int npme::pool_reserve(int device, size_t bytes) {
  cudaMemPool_t pool;
  std::string err;
  {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (pool_get(device, &pool, err)) return NPME_ECUDA;
  }
  size_t cur = 0;
  cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &cur);
  if (cur < bytes) {
    // one allocation of the difference, freed at once: the pool keeps the
    // memory (its release threshold is unlimited) and hands it out later
    cudaStream_t st = nullptr;
    void *q = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess) {
      if (cudaMallocFromPoolAsync(&q, bytes - cur, pool, st) == cudaSuccess) cudaFreeAsync(q, st);
      cudaStreamSynchronize(st);
      cudaStreamDestroy(st);
    }
    cudaGetLastError();  // not enough memory: the pool grows on demand instead
  }
  return NPME_OK;
}

void npme::pool_unreserve(int device) { pool_put(device); }

double npme::compact_extent(double X0, double del, long order, long N) {
  return min_x_compact(X0, del, order, N);
}

int npme::handle_buffer(npme_handle *h, void **field, size_t bytes) {
  return dalloc(h, field, bytes);
}

int npme::record_error(npme_handle *h, int code, const std::string &msg) {
  return fail(h, code, msg);
}

namespace {

int check_params(npme_handle *h, const npme_params &p) {
  if (!(p.Rdir > 0)) return fail(h, NPME_EINVAL, "Rdir must be > 0");
  if (p.funcType < 0 || p.funcType > 3) return fail(h, NPME_EINVAL, "unknown funcType");
  if (p.funcType == NPME_FUNC_USER && p.EwaldSplit != NPME_SPLIT_DERIVMATCH)
    return fail(h, NPME_EINVAL, "a user kernel brings its own split (EwaldSplit DerivMatch)");
  if (p.EwaldSplit < 0 || p.EwaldSplit > 1) return fail(h, NPME_EINVAL, "unknown EwaldSplit");
  if (p.EwaldSplit == NPME_SPLIT_LAPLACE_ORIG && p.funcType != NPME_FUNC_LAPLACE)
    return fail(h, NPME_EINVAL, "EwaldSplit LaplaceOrig requires funcType Laplace");
  if (p.EwaldSplit == NPME_SPLIT_LAPLACE_ORIG && !(p.tol > 0 && p.tol < 1))
    return fail(h, NPME_EINVAL, "tol must be in (0, 1)");
  if (p.EwaldSplit == NPME_SPLIT_DERIVMATCH && (p.nDeriv < 2 || p.nDeriv > npme::kMaxDeriv))
    return fail(h, NPME_EINVAL, "nDeriv must be in [2, 15]");
  if (p.BnOrder < 4 || p.BnOrder > 16 || (p.BnOrder & 1))
    return fail(h, NPME_EINVAL, "BnOrder must be even and in [4, 16]");
  const long Ns[3] = {p.N1, p.N2, p.N3};
  for (int d = 0; d < 3; d++) {
    if (Ns[d] % 4 != 0 || Ns[d] < 4)  // src/RecSumSupportFunctions.cpp:42-58
      return fail(h, NPME_EINVAL, "N1, N2, N3 must be positive multiples of 4");
    if (p.BnOrder >= Ns[d] / 4)  // src/RecSumSupportFunctions.cpp:61-79
      return fail(h, NPME_EINVAL, "BnOrder must be < N/4 on every axis");
    if (Ns[d] > 2048) return fail(h, NPME_EINVAL, "N1, N2, N3 must be <= 2048");
  }
  if (p.nNeigh < 1 || p.nNeigh > 4) return fail(h, NPME_EINVAL, "nNeigh must be in [1, 4]");
  if (p.precision != NPME_PREC_FP32 && p.precision != NPME_PREC_FP64)
    return fail(h, NPME_EINVAL, "unknown precision");
  return NPME_OK;
}

// Derived state of the parameters: kernel kind, precision and the splitting
// coefficients (host FP64).
int apply_params(npme_handle *h) {
  h->user_kernel = h->p.funcType == NPME_FUNC_USER;
  h->complex_kernel = h->user_kernel ? h->uops.complex_kernel != 0
                                     : h->p.funcType == NPME_FUNC_HELMHOLTZ;
  h->fp32 = h->p.precision == NPME_PREC_FP32;
  memset(h->a_r, 0, sizeof(h->a_r));
  memset(h->a_i, 0, sizeof(h->a_i));
  memset(h->b_r, 0, sizeof(h->b_r));
  memset(h->b_i, 0, sizeof(h->b_i));
  h->beta = 0;
  if (h->user_kernel) {  // the caller's functors define the split
    h->fself_r = h->uops.direct ? h->uops.fself : 0.0;
    h->fself_i = h->uops.direct ? h->uops.fself_i : 0.0;
  } else if (h->p.EwaldSplit == NPME_SPLIT_DERIVMATCH) {
    std::complex<double> a[32], b[32];
    dm_coefficients(h->p, a, b);
    for (int i = 0; i <= h->p.nDeriv; i++) {
      h->a_r[i] = a[i].real(), h->a_i[i] = a[i].imag();
      h->b_r[i] = b[i].real(), h->b_i[i] = b[i].imag();
    }
    // f_LR(0) = a[0] (src/Interface.cpp:1946-1952)
    h->fself_r = h->a_r[0];
    h->fself_i = h->a_i[0];
  } else {
    h->beta = orig_beta(h->p.Rdir, h->p.tol);
    if (h->beta <= 0) return fail(h, NPME_EINVAL, "original-Ewald beta did not converge");
    h->fself_r = 2.0 * h->beta / std::sqrt(M_PI);  // beta erf(beta r)/(beta r) at r = 0
    h->fself_i = 0;
  }
  return NPME_OK;
}

void fill_default_del(npme_params &p) {
  if (p.del1 <= 0) p.del1 = p.Rdir;
  if (p.del2 <= 0) p.del2 = p.Rdir;
  if (p.del3 <= 0) p.del3 = p.Rdir;
}

}  // namespace

// Set-up in three stages: per handle, the checks, coordinates and box
// (setup_prepare); for all handles at once, the geometry on the device
// (npme::setup_geometry), then per handle the FFT plans and for all handles
// the kernel transforms (npme::build_kernel_transforms); then one wait and
// the counts (npme::finish_setup).
static int setup_prepare(npme_handle *h, size_t n, const double *coord) {
  if (!h) return fail(nullptr, NPME_EINVAL, "null handle");
  if (h->user_kernel && !h->uops.direct)
    return fail(h, NPME_ESTATE, "user kernel: npme_gpu_set_user_kernel before setup");
  if (!coord && n) return fail(h, NPME_EINVAL, "null coord");
  if (n == 0) return fail(h, NPME_EINVAL, "nCharge must be > 0");
  if (n >= (size_t)1 << 31) return fail(h, NPME_EINVAL, "nCharge must be < 2^31");
  CK(cudaSetDevice(h->device));
  {
    // load the no-allocation entry point's static scratch now, while the
    // caller allows allocation (a failure shows up in that entry point)
    std::string ignored;
    npme::noalloc_preload(ignored);
  }
  // A handle that was set up before keeps its buffers (grown when needed),
  // its FFT plans (the FFT box is a handle parameter) and its kernel-transform
  // scratch: only the geometry-dependent state is rebuilt (ResetCoord,
  // src/Interface.cpp:1958-1987).
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->stream2) cudaStreamSynchronize(h->stream2);
  h->ready = false;
  h->setup_gen++;  // a captured CalcV belongs to the previous geometry
  h->n = n;
  const npme_params &p = h->p;
  // box (src/RecSumSupportFunctions.cpp:182-201, 276-296) from the points'
  // bounding box
  double mx[3], mn[3];
  int rc = npme::device_bbox(h, coord, mn, mx);
  if (rc) return rc;
  for (int d = 0; d < 3; d++) h->bmin[d] = mn[d], h->bmax[d] = mx[d];
  const long Ns[3] = {p.N1, p.N2, p.N3};
  const double dels[3] = {p.del1, p.del2, p.del3};
  for (int d = 0; d < 3; d++) {
    const double X0 = mx[d] - mn[d], R0 = 0.5 * (mx[d] + mn[d]);
    const double X = min_x_compact(X0, dels[d], p.BnOrder, Ns[d]);
    h->box[d] = X;
    h->box[3 + d] = R0 + 0.5 * (X0 - X);
    h->box[6 + d] = 2 * (X + dels[d]);
    h->grid.N[d] = Ns[d];
    h->grid.H[d] = Ns[d] / 2;
    h->grid.nb[d] = (Ns[d] / 2 + npme::kBrick - 1) / npme::kBrick;
  }
  h->grid.order = p.BnOrder;
  // the reference's cells of edge >= Rdir / nNeigh (reported by
  // npme_gpu_get_info; the direct sum walks warp groups instead)
  const double target = p.Rdir / p.nNeigh;
  for (int d = 0; d < 3; d++) {
    const double ext = mx[d] - mn[d];
    int nc = (int)std::floor(ext / target);
    nc = std::max(1, std::min(nc, 1 << 16));
    h->cells.nc[d] = nc;
    h->cells.edge[d] = (nc == 1) ? std::max(ext, target) : ext / nc;
    h->cells.origin[d] = mn[d];
  }
  h->cells.reach = p.nNeigh;
  // the built-in kernels evaluate every pair once unless NPME_PAIRS_ONCE=0
  {
    const char *e = std::getenv("NPME_PAIRS_ONCE");
    h->use_sym = !(e && e[0] == '0');
  }
  return NPME_OK;
}

int npme::setup_many(npme_handle **hs, int R, const size_t *n, const double *const *coord,
                     int *status) {
  std::vector<int> st(R, NPME_OK);
  // per handle: checks, coordinates, box
  for (int r = 0; r < R; r++) {
    npme::StepTimer t("set-up: checks, coordinates, box", n[r]);
    st[r] = setup_prepare(hs[r], n[r], coord[r]);
  }
  // the geometry of the prepared handles, one pass per precision
  for (int prec = 0; prec < 2; prec++) {
    std::vector<npme_handle *> group;
    std::vector<int> idx;
    for (int r = 0; r < R; r++)
      if (!st[r] && hs[r]->fp32 == (prec == 0)) group.push_back(hs[r]), idx.push_back(r);
    if (group.empty()) continue;
    npme_handle *owner = group[0];
    int rc;
    {
      npme::StepTimer t("set-up: geometry enqueue", group.size());
      rc = npme::setup_geometry(group.data(), (int)group.size(), owner->stream);
    }
    if (rc) {
      for (size_t k = 0; k < group.size(); k++) {
        if (group[k] != owner) group[k]->err = owner->err;
        st[idx[k]] = rc;
      }
      continue;
    }
    std::vector<npme_handle *> kt;
    std::vector<int> kidx;
    for (size_t k = 0; k < group.size(); k++) {
      st[idx[k]] = npme::prepare_plans(group[k]);
      if (!st[idx[k]]) kt.push_back(group[k]), kidx.push_back(idx[k]);
    }
    if (!kt.empty()) {
      npme::StepTimer t("set-up: kernel transforms enqueue", kt.size());
      std::vector<int> kst(kt.size(), NPME_OK);
      npme::build_kernel_transforms(kt.data(), (int)kt.size(), owner, kst.data());
      for (size_t k = 0; k < kt.size(); k++) st[kidx[k]] = kst[k];
    }
    npme::StepTimer t_wait("set-up: wait for the device and read the counts", group.size());
    // the owner's stream carries the shared passes; every handle's stream
    // its own transform: CalcV may be enqueued on any stream, so the set-up
    // completes here (and the counts arrive)
    for (size_t k = 0; k < group.size(); k++) {
      npme_handle *h = group[k];
      const cudaError_t e = cudaStreamSynchronize(h->stream);
      if (e != cudaSuccess && !st[idx[k]])
        st[idx[k]] = fail(h, NPME_ECUDA, std::string("set-up: ") + cudaGetErrorString(e));
    }
    for (size_t k = 0; k < group.size(); k++)
      if (!st[idx[k]]) st[idx[k]] = npme::finish_setup(group[k], owner, (int)k);
  }
  int all = NPME_OK;
  for (int r = 0; r < R; r++) {
    if (st[r] && hs[r]) release(hs[r]);
    if (!st[r]) hs[r]->ready = true;
    if (status) status[r] = st[r];
    if (st[r] && !all) all = st[r];
  }
  return all;
}

extern "C" {

void npme_gpu_default_params(npme_params *p) {
  if (!p) return;
  memset(p, 0, sizeof(*p));
  p->funcType = NPME_FUNC_LAPLACE;
  p->EwaldSplit = NPME_SPLIT_DERIVMATCH;
  p->alpha = -1.0;
  p->Rdir = 0.0;      // required
  p->tol = 1.0e-6;    // src/Constant.h:50
  p->BnOrder = 8;     // src/Constant.h:49
  p->nDeriv = 8;      // src/Interface.cpp:452-455 for BnOrder 8
  p->n1 = p->n2 = p->n3 = 16;
  p->a1 = p->a2 = p->a3 = 4.0;    // src/Interface.cpp:97-99
  p->del1 = p->del2 = p->del3 = -1.0;  // < 0 means Rdir (src/Interface.cpp:243-245)
  p->nNeigh = 2;        // src/Constant.h:52
  p->nCellClust1D = 3;  // src/Constant.h:53
  p->useCompactF = 1;
  p->precision = NPME_PREC_FP32;
  p->device = 0;
}

int npme_gpu_create(const npme_params *p, npme_handle **out) {
  if (!p || !out) return fail(nullptr, NPME_EINVAL, "null argument");
  *out = nullptr;
  npme_handle *h = new (std::nothrow) npme_handle;
  if (!h) return fail(nullptr, NPME_ENOMEM, "host allocation failed");
  h->p = *p;
  fill_default_del(h->p);
  int rc = check_params(h, h->p);
  if (rc) {
    set_global_err(h->err);
    delete h;
    return rc;
  }
  h->device = p->device;
  cudaError_t e = cudaSetDevice(h->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->stream2, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming);
  for (int i = 0; i < 10 && e == cudaSuccess; i++) e = cudaEventCreate(&h->timing.ev[i]);
  if (e != cudaSuccess) {
    set_global_err(std::string("CUDA initialisation failed: ") + cudaGetErrorString(e));
    npme_gpu_destroy(h);
    return NPME_ECUDA;
  }
  if ((rc = pool_acquire(h))) {
    set_global_err(h->err);
    npme_gpu_destroy(h);
    return rc;
  }
  if ((rc = apply_params(h))) {
    set_global_err(h->err);
    npme_gpu_destroy(h);
    return rc;
  }
  *out = h;
  return NPME_OK;
}

int npme_gpu_set_params(npme_handle *h, const npme_params *p) {
  if (!h) return fail(nullptr, NPME_EINVAL, "null handle");
  if (!p) return fail(h, NPME_EINVAL, "null params");
  if (p->device != h->device) return fail(h, NPME_EINVAL, "set_params cannot change the device");
  npme_params q = *p;
  fill_default_del(q);
  int rc = check_params(h, q);
  if (rc) return rc;
  CK(cudaSetDevice(h->device));
  // work already enqueued may still read the handle's buffers and plans
  if (h->stream) CK(cudaStreamSynchronize(h->stream));
  if (h->stream2) CK(cudaStreamSynchronize(h->stream2));
  const npme_params old = h->p;
  h->p = q;
  if ((rc = apply_params(h))) {
    h->p = old;
    apply_params(h);
    return rc;
  }
  h->ready = false;  // buffers and plans are kept; setup rebuilds the rest
  h->setup_gen++;
  return NPME_OK;
}

int npme_gpu_set_user_kernel(npme_handle *h, const npme_user_ops *ops) {
  if (!h) return fail(nullptr, NPME_EINVAL, "null handle");
  if (!ops || !ops->direct || !ops->sample_lr || !ops->exact)
    return fail(h, NPME_EINVAL, "incomplete user kernel table");
  if (!h->user_kernel) return fail(h, NPME_EINVAL, "the handle's funcType is not NPME_FUNC_USER");
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->stream2) cudaStreamSynchronize(h->stream2);
  h->uops = *ops;
  h->fself_r = ops->fself, h->fself_i = ops->fself_i;
  h->complex_kernel = ops->complex_kernel != 0;
  h->ready = false;  // the kernel transform depends on f_LR: set up again
  h->setup_gen++;
  return NPME_OK;
}

int npme_gpu_setup(npme_handle *h, size_t n, const double *coord) {
  if (!h) return fail(nullptr, NPME_EINVAL, "null handle");
  return npme::setup_many(&h, 1, &n, &coord, nullptr);
}


static void tmark(npme_handle *h, int i, cudaStream_t s) {
  if (h->timing.enabled) cudaEventRecord(h->timing.ev[i], s);
}

// Enqueues one CalcV on stream s (the launches; no checks).
static int enqueue_calcv(npme_handle *h, double *d_V, const double *d_charge, cudaStream_t s) {
  h->launches = 0;
  tmark(h, 0, s);
  npme::launch_gather_charges(h, d_charge, s);
  CK(cudaGetLastError());  // launch errors are checked before cuFFT runs
  tmark(h, 1, s);
  // the direct sum runs on stream2 beside the reciprocal sum; in the serial
  // timing mode it starts after the reciprocal chain, so that each stage's
  // events time that stage alone
  const bool serial = h->timing.enabled && h->timing.serial;
  h->merge_pending = false;
  auto fork_direct = [&]() -> int {
    CK(cudaEventRecord(h->ev_fork, s));
    CK(cudaStreamWaitEvent(h->stream2, h->ev_fork, 0));
    tmark(h, 8, h->stream2);
    if (npme::launch_direct(h, d_charge, d_V, h->stream2))
      return fail(h, NPME_ECUDA, "direct-sum launch of the caller-defined kernel failed");
    CK(cudaGetLastError());
    tmark(h, 9, h->stream2);
    CK(cudaEventRecord(h->ev_join, h->stream2));
    return NPME_OK;
  };
  int frc;
  if (!serial && (frc = fork_direct())) return frc;
  if (npme::grid_clear(h, s)) return fail(h, NPME_ECUDA, "clearing the spread grid failed");
  npme::launch_spread(h, s);
  CK(cudaGetLastError());
  tmark(h, 2, s);
  if ((frc = npme::fft_forward(h, s))) return frc;
  tmark(h, 3, s);
  npme::launch_multiply(h, s);
  CK(cudaGetLastError());
  tmark(h, 4, s);
  if ((frc = npme::fft_inverse(h, s))) return frc;
  tmark(h, 5, s);
  if (serial && (frc = fork_direct())) return frc;
  CK(cudaStreamWaitEvent(s, h->ev_join, 0));
  tmark(h, 6, s);
  npme::launch_interp(h, d_V, s);
  tmark(h, 7, s);
  h->timing_pending = h->timing.enabled;
  CK(cudaGetLastError());
  return NPME_OK;
}

namespace {

void drop_graph(npme_handle *h) {
  if (h->graph) cudaGraphExecDestroy(h->graph);
  h->graph = nullptr;
  h->graph_V = nullptr, h->graph_q = nullptr;
}

// Captures one CalcV on the handle's stream (thread-local capture mode, so
// other threads of the process stay free to allocate) and instantiates it.
// On any failure the capture is ended and discarded and the call is enqueued
// as plain launches instead; the failure is not an error of the call.
bool capture_calcv(npme_handle *h, double *d_V, const double *d_charge) {
  cudaStream_t cs = h->stream;
  if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  const int rc = enqueue_calcv(h, d_V, d_charge, cs);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(cs, &g);
  cudaGraphExec_t x = nullptr;
  if (!rc && e == cudaSuccess && g) e = cudaGraphInstantiate(&x, g, 0);
  if (g) cudaGraphDestroy(g);
  if (rc || e != cudaSuccess || !x) {
    if (x) cudaGraphExecDestroy(x);
    cudaGetLastError();
    return false;
  }
  drop_graph(h);
  h->graph = x;
  h->graph_gen = h->setup_gen;
  h->graph_V = d_V, h->graph_q = d_charge;
  h->graph_launches = h->launches;
  return true;
}

}  // namespace

int npme_gpu_calcv_device(npme_handle *h, double *d_V, const double *d_charge, void *stream) {
  if (!h) return fail(nullptr, NPME_EINVAL, "null handle");
  if (!h->ready) return fail(h, NPME_ESTATE, "calcv before setup");
  if (!d_V || !d_charge) return fail(h, NPME_EINVAL, "null buffer");
  CK(cudaSetDevice(h->device));
  cudaStream_t s = (cudaStream_t)stream;  // NULL: the default stream
  // Graph replay: the launches of a CalcV depend only on the set-up and the
  // two buffers, so the second call with the same buffers after a set-up is
  // captured and later ones launch the graph (caller-defined kernels and the
  // timing mode always run as plain launches).
  if (h->graph_enabled && !h->timing.enabled && !h->user_kernel) {
    if (h->graph && h->graph_gen == h->setup_gen && h->graph_V == d_V && h->graph_q == d_charge) {
      CK(cudaGraphLaunch(h->graph, s));
      h->launches = h->graph_launches;
      return NPME_OK;
    }
    if (h->seen_gen == h->setup_gen && h->seen_V == d_V && h->seen_q == d_charge &&
        h->nograph_gen != h->setup_gen) {
      if (capture_calcv(h, d_V, d_charge)) {
        CK(cudaGraphLaunch(h->graph, s));
        h->launches = h->graph_launches;
        return NPME_OK;
      }
      h->nograph_gen = h->setup_gen;  // not capturable: plain launches until the next set-up
    }
    h->seen_gen = h->setup_gen, h->seen_V = d_V, h->seen_q = d_charge;
  }
  return enqueue_calcv(h, d_V, d_charge, s);
}

// Reads the stage events of the last timed calcv (waits for its last event).
static void collect_timing(npme_handle *h) {
  if (!h->timing.enabled || !h->timing_pending) return;
  h->timing_pending = false;
  cudaEvent_t *e = h->timing.ev;
  if (cudaEventSynchronize(e[7]) != cudaSuccess || cudaEventSynchronize(e[9]) != cudaSuccess)
    return;
  float ms;
  // gather, spread, fft, multiply, ifft, direct, interp, total
  cudaEventElapsedTime(&ms, e[0], e[1]); h->stage_ms[0] = ms;
  cudaEventElapsedTime(&ms, e[1], e[2]); h->stage_ms[1] = ms;
  cudaEventElapsedTime(&ms, e[2], e[3]); h->stage_ms[2] = ms;
  cudaEventElapsedTime(&ms, e[3], e[4]); h->stage_ms[3] = ms;
  cudaEventElapsedTime(&ms, e[4], e[5]); h->stage_ms[4] = ms;
  cudaEventElapsedTime(&ms, e[8], e[9]); h->stage_ms[5] = ms;
  cudaEventElapsedTime(&ms, e[6], e[7]); h->stage_ms[6] = ms;
  cudaEventElapsedTime(&ms, e[0], e[7]); h->stage_ms[7] = ms;
}

static int calcv_host(npme_handle *h, double *V, size_t n, const double *charge, bool cplx) {
  if (!h) return fail(nullptr, NPME_EINVAL, "null handle");
  if (!h->ready) return fail(h, NPME_ESTATE, "calcv before setup");
  if (cplx != h->complex_kernel)
    return fail(h, NPME_EINVAL, cplx ? "complex call on a real kernel"
                                     : "real call on a complex kernel");
  if (n != h->n) return fail(h, NPME_EINVAL, "nCharge differs from setup");
  if (!V || !charge) return fail(h, NPME_EINVAL, "null buffer");
  CK(cudaSetDevice(h->device));
  const int C = cplx ? 2 : 1;
  CK(cudaMemcpyAsync(h->d_q_in, charge, sizeof(double) * C * n, cudaMemcpyHostToDevice,
                     h->stream));
  int rc = npme_gpu_calcv_device(h, h->d_V, h->d_q_in, h->stream);
  if (rc) return rc;
  CK(cudaMemcpyAsync(V, h->d_V, sizeof(double) * 4 * C * n, cudaMemcpyDeviceToHost,
                     h->stream));
  CK(cudaStreamSynchronize(h->stream));
  collect_timing(h);
  return NPME_OK;
}

int npme_gpu_calcv_real(npme_handle *h, double *V, size_t n, const double *charge,
                        const double *coord) {
  (void)coord;
  return calcv_host(h, V, n, charge, false);
}

int npme_gpu_calcv_complex(npme_handle *h, double *V, size_t n, const double *charge,
                           const double *coord) {
  (void)coord;
  return calcv_host(h, V, n, charge, true);
}

static int exact_host(npme_handle *h, double *V, size_t n, const double *charge, bool cplx) {
  if (!h) return fail(nullptr, NPME_EINVAL, "null handle");
  if (!h->ready) return fail(h, NPME_ESTATE, "calcv_exact before setup");
  if (cplx != h->complex_kernel) return fail(h, NPME_EINVAL, "charge type mismatch");
  if (n != h->n) return fail(h, NPME_EINVAL, "nCharge differs from setup");
  if (!V || !charge) return fail(h, NPME_EINVAL, "null buffer");
  CK(cudaSetDevice(h->device));
  const int C = cplx ? 2 : 1;
  CK(cudaMemcpyAsync(h->d_q_in, charge, sizeof(double) * C * n, cudaMemcpyHostToDevice,
                     h->stream));
  h->launches = 0;
  if (npme::launch_exact(h, h->d_q_in, h->d_V, h->stream))
    return fail(h, NPME_ECUDA, "exact-sum launch of the caller-defined kernel failed");
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(V, h->d_V, sizeof(double) * 4 * C * n, cudaMemcpyDeviceToHost,
                     h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return NPME_OK;
}

int npme_gpu_calcv_exact_subset(npme_handle *h, double *V, size_t m,
                                const unsigned int *targets, const double *charge) {
  if (!h) return fail(nullptr, NPME_EINVAL, "null handle");
  if (!h->ready) return fail(h, NPME_ESTATE, "calcv_exact_subset before setup");
  if (!V || !targets || !charge) return fail(h, NPME_EINVAL, "null buffer");
  if (m == 0) return NPME_OK;
  if (m > h->n) return fail(h, NPME_EINVAL, "more targets than points");
  for (size_t t = 0; t < m; t++)
    if (targets[t] >= h->n) return fail(h, NPME_EINVAL, "target index out of range");
  CK(cudaSetDevice(h->device));
  const int C = h->complex_kernel ? 2 : 1;
  int rc;
  if ((rc = dalloc(h, &h->d_tidx, sizeof(uint32_t) * m))) return rc;
  CK(cudaMemcpyAsync(h->d_tidx, targets, sizeof(uint32_t) * m, cudaMemcpyHostToDevice,
                     h->stream));
  CK(cudaMemcpyAsync(h->d_q_in, charge, sizeof(double) * C * h->n, cudaMemcpyHostToDevice,
                     h->stream));
  h->launches = 0;
  if (npme::launch_exact(h, h->d_q_in, h->d_V, h->stream, h->d_tidx, (long)m))
    return fail(h, NPME_ECUDA, "exact-sum launch of the caller-defined kernel failed");
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(V, h->d_V, sizeof(double) * 4 * C * m, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return NPME_OK;
}

int npme_gpu_calcv_exact_real(npme_handle *h, double *V, size_t n, const double *charge,
                              const double *coord) {
  (void)coord;
  return exact_host(h, V, n, charge, false);
}

int npme_gpu_calcv_exact_complex(npme_handle *h, double *V, size_t n, const double *charge,
                                 const double *coord) {
  (void)coord;
  return exact_host(h, V, n, charge, true);
}

int npme_gpu_direct_sum_device(npme_handle *h, double *d_V, const double *d_charge,
                               void *stream) {
  if (!h) return fail(nullptr, NPME_EINVAL, "null handle");
  if (!h->ready) return fail(h, NPME_ESTATE, "direct_sum before setup");
  if (!d_V || !d_charge) return fail(h, NPME_EINVAL, "null buffer");
  CK(cudaSetDevice(h->device));
  cudaStream_t s = (cudaStream_t)stream;  // NULL: the default stream
  h->launches = 0;
  npme::launch_gather_direct(h, d_charge, h->d_qc, s);
  npme::DirectArgs a{h->d_qc, d_charge, 0.0, 0.0, d_V};
  if (npme::launch_direct_args(h, a, s))
    return fail(h, NPME_ECUDA, "direct-sum launch of the caller-defined kernel failed");
  CK(cudaGetLastError());
  return NPME_OK;
}

int npme_gpu_count_pairs(npme_handle *h, unsigned long long *unordered_pairs) {
  if (!h || !unordered_pairs) return fail(h, NPME_EINVAL, "null argument");
  if (!h->ready) return fail(h, NPME_ESTATE, "count_pairs before setup");
  CK(cudaSetDevice(h->device));
  unsigned long long *d_count = nullptr;
  CK(cudaMalloc(&d_count, sizeof(unsigned long long)));
  cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), h->stream);
  npme::launch_count_pairs(h, d_count, h->stream);
  unsigned long long ordered = 0;
  cudaError_t e = cudaMemcpyAsync(&ordered, d_count, sizeof(ordered), cudaMemcpyDeviceToHost,
                                  h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(d_count);
  if (e != cudaSuccess) return fail(h, NPME_ECUDA, cudaGetErrorString(e));
  *unordered_pairs = ordered / 2;
  return NPME_OK;
}

int npme_gpu_set_graph(npme_handle *h, int enable) {
  if (!h) return fail(nullptr, NPME_EINVAL, "null handle");
  if (enable < 0 || enable > 1) return fail(h, NPME_EINVAL, "graph mode must be 0 or 1");
  h->graph_enabled = enable != 0;
  return NPME_OK;
}

int npme_gpu_set_timing(npme_handle *h, int enable) {
  if (!h) return fail(nullptr, NPME_EINVAL, "null handle");
  if (enable < 0 || enable > 2) return fail(h, NPME_EINVAL, "timing mode must be 0, 1 or 2");
  h->timing.enabled = enable != 0;
  h->timing.serial = enable == 2;
  return NPME_OK;
}

int npme_gpu_get_info(const npme_handle *hc, npme_info *info) {
  if (!hc || !info) return fail(nullptr, NPME_EINVAL, "null argument");
  // the stage-time cache is filled lazily: reading it is logically const
  npme_handle *h = const_cast<npme_handle *>(hc);
  collect_timing(h);
  memset(info, 0, sizeof(*info));
  info->nCharge = h->n;
  info->X = h->box[0], info->Y = h->box[1], info->Z = h->box[2];
  for (int d = 0; d < 3; d++) info->R[d] = h->box[3 + d], info->L[d] = h->box[6 + d];
  info->fself_r = h->fself_r, info->fself_i = h->fself_i;
  for (int i = 0; i < 32; i++) info->dm_a_r[i] = h->a_r[i], info->dm_a_i[i] = h->a_i[i];
  info->nDeriv = h->p.nDeriv;
  info->nCells = (long)h->cells.nc[0] * h->cells.nc[1] * h->cells.nc[2];
  info->nBricks = h->n_bricks;
  info->nNonEmptyBricks = h->n_nonempty;
  info->deviceBytes = h->dev_bytes;
  for (int i = 0; i < 8; i++) info->stage_ms[i] = h->stage_ms[i];
  info->launches = h->launches;
  info->nGroups = h->n_groups;
  info->candidatesPerPoint = h->cand_per_point;
  info->pairsOnce = npme::pairs_once(h) ? 1 : 0;
  info->pairsOnceCandidatesPerPoint = h->hcand_per_point;
  return NPME_OK;
}

int npme_gpu_last_error(const npme_handle *h, char *buf, size_t len) {
  if (!buf || len == 0) return NPME_EINVAL;
  std::string s;
  if (h) s = h->err;
  else {
    std::lock_guard<std::mutex> lk(g_err_mu);
    s = g_err;
  }
  strncpy(buf, s.c_str(), len - 1);
  buf[len - 1] = 0;
  return NPME_OK;
}

int npme_gpu_destroy(npme_handle *h) {
  if (!h) return NPME_OK;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->stream2) cudaStreamSynchronize(h->stream2);
  if (h->graph) cudaGraphExecDestroy(h->graph);
  release(h);
  pool_release(h);
  npme::pinned_return((void **)&h->h_fstage, &h->fstage_cap);
  npme::pinned_return(&h->h_counts, &h->counts_cap);
  npme::pinned_return(&h->h_desc, &h->desc_cap);
  npme::pinned_return(&h->h_ktdesc, &h->ktdesc_cap);
  if (h->stream) cudaStreamDestroy(h->stream);
  if (h->stream2) cudaStreamDestroy(h->stream2);
  if (h->ev_fork) cudaEventDestroy(h->ev_fork);
  if (h->ev_join) cudaEventDestroy(h->ev_join);
  for (int i = 0; i < 10; i++)
    if (h->timing.ev[i]) cudaEventDestroy(h->timing.ev[i]);
  delete h;
  return NPME_OK;
}

}  // extern "C"
