// C ABI of npme_b200 (include/npme_gpu.h): parameter handling, set-up
// (derivative-match coefficients, box, point binning, buffers, FFT plans,
// kernel transform) and the CalcV orchestration on CUDA streams.
#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "internal.h"

using npme::BrickPoint;

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

// src/RecSumSupportFunctions.h:123-127
long start_index(double w) { return w < 0 ? (long)(-w) + 1 : (long)(-w); }

// Device memory of all handles comes from one stream-ordered pool per device
// (cudaMallocFromPoolAsync / cudaFreeAsync on the handle's stream).  Unlike
// cudaMalloc / cudaFree, neither synchronises the device, so a handle that
// grows its buffers during set-up does not stall the CalcV of other handles
// running meanwhile; freed blocks stay in the pool for the next handle.  The
// pool returns its memory to the device when the last handle of the device
// is destroyed.
std::mutex g_pool_mu;
std::map<int, std::pair<cudaMemPool_t, int>> g_pools;  // device -> (pool, live handles)

int pool_acquire(npme_handle *h) {
  std::lock_guard<std::mutex> lk(g_pool_mu);
  auto it = g_pools.find(h->device);
  if (it == g_pools.end()) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = h->device;
    cudaMemPool_t pool;
    cudaError_t e = cudaMemPoolCreate(&pool, &props);
    if (e != cudaSuccess)
      return fail(h, NPME_ECUDA, std::string("cudaMemPoolCreate: ") + cudaGetErrorString(e));
    unsigned long long keep = ~0ull;  // keep freed blocks for reuse
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    it = g_pools.emplace(h->device, std::make_pair(pool, 0)).first;
  }
  it->second.second++;
  h->pool = it->second.first;
  return NPME_OK;
}

void pool_release(npme_handle *h) {
  if (!h->pool) return;
  std::lock_guard<std::mutex> lk(g_pool_mu);
  auto it = g_pools.find(h->device);
  if (it != g_pools.end() && --it->second.second == 0) cudaMemPoolTrimTo(it->second.first, 0);
  h->pool = nullptr;
}

// Frees every device buffer of the handle (stream-ordered; the caller has
// synchronised the handle's streams).
void release(npme_handle *h) {
  h->pf = h->pi = nullptr;  // shared plans stay in the process-wide cache
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
// the order of the handle's stream.
template <typename P>
int dalloc(npme_handle *h, P **ptr, size_t bytes) {
  if (bytes == 0) bytes = 16;
  size_t &cap = h->caps[(void *)ptr];
  if (*ptr && cap >= bytes) return NPME_OK;
  if (*ptr) {
    cudaFreeAsync(*ptr, h->stream);
    h->dev_bytes -= cap;
    *ptr = nullptr;
    cap = 0;
  }
  cudaError_t e = cudaMallocFromPoolAsync((void **)ptr, bytes, h->pool, h->stream);
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

// Host threads for the set-up of an n-point system: the machine's cores
// shared among the set-ups running at the same time (a serving process runs
// several on its own threads), one for small systems.
std::atomic<int> g_active_setups{0};

#ifndef NPME_SETUP_THREADS_MAX
#define NPME_SETUP_THREADS_MAX 16
#endif

int setup_threads(size_t n) {
  if (n < 50000) return 1;
  const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
  return std::max(1, std::min(NPME_SETUP_THREADS_MAX, hw / std::max(1, g_active_setups.load())));
}

// fn(begin, end) over [0, count) split into contiguous ranges, one host
// thread each; the thread count follows `work` (points handled; default
// count), the calling thread alone for small systems.
template <class F>
void parallel_ranges(size_t count, F fn, size_t work = 0) {
  const int nt = (int)std::min<size_t>(setup_threads(work ? work : count),
                                       std::max<size_t>(1, count));
  if (nt <= 1) {
    fn((size_t)0, count);
    return;
  }
  std::vector<std::thread> pool;
  for (int t = 0; t < nt; t++)
    pool.emplace_back(fn, count * t / nt, count * (t + 1) / nt);
  for (auto &th : pool) th.join();
}

// Sorts the points by xy column (`col`, ncol columns), then by (z, index)
// inside each column.  Fills the permutation, the column starts and the
// sorted z.
void column_sort(const double *coord, size_t n, long ncol, const std::vector<int> &col,
                 std::vector<uint32_t> &order, std::vector<long> &cstart,
                 std::vector<double> &zs) {
  // counting sort by column (stable), then each column by (z, index)
  cstart.assign(ncol + 1, 0);
  for (size_t i = 0; i < n; i++) cstart[col[i] + 1]++;
  for (long c = 0; c < ncol; c++) cstart[c + 1] += cstart[c];
  order.resize(n);
  {
    std::vector<long> fill(cstart.begin(), cstart.end() - 1);
    for (size_t i = 0; i < n; i++) order[fill[col[i]]++] = (uint32_t)i;
  }
  zs.resize(n);
  auto sort_columns = [&](long c0, long c1) {
    std::vector<std::pair<double, uint32_t>> zc;
    for (long c = c0; c < c1; c++) {
      const long b = cstart[c], e1 = cstart[c + 1];
      zc.resize(e1 - b);
      for (long k = b; k < e1; k++) zc[k - b] = {coord[3 * (size_t)order[k] + 2], order[k]};
      std::sort(zc.begin(), zc.end());
      for (long k = b; k < e1; k++) zs[k] = zc[k - b].first, order[k] = zc[k - b].second;
    }
  };
  const int nt = setup_threads(n);
  if (nt == 1) {
    sort_columns(0, ncol);
  } else {
    std::vector<std::thread> pool;
    for (int t = 0; t < nt; t++) pool.emplace_back(sort_columns, ncol * t / nt, ncol * (t + 1) / nt);
    for (auto &th : pool) th.join();
  }
}

// gpos[k] = coord[gorder[k]], spos[k] = coord[sorder[k]] (FP64, w unused)
__global__ void gather_positions_kernel(const double *__restrict__ coord,
                                        const uint32_t *__restrict__ gorder,
                                        const uint32_t *__restrict__ sorder, long n,
                                        double4 *__restrict__ gpos, double4 *__restrict__ spos) {
  const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const double *x = coord + 3 * (long)gorder[k];
  gpos[k] = make_double4(x[0], x[1], x[2], 0.0);
  const double *y = coord + 3 * (long)sorder[k];
  spos[k] = make_double4(y[0], y[1], y[2], 0.0);
}

#ifndef NPME_SOURCE_SPLIT
#define NPME_SOURCE_SPLIT 2
#endif

// Warp groups for the FP32 direct sum.  Targets are binned into xy columns
// of edge e ~ (32 / density)^(1/3) and sorted by z inside each column; each
// run of 32 consecutive points of a column is one group (a compact, roughly
// cubic cluster).  Sources are binned the same way into finer columns (edge
// e / NPME_SOURCE_SPLIT) and sorted by z.  For every group the source
// segments are the z ranges of the fine columns that can hold a point within
// Rdir of the group's bounding box: |dz| <= sqrt(Rdir^2 - d_xy^2), d_xy the
// distance from the bounding box to the column in the xy plane; finer source
// columns bound that distance more tightly, so fewer sources are staged per
// group.  Geometry is fixed between CalcV calls (the reference's contract),
// so this is set-up work.  Returns the group-order permutation of the
// targets in `order` and the source-order permutation in `sorder`.
int build_groups(npme_handle *h, const double *coord, std::vector<uint32_t> &order,
                 std::vector<uint32_t> &sorder) {
  const size_t n = h->n;
  const double R = h->p.Rdir, R2 = R * R;
  double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
  for (size_t i = 0; i < n; i++)
    for (int d = 0; d < 3; d++) {
      mn[d] = std::min(mn[d], coord[3 * i + d]);
      mx[d] = std::max(mx[d], coord[3 * i + d]);
    }
  // column edge from the mean density of the bounding box (degenerate axes
  // are given a nominal thickness of Rdir / 4)
  double vol = 1.0;
  for (int d = 0; d < 3; d++) vol *= std::max(mx[d] - mn[d], 0.25 * R);
  double e = std::cbrt(32.0 * vol / (double)n);
  e = std::max(e, 1e-3 * R);
  constexpr int S = NPME_SOURCE_SPLIT;
  int nc[2], ns[2];
  double edge[2], sedge[2];
  for (int d = 0; d < 2; d++) {
    const double ext = mx[d] - mn[d];
    nc[d] = std::max(1, std::min((int)std::ceil(ext / e), 1 << 14));
    edge[d] = std::max(ext / nc[d], 1e-12);
    ns[d] = nc[d] * S;
    sedge[d] = edge[d] / S;
  }
  // every fine column lies inside one coarse column: a point's fine column
  // is its coarse column's sub-column
  std::vector<int> ccol(n), scol(n);
  for (size_t i = 0; i < n; i++) {
    int cs[2], ss[2];
    for (int d = 0; d < 2; d++) {
      const double u = coord[3 * i + d] - mn[d];
      cs[d] = std::min(nc[d] - 1, std::max(0, (int)(u / edge[d])));
      ss[d] = cs[d] * S + std::min(S - 1, std::max(0, (int)((u - cs[d] * edge[d]) / sedge[d])));
    }
    ccol[i] = cs[0] * nc[1] + cs[1];
    scol[i] = ss[0] * ns[1] + ss[1];
  }
  std::vector<long> cstart, sstart;
  std::vector<double> zt, zs;
  const long ncol = (long)nc[0] * nc[1];
  column_sort(coord, n, ncol, ccol, order, cstart, zt);
  column_sort(coord, n, (long)ns[0] * ns[1], scol, sorder, sstart, zs);
  // position of each source in the coarse (group) order: increasing inside
  // a fine column, since both orders sort a column by (z, index)
  const bool half = true;
  std::vector<uint32_t> fcpos;
  if (half) {
    std::vector<uint32_t> cpos(n);
    for (size_t k = 0; k < n; k++) cpos[order[k]] = (uint32_t)k;
    fcpos.resize(n);
    for (size_t k = 0; k < n; k++) fcpos[k] = cpos[sorder[k]];
  }

  // Per coarse column: the fine columns that can hold a source within R of
  // the column's points, each with a pair of cursors into its z-sorted
  // sources.  The groups of a column come in increasing z, so the cursors
  // only creep forward (a few steps per group, either direction as the
  // window half-height varies) instead of a binary search per group and
  // column, and the column's source z values stay in cache.  Coarse columns
  // are independent: large systems split them over host threads, each
  // filling its own lists, concatenated in column order afterwards.
  struct Part {
    std::vector<int4> groups, hgroups;
    std::vector<double4> cen;
    std::vector<int2> segs, hsegs;
    std::vector<long> work, hwork;  // sources staged per group (launch order)
    double cand = 0, hcand = 0;
  };
  auto build_part = [&](long c_begin, long c_end, Part &out) {
    std::vector<long> nb_col, nb_cc, pa, pb;
    std::vector<int> nb_s0, nb_s1;
    std::vector<double> dxv, dyv;
    for (long c = c_begin; c < c_end; c++) {
      if (cstart[c] == cstart[c + 1]) continue;
      double cl[2] = {1e300, 1e300}, ch[2] = {-1e300, -1e300};
      for (long k = cstart[c]; k < cstart[c + 1]; k++)
        for (int d = 0; d < 2; d++) {
          const double x = coord[3 * (size_t)order[k] + d];
          cl[d] = std::min(cl[d], x);
          ch[d] = std::max(ch[d], x);
        }
      int lo[2], hi[2];
      for (int d = 0; d < 2; d++) {
        lo[d] = (int)std::max(0.0, std::floor((cl[d] - R - mn[d]) / sedge[d]));
        hi[d] = (int)std::min((double)(ns[d] - 1), std::floor((ch[d] + R - mn[d]) / sedge[d]));
      }
      nb_col.clear(), nb_cc.clear(), nb_s0.clear(), nb_s1.clear();
      for (int s0 = lo[0]; s0 <= hi[0]; s0++)
        for (int s1 = lo[1]; s1 <= hi[1]; s1++) {
          const long sc = (long)s0 * ns[1] + s1;
          if (sstart[sc] == sstart[sc + 1]) continue;
          nb_col.push_back(sc), nb_s0.push_back(s0 - lo[0]), nb_s1.push_back(s1 - lo[1]);
          nb_cc.push_back((long)(s0 / S) * nc[1] + s1 / S);
        }
      pa.assign(nb_col.size(), 0), pb.assign(nb_col.size(), 0);
      for (size_t t = 0; t < nb_col.size(); t++) pa[t] = pb[t] = sstart[nb_col[t]];
      dxv.resize(hi[0] - lo[0] + 1), dyv.resize(hi[1] - lo[1] + 1);
      for (long p0 = cstart[c]; p0 < cstart[c + 1]; p0 += 32) {
        const long p1 = std::min(p0 + 32, cstart[c + 1]);
        double bl[3] = {1e300, 1e300, 1e300}, bh[3] = {-1e300, -1e300, -1e300};
        for (long k = p0; k < p1; k++)
          for (int d = 0; d < 3; d++) {
            const double x = coord[3 * (size_t)order[k] + d];
            bl[d] = std::min(bl[d], x);
            bh[d] = std::max(bh[d], x);
          }
        // squared xy distances from the bounding box to each fine column
        for (size_t u = 0; u < dxv.size(); u++) {
          const double l0 = mn[0] + (lo[0] + (long)u) * sedge[0], h0 = l0 + sedge[0];
          const double d = std::max(0.0, std::max(l0 - bh[0], bl[0] - h0));
          dxv[u] = d * d;
        }
        for (size_t u = 0; u < dyv.size(); u++) {
          const double l1 = mn[1] + (lo[1] + (long)u) * sedge[1], h1 = l1 + sedge[1];
          const double d = std::max(0.0, std::max(l1 - bh[1], bl[1] - h1));
          dyv[u] = d * d;
        }
        const int seg0 = (int)out.segs.size(), hseg0 = (int)out.hsegs.size();
        long gwork = 0, hwork = 0;
        for (size_t t = 0; t < nb_col.size(); t++) {
          const double d2 = dxv[nb_s0[t]] + dyv[nb_s1[t]];
          if (d2 > R2) continue;
          const double hz = std::sqrt(R2 - d2), zlo = bl[2] - hz, zhi = bh[2] + hz;
          const long zb = sstart[nb_col[t]], ze = sstart[nb_col[t] + 1];
          long a = pa[t], b = pb[t];
          // a: first source with z >= zlo; b: first source with z > zhi
          while (a < ze && zs[a] < zlo) a++;
          while (a > zb && zs[a - 1] >= zlo) a--;
          while (b < ze && zs[b] <= zhi) b++;
          while (b > zb && zs[b - 1] > zhi) b--;
          pa[t] = a, pb[t] = b;
          if (b > a) {
            out.segs.push_back(make_int2((int)a, (int)(b - a)));
            out.cand += (double)(b - a) * (double)(p1 - p0);
            gwork += b - a;
          }
          // half shell: later coarse columns whole, the group's own column
          // from the first point after the group
          if (half && b > a && nb_cc[t] >= c) {
            long a2 = a;
            if (nb_cc[t] == c)
              a2 = std::lower_bound(fcpos.begin() + a, fcpos.begin() + b, (uint32_t)p1) -
                   fcpos.begin();
            if (b > a2) {
              out.hsegs.push_back(make_int2((int)a2, (int)(b - a2)));
              out.hcand += (double)(b - a2) * (double)(p1 - p0);
              hwork += b - a2;
            }
          }
        }
        out.groups.push_back(make_int4((int)p0, (int)(p1 - p0), seg0, (int)out.segs.size()));
        out.work.push_back(gwork);
        if (half) {
          out.hgroups.push_back(
              make_int4((int)p0, (int)(p1 - p0), hseg0, (int)out.hsegs.size()));
          out.hwork.push_back(hwork);
        }
        // centre and half-diagonal of the bounding box
        out.cen.push_back(make_double4(
            0.5 * (bl[0] + bh[0]), 0.5 * (bl[1] + bh[1]), 0.5 * (bl[2] + bh[2]),
            0.5 * std::sqrt((bh[0] - bl[0]) * (bh[0] - bl[0]) + (bh[1] - bl[1]) * (bh[1] - bl[1]) +
                            (bh[2] - bl[2]) * (bh[2] - bl[2]))));
      }
    }
  };
  const int nthreads = setup_threads(n);
  std::vector<Part> parts(nthreads);
  if (nthreads == 1) {
    build_part(0, ncol, parts[0]);
  } else {
    std::vector<std::thread> pool;
    for (int t = 0; t < nthreads; t++)
      pool.emplace_back(build_part, ncol * t / nthreads, ncol * (t + 1) / nthreads,
                        std::ref(parts[t]));
    for (auto &th : pool) th.join();
  }
  // group records with segment indices made global; the segment lists stay
  // in their parts and are uploaded part by part (no host concatenation)
  std::vector<int4> groups, hgroups;
  std::vector<double4> cen;
  std::vector<long> work, hwork;
  size_t nsegs = 0, nhsegs = 0;
  double cand = 0, hcand = 0;
  for (Part &pt : parts) {
    const int base = (int)nsegs, hbase = (int)nhsegs;
    for (int4 g : pt.groups) groups.push_back(make_int4(g.x, g.y, g.z + base, g.w + base));
    for (int4 g : pt.hgroups) hgroups.push_back(make_int4(g.x, g.y, g.z + hbase, g.w + hbase));
    cen.insert(cen.end(), pt.cen.begin(), pt.cen.end());
    work.insert(work.end(), pt.work.begin(), pt.work.end());
    hwork.insert(hwork.end(), pt.hwork.begin(), pt.hwork.end());
    nsegs += pt.segs.size(), nhsegs += pt.hsegs.size();
    cand += pt.cand, hcand += pt.hcand;
  }
  // group records hold segment indices as int
  if (nsegs >= ((size_t)1 << 31) || nhsegs >= ((size_t)1 << 31))
    return fail(h, NPME_EINVAL, "too many direct-sum source segments (2^31)");
  // heaviest groups first, so the last wave of the launch holds the light
  // ones (each list by its own work)
  auto by_work = [](std::vector<int4> &gl, const std::vector<long> &wk,
                    const std::vector<double4> &cin, std::vector<double4> &cout) {
    std::vector<uint32_t> go(gl.size());
    for (size_t g = 0; g < go.size(); g++) go[g] = (uint32_t)g;
    std::stable_sort(go.begin(), go.end(), [&](uint32_t a, uint32_t b) { return wk[a] > wk[b]; });
    std::vector<int4> g2(gl.size());
    cout.resize(gl.size());
    for (size_t g = 0; g < go.size(); g++) g2[g] = gl[go[g]], cout[g] = cin[go[g]];
    gl.swap(g2);
  };
  std::vector<double4> gcen, hcen;
  by_work(groups, work, cen, gcen);
  if (half) by_work(hgroups, hwork, cen, hcen);
  cen.swap(gcen);
  h->n_groups = (long)groups.size();
  h->n_segs = (long)nsegs;
  h->cand_per_point = cand / (double)n;
  h->n_hgroups = (long)hgroups.size();
  h->n_hsegs = (long)nhsegs;
  h->hcand_per_point = hcand / (double)n;
  // heads of offsets up to ~the group half-diagonal carry ~6e-8 e absolute
  // error; below r = e/4 the relative error would exceed ~1e-6, so refine
  h->refine2 = (0.25 * e) * (0.25 * e);
  int rc;
  if ((rc = dalloc(h, &h->d_coord, sizeof(double) * 3 * n))) return rc;
  if ((rc = dalloc(h, &h->d_gpos, sizeof(double4) * n))) return rc;
  if ((rc = dalloc(h, &h->d_spos, sizeof(double4) * n))) return rc;
  if ((rc = dalloc(h, &h->d_cperm, sizeof(uint32_t) * n))) return rc;
  if ((rc = dalloc(h, &h->d_sperm, sizeof(uint32_t) * n))) return rc;
  if ((rc = dalloc(h, &h->d_groups, sizeof(int4) * groups.size()))) return rc;
  if ((rc = dalloc(h, &h->d_gcen, sizeof(double4) * cen.size()))) return rc;
  if ((rc = dalloc(h, &h->d_segs, sizeof(int2) * std::max<size_t>(1, nsegs)))) return rc;
  // target and source positions are gathered on the device from the
  // caller's coordinates and the two orders
  CK(cudaMemcpyAsync(h->d_coord, coord, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d_cperm, order.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice,
                     h->stream));
  CK(cudaMemcpyAsync(h->d_sperm, sorder.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice,
                     h->stream));
  gather_positions_kernel<<<(unsigned)((n + 255) / 256), 256, 0, h->stream>>>(
      h->d_coord, h->d_cperm, h->d_sperm, (long)n, h->d_gpos, h->d_spos);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(h->d_groups, groups.data(), sizeof(int4) * groups.size(),
                     cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d_gcen, cen.data(), sizeof(double4) * cen.size(), cudaMemcpyHostToDevice,
                     h->stream));
  {
    size_t off = 0;
    for (const Part &pt : parts) {
      if (!pt.segs.empty())
        CK(cudaMemcpyAsync(h->d_segs + off, pt.segs.data(), sizeof(int2) * pt.segs.size(),
                           cudaMemcpyHostToDevice, h->stream));
      off += pt.segs.size();
    }
  }
  if (half) {
    if ((rc = dalloc(h, &h->d_hgroups, sizeof(int4) * hgroups.size()))) return rc;
    if ((rc = dalloc(h, &h->d_hcen, sizeof(double4) * hcen.size()))) return rc;
    if ((rc = dalloc(h, &h->d_hsegs, sizeof(int2) * std::max<size_t>(1, nhsegs)))) return rc;
    if (h->fp32) {
      const size_t nv = (h->complex_kernel ? 2 : 1) * n;  // float4 per source (two if complex)
      if ((rc = dalloc(h, &h->d_vsrc, sizeof(float4) * nv))) return rc;
      CK(cudaMemsetAsync(h->d_vsrc, 0, sizeof(float4) * nv, h->stream));
    } else {
      if ((rc = dalloc(h, &h->d_vsrc64, sizeof(double) * 4 * n))) return rc;
      CK(cudaMemsetAsync(h->d_vsrc64, 0, sizeof(double) * 4 * n, h->stream));
    }
    CK(cudaMemcpyAsync(h->d_hgroups, hgroups.data(), sizeof(int4) * hgroups.size(),
                       cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->d_hcen, hcen.data(), sizeof(double4) * hcen.size(),
                       cudaMemcpyHostToDevice, h->stream));
    size_t off = 0;
    for (const Part &pt : parts) {
      if (!pt.hsegs.empty())
        CK(cudaMemcpyAsync(h->d_hsegs + off, pt.hsegs.data(), sizeof(int2) * pt.hsegs.size(),
                           cudaMemcpyHostToDevice, h->stream));
      off += pt.hsegs.size();
    }
  }
  return NPME_OK;
}

template <typename T>
int upload_points(npme_handle *h, const double *coord) {
  const size_t n = h->n;
  const npme::GridGeom &g = h->grid;
  const double *R = h->box + 3, *L = h->box + 6;
  const int P = g.order;
  // --- brick order for spread / interpolation ---
  std::vector<BrickPoint<T>> pts(n);
  std::vector<int> bid(n);
  // the first point (lowest index) whose stencil leaves the octant, and its axis
  std::atomic<long> bad{(long)n};
  std::atomic<int> bad_axis{0};
  parallel_ranges(n, [&](size_t i0, size_t i1) {
    for (size_t i = i0; i < i1; i++) {
      uint32_t g0[3];
      T u[3];
      for (int d = 0; d < 3; d++) {
        const double w = (double)g.N[d] / L[d] * (coord[3 * i + d] - R[d]);
        const long ms = start_index(w);
        const long o = ms + g.N[d] / 4;
        if (o < 0 || o + P - 1 > g.H[d] - 1) {
          long cur = bad.load();
          while ((long)i < cur && !bad.compare_exchange_weak(cur, (long)i)) {
          }
          if (bad.load() == (long)i) bad_axis = d;
          return;
        }
        g0[d] = (uint32_t)o;
        u[d] = (T)(w + (double)ms);
      }
      BrickPoint<T> &bp = pts[i];
      bp.u[0] = u[0], bp.u[1] = u[1], bp.u[2] = u[2];
      bp.g0 = (g0[0] << 20) | (g0[1] << 10) | g0[2];
      bp.orig = (uint32_t)i;
      bid[i] = (int)(((g0[0] / npme::kBrick) * g.nb[1] + g0[1] / npme::kBrick) * g.nb[2] +
                     g0[2] / npme::kBrick);
    }
  });
  if (bad.load() < (long)n)
    return fail(h, NPME_EINVAL,
                "point " + std::to_string(bad.load()) + " has a B-spline stencil outside the "
                "charge octant (axis " + std::to_string(bad_axis.load()) + ")");
  const long nbt = g.nb[0] * g.nb[1] * g.nb[2];
  std::vector<int> bstart(nbt + 1, 0);
  for (size_t i = 0; i < n; i++) bstart[bid[i] + 1]++;
  for (long b = 0; b < nbt; b++) bstart[b + 1] += bstart[b];
  std::vector<int> fillp(bstart.begin(), bstart.end() - 1);
  std::vector<BrickPoint<T>> sorted(n);
  for (size_t i = 0; i < n; i++) sorted[fillp[bid[i]]++] = pts[i];
  std::vector<int> blist;
  for (long b = 0; b < nbt; b++)
    if (bstart[b + 1] > bstart[b]) blist.push_back((int)b);
  // inside a brick, points sorted by the shared-memory bank of their stencil
  // origin in the brick's tile (the kernels give the lanes of a warp points
  // of different banks; see brick_point in bodies.cuh)
  {
    const int TL = npme::kBrick + P - 1;
    const int words = (int)(sizeof(T) / 4) * (h->complex_kernel ? 2 : 1);
    const int nkeys = 32 / words;
    parallel_ranges(blist.size(), [&](size_t k0, size_t k1) {
    std::vector<BrickPoint<T>> tmp;
    int cnt[32];
    for (size_t kb = k0; kb < k1; kb++) {
      const int b = blist[kb];
      const int beg = bstart[b], end = bstart[b + 1];
      const long b3 = b % g.nb[2], b2 = (b / g.nb[2]) % g.nb[1], b1 = b / (g.nb[2] * g.nb[1]);
      auto key = [&](const BrickPoint<T> &pt) {
        const long l1 = (long)(pt.g0 >> 20) - b1 * npme::kBrick;
        const long l2 = (long)((pt.g0 >> 10) & 1023u) - b2 * npme::kBrick;
        const long l3 = (long)(pt.g0 & 1023u) - b3 * npme::kBrick;
        return (int)(((l1 * TL + l2) * TL + l3) % nkeys);
      };
      tmp.assign(sorted.begin() + beg, sorted.begin() + end);
      std::fill(cnt, cnt + 32, 0);
      for (const auto &pt : tmp) cnt[key(pt)]++;
      int acc = beg;
      for (int k = 0; k < nkeys; k++) {
        const int c = cnt[k];
        cnt[k] = acc;
        acc += c;
      }
      for (const auto &pt : tmp) sorted[cnt[key(pt)]++] = pt;
    }
    }, n);
  }
  h->n_bricks = nbt;
  h->n_nonempty = (long)blist.size();

  std::vector<uint32_t> cperm;  // group order -> caller index (build_groups)
  const int C = h->complex_kernel ? 2 : 1;
  int rc;
  // the direct sum walks warp groups: targets in group order, sources
  // (and their gathered charges) in fine-column order
  std::vector<uint32_t> sperm;
  if ((rc = build_groups(h, coord, cperm, sperm))) return rc;
  if ((rc = dalloc(h, (BrickPoint<T> **)&h->d_bpts, sizeof(BrickPoint<T>) * n))) return rc;
  if ((rc = dalloc(h, &h->d_brick_start, sizeof(int) * (nbt + 1)))) return rc;
  if ((rc = dalloc(h, &h->d_brick_list, sizeof(int) * std::max<size_t>(1, blist.size()))))
    return rc;
  if ((rc = dalloc(h, (T **)&h->d_qb, sizeof(T) * C * n))) return rc;
  if ((rc = dalloc(h, (T **)&h->d_qc, sizeof(T) * C * n))) return rc;
  if ((rc = dalloc(h, &h->d_q_in, sizeof(double) * C * n))) return rc;
  if ((rc = dalloc(h, &h->d_V, sizeof(double) * 4 * C * n))) return rc;
  CK(cudaMemcpyAsync(h->d_bpts, sorted.data(), sizeof(BrickPoint<T>) * n, cudaMemcpyHostToDevice,
                     h->stream));
  CK(cudaMemcpyAsync(h->d_brick_start, bstart.data(), sizeof(int) * (nbt + 1),
                     cudaMemcpyHostToDevice, h->stream));
  if (!blist.empty())
    CK(cudaMemcpyAsync(h->d_brick_list, blist.data(), sizeof(int) * blist.size(),
                       cudaMemcpyHostToDevice, h->stream));
  // charges of the direct sum are gathered into its source order
  h->d_dperm = h->d_sperm;

  // --- grids ---
  const long *N = g.N;
  const size_t Ntot = (size_t)N[0] * N[1] * N[2];
  const size_t Mtot = (size_t)(N[0] / 2 + 1) * (N[1] / 2 + 1) * (N[2] / 2 + 1);
  if (h->complex_kernel) {
    if ((rc = dalloc(h, (T **)&h->d_grid, sizeof(T) * 2 * Ntot))) return rc;
    if ((rc = dalloc(h, (T **)&h->d_G, sizeof(T) * 2 * Mtot))) return rc;
  } else {
    if ((rc = dalloc(h, (T **)&h->d_grid, sizeof(T) * Ntot))) return rc;
    if ((rc = dalloc(h, (T **)&h->d_kgrid, sizeof(T) * 2 * (size_t)N[0] * N[1] * (N[2] / 2 + 1))))
      return rc;
    if ((rc = dalloc(h, (T **)&h->d_G, sizeof(T) * Mtot))) return rc;
  }
  return NPME_OK;
}

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
  if (p.BnOrder < 4 || p.BnOrder > 12 || (p.BnOrder & 1))
    return fail(h, NPME_EINVAL, "BnOrder must be even and in [4, 12]");
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
  return NPME_OK;
}

static int setup_impl(npme_handle *h, size_t n, const double *coord);

int npme_gpu_setup(npme_handle *h, size_t n, const double *coord) {
  g_active_setups++;
  const int rc = setup_impl(h, n, coord);
  g_active_setups--;
  return rc;
}

static int setup_impl(npme_handle *h, size_t n, const double *coord) {
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
  h->n = n;
  const npme_params &p = h->p;
  // box (src/RecSumSupportFunctions.cpp:182-201, 276-296)
  double mx[3] = {-1e300, -1e300, -1e300}, mn[3] = {1e300, 1e300, 1e300};
  for (size_t i = 0; i < n; i++)
    for (int d = 0; d < 3; d++) {
      const double x = coord[3 * i + d];
      if (!std::isfinite(x)) return fail(h, NPME_EINVAL, "non-finite coordinate");
      mx[d] = std::max(mx[d], x);
      mn[d] = std::min(mn[d], x);
    }
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
  int rc = h->fp32 ? upload_points<float>(h, coord) : upload_points<double>(h, coord);
  if (rc) {
    release(h);
    return rc;
  }
  if ((rc = npme::prepare_plans(h))) {
    release(h);
    return rc;
  }
  if ((rc = npme::build_kernel_transform(h))) {
    release(h);
    return rc;
  }
  h->ready = true;
  return NPME_OK;
}

static void tmark(npme_handle *h, int i, cudaStream_t s) {
  if (h->timing.enabled) cudaEventRecord(h->timing.ev[i], s);
}

int npme_gpu_calcv_device(npme_handle *h, double *d_V, const double *d_charge, void *stream) {
  if (!h) return fail(nullptr, NPME_EINVAL, "null handle");
  if (!h->ready) return fail(h, NPME_ESTATE, "calcv before setup");
  if (!d_V || !d_charge) return fail(h, NPME_EINVAL, "null buffer");
  CK(cudaSetDevice(h->device));
  cudaStream_t s = (cudaStream_t)stream;  // NULL: the default stream
  h->launches = 0;
  const size_t gbytes = (h->fp32 ? 4 : 8) * (h->complex_kernel ? 2 : 1) *
                        (size_t)h->grid.N[0] * h->grid.N[1] * h->grid.N[2];
  tmark(h, 0, s);
  npme::launch_gather_charges(h, d_charge, s);
  CK(cudaGetLastError());  // launch errors are checked before cuFFT runs
  tmark(h, 1, s);
  // the direct sum runs on stream2 beside the reciprocal sum; in the serial
  // timing mode it starts after the reciprocal chain, so that each stage's
  // events time that stage alone
  const bool serial = h->timing.enabled && h->timing.serial;
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
  CK(cudaMemsetAsync(h->d_grid, 0, gbytes, s));
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
  release(h);
  pool_release(h);
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
