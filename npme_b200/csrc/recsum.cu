// Reciprocal sum on the B200: kernel transform (set-up), charge spreading,
// Fourier-space multiply and potential interpolation.  The FFTs themselves
// are cuFFT calls issued from npme_gpu.cu.
//
// Grid convention: the charge octant of the reference's compact grid
// (m in [-N/4, N/4), src/RecSumSupportFunctions.h:100-113) is stored at grid
// index g = m + N/4 in [0, N/2) of a zero-padded N1 x N2 x N3 box.  The
// convolution is cyclic on the full box and both input and output are
// shifted by the same N/4, so theta on the octant equals the reference's
// theta (src/RecSumV.cpp:766-840) without its 8 even/odd half transforms.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <mutex>
#include <type_traits>
#include <vector>

#include "bodies.cuh"
#include "internal.h"

namespace npme {

// ---------------------------------------------------------------------------
// Kernel transform (FP64): sample the smooth kernel f_LR on the (N/2+1)^3
// octant with the 8-image Fourier-extension window (src/RecSumGrid.cpp:45-162,
// 388-424), transform each axis by the even-extension DFT (src/RecSumGrid.cpp:
// 470-582, a DCT-I), then fold in lambda^2 and 1/(N1 N2 N3)
// (src/RecSumV.cpp:639-707).

struct LRKernel {
  int func, split, nder;
  double R2, alpha, beta, k0r, k0i;
  double ar[32], ai[32];  // unscaled a_n (coefficients of r^(2n))
};

__device__ double2 lr_eval(const LRKernel &k, double r2) {
  if (k.split == 1) {  // beta erf(beta r)/(beta r)
    const double x = sqrt(r2) * k.beta;
    double v;
    if (x < 1e-3) {
      const double x2 = x * x;
      v = 1.1283791670955126 * (1.0 - x2 / 3.0 + x2 * x2 / 10.0);
    } else {
      v = erf(x) / x;
    }
    return make_double2(k.beta * v, 0.0);
  }
  if (r2 > k.R2) {
    const double r = sqrt(r2);
    if (k.func == 0) return make_double2(1.0 / r, 0.0);
    if (k.func == 1) return make_double2(pow(r2, 0.5 * k.alpha), 0.0);
    double s, c;
    sincos(k.k0r * r, &s, &c);
    const double d = exp(-k.k0i * r) / r;
    return make_double2(c * d, s * d);
  }
  double pr = k.ar[k.nder], pi = k.ai[k.nder];
  for (int n = k.nder - 1; n >= 0; n--) {
    pr = fma(pr, r2, k.ar[n]);
    pi = fma(pi, r2, k.ai[n]);
  }
  return make_double2(pr, pi);
}

struct BuiltinLR {
  LRKernel k;
  __device__ double2 operator()(double r2) const { return lr_eval(k, r2); }
};

// The same, reading the parameters where they lie (a batch's descriptors in
// global memory) instead of copying them
struct BuiltinLRRef {
  const LRKernel *k;
  __device__ double2 operator()(double r2) const { return lr_eval(*k, r2); }
};

// CPLX: complex samples (double2); else the real part only (double), for
// the real kernels, whose transform then runs in real arithmetic.
template <bool CPLX>
__global__ void sample_fhat_kernel(LRKernel k, int M1, int M2, int M3,
                                   const double *__restrict__ ax,  // 4*M per axis: x1,x2,T1,T2
                                   const double *__restrict__ ay,
                                   const double *__restrict__ az, void *out) {
  const long total = (long)M1 * M2 * M3;
  const BuiltinLR lr{k};
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    const double2 f = fhat_sample_body(lr, idx, M1, M2, M3, ax, ay, az);
    if (CPLX) static_cast<double2 *>(out)[idx] = f;
    else static_cast<double *>(out)[idx] = f.x;
  }
}

// The DCT-I along one axis of the M1 x M2 x M3 compact octant,
//   out[k] = f[0] + (-1)^k f[M-1] + 2 sum_{j=1}^{M-2} f[j] cos(2 pi j k / N),
// is the matrix product out[k, line] = sum_j C[k, j] f[j, line] over all
// lines of that axis, with C[k, j] = c_j cos(2 pi (j k mod N) / N), c_0 =
// c_{M-1} = 1, else 2 (cos(pi k) = (-1)^k for j = M - 1 = N/2).

// C (M x M, row k) from the cosine table cosN[m] = cos(2 pi m / N)
__global__ void dct1_matrix_kernel(const double *__restrict__ cosN, int M, int N,
                                   double *__restrict__ C) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)M * M) return;
  const int k = (int)(t / M), j = (int)(t - (long)k * M);
  const double c = (j == 0 || j == M - 1) ? 1.0 : 2.0;
  C[t] = c * cosN[(int)(((long)j * k) % N)];
}

// Offset of element j of line `line` along axis `ax`.
__device__ __forceinline__ long dct_addr(int ax, long line, int j, int M2, int M3) {
  if (ax == 0) return line + (long)j * M2 * M3;        // lines (i2, i3)
  if (ax == 1) return (line / M3) * (long)M2 * M3 + line % M3 + (long)j * M3;  // (i1, i3)
  return line * M3 + j;                                 // lines (i1, i2)
}

// Tiled FP64 GEMM: a CTA computes 64 outputs k for 32 lines; tiles of C
// (64 x 16) and of the input (16 x 32) pass through shared memory.  CPLX:
// complex lines (double2); else real lines (double), half the work.
constexpr int kDctK = 64, kDctL = 32, kDctJ = 16;
template <bool CPLX>
__global__ void __launch_bounds__(256) dct1_gemm_kernel(const void *__restrict__ in_,
                                                        void *__restrict__ out_,
                                                        const double *__restrict__ C, int ax,
                                                        int M, long nlines, int M2, int M3) {
  using V = typename std::conditional<CPLX, double2, double>::type;
  const V *__restrict__ in = static_cast<const V *>(in_);
  V *__restrict__ out = static_cast<V *>(out_);
  __shared__ double Cs[kDctK][kDctJ + 1];
  __shared__ V Fs[kDctJ][kDctL];
  const int tl = threadIdx.x & 31, tk = threadIdx.x >> 5;  // line in tile, k group
  const long l0 = (long)blockIdx.x * kDctL;
  const int k0 = blockIdx.y * kDctK;
  double ar[8], ai[8];
#pragma unroll
  for (int r = 0; r < 8; r++) ar[r] = ai[r] = 0.0;
  for (int j0 = 0; j0 < M; j0 += kDctJ) {
    for (int t = threadIdx.x; t < kDctK * kDctJ; t += 256) {
      const int kk = t / kDctJ, jj = t % kDctJ;
      Cs[kk][jj] = (k0 + kk < M && j0 + jj < M) ? C[(long)(k0 + kk) * M + j0 + jj] : 0.0;
    }
    for (int t = threadIdx.x; t < kDctJ * kDctL; t += 256) {
      const int jj = t / kDctL, ll = t % kDctL;
      const long line = l0 + ll;
      Fs[jj][ll] = (line < nlines && j0 + jj < M) ? in[dct_addr(ax, line, j0 + jj, M2, M3)] : V{};
    }
    __syncthreads();
#pragma unroll
    for (int jj = 0; jj < kDctJ; jj++) {
      const V f = Fs[jj][tl];
#pragma unroll
      for (int r = 0; r < 8; r++) {
        const double c = Cs[tk + 8 * r][jj];
        if constexpr (CPLX) {
          ar[r] = fma(c, f.x, ar[r]);
          ai[r] = fma(c, f.y, ai[r]);
        } else {
          ar[r] = fma(c, f, ar[r]);
        }
      }
    }
    __syncthreads();
  }
  const long line = l0 + tl;
  if (line >= nlines) return;
#pragma unroll
  for (int r = 0; r < 8; r++) {
    const int k = k0 + tk + 8 * r;
    if (k >= M) continue;
    if constexpr (CPLX) out[dct_addr(ax, line, k, M2, M3)] = make_double2(ar[r], ai[r]);
    else out[dct_addr(ax, line, k, M2, M3)] = ar[r];
  }
}

// The same transform with the CTA's whole panel staged at once: the 64 rows
// k0.. of C (all M columns) and its 32 lines (all M elements) go to shared
// memory in one load phase, then every thread runs its 8 outputs over all j.
// The per-output sums run over j in the same order as the tiled kernel (whose
// padding adds exact zeros), so both give the same values; this one pays the
// load latency once instead of once per 16 columns, which is what bounds the
// transform at the small FFT boxes of a serving stream.  Used while the panel
// fits the shared memory of a CTA (on B200: M <= 299 real, 223 complex).
template <bool CPLX>
__device__ __forceinline__ void dct1_panel_body(const void *__restrict__ in_,
                                                void *__restrict__ out_,
                                                const double *__restrict__ C, int ax, int M,
                                                long nlines, int M2, int M3, long bx, int by,
                                                double2 *dct_panel) {
  using V = typename std::conditional<CPLX, double2, double>::type;
  const V *__restrict__ in = static_cast<const V *>(in_);
  V *__restrict__ out = static_cast<V *>(out_);
  // Fs rows padded by one element: the loads along j (lines of the last
  // axis) then store to different banks
  constexpr int FL = kDctL + 1;
  double *Cs = reinterpret_cast<double *>(dct_panel);        // [kDctK][M]
  V *Fs = reinterpret_cast<V *>(Cs + (long)kDctK * M);       // [M][FL]
  const int tl = threadIdx.x & 31, tk = threadIdx.x >> 5;
  const long l0 = bx * kDctL;
  const int k0 = by * kDctK;
  const int krows = min(kDctK, M - k0);
  for (int t = threadIdx.x; t < kDctK * M; t += 256)
    Cs[t] = t < krows * M ? C[(long)k0 * M + t] : 0.0;  // rows k0.. are contiguous
  for (int t = threadIdx.x; t < M * kDctL; t += 256) {
    // consecutive threads on consecutive addresses: along j for lines of the
    // last axis (contiguous), along the lines otherwise
    int jj, ll;
    if (ax == 2) ll = t / M, jj = t - ll * M;
    else jj = t / kDctL, ll = t - jj * kDctL;
    const long line = l0 + ll;
    Fs[jj * FL + ll] = line < nlines ? in[dct_addr(ax, line, jj, M2, M3)] : V{};
  }
  __syncthreads();
  double ar[8], ai[8];
#pragma unroll
  for (int r = 0; r < 8; r++) ar[r] = ai[r] = 0.0;
  for (int j = 0; j < M; j++) {
    const V f = Fs[j * FL + tl];
#pragma unroll
    for (int r = 0; r < 8; r++) {
      const double c = Cs[(tk + 8 * r) * M + j];
      if constexpr (CPLX) {
        ar[r] = fma(c, f.x, ar[r]);
        ai[r] = fma(c, f.y, ai[r]);
      } else {
        ar[r] = fma(c, f, ar[r]);
      }
    }
  }
  const long line = l0 + tl;
  if (line >= nlines) return;
#pragma unroll
  for (int r = 0; r < 8; r++) {
    const int k = k0 + tk + 8 * r;
    if (k >= M) continue;
    if constexpr (CPLX) out[dct_addr(ax, line, k, M2, M3)] = make_double2(ar[r], ai[r]);
    else out[dct_addr(ax, line, k, M2, M3)] = ar[r];
  }
}

template <bool CPLX>
__global__ void __launch_bounds__(256) dct1_panel_kernel(const void *__restrict__ in,
                                                         void *__restrict__ out,
                                                         const double *__restrict__ C, int ax,
                                                         int M, long nlines, int M2, int M3) {
  extern __shared__ double2 dct_panel[];
  dct1_panel_body<CPLX>(in, out, C, ax, M, nlines, M2, M3, blockIdx.x, blockIdx.y, dct_panel);
}

// Shared memory of a dct1_panel_kernel CTA, or 0 when the panel does not fit
// the limit.
static size_t dct_panel_bytes(int M, bool cplx, size_t limit) {
  const size_t b = sizeof(double) * (size_t)M * (kDctK + (cplx ? 2 : 1) * (kDctL + 1));
  return b <= limit ? b : 0;
}

// G = F * lambda^2 products / volume.  CPLX_IN: F complex (double2), else
// real (double); CPLX: the complex kernel's (re, im) output, else the real
// part only.
template <typename T, bool CPLX, bool CPLX_IN>
__device__ __forceinline__ void scale_fhat_body(const void *__restrict__ F_, long idx, int M2,
                                                int M3, const double *__restrict__ l1,
                                                const double *__restrict__ l2,
                                                const double *__restrict__ l3, double inv_vol,
                                                T *G) {
  const int i3 = idx % M3, i2 = (idx / M3) % M2, i1 = idx / ((long)M2 * M3);
  const double s = l1[i1] * l2[i2] * l3[i3] * inv_vol;
  const double2 F = CPLX_IN ? static_cast<const double2 *>(F_)[idx]
                            : make_double2(static_cast<const double *>(F_)[idx], 0.0);
  if (CPLX) {
    G[2 * idx] = (T)(F.x * s);
    G[2 * idx + 1] = (T)(F.y * s);
  } else {
    G[idx] = (T)(F.x * s);
  }
}

template <typename T, bool CPLX, bool CPLX_IN>
__global__ void scale_fhat_kernel(const void *__restrict__ F_, int M1, int M2, int M3,
                                  const double *__restrict__ l1, const double *__restrict__ l2,
                                  const double *__restrict__ l3, double inv_vol, T *G) {
  const long total = (long)M1 * M2 * M3;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x)
    scale_fhat_body<T, CPLX, CPLX_IN>(F_, idx, M2, M3, l1, l2, l3, inv_vol, G);
}

// Host B-spline (same recurrence as the device one) for lambda^2.
static double bspline_host(int n, double w) {
  if (w < 0.0 || w >= (double)n) return 0.0;
  const int i0 = (int)std::floor(w);
  const double u = w - i0;
  double c[64];
  c[0] = 1.0;
  for (int j = 1; j < n; j++)
    for (int k = j; k >= 0; k--) {
      const double x = u + k;
      const double left = (k <= j - 1) ? c[k] : 0.0;
      const double right = (k >= 1) ? c[k - 1] : 0.0;
      c[k] = (x * left + ((double)(j + 1) - x) * right) / (double)j;
    }
  return c[i0];
}

// |1/sum_p B_n(p) exp(-2 pi i k p / N)|^2 for k = 0..N/2 (src/RecSumV.cpp:565-581)
static void lambda2_host(long N, int order, std::vector<double> &out) {
  std::vector<double> b(order + 1);
  for (int p = 0; p <= order; p++) b[p] = bspline_host(order, p);
  out.resize(N / 2 + 1);
  for (long k = 0; k <= N / 2; k++) {
    const double z = (double)k / (double)N;
    double dr = 0, di = 0;
    for (int p = 0; p <= order; p++) {
      dr += b[p] * std::cos(2.0 * M_PI * z * p);
      di -= b[p] * std::sin(2.0 * M_PI * z * p);
    }
    out[k] = 1.0 / (dr * dr + di * di);
  }
}

// lambda^2 (per N and order) and cos(2 pi m / N) (per N) of every axis a
// process has seen: a serving process meets the same few FFT lengths again
// and again, and the kernel transform of each request needs them.
struct AxisTables {
  std::vector<double> lam, cosines;
};
static std::mutex g_axis_mu;
static std::map<std::pair<long, int>, std::shared_ptr<const AxisTables>> g_axis_tables;

static std::shared_ptr<const AxisTables> axis_tables(long N, int order) {
  std::lock_guard<std::mutex> lk(g_axis_mu);
  auto &slot = g_axis_tables[std::make_pair(N, order)];
  if (!slot) {
    auto t = std::make_shared<AxisTables>();
    lambda2_host(N, order, t->lam);
    t->cosines.resize(N);
    for (long m = 0; m < N; m++) t->cosines[m] = std::cos(2.0 * M_PI * (double)m / (double)N);
    slot = t;
  }
  return slot;
}

static double hramp(double x, double a) {
  const double erf_max = 6.0;
  if (x < -1.0) return 0.0;
  if (x > 1.0) return 1.0;
  const double z = erf_max / a, xMax = z / std::sqrt(1.0 + z * z);
  if (x >= xMax) return 1.0;
  if (x <= -xMax) return 0.0;
  return 0.5 * (1.0 + std::erf(a * x / std::sqrt(1.0 - x * x)));
}

// Top-hat window of half width X falling to 0 at Xmax (src/RecSumGrid.cpp:1124-1170)
static double tsmooth(double x, double X, double Xmax, double a) {
  const double del = (Xmax - X) * 0.5;
  if (x < -X) return hramp((x + X + del) / del, a);
  if (x <= X) return 1.0;
  return hramp((-x + X + del) / del, a);
}

// x1, x2, T1, T2 for one axis (src/RecSumGrid.cpp:1181-1212)
static void window_axis(long N, double X, double del, double a, std::vector<double> &v) {
  const long M = N / 2 + 1;
  const double Xmax = X + del, h = 2 * Xmax / N;
  v.assign(4 * M, 0.0);
  for (long i = 0; i < M; i++) {
    const double x1 = i * h;
    double x2, T1, T2;
    if (x1 > X) {
      T1 = tsmooth(x1, X, 2 * Xmax - X, a);
      x2 = x1 - 2 * Xmax;
      T2 = tsmooth(x2, X, 2 * Xmax - X, a);
    } else if (x1 > -X) {
      T1 = 1.0, x2 = 1.0, T2 = 0.0;
    } else {
      T1 = tsmooth(x1, X, 2 * Xmax - X, a);
      x2 = x1 + 2 * Xmax;
      T2 = tsmooth(x2, X, 2 * Xmax - X, a);
    }
    v[i] = x1, v[M + i] = x2, v[2 * M + i] = T1, v[3 * M + i] = T2;
  }
}

#define NPME_CK(call)                                          \
  do {                                                         \
    cudaError_t e_ = (call);                                   \
    if (e_ != cudaSuccess) {                                   \
      h->err = std::string(#call) + ": " + cudaGetErrorString(e_); \
      return NPME_ECUDA;                                       \
    }                                                          \
  } while (0)

// DCT-I matrices, one per (device, FFT length) for the whole process, like
// the FFT plans: a serving process meets the same few lengths again and
// again, while its handles move between lengths.  Built on the stream of the
// first handle that needs one; later users wait for that construction's
// event (complete long before, as a rule) and share the matrix read-only.
// Never freed: M x M doubles per length seen (133 KB at N = 256).
namespace {
struct DctMatrix {
  double *d = nullptr;
  cudaEvent_t built = nullptr;
};
std::mutex g_dct_mu;
std::map<std::pair<int, long>, DctMatrix> g_dct;
}  // namespace

static int dct_matrix(npme_handle *h, cudaStream_t s, long N, const double *d_cos,
                      double **out) {
  std::lock_guard<std::mutex> lk(g_dct_mu);
  DctMatrix &m = g_dct[std::make_pair(h->device, N)];
  if (!m.d) {
    const long M = N / 2 + 1;
    cudaError_t e = cudaMalloc(&m.d, sizeof(double) * M * M);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&m.built, cudaEventDisableTiming);
    if (e == cudaSuccess) {
      dct1_matrix_kernel<<<(unsigned)((M * M + 255) / 256), 256, 0, s>>>(d_cos, (int)M, (int)N, m.d);
      e = cudaEventRecord(m.built, s);
    }
    if (e != cudaSuccess) {
      if (m.d) cudaFree(m.d);
      if (m.built) cudaEventDestroy(m.built);
      m = DctMatrix{};
      cudaGetLastError();
      h->err = std::string("DCT matrix: ") + cudaGetErrorString(e);
      return NPME_ECUDA;
    }
  } else if (cudaStreamWaitEvent(s, m.built, 0) != cudaSuccess) {
    h->err = "DCT matrix: stream wait failed";
    return NPME_ECUDA;
  }
  *out = m.d;
  return NPME_OK;
}

// One handle's kernel transform as its launches see it.
struct KtSys {
  LRKernel k;
  const double *ax[3];   // window tables x1, x2, T1, T2 per axis
  const double *lam[3];  // lambda^2 per axis
  const double *C[3];    // DCT-I matrix per axis
  void *ft0, *ft1;       // scratch octants
  void *G;               // output: the handle's d_G
  double inv_vol;
  int M[3];
  long start;            // first element in a batch's concatenated octants
  long tile0[3];         // first DCT tile in the batch, per axis
};

// Host side of a handle's kernel transform: scratch, per-axis tables copied
// to the device on stream s, the DCT-I matrices, and the descriptor of its
// launches.  Buffers come from the handle's stream; when s is another
// stream, s waits for them.
static int kt_prepare(npme_handle *h, cudaStream_t s, KtSys *d) {
  const long *N = h->grid.N;
  const int M1 = N[0] / 2 + 1, M2 = N[1] / 2 + 1, M3 = N[2] / 2 + 1;
  const long MT = (long)M1 * M2 * M3;
  const double dels[3] = {h->p.del1, h->p.del2, h->p.del3};
  const double as[3] = {h->p.a1, h->p.a2, h->p.a3};
  std::vector<double> ax[3];
  std::shared_ptr<const AxisTables> tab[3];
  for (int a = 0; a < 3; a++) {
    window_axis(N[a], h->box[a], dels[a], as[a], ax[a]);
    tab[a] = axis_tables(N[a], h->grid.order);
  }
  LRKernel &k = d->k;
  k = LRKernel{};
  k.func = h->p.funcType;
  k.split = h->p.EwaldSplit;
  k.nder = h->p.nDeriv;
  k.R2 = h->p.Rdir * h->p.Rdir;
  k.alpha = h->p.alpha;
  k.beta = h->beta;
  k.k0r = h->p.k0_r;
  k.k0i = h->p.k0_i;
  for (int i = 0; i <= k.nder && i < 32; i++) k.ar[i] = h->a_r[i], k.ai[i] = h->a_i[i];
  // scratch kept by the handle, so a new geometry on the same handle reuses it
  int rc = NPME_OK;
  if ((rc = handle_buffer(h, (void **)&h->d_ft0, sizeof(double2) * MT)) ||
      (rc = handle_buffer(h, (void **)&h->d_ft1, sizeof(double2) * MT)))
    return rc;
  // the per-axis tables (window x1, x2, T1, T2; lambda^2; cosines of the
  // DCT) go through one pinned staging block kept by the handle, in one
  // asynchronous copy; the next set-up on the handle waits for the copy
  // before it refills the block
  size_t off[3][3], total = 0;
  for (int a = 0; a < 3; a++) {
    off[a][0] = total, total += ax[a].size();
    off[a][1] = total, total += tab[a]->lam.size();
    off[a][2] = total, total += (size_t)N[a];
  }
  if ((rc = pinned_block(h, (void **)&h->h_fstage, &h->fstage_cap, sizeof(double) * total)))
    return rc;
  for (int a = 0; a < 3; a++) {
    std::copy(ax[a].begin(), ax[a].end(), h->h_fstage + off[a][0]);
    std::copy(tab[a]->lam.begin(), tab[a]->lam.end(), h->h_fstage + off[a][1]);
    std::copy(tab[a]->cosines.begin(), tab[a]->cosines.end(), h->h_fstage + off[a][2]);
  }
  if ((rc = handle_buffer(h, (void **)&h->d_ftab, sizeof(double) * total))) return rc;
  if (s != h->stream) {
    NPME_CK(cudaEventRecord(h->ev_fork, h->stream));
    NPME_CK(cudaStreamWaitEvent(s, h->ev_fork, 0));
  }
  NPME_CK(cudaMemcpyAsync(h->d_ftab, h->h_fstage, sizeof(double) * total, cudaMemcpyHostToDevice,
                          s));
  for (int a = 0; a < 3; a++) {
    h->d_fax[a] = h->d_ftab + off[a][0];
    h->d_flam[a] = h->d_ftab + off[a][1];
    h->d_fcos[a] = h->d_ftab + off[a][2];
    d->ax[a] = h->d_fax[a];
    d->lam[a] = h->d_flam[a];
    double *C = nullptr;
    if ((rc = dct_matrix(h, s, N[a], h->d_fcos[a], &C))) return rc;
    d->C[a] = C;
  }
  d->ft0 = h->d_ft0, d->ft1 = h->d_ft1, d->G = h->d_G;
  d->inv_vol = 1.0 / ((double)N[0] * N[1] * N[2]);
  d->M[0] = M1, d->M[1] = M2, d->M[2] = M3;
  d->start = 0;
  d->tile0[0] = d->tile0[1] = d->tile0[2] = 0;
  return NPME_OK;
}

// DCT tiles of one axis: (lines / 32) x (outputs / 64)
static long kt_tiles(const KtSys &d, int a, long *nx) {
  const int M = d.M[a];
  const long nlines = (long)d.M[0] * d.M[1] * d.M[2] / M;
  *nx = (nlines + kDctL - 1) / kDctL;
  return *nx * ((M + kDctK - 1) / kDctK);
}

// Batched stages: every handle of a set-up pass is a system with its own
// octant; element and tile indices run over the concatenation of the
// systems' octants and tiles, mapped back by binary search over their starts.
__device__ __forceinline__ int kt_owner_elem(const KtSys *__restrict__ d, int R, long idx) {
  int lo = 0, hi = R - 1;
  while (lo < hi) {
    const int m = (lo + hi + 1) >> 1;
    if (d[m].start <= idx) lo = m;
    else hi = m - 1;
  }
  return lo;
}

__device__ __forceinline__ int kt_owner_tile(const KtSys *__restrict__ d, int R, int a, long t) {
  int lo = 0, hi = R - 1;
  while (lo < hi) {
    const int m = (lo + hi + 1) >> 1;
    if (d[m].tile0[a] <= t) lo = m;
    else hi = m - 1;
  }
  return lo;
}

template <bool CPLX>
__global__ void batch_sample_fhat_kernel(const KtSys *__restrict__ d, int R, long total) {
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    const KtSys &D = d[kt_owner_elem(d, R, idx)];
    const long i = idx - D.start;
    const BuiltinLRRef lr{&D.k};
    const double2 f = fhat_sample_body(lr, i, D.M[0], D.M[1], D.M[2], D.ax[0], D.ax[1], D.ax[2]);
    if (CPLX) static_cast<double2 *>(D.ft0)[i] = f;
    else static_cast<double *>(D.ft0)[i] = f.x;
  }
}

// Axis a of every system: pass 0 reads ft0 and writes ft1, pass 1 back,
// pass 2 ft0 -> ft1 again (the single-system order).
template <bool CPLX>
__global__ void __launch_bounds__(256) batch_dct1_panel_kernel(const KtSys *__restrict__ d, int R,
                                                               int a) {
  extern __shared__ double2 dct_panel[];
  const KtSys &D = d[kt_owner_tile(d, R, a, blockIdx.x)];
  const long t = blockIdx.x - D.tile0[a];
  const int M = D.M[a];
  const long nlines = (long)D.M[0] * D.M[1] * D.M[2] / M;
  const long nx = (nlines + kDctL - 1) / kDctL;
  const void *src = (a == 1) ? D.ft1 : D.ft0;
  void *dst = (a == 1) ? D.ft0 : D.ft1;
  dct1_panel_body<CPLX>(src, dst, D.C[a], a, M, nlines, D.M[1], D.M[2], t % nx, (int)(t / nx),
                        dct_panel);
}

template <typename T, bool CPLX, bool CPLX_IN>
__global__ void batch_scale_fhat_kernel(const KtSys *__restrict__ d, int R, long total) {
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    const KtSys &D = d[kt_owner_elem(d, R, idx)];
    // after three passes the transform is in ft1
    scale_fhat_body<T, CPLX, CPLX_IN>(D.ft1, idx - D.start, D.M[1], D.M[2], D.lam[0], D.lam[1],
                                      D.lam[2], D.inv_vol, (T *)D.G);
  }
}

// The panel kernels' dynamic shared-memory limit, raised once per device to
// the device's opt-in maximum.  The size a launch needs varies with M, and a
// cudaFuncSetAttribute before each launch would race between host threads
// that set up handles at the same time (one lowering the limit under
// another's launch).  The handle's device is current.
static int dct_panel_limit(npme_handle *h, size_t *limit) {
  static std::mutex mu;
  static std::map<int, size_t> done;
  std::lock_guard<std::mutex> lk(mu);
  auto it = done.find(h->device);
  if (it == done.end()) {
    int optin = 0;
    cudaError_t e =
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device);
    const void *kernels[4] = {(const void *)dct1_panel_kernel<true>,
                              (const void *)dct1_panel_kernel<false>,
                              (const void *)batch_dct1_panel_kernel<true>,
                              (const void *)batch_dct1_panel_kernel<false>};
    for (int i = 0; i < 4 && e == cudaSuccess; i++)
      e = cudaFuncSetAttribute(kernels[i], cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
    if (e != cudaSuccess) {
      h->err = std::string("DCT panel limit: ") + cudaGetErrorString(e);
      return NPME_ECUDA;
    }
    it = done.emplace(h->device, (size_t)optin).first;
  }
  *limit = it->second;
  return NPME_OK;
}

// The launches of one handle's transform on stream s.
static int kt_launch_one(npme_handle *h, const KtSys &d, cudaStream_t s) {
  const int M1 = d.M[0], M2 = d.M[1], M3 = d.M[2];
  const long MT = (long)M1 * M2 * M3;
  const int threads = 256, blocks = 148 * 8;
  // the built-in real kernels sample and transform real values; complex
  // kernels and caller-defined ones (whose sampler writes complex values)
  // run the complex transform
  const bool cplx_ft = h->complex_kernel || h->user_kernel;
  int rc = NPME_OK;
  if (h->user_kernel) {
    if ((rc = h->uops.sample_lr(h, M1, M2, M3, d.ax[0], d.ax[1], d.ax[2], (double2 *)d.ft0, s)))
      return rc;
  } else if (cplx_ft) {
    sample_fhat_kernel<true><<<blocks, threads, 0, s>>>(d.k, M1, M2, M3, d.ax[0], d.ax[1],
                                                        d.ax[2], d.ft0);
  } else {
    sample_fhat_kernel<false><<<blocks, threads, 0, s>>>(d.k, M1, M2, M3, d.ax[0], d.ax[1],
                                                         d.ax[2], d.ft0);
  }
  void *src = d.ft0, *dst = d.ft1;
  size_t limit = 0;
  if ((rc = dct_panel_limit(h, &limit))) return rc;
  for (int a = 0; a < 3; a++) {
    const int M = d.M[a];
    const double *C = d.C[a];
    long nx;
    kt_tiles(d, a, &nx);
    const long nlines = MT / M;
    const dim3 grid((unsigned)nx, (unsigned)((M + kDctK - 1) / kDctK));
    const size_t pb = dct_panel_bytes(M, cplx_ft, limit);
    if (pb && cplx_ft) {
      dct1_panel_kernel<true><<<grid, 256, pb, s>>>(src, dst, C, a, M, nlines, M2, M3);
    } else if (pb) {
      dct1_panel_kernel<false><<<grid, 256, pb, s>>>(src, dst, C, a, M, nlines, M2, M3);
    } else if (cplx_ft) {
      dct1_gemm_kernel<true><<<grid, 256, 0, s>>>(src, dst, C, a, M, nlines, M2, M3);
    } else {
      dct1_gemm_kernel<false><<<grid, 256, 0, s>>>(src, dst, C, a, M, nlines, M2, M3);
    }
    std::swap(src, dst);
  }
  const double *const *l = d.lam;
#define NPME_SCALE(T, CX, CI)                                                               \
  scale_fhat_kernel<T, CX, CI><<<blocks, threads, 0, s>>>(src, M1, M2, M3, l[0], l[1], l[2], \
                                                          d.inv_vol, (T *)d.G)
  if (h->fp32) {
    if (h->complex_kernel) NPME_SCALE(float, true, true);
    else if (cplx_ft) NPME_SCALE(float, false, true);
    else NPME_SCALE(float, false, false);
  } else {
    if (h->complex_kernel) NPME_SCALE(double, true, true);
    else if (cplx_ft) NPME_SCALE(double, false, true);
    else NPME_SCALE(double, false, false);
  }
#undef NPME_SCALE
  // launch errors now; set-up waits for the stream before it returns
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    h->err = std::string("kernel transform: ") + cudaGetErrorString(e);
    rc = NPME_ECUDA;
  }
  return rc;
}

int build_kernel_transform(npme_handle *h) {
  KtSys d;
  const int rc = kt_prepare(h, h->stream, &d);
  return rc ? rc : kt_launch_one(h, d, h->stream);
}

// Layout of one class of handles (the same precision and kernel type,
// built-in kernels) in a batch: element and tile starts, the largest panel.
// False when a panel does not fit a CTA or a launch would need 2^31 blocks
// or more: then the class goes handle by handle (tiled transform).
static bool kt_layout(std::vector<KtSys> &ds, bool cplx, size_t limit, long *total,
                      long tiles[3], size_t *pb) {
  *total = 0, tiles[0] = tiles[1] = tiles[2] = 0, *pb = 0;
  for (KtSys &d : ds) {
    d.start = *total;
    *total += (long)d.M[0] * d.M[1] * d.M[2];
    for (int a = 0; a < 3; a++) {
      long nx;
      d.tile0[a] = tiles[a];
      tiles[a] += kt_tiles(d, a, &nx);
      const size_t b = dct_panel_bytes(d.M[a], cplx, limit);
      if (!b) return false;
      *pb = std::max(*pb, b);
    }
  }
  return tiles[0] < (1L << 31) && tiles[1] < (1L << 31) && tiles[2] < (1L << 31);
}

// One launch per stage for a class whose descriptors are at dd on the
// device.
static void kt_launch_class(const KtSys *dd, int R, bool cplx, bool fp32, long total,
                            const long tiles[3], size_t pb, cudaStream_t s) {
  const unsigned eb = (unsigned)std::min<long>((total + 255) / 256, 148 * 8);
  if (cplx) batch_sample_fhat_kernel<true><<<eb, 256, 0, s>>>(dd, R, total);
  else batch_sample_fhat_kernel<false><<<eb, 256, 0, s>>>(dd, R, total);
  for (int a = 0; a < 3; a++) {
    if (cplx) batch_dct1_panel_kernel<true><<<(unsigned)tiles[a], 256, pb, s>>>(dd, R, a);
    else batch_dct1_panel_kernel<false><<<(unsigned)tiles[a], 256, pb, s>>>(dd, R, a);
  }
  if (fp32) {
    if (cplx) batch_scale_fhat_kernel<float, true, true><<<eb, 256, 0, s>>>(dd, R, total);
    else batch_scale_fhat_kernel<float, false, false><<<eb, 256, 0, s>>>(dd, R, total);
  } else {
    if (cplx) batch_scale_fhat_kernel<double, true, true><<<eb, 256, 0, s>>>(dd, R, total);
    else batch_scale_fhat_kernel<double, false, false><<<eb, 256, 0, s>>>(dd, R, total);
  }
}

// The kernel transforms of a set-up pass (one precision), on the owner's
// stream: a class of two or more handles (built-in real kernels, built-in
// complex kernels) in one launch per stage, caller-defined kernels and
// classes of one handle by handle on their own streams.  One launch per
// stage instead of five per handle: about 4 % more served capacity at the
// best passes of a serving stream.
void build_kernel_transforms(npme_handle **hs, int R, npme_handle *owner, int *status) {
  npme_handle *h = owner;  // errors of the shared steps are recorded on the owner
  const cudaStream_t s = owner->stream;
  std::vector<int> cls(R, -1);
  int count[2] = {0, 0};
  for (int r = 0; r < R; r++)
    if (!hs[r]->user_kernel) cls[r] = hs[r]->complex_kernel ? 1 : 0, count[cls[r]]++;
  for (int r = 0; r < R; r++) {
    if (cls[r] >= 0 && count[cls[r]] >= 2) continue;
    cls[r] = -1;
    status[r] = build_kernel_transform(hs[r]);
  }
  size_t limit = 0;
  int rc = NPME_OK;
  const bool any = std::any_of(cls.begin(), cls.end(), [](int c) { return c >= 0; });
  if (!any) return;
  if ((rc = dct_panel_limit(h, &limit))) {
    for (int r = 0; r < R; r++)
      if (cls[r] >= 0) status[r] = rc, hs[r]->err = h->err;
    return;
  }
  // every class's descriptors, in one staging block and one copy (two
  // classes must not share a pinned block that an earlier copy still reads)
  std::vector<KtSys> ds[2];
  std::vector<int> at[2];
  for (int r = 0; r < R; r++) {
    if (cls[r] < 0) continue;
    KtSys d;
    status[r] = kt_prepare(hs[r], s, &d);
    if (!status[r]) ds[cls[r]].push_back(d), at[cls[r]].push_back(r);
  }
  long total[2] = {0, 0}, tiles[2][3];
  size_t pb[2] = {0, 0};
  bool batched[2] = {false, false};
  for (int c = 0; c < 2; c++) {
    if (ds[c].empty()) continue;
    batched[c] = kt_layout(ds[c], c == 1, limit, &total[c], tiles[c], &pb[c]);
    if (!batched[c])
      for (size_t k = 0; k < ds[c].size(); k++)
        status[at[c][k]] = kt_launch_one(hs[at[c][k]], ds[c][k], s);
  }
  const size_t n0 = batched[0] ? ds[0].size() : 0, n1 = batched[1] ? ds[1].size() : 0;
  if (n0 + n1 == 0) return;
  const size_t bytes = sizeof(KtSys) * (n0 + n1);
  auto fail_all = [&](int code) {
    for (int c = 0; c < 2; c++)
      if (batched[c])
        for (int r : at[c]) {
          status[r] = code;
          if (hs[r] != h) hs[r]->err = h->err;
        }
  };
  if ((rc = pinned_block(h, &h->h_ktdesc, &h->ktdesc_cap, bytes)) ||
      (rc = handle_buffer(h, &h->d_ktdesc, bytes)))
    return fail_all(rc);
  KtSys *hd = static_cast<KtSys *>(h->h_ktdesc);
  if (n0) std::copy(ds[0].begin(), ds[0].end(), hd);
  if (n1) std::copy(ds[1].begin(), ds[1].end(), hd + n0);
  cudaError_t e = cudaMemcpyAsync(h->d_ktdesc, hd, bytes, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) {
    const KtSys *dd = static_cast<const KtSys *>(h->d_ktdesc);
    const bool fp32 = owner->fp32;
    if (n0) kt_launch_class(dd, (int)n0, false, fp32, total[0], tiles[0], pb[0], s);
    if (n1) kt_launch_class(dd + n0, (int)n1, true, fp32, total[1], tiles[1], pb[1], s);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    h->err = std::string("kernel transform: ") + cudaGetErrorString(e);
    return fail_all(NPME_ECUDA);
  }
}

// ---------------------------------------------------------------------------
// Per-call charge gather into brick order (spread/interp) and the direct
// sum's source order, converted to the bulk precision.

template <typename T, bool CPLX>
__global__ void gather_kernel(const double *__restrict__ q, const BrickPoint<T> *__restrict__ bp,
                              const uint32_t *__restrict__ dperm, T *__restrict__ qb,
                              T *__restrict__ qc, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x)
    gather_body<T, CPLX>(q, bp, dperm, qb, qc, i);
}

void launch_gather_charges(npme_handle *h, const double *d_q, cudaStream_t s) {
  const int threads = 256;
  const int blocks = (int)std::min<long>((h->n + threads - 1) / threads, 148 * 16);
  if (h->fp32) {
    if (h->complex_kernel)
      gather_kernel<float, true><<<blocks, threads, 0, s>>>(
          d_q, (const BrickPoint<float> *)h->d_bpts, h->d_dperm, (float *)h->d_qb,
          (float *)h->d_qc, (long)h->n);
    else
      gather_kernel<float, false><<<blocks, threads, 0, s>>>(
          d_q, (const BrickPoint<float> *)h->d_bpts, h->d_dperm, (float *)h->d_qb,
          (float *)h->d_qc, (long)h->n);
  } else {
    if (h->complex_kernel)
      gather_kernel<double, true><<<blocks, threads, 0, s>>>(
          d_q, (const BrickPoint<double> *)h->d_bpts, h->d_dperm, (double *)h->d_qb,
          (double *)h->d_qc, (long)h->n);
    else
      gather_kernel<double, false><<<blocks, threads, 0, s>>>(
          d_q, (const BrickPoint<double> *)h->d_bpts, h->d_dperm, (double *)h->d_qb,
          (double *)h->d_qc, (long)h->n);
  }
  h->launches++;
}

// Charges into the direct-sum order only (the bare short-range sum).
template <typename T, bool CPLX>
__global__ void gather_one_kernel(const double *__restrict__ q,
                                  const uint32_t *__restrict__ perm, T *__restrict__ dst,
                                  long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    const long o = perm[i];
    if (CPLX) {
      dst[2 * i] = (T)q[2 * o];
      dst[2 * i + 1] = (T)q[2 * o + 1];
    } else {
      dst[i] = (T)q[o];
    }
  }
}

void launch_gather_direct(npme_handle *h, const double *d_q, void *d_qdst, cudaStream_t s) {
  const int threads = 256;
  const int blocks = (int)std::min<long>((h->n + threads - 1) / threads, 148 * 16);
  const long n = (long)h->n;
  if (h->fp32) {
    if (h->complex_kernel)
      gather_one_kernel<float, true><<<blocks, threads, 0, s>>>(d_q, h->d_dperm, (float *)d_qdst, n);
    else
      gather_one_kernel<float, false><<<blocks, threads, 0, s>>>(d_q, h->d_dperm, (float *)d_qdst, n);
  } else {
    if (h->complex_kernel)
      gather_one_kernel<double, true><<<blocks, threads, 0, s>>>(d_q, h->d_dperm, (double *)d_qdst, n);
    else
      gather_one_kernel<double, false><<<blocks, threads, 0, s>>>(d_q, h->d_dperm, (double *)d_qdst, n);
  }
  h->launches++;
}

// ---------------------------------------------------------------------------
// Spread (src/RecSumQ.cpp:184-314): Q[g] += q B1 B2 B3.  One CTA per
// non-empty brick of kBrick^3 stencil origins.  The CTA accumulates its
// points' stencils into a shared-memory tile of (kBrick + P - 1)^3 grid
// points with shared atomics (FP32: 64-bit fixed point in two native
// 32-bit integer atomics, spread_brick_fixed), then adds the tile to the
// global grid (global atomics only where tiles of neighbouring bricks
// overlap: one add per tile point instead of one per stencil point).  Complex charges are spread
// without conjugation; with the cyclic convolution used here that gives the
// reference's theta for conj(q) spreading (src/RecSumQ.cpp:337) because the
// reference conjugates twice (src/RecSumV.cpp:672).

template <typename T, int P, bool CPLX>
__global__ void __launch_bounds__(256) spread_kernel(
    const int *__restrict__ brick_list, const int *__restrict__ brick_start,
    const BrickPoint<T> *__restrict__ bp, const T *__restrict__ q, T *__restrict__ grid,
    int nb2, int nb3, long N1, long N2, long N3) {
  extern __shared__ unsigned char smem_raw[];
  if constexpr (std::is_same<T, float>::value)
    spread_brick_fixed<P, CPLX>(brick_list[blockIdx.x], brick_start, bp, q, grid, nb2, nb3, N1,
                                N2, N3, reinterpret_cast<int *>(smem_raw));
  else
    spread_brick_body<T, P, CPLX>(brick_list[blockIdx.x], brick_start, bp, q, grid, nb2, nb3, N1,
                                  N2, N3, reinterpret_cast<T *>(smem_raw));
}

template <typename T, bool CPLX, int P>
static void spread_dispatch(npme_handle *h, cudaStream_t s) {
  constexpr int TL = kBrick + P - 1;
  // FP32: two int words per tile value; FP64: one double
  const size_t smem = (sizeof(T) == 4 ? 8 : sizeof(T)) * TL * TL * TL * (CPLX ? 2 : 1);
  auto kern = spread_kernel<T, P, CPLX>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  kern<<<(unsigned)h->n_nonempty, 256, smem, s>>>(
      h->d_brick_list, h->d_brick_start, (const BrickPoint<T> *)h->d_bpts,
      (const T *)h->d_qb, (T *)h->d_grid, (int)h->grid.nb[1], (int)h->grid.nb[2],
      h->grid.N[0], h->grid.N[1], h->grid.N[2]);
}

template <typename T, bool CPLX>
static void spread_order(npme_handle *h, cudaStream_t s) {
  switch (h->grid.order) {
    case 4: spread_dispatch<T, CPLX, 4>(h, s); break;
    case 6: spread_dispatch<T, CPLX, 6>(h, s); break;
    case 8: spread_dispatch<T, CPLX, 8>(h, s); break;
    case 10: spread_dispatch<T, CPLX, 10>(h, s); break;
    case 12: spread_dispatch<T, CPLX, 12>(h, s); break;
    case 14: spread_dispatch<T, CPLX, 14>(h, s); break;
    case 16: spread_dispatch<T, CPLX, 16>(h, s); break;
  }
}

void launch_spread(npme_handle *h, cudaStream_t s) {
  if (h->n_nonempty == 0) return;
  if (h->fp32) {
    if (h->complex_kernel) spread_order<float, true>(h, s);
    else spread_order<float, false>(h, s);
  } else {
    if (h->complex_kernel) spread_order<double, true>(h, s);
    else spread_order<double, false>(h, s);
  }
  h->launches++;
}

// ---------------------------------------------------------------------------
// Fourier-space multiply by the kernel transform G (compact octant storage,
// |k| folding as in src/RecSumV.cpp:639-707).  Real kernels: R2C half
// spectrum N1 x N2 x (N3/2+1), G real.  Complex kernels: full N^3 spectrum,
// G complex.

template <typename T>
__global__ void multiply_real_kernel(typename Vec2<T>::type *__restrict__ X,
                                     const T *__restrict__ G, int N1, int N2, int N3h, int M2,
                                     int M3) {
  const int rows = N1 * N2, lane = threadIdx.x & 31;
  for (int r = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); r < rows;
       r += (int)((gridDim.x * blockDim.x) >> 5))
    multiply_real_row<T>(X, G, r, N1, N2, N3h, M2, M3, lane);
}

template <typename T>
__global__ void multiply_cplx_kernel(typename Vec2<T>::type *__restrict__ X,
                                     const typename Vec2<T>::type *__restrict__ G, int N1, int N2,
                                     int N3, int M2, int M3) {
  const int rows = N1 * N2, lane = threadIdx.x & 31;
  for (int r = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); r < rows;
       r += (int)((gridDim.x * blockDim.x) >> 5))
    multiply_cplx_row<T>(X, G, r, N1, N2, N3, M2, M3, lane);
}

void launch_multiply(npme_handle *h, cudaStream_t s) {
  const long *N = h->grid.N;
  const int M2 = N[1] / 2 + 1, M3 = N[2] / 2 + 1;
  // one warp per spectrum row, 8 rows per CTA, as many CTAs as rows need
  // (at most 148 x 16, each then looping)
  const int threads = 256;
  const int blocks = (int)std::min<long>(148 * 16, (N[0] * N[1] + 7) / 8);
  if (h->complex_kernel) {
    if (h->fp32)
      multiply_cplx_kernel<float><<<blocks, threads, 0, s>>>(
          (float2 *)h->d_grid, (const float2 *)h->d_G, (int)N[0], (int)N[1], (int)N[2], M2, M3);
    else
      multiply_cplx_kernel<double><<<blocks, threads, 0, s>>>(
          (double2 *)h->d_grid, (const double2 *)h->d_G, (int)N[0], (int)N[1], (int)N[2], M2,
          M3);
  } else {
    if (h->fp32)
      multiply_real_kernel<float><<<blocks, threads, 0, s>>>(
          (float2 *)h->d_kgrid, (const float *)h->d_G, (int)N[0], (int)N[1],
          (int)(N[2] / 2 + 1), M2, M3);
    else
      multiply_real_kernel<double><<<blocks, threads, 0, s>>>(
          (double2 *)h->d_kgrid, (const double *)h->d_G, (int)N[0], (int)N[1],
          (int)(N[2] / 2 + 1), M2, M3);
  }
  h->launches++;
}

// ---------------------------------------------------------------------------
// Interpolation (src/RecSumV.cpp:201-306, 308-434): V += sum theta B1 B2 B3,
// dV/dx_d += (N_d / L_d) sum theta dB_d ..., real kernels keep the real part
// (src/RecSumV.cpp:395-398).  One CTA per non-empty brick, which reads the
// brick's theta tile into shared memory; V is accumulated into the
// caller-order output, which already holds the direct sum.

template <typename T, int P, bool CPLX>
__global__ void __launch_bounds__(256) interp_kernel(
    const int *__restrict__ brick_list, const int *__restrict__ brick_start,
    const BrickPoint<T> *__restrict__ bp, const T *__restrict__ theta, double *__restrict__ V,
    int nb2, int nb3, long N1, long N2, long N3, T c1, T c2, T c3, void *vsrc, double vs,
    double gs) {
  extern __shared__ unsigned char smem_raw[];
  interp_brick_body<T, P, CPLX>(brick_list[blockIdx.x], brick_start, bp, theta, V, nb2, nb3, N1,
                                N2, N3, c1, c2, c3, reinterpret_cast<T *>(smem_raw), vsrc, vs,
                                gs);
}

template <typename T, bool CPLX, int P>
static void interp_dispatch(npme_handle *h, double *d_V, cudaStream_t s) {
  constexpr int TL = kBrick + P - 1;
  const size_t smem = sizeof(T) * TL * TL * TL * (CPLX ? 2 : 1);
  const double *L = h->box + 6;
  auto kern = interp_kernel<T, P, CPLX>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  kern<<<(unsigned)h->n_nonempty, 256, smem, s>>>(
      h->d_brick_list, h->d_brick_start, (const BrickPoint<T> *)h->d_bpts, (const T *)h->d_grid,
      d_V, (int)h->grid.nb[1], (int)h->grid.nb[2], h->grid.N[0], h->grid.N[1], h->grid.N[2],
      (T)(h->grid.N[0] / L[0]), (T)(h->grid.N[1] / L[1]), (T)(h->grid.N[2] / L[2]),
      h->merge_pending ? (h->fp32 ? (void *)h->d_vsrc : (void *)h->d_vsrc64) : nullptr,
      h->merge_vs, h->merge_gs);
}

template <typename T, bool CPLX>
static void interp_order(npme_handle *h, double *d_V, cudaStream_t s) {
  switch (h->grid.order) {
    case 4: interp_dispatch<T, CPLX, 4>(h, d_V, s); break;
    case 6: interp_dispatch<T, CPLX, 6>(h, d_V, s); break;
    case 8: interp_dispatch<T, CPLX, 8>(h, d_V, s); break;
    case 10: interp_dispatch<T, CPLX, 10>(h, d_V, s); break;
    case 12: interp_dispatch<T, CPLX, 12>(h, d_V, s); break;
    case 14: interp_dispatch<T, CPLX, 14>(h, d_V, s); break;
    case 16: interp_dispatch<T, CPLX, 16>(h, d_V, s); break;
  }
}

void launch_interp(npme_handle *h, double *d_V, cudaStream_t s) {
  if (h->n_nonempty == 0) return;
  if (h->fp32) {
    if (h->complex_kernel) interp_order<float, true>(h, d_V, s);
    else interp_order<float, false>(h, d_V, s);
  } else {
    if (h->complex_kernel) interp_order<double, true>(h, d_V, s);
    else interp_order<double, false>(h, d_V, s);
  }
  h->merge_pending = false;  // folded in (and cleared) by this launch
  h->launches++;
}

}  // namespace npme
