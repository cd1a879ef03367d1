// Internal declarations of npme_b200: the handle and the kernel launchers.
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>
#include <stdint.h>

#include <chrono>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/npme_gpu.h"
#include "common.cuh"

namespace npme {

// Brick edge (grid points) of the spread tiles.
constexpr int kBrick = 8;
// Warps (one group of 32 targets each) per CTA of the direct sums.
constexpr int kGroupWarps = 4;
// Scratch buffers the device set-up keeps on a handle (setup.cu).
constexpr int kSetupScratch = 48;

// Geometry of the reciprocal-space grid and of the brick decomposition.
struct GridGeom {
  long N[3];      // full FFT box
  long H[3];      // charge octant N/2
  long nb[3];     // bricks per axis over the octant
  int order;
};

// Cells of edge >= Rdir / nNeigh over the points' bounding box (the
// reference's cell geometry, reported by npme_gpu_get_info).
struct CellGeom {
  int nc[3];       // cells per axis
  double origin[3];
  double edge[3];  // cell edge >= Rdir / nNeigh
  int reach;       // neighbour cells per direction = nNeigh
};

// One spread/interp record per point in brick order.  g0 packs the three
// stencil origins (10 bits each, grid index in the octant).
template <typename T>
struct BrickPoint {
  T u[3];
  uint32_t g0;
  uint32_t orig;  // caller's index
};

struct Timing {
  bool enabled = false;
  bool serial = false;  // the direct sum after the reciprocal chain (stage attribution)
  cudaEvent_t ev[10] = {};
};

// A cuFFT plan shared by every handle with the same FFT box and type (fft.cu).
struct FFTPlan {
  cufftHandle plan = 0;
  int type = 0;
  size_t work = 0;  // work-area bytes the caller provides
  std::mutex mu;    // guards stream / work-area binding + enqueue
};

}  // namespace npme

struct npme_handle {
  npme_params p;
  int device = 0;
  bool complex_kernel = false;
  bool user_kernel = false;  // funcType NPME_FUNC_USER: launches from uops
  npme_user_ops uops = {};
  bool fp32 = true;
  bool ready = false;
  std::string err;

  // set-up state
  size_t n = 0;
  double box[9];  // X Y Z R[3] L[3]
  double bmin[3], bmax[3];  // bounding box of the points
  double fself_r = 0, fself_i = 0;
  double a_r[32], a_i[32], b_r[32], b_i[32];
  double beta = 0;
  npme::GridGeom grid;
  npme::CellGeom cells;
  long n_bricks = 0, n_nonempty = 0;

  cudaStream_t stream = nullptr;
  cudaStream_t stream2 = nullptr;  // direct sum runs here, overlapped with the FFTs
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // shared plans (not owned): (y, z) slab transforms forward and inverse,
  // and the transforms along x (fft.cu)
  npme::FFTPlan *pf = nullptr, *pi = nullptr, *px = nullptr;
  void *d_work = nullptr;                        // this handle's cuFFT work area
  cudaMemPool_t pool = nullptr;                  // device memory pool (shared, not owned)

  // device buffers (all allocated in setup; calcv allocates nothing)
  double *d_coord = nullptr;     // original order, FP64 (exact sum, FP64 direct)
  void *d_bpts = nullptr;        // BrickPoint<T>[n]
  int *d_brick_start = nullptr;  // [n_bricks + 1]
  int *d_brick_list = nullptr;   // non-empty brick ids
  uint32_t *d_cperm = nullptr;   // group order (direct-sum targets) -> caller index
  void *d_qb = nullptr;          // charges in brick order (T or T2)
  void *d_qc = nullptr;          // charges in the direct sum's source order (T or T2)
  void *d_grid = nullptr;        // spread grid, real N1 N2 N3 (or complex)
  void *d_kgrid = nullptr;       // transformed grid N1 N2 (N3/2+1) complex (real kernels)
  void *d_theta = nullptr;       // theta, same layout as d_grid (real kernels)
  void *d_G = nullptr;           // kernel transform on the octant (N/2+1)^3, T or T2
  double *d_q_in = nullptr;      // staging for host charges (n or 2n doubles)
  double *d_V = nullptr;         // staging for host output (4n or 8n doubles)
  double *d_V_exact = nullptr;
  int *d_err = nullptr;          // device error flag
  uint32_t *d_tidx = nullptr;    // target list of the exact subset sum
  size_t dev_bytes = 0;
  std::map<void *, size_t> caps;  // pointer field -> capacity of its buffer
  // kernel-transform construction scratch (kept to reuse across set-ups)
  double2 *d_ft0 = nullptr, *d_ft1 = nullptr;
  double *d_ftab = nullptr;    // per-axis tables of the transform, one block:
  double *d_fax[3] = {nullptr, nullptr, nullptr};   //   windows (views into d_ftab)
  double *d_flam[3] = {nullptr, nullptr, nullptr};  //   lambda^2
  double *d_fcos[3] = {nullptr, nullptr, nullptr};  //   cos(2 pi m / N)
  // pinned host staging (pinned_block; back to the process-wide cache at
  // destroy), capacities in bytes
  double *h_fstage = nullptr;  // the kernel transform's per-axis tables
  void *h_counts = nullptr;    // set-up counts of the batches this handle owned
  void *h_desc = nullptr;      // set-up descriptors of those batches
  void *h_ktdesc = nullptr;    // kernel-transform descriptors of those batches
  size_t fstage_cap = 0, counts_cap = 0, desc_cap = 0, ktdesc_cap = 0;
  void *d_ktdesc = nullptr;    // the same on the device
  // device set-up scratch (sort keys, counts, group records), kept to reuse
  void *d_su[npme::kSetupScratch] = {};

  // direct sum (both precisions): warp groups of <= 32 z-sorted points of
  // one xy column and, per group, the source segments (neighbour-column z
  // ranges) that can hold a point within Rdir of the group.  Built once per
  // geometry.
  long n_groups = 0, n_segs = 0;
  double cand_per_point = 0;     // staged source candidates per target point
  double refine2 = 0;            // r^2 below which pair differences are refined
  double4 *d_gpos = nullptr;     // targets in group order, FP64 positions
  double4 *d_spos = nullptr;     // sources in fine-column order, FP64 positions
  uint32_t *d_sperm = nullptr;   // source order -> caller index
  uint32_t *d_bperm = nullptr;   // brick order position -> caller index
  const uint32_t *d_dperm = nullptr;  // gather order of the direct-sum charges (d_sperm or d_cperm)
  int4 *d_groups = nullptr;      // (first point, count, first segment, end segment)
  double4 *d_gcen = nullptr;     // group frame origin (bbox centre)
  int2 *d_segs = nullptr;        // (first point, count)
  // real-kernel direct sum with every pair evaluated once: the same groups
  // with their half-shell segments (sources in later coarse columns, or later
  // in the group's own column), ordered by their own work
  bool use_sym = true;
  long n_hgroups = 0, n_hsegs = 0;
  double hcand_per_point = 0;    // half-shell candidates per target point
  int4 *d_hgroups = nullptr;
  double4 *d_hcen = nullptr;
  int2 *d_hsegs = nullptr;
  // the source-side sums are indexed by the source point's position in the
  // brick order (spos[k].w holds it), so that the interpolation, which visits
  // the points in that order, can fold them into V
  float4 *d_vsrc = nullptr;      // FP32: source-side sums (two float4 if complex), kept zero
  double *d_vsrc64 = nullptr;    // FP64: source-side sums [n][4], kept zero
  // CalcV leaves the source-side sums of its pair-once walk to the
  // interpolation (scale vs for the potential, gs for the gradient)
  bool merge_pending = false;
  double merge_vs = 1.0, merge_gs = 1.0;

  npme::Timing timing;
  bool timing_pending = false;
  float stage_ms[8] = {0};
  int launches = 0;

  // CalcV replayed as a CUDA graph: captured at the second call with the
  // same device buffers after a set-up, launched as one graph from then on.
  // setup_gen counts set-ups and parameter changes; a graph belongs to one.
  bool graph_enabled = true;
  cudaGraphExec_t graph = nullptr;
  unsigned long long setup_gen = 1, graph_gen = 0, seen_gen = 0, nograph_gen = 0;
  double *graph_V = nullptr, *seen_V = nullptr;
  const double *graph_q = nullptr, *seen_q = nullptr;
  int graph_launches = 0;
};

namespace npme {

// npme_gpu.cu: capacity-tracked device buffer owned by the handle
int handle_buffer(npme_handle *h, void **field, size_t bytes);
// npme_gpu.cu: pinned host block of at least `bytes` in *block (capacity in
// *cap); the block held before, if any, goes back to the process-wide cache,
// so the caller makes sure no copy from or to it is still in flight.  Blocks
// come from and return to that cache: cudaFreeHost synchronises the whole
// device and cudaHostAlloc pins pages, both too slow for a server that
// creates and retires handles while other requests run.
int pinned_block(npme_handle *h, void **block, size_t *cap, size_t bytes);
// returns a handle's pinned block to the cache (destroy)
void pinned_return(void **block, size_t *cap);
// PME-corrected half extent X of a box of half extent X0 for an N-point FFT
// axis (src/RecSumSupportFunctions.cpp:137-147)
double compact_extent(double X0, double del, long order, long N);

// setup.cu: the caller's coordinates to d_coord, their bounding box (and
// the non-finite check) read back into mn / mx
int device_bbox(npme_handle *h, const double *coord, double mn[3], double mx[3]);
// brick order, direct-sum orders, warp groups and segments, buffers of R
// handles of one precision in one pass on stream s (each with its box, grid
// geometry and bmin / bmax set, its coordinates on its own stream); hs[0]
// owns the scratch.  Enqueued without waiting: the counts reach
// hs[0]->h_counts with the caller's synchronisation.
int setup_geometry(npme_handle **hs, int R, cudaStream_t s);
// after that synchronisation: system r's counts (from owner) into handle h,
// and its stencil check
int finish_setup(npme_handle *h, const npme_handle *owner, int r);
// Sets up R handles (npme_gpu_setup's work for each, geometry in shared
// passes); status[r] is each handle's result (its message in h->err).
// Returns NPME_OK when every handle was set up.
int setup_many(npme_handle **hs, int R, const size_t *n, const double *const *coord,
               int *status);

// fft.cu
int prepare_plans(npme_handle *h);
// zeroes what the spread adds into and the forward transform reads
int grid_clear(npme_handle *h, cudaStream_t s);
int fft_forward(npme_handle *h, cudaStream_t s);
int fft_inverse(npme_handle *h, cudaStream_t s);

// recsum.cu
int build_kernel_transform(npme_handle *h);  // F-hat, lambda^2 -> d_G
// The kernel transforms of several handles (one precision), on the owner's
// stream: one launch per stage for every class of two or more handles with
// a built-in kernel (real, complex), the rest one by one on their own
// streams.  status[k] gets each handle's result.
void build_kernel_transforms(npme_handle **hs, int R, npme_handle *owner, int *status);
void launch_gather_charges(npme_handle *h, const double *d_q, cudaStream_t s);
void launch_spread(npme_handle *h, cudaStream_t s);
void launch_multiply(npme_handle *h, cudaStream_t s);
void launch_interp(npme_handle *h, double *d_V, cudaStream_t s);

// direct.cu
// One direct-sum launch: charges already in the direct-sum source order
// (fine-column order for FP32 bulk, cell order for FP64), the caller's
// charges and the self term f_LR(0) q to subtract from V (zero for the bare
// short-range sum), and the output.
struct DirectArgs {
  const void *q;          // charges gathered into the direct-sum source order
  const double *qcaller;  // caller-order charges (the self term)
  double fself_r, fself_i;
  double *V;
  // built-in pair-once walks: leave the source-side sums for the
  // interpolation instead of merging them (sets h->merge_pending)
  bool defer_merge = false;
};
// status `code` with `msg` recorded on the handle (or, for a null handle, as
// the library's last error), as every entry point reports failures
int record_error(npme_handle *h, int code, const std::string &msg);
// loads the static scratch of npme_gpu_direct_sum_device_noalloc onto the
// current device (noalloc.cu)
int noalloc_preload(std::string &err);
// true when the direct sum takes the pair-once form (FP32 real DM kernels
// with the half-shell lists built)
bool pairs_once(const npme_handle *h);
// V[caller(s)] += the source-side sums of the pair-once walk (times vs for
// the potential, gs for the gradient; FP32 real, FP32 complex or FP64 by the
// handle), and zeroes them for the next call
void launch_merge_source(npme_handle *h, double *V, cudaStream_t s, double vs, double gs);
// Both return NPME_OK, or the status a caller-defined kernel's launcher
// reported (its launch error is not left pending for cudaGetLastError).
int launch_direct(npme_handle *h, const double *d_q, double *d_V, cudaStream_t s);
int launch_direct_args(npme_handle *h, const DirectArgs &a, cudaStream_t s);
// caller-order charges (double) -> direct-sum order in the bulk precision
void launch_gather_direct(npme_handle *h, const double *d_q, void *d_qdst, cudaStream_t s);
// exact O(N^2) sum; with d_tidx, only for the nt targets listed (output row t
// = target d_tidx[t]); returns NPME_OK or a caller-defined kernel's status
int launch_exact(npme_handle *h, const double *d_q, double *d_V, cudaStream_t s,
                  const uint32_t *d_tidx = nullptr, long nt = 0);
void launch_count_pairs(npme_handle *h, unsigned long long *d_count, cudaStream_t s);
template <typename T>
PairCoef<T> make_pair_coef(const npme_handle *h);

// Device memory reservation for a server: the device's stream-ordered pool
// (which every handle allocates from) is grown to hold at least `bytes`, and
// the reservation counts as one live user of the pool, so the pool keeps the
// memory until pool_unreserve.  Growing the pool while kernels run stalls the
// driver for every host thread (tenths of a second at a time under a serving
// load), so a server grows it once, at creation.  Best effort: without the
// memory the pool grows on demand.
int pool_reserve(int device, size_t bytes);
void pool_unreserve(int device);

// Slow-step log of the serving queue and of set-up: with NPME_SERVER_TRACE
// set in the environment, a step that takes longer than 5 ms is reported on
// stderr with its name and how many requests or systems it served.  Off by
// default (one check of a cached flag per step).
bool step_trace_on();
struct StepTimer {
  const char *name;
  size_t count;
  std::chrono::steady_clock::time_point t0;
  bool on;
  StepTimer(const char *step, size_t n)
      : name(step), count(n), t0(std::chrono::steady_clock::now()), on(step_trace_on()) {}
  ~StepTimer();
};

}  // namespace npme
