// The reciprocal sum's transforms with cuFFT, pruned to the charge octant,
// and the plans they share across handles.
//
// The spread grid is the zero-padded box N1 x N2 x N3 whose charges all lie
// in the octant [0, N1/2) x [0, N2/2) x [0, N3/2), and the interpolation
// reads theta only on that octant.  So the forward transform is a batched 2D
// transform over (y, z) of the N1/2 slabs x < N1/2 only (the other slabs are
// zero), followed by 1D transforms along x over the whole spectrum; the
// inverse is the 1D transforms along x, then the 2D transforms of the slabs
// x < N1/2 only.  Against a full 3D transform this skips half of the (y, z)
// work in each direction.  Real kernels: 2D R2C / C2R over (y, z) (spectrum
// N1 x N2 x (N3/2+1)), 1D C2C along x; complex kernels: 2D and 1D C2C in
// place.  The slabs the 2D pass does not write must be zero before the x
// pass: the spectrum's upper slabs (real kernels, cleared here) or the grid's
// (complex kernels, cleared with the grid before the spread).
//
// A plan depends only on (device, kind, transform type, N1, N2, N3, points
// per slab); creating one costs milliseconds, so handles that see the same
// FFT box share it.  Plans are made without a work area of their own
// (cufftSetAutoAllocation(0)); every handle owns a work buffer and each
// execution binds the plan to the caller's stream and work buffer under the
// plan's mutex.  cuFFT reads both when it enqueues the transform, so
// executions of one plan by different handles on different streams never
// share scratch memory.
#include <cufft.h>

#include <algorithm>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>

#include "internal.h"

namespace npme {

namespace {
std::mutex g_plans_mu;
std::map<std::tuple<int, int, int, long, long, long, long>, std::unique_ptr<FFTPlan>> g_plans;

enum PlanKind { kSlabs2D = 1, kAlongX = 2 };

bool is_real_to_complex(int type) { return type == CUFFT_R2C || type == CUFFT_D2Z; }
bool is_complex_to_real(int type) { return type == CUFFT_C2R || type == CUFFT_Z2D; }

// kSlabs2D: 2D transforms over (y, z) of the N1/2 slabs x < N1/2.
// kAlongX: 1D transforms of length N1 along x, one per (y, z) point of the
// spectrum (stride = points per slab, consecutive batches adjacent).
cufftResult make_plan(FFTPlan *p, int kind, int type, long N1, long N2, long N3,
                      long slab_points) {
  if (kind == kSlabs2D) {
    int n[2] = {(int)N2, (int)N3};
    const long real_slab = N2 * N3, cplx_slab = N2 * (N3 / 2 + 1);
    int rembed[2] = {(int)N2, (int)N3}, cembed[2] = {(int)N2, (int)(N3 / 2 + 1)};
    if (is_real_to_complex(type))
      return cufftMakePlanMany(p->plan, 2, n, rembed, 1, (int)real_slab, cembed, 1, (int)cplx_slab,
                               (cufftType)type, (int)(N1 / 2), &p->work);
    if (is_complex_to_real(type))
      return cufftMakePlanMany(p->plan, 2, n, cembed, 1, (int)cplx_slab, rembed, 1, (int)real_slab,
                               (cufftType)type, (int)(N1 / 2), &p->work);
    return cufftMakePlanMany(p->plan, 2, n, rembed, 1, (int)real_slab, rembed, 1, (int)real_slab,
                             (cufftType)type, (int)(N1 / 2), &p->work);
  }
  int n[1] = {(int)N1}, embed[1] = {(int)N1};
  return cufftMakePlanMany(p->plan, 1, n, embed, (int)slab_points, 1, embed, (int)slab_points, 1,
                           (cufftType)type, (int)slab_points, &p->work);
}

FFTPlan *plan_get(int device, int kind, int type, long N1, long N2, long N3, long slab_points,
                  std::string &err) {
  std::lock_guard<std::mutex> lk(g_plans_mu);
  // the points per slab tell a real kernel's spectrum from a complex grid of
  // the same box (both transform along x with C2C)
  auto key = std::make_tuple(device, kind, type, N1, N2, N3, slab_points);
  auto it = g_plans.find(key);
  if (it != g_plans.end()) return it->second.get();
  std::unique_ptr<FFTPlan> p(new FFTPlan);
  cufftResult r = cufftCreate(&p->plan);
  if (r == CUFFT_SUCCESS) r = cufftSetAutoAllocation(p->plan, 0);
  if (r == CUFFT_SUCCESS) r = make_plan(p.get(), kind, type, N1, N2, N3, slab_points);
  if (r != CUFFT_SUCCESS) {
    err = "cuFFT plan " + std::to_string(N1) + "x" + std::to_string(N2) + "x" +
          std::to_string(N3) + " (kind " + std::to_string(kind) + ") failed: " +
          std::to_string((int)r);
    cufftDestroy(p->plan);
    return nullptr;
  }
  p->type = type;
  FFTPlan *raw = p.get();
  g_plans[key] = std::move(p);
  return raw;
}

// Enqueues plan p on stream s with the handle's work area; dir is used by
// the complex-to-complex types.
cufftResult exec(FFTPlan *p, npme_handle *h, cudaStream_t s, void *in, void *out, int dir) {
  std::lock_guard<std::mutex> lk(p->mu);
  cufftResult r = cufftSetStream(p->plan, s);
  if (r == CUFFT_SUCCESS) r = cufftSetWorkArea(p->plan, h->d_work);
  if (r != CUFFT_SUCCESS) return r;
  switch (p->type) {
    case CUFFT_R2C: return cufftExecR2C(p->plan, (cufftReal *)in, (cufftComplex *)out);
    case CUFFT_D2Z: return cufftExecD2Z(p->plan, (cufftDoubleReal *)in, (cufftDoubleComplex *)out);
    case CUFFT_C2R: return cufftExecC2R(p->plan, (cufftComplex *)in, (cufftReal *)out);
    case CUFFT_Z2D: return cufftExecZ2D(p->plan, (cufftDoubleComplex *)in, (cufftDoubleReal *)out);
    case CUFFT_C2C: return cufftExecC2C(p->plan, (cufftComplex *)in, (cufftComplex *)out, dir);
    case CUFFT_Z2Z:
      return cufftExecZ2Z(p->plan, (cufftDoubleComplex *)in, (cufftDoubleComplex *)out, dir);
    default: return CUFFT_INVALID_TYPE;
  }
}

int fft_fail(npme_handle *h, const char *what, cufftResult r) {
  h->err = std::string("cuFFT ") + what + " failed: " + std::to_string((int)r);
  return NPME_ECUDA;
}

}  // namespace

// Bytes of one complex element of the handle's spectrum (real kernels) or
// grid (complex kernels).
static size_t cplx_bytes(const npme_handle *h) { return h->fp32 ? 8 : 16; }

int grid_clear(npme_handle *h, cudaStream_t s) {
  const long *N = h->grid.N;
  // real kernels: only the slabs x < N1/2 feed the transform; complex
  // kernels: the whole grid (the upper slabs hold the last inverse pass)
  const size_t bytes = h->complex_kernel ? cplx_bytes(h) * (size_t)N[0] * N[1] * N[2]
                                         : (h->fp32 ? 4 : 8) * (size_t)(N[0] / 2) * N[1] * N[2];
  return cudaMemsetAsync(h->d_grid, 0, bytes, s) == cudaSuccess ? NPME_OK : NPME_ECUDA;
}

// Forward transform of the handle's spread grid: into the spectrum buffer
// (real kernels) or in place (complex kernels).
int fft_forward(npme_handle *h, cudaStream_t s) {
  cufftResult r;
  const long *N = h->grid.N;
  if (h->complex_kernel) {
    if ((r = exec(h->pf, h, s, h->d_grid, h->d_grid, CUFFT_FORWARD)) != CUFFT_SUCCESS)
      return fft_fail(h, "forward (y, z) slabs", r);
    if ((r = exec(h->px, h, s, h->d_grid, h->d_grid, CUFFT_FORWARD)) != CUFFT_SUCCESS)
      return fft_fail(h, "forward along x", r);
    return NPME_OK;
  }
  if ((r = exec(h->pf, h, s, h->d_grid, h->d_kgrid, CUFFT_FORWARD)) != CUFFT_SUCCESS)
    return fft_fail(h, "forward (y, z) slabs", r);
  // the spectrum's slabs x >= N1/2 start the x pass at zero
  const size_t slab = cplx_bytes(h) * (size_t)N[1] * (N[2] / 2 + 1);
  if (cudaMemsetAsync((char *)h->d_kgrid + slab * (N[0] / 2), 0, slab * (N[0] - N[0] / 2), s) !=
      cudaSuccess) {
    h->err = "clearing the upper spectrum slabs failed";
    return NPME_ECUDA;
  }
  if ((r = exec(h->px, h, s, h->d_kgrid, h->d_kgrid, CUFFT_FORWARD)) != CUFFT_SUCCESS)
    return fft_fail(h, "forward along x", r);
  return NPME_OK;
}

// Inverse transform back onto the grid (theta on the slabs x < N1/2).
int fft_inverse(npme_handle *h, cudaStream_t s) {
  cufftResult r;
  if (h->complex_kernel) {
    if ((r = exec(h->px, h, s, h->d_grid, h->d_grid, CUFFT_INVERSE)) != CUFFT_SUCCESS)
      return fft_fail(h, "inverse along x", r);
    if ((r = exec(h->pi, h, s, h->d_grid, h->d_grid, CUFFT_INVERSE)) != CUFFT_SUCCESS)
      return fft_fail(h, "inverse (y, z) slabs", r);
    return NPME_OK;
  }
  if ((r = exec(h->px, h, s, h->d_kgrid, h->d_kgrid, CUFFT_INVERSE)) != CUFFT_SUCCESS)
    return fft_fail(h, "inverse along x", r);
  if ((r = exec(h->pi, h, s, h->d_kgrid, h->d_grid, CUFFT_INVERSE)) != CUFFT_SUCCESS)
    return fft_fail(h, "inverse (y, z) slabs", r);
  return NPME_OK;
}

// Looks up the handle's plans and sizes its work buffer.
int prepare_plans(npme_handle *h) {
  const long *N = h->grid.N;
  int tf, ti, tx;
  long slab_points;
  if (h->complex_kernel) {
    tf = ti = tx = h->fp32 ? CUFFT_C2C : CUFFT_Z2Z;
    slab_points = N[1] * N[2];
  } else {
    tf = h->fp32 ? CUFFT_R2C : CUFFT_D2Z;
    ti = h->fp32 ? CUFFT_C2R : CUFFT_Z2D;
    tx = h->fp32 ? CUFFT_C2C : CUFFT_Z2Z;
    slab_points = N[1] * (N[2] / 2 + 1);
  }
  h->pf = plan_get(h->device, kSlabs2D, tf, N[0], N[1], N[2], slab_points, h->err);
  h->pi = h->pf ? plan_get(h->device, kSlabs2D, ti, N[0], N[1], N[2], slab_points, h->err)
                : nullptr;
  h->px = h->pi ? plan_get(h->device, kAlongX, tx, N[0], N[1], N[2], slab_points, h->err)
                : nullptr;
  if (!h->pf || !h->pi || !h->px) return NPME_ECUDA;
  const size_t work = std::max(h->pf->work, std::max(h->pi->work, h->px->work));
  return handle_buffer(h, &h->d_work, work);
}

}  // namespace npme
