// cuFFT plans shared by all handles of a process.
//
// A plan depends only on (device, transform type, N1, N2, N3); creating one
// costs milliseconds, so handles that see the same FFT box share it.  Plans
// are made without a work area of their own (cufftSetAutoAllocation(0));
// every handle owns a work buffer and each execution binds the plan to the
// caller's stream and work buffer under the plan's mutex.  cuFFT reads both
// when it enqueues the transform, so executions of one plan by different
// handles on different streams never share scratch memory.
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
std::map<std::tuple<int, int, long, long, long>, std::unique_ptr<FFTPlan>> g_plans;
}  // namespace

FFTPlan *plan_get(int device, int type, long N1, long N2, long N3, std::string &err) {
  std::lock_guard<std::mutex> lk(g_plans_mu);
  auto key = std::make_tuple(device, type, N1, N2, N3);
  auto it = g_plans.find(key);
  if (it != g_plans.end()) return it->second.get();
  std::unique_ptr<FFTPlan> p(new FFTPlan);
  cufftResult r = cufftCreate(&p->plan);
  if (r == CUFFT_SUCCESS) r = cufftSetAutoAllocation(p->plan, 0);
  if (r == CUFFT_SUCCESS)
    r = cufftMakePlan3d(p->plan, (int)N1, (int)N2, (int)N3, (cufftType)type, &p->work);
  if (r != CUFFT_SUCCESS) {
    err = "cuFFT plan " + std::to_string(N1) + "x" + std::to_string(N2) + "x" +
          std::to_string(N3) + " failed: " + std::to_string((int)r);
    cufftDestroy(p->plan);
    return nullptr;
  }
  p->type = type;
  FFTPlan *raw = p.get();
  g_plans[key] = std::move(p);
  return raw;
}

// Forward transform of the handle's spread grid: R2C into the spectrum
// buffer (real kernels) or C2C in place (complex kernels).
int fft_forward(npme_handle *h, cudaStream_t s) {
  FFTPlan *p = h->pf;
  std::lock_guard<std::mutex> lk(p->mu);
  cufftResult r = cufftSetStream(p->plan, s);
  if (r == CUFFT_SUCCESS) r = cufftSetWorkArea(p->plan, h->d_work);
  if (r == CUFFT_SUCCESS) {
    switch (p->type) {
      case CUFFT_R2C:
        r = cufftExecR2C(p->plan, (cufftReal *)h->d_grid, (cufftComplex *)h->d_kgrid);
        break;
      case CUFFT_D2Z:
        r = cufftExecD2Z(p->plan, (cufftDoubleReal *)h->d_grid, (cufftDoubleComplex *)h->d_kgrid);
        break;
      case CUFFT_C2C:
        r = cufftExecC2C(p->plan, (cufftComplex *)h->d_grid, (cufftComplex *)h->d_grid,
                         CUFFT_FORWARD);
        break;
      case CUFFT_Z2Z:
        r = cufftExecZ2Z(p->plan, (cufftDoubleComplex *)h->d_grid,
                         (cufftDoubleComplex *)h->d_grid, CUFFT_FORWARD);
        break;
      default: r = CUFFT_INVALID_TYPE;
    }
  }
  if (r != CUFFT_SUCCESS) {
    h->err = "cuFFT forward transform failed: " + std::to_string((int)r);
    return NPME_ECUDA;
  }
  return NPME_OK;
}

// Inverse transform back onto the grid (theta): C2R / Z2D or C2C in place.
int fft_inverse(npme_handle *h, cudaStream_t s) {
  FFTPlan *p = h->pi;
  std::lock_guard<std::mutex> lk(p->mu);
  cufftResult r = cufftSetStream(p->plan, s);
  if (r == CUFFT_SUCCESS) r = cufftSetWorkArea(p->plan, h->d_work);
  if (r == CUFFT_SUCCESS) {
    switch (p->type) {
      case CUFFT_C2R:
        r = cufftExecC2R(p->plan, (cufftComplex *)h->d_kgrid, (cufftReal *)h->d_grid);
        break;
      case CUFFT_Z2D:
        r = cufftExecZ2D(p->plan, (cufftDoubleComplex *)h->d_kgrid, (cufftDoubleReal *)h->d_grid);
        break;
      case CUFFT_C2C:
        r = cufftExecC2C(p->plan, (cufftComplex *)h->d_grid, (cufftComplex *)h->d_grid,
                         CUFFT_INVERSE);
        break;
      case CUFFT_Z2Z:
        r = cufftExecZ2Z(p->plan, (cufftDoubleComplex *)h->d_grid,
                         (cufftDoubleComplex *)h->d_grid, CUFFT_INVERSE);
        break;
      default: r = CUFFT_INVALID_TYPE;
    }
  }
  if (r != CUFFT_SUCCESS) {
    h->err = "cuFFT inverse transform failed: " + std::to_string((int)r);
    return NPME_ECUDA;
  }
  return NPME_OK;
}

// Looks up the handle's two plans and sizes its work buffer.
int prepare_plans(npme_handle *h) {
  const long *N = h->grid.N;
  int tf, ti;
  if (h->complex_kernel) tf = ti = h->fp32 ? CUFFT_C2C : CUFFT_Z2Z;
  else tf = h->fp32 ? CUFFT_R2C : CUFFT_D2Z, ti = h->fp32 ? CUFFT_C2R : CUFFT_Z2D;
  h->pf = plan_get(h->device, tf, N[0], N[1], N[2], h->err);
  h->pi = h->pf ? plan_get(h->device, ti, N[0], N[1], N[2], h->err) : nullptr;
  if (!h->pf || !h->pi) return NPME_ECUDA;
  const size_t work = std::max(h->pf->work, h->pi->work);
  return handle_buffer(h, &h->d_work, work);
}

}  // namespace npme
