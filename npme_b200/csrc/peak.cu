// FP32 FMA-pipe throughput of this GPU, measured: the denominator of the
// direct sum's roofline fraction (the direct sum is bound by the FP32 pipe,
// and the device reports no measured FP32 peak of its own).  Built as its own
// small library (libnpme_peak.so), outside the solver's C ABI.
//
// Every thread runs kChains independent FMA chains (scalar fmaf, or the
// two-wide __ffma2_rn the direct sum uses) for `iters` steps; the grid fills
// every SM with 8 CTAs of 256 threads.  Flops = 2 per FMA lane-operation.
#include <cuda_runtime.h>

namespace {

constexpr int kChains = 8;

__global__ void __launch_bounds__(256) fma_scalar_kernel(float *out, int iters, float a, float b) {
  float x[kChains];
#pragma unroll
  for (int c = 0; c < kChains; c++) x[c] = threadIdx.x * 1e-6f + c;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int u = 0; u < 16; u++)
#pragma unroll
      for (int c = 0; c < kChains; c++) x[c] = fmaf(x[c], a, b);
  }
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < kChains; c++) s += x[c];
  if (s == 12345.f) out[threadIdx.x] = s;  // keeps the chains live
}

__global__ void __launch_bounds__(256) fma_packed_kernel(float *out, int iters, float a, float b) {
  float2 x[kChains];
#pragma unroll
  for (int c = 0; c < kChains; c++) x[c] = make_float2(threadIdx.x * 1e-6f + c, c + 0.5f);
  const float2 a2 = make_float2(a, a), b2 = make_float2(b, b);
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int u = 0; u < 16; u++)
#pragma unroll
      for (int c = 0; c < kChains; c++) x[c] = __ffma2_rn(x[c], a2, b2);
  }
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < kChains; c++) s += x[c].x + x[c].y;
  if (s == 12345.f) out[threadIdx.x] = s;
}

}  // namespace

// Best of `reps` timed launches of each form (after one warm-up launch);
// *tflops = the larger of the two, *ms = that launch's duration.  Returns 0,
// or the CUDA error code.
extern "C" int npme_peak_fp32(int device, int iters, int reps, double *tflops, double *ms) {
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return (int)e;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const int blocks = sms * 8, threads = 256;
  float *out = nullptr;
  if ((e = cudaMalloc(&out, sizeof(float) * threads)) != cudaSuccess) return (int)e;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  double best = 0.0, best_ms = 0.0;
  for (int form = 0; form < 2; form++) {
    // lane-operations per FMA instruction: 1 (scalar) or 2 (packed)
    const double lanes = form ? 2.0 : 1.0;
    const double flops = 2.0 * lanes * kChains * 16.0 * iters * (double)blocks * threads;
    for (int r = 0; r <= reps; r++) {
      cudaEventRecord(a);
      if (form) fma_packed_kernel<<<blocks, threads>>>(out, iters, 0.999999f, 1e-7f);
      else fma_scalar_kernel<<<blocks, threads>>>(out, iters, 0.999999f, 1e-7f);
      cudaEventRecord(b);
      if ((e = cudaEventSynchronize(b)) != cudaSuccess) break;
      float t = 0.f;
      cudaEventElapsedTime(&t, a, b);
      if (r > 0 && t > 0.f && flops / (t * 1e-3) / 1e12 > best) {
        best = flops / (t * 1e-3) / 1e12;
        best_ms = t;
      }
    }
    if (e != cudaSuccess) break;
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(out);
  *tflops = best;
  *ms = best_ms;
  return (int)e;
}
