// Measurement helpers exported next to the RHS entry points:
//
//  b200bssn_plan_profile  evaluates a plan once with CUDA events between its
//                         launches and reports the summed device time of the
//                         derivative and the algebra kernels (the bench's live
//                         per-kernel timing).
//  b200bssn_fma_peak      measures the FP64 or FP32 FMA throughput of the device
//                         with independent FMA chains (the roofline denominator
//                         for the algebra kernel, which is bound by the FP pipes).
#include <cuda_runtime.h>

#include <vector>

#include "b200bssn.h"

namespace {

template <typename T, int CHAINS>
__global__ void __launch_bounds__(256) fma_chains(T* out, int iters, T a, T b) {
  T acc[CHAINS];
#pragma unroll
  for (int c = 0; c < CHAINS; ++c) acc[c] = (T)(threadIdx.x + c);
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int r = 0; r < 16; ++r) {
#pragma unroll
      for (int c = 0; c < CHAINS; ++c) acc[c] = fma(acc[c], a, b);
    }
  }
  T s = 0;
#pragma unroll
  for (int c = 0; c < CHAINS; ++c) s += acc[c];
  if (s == (T)-12345.678) out[blockIdx.x] = s;  // keeps the chains alive
}

}  // namespace

extern "C" int b200bssn_fma_peak(int device, uint32_t precision, double* tflops) {
  if (!tflops || (precision != B200BSSN_FP64 && precision != B200BSSN_MIXED))
    return B200BSSN_ERR_INVALID_ARGUMENT;
  if (cudaSetDevice(device) != cudaSuccess) return B200BSSN_ERR_NO_DEVICE;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const int blocks = sms * 8, threads = 256, iters = 2048;
  constexpr int kChains = 8;
  void* out = nullptr;
  if (cudaMalloc(&out, blocks * sizeof(double)) != cudaSuccess) return B200BSSN_ERR_OUT_OF_MEMORY;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best_ms = 1e30f;
  for (int rep = 0; rep < 4; ++rep) {
    cudaEventRecord(e0);
    if (precision == B200BSSN_FP64)
      fma_chains<double, kChains><<<blocks, threads>>>((double*)out, iters, 0.999999, 1e-7);
    else
      fma_chains<float, kChains><<<blocks, threads>>>((float*)out, iters, 0.9999f, 1e-4f);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && ms < best_ms) best_ms = ms;
  }
  cudaError_t err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (err != cudaSuccess) return B200BSSN_ERR_CUDA;
  const double flops = 2.0 * kChains * 16.0 * iters * (double)blocks * threads;
  *tflops = flops / (best_ms * 1e-3) / 1e12;
  return B200BSSN_OK;
}
