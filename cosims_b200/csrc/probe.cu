// probe.cu -- measured vector-pipe peaks of the device, for roofline reports.
//
// The trajectory kernels are bound by the FP32 (mixed form) or FP64 (plain
// form) pipes, not by HBM or the tensor cores; this measures each pipe's FMA
// throughput on the device in use (independent FMA chains, every SM full).
#include <cuda_runtime.h>
#include "capi_internal.h"

namespace cosims {

template <typename T>
__global__ void __launch_bounds__(256) fma_chains(T *out, int iters, T b, T c) {
  T a0 = (T)(threadIdx.x * 1e-3), a1 = a0 + (T)1, a2 = a0 + (T)2, a3 = a0 + (T)3;
  T a4 = a0 + (T)4, a5 = a0 + (T)5, a6 = a0 + (T)6, a7 = a0 + (T)7;
#pragma unroll 4
  for (int i = 0; i < iters; i++) {
    a0 = fma(a0, b, c); a1 = fma(a1, b, c); a2 = fma(a2, b, c); a3 = fma(a3, b, c);
    a4 = fma(a4, b, c); a5 = fma(a5, b, c); a6 = fma(a6, b, c); a7 = fma(a7, b, c);
  }
  T s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
  if (s == (T)-1) out[blockIdx.x] = s;   // never true; keeps the chains live
}

template <typename T>
static cosims_status measure(int sm, T b, T c, double *tflops) {
  T *out = nullptr;
  cudaError_t e = cudaMalloc((void **)&out, sizeof(T) * sm * 8);
  if (e != cudaSuccess) return cuda_fail(e, "probe allocation");
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  const int grid = sm * 8, block = 256, iters = sizeof(T) == 4 ? 1 << 16 : 1 << 14;
  fma_chains<T><<<grid, block>>>(out, 256, b, c);   // warm-up
  float best = 1e30f;
  for (int r = 0; r < 3; r++) {
    cudaEventRecord(t0);
    fma_chains<T><<<grid, block>>>(out, iters, b, c);
    cudaEventRecord(t1);
    cudaEventSynchronize(t1);
    float ms = 0;
    cudaEventElapsedTime(&ms, t0, t1);
    best = ms < best ? ms : best;
  }
  e = cudaGetLastError();
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  cudaFree(out);
  if (e != cudaSuccess) return cuda_fail(e, "probe kernel");
  const double flops = 2.0 * 8.0 * (double)iters * (double)grid * block;
  *tflops = flops / (best * 1e-3) / 1e12;
  return COSIMS_OK;
}

}  // namespace cosims

extern "C" cosims_status cosims_probe_peaks(int32_t device, double *fp32_tflops,
                                            double *fp64_tflops) {
  using namespace cosims;
  int sm = 0, smem = 0;
  cosims_status st = check_device(device, &sm, &smem);
  if (st != COSIMS_OK) return st;
  DeviceGuard g(device);
  if (fp32_tflops) {
    st = measure<float>(sm, 0.999999f, 1e-7f, fp32_tflops);
    if (st != COSIMS_OK) return st;
  }
  if (fp64_tflops) st = measure<double>(sm, 0.999999, 1e-7, fp64_tflops);
  return st;
}
