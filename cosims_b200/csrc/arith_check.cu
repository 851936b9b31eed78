// arith_check.cu -- self-check of the branch-free division and square root
// (exact_arith.cuh) against CUDA's IEEE operators, bit for bit.
//
// The plain form relies on div_rn_pos and sqrt_rn reproducing IEEE round to
// nearest exactly inside their valid range.  cosims_check_exact_arith draws n
// operand pairs per class from a counter-based hash: operands spread over the
// whole valid exponent range, operands of the force loops' physical ranges
// (squared distances of 0.5 to 1e5 A^2 and their powers, LJ and charge
// numerators of either sign), and mantissa edge cases (powers of two,
// all-ones mantissas, zero dividends).  It counts the results that differ
// from `a / b` and `sqrt(x)` in any bit.
#include <cuda_runtime.h>
#include "capi_internal.h"
#include "exact_arith.cuh"

namespace cosims {
namespace {

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;                 // splitmix64 (Steele, Lea, Flood, 2014)
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// A double with a random 52-bit mantissa and exponent e (unbiased).
__device__ __forceinline__ double with_exp(unsigned long long bits, int e) {
  const unsigned long long m = bits & 0x000FFFFFFFFFFFFFull;
  return __longlong_as_double((long long)(((unsigned long long)(e + 1023) << 52) | m));
}

__device__ __forceinline__ double uniform01(unsigned long long bits) {
  return (double)(bits >> 11) * 0x1p-53;
}

__global__ void arith_check_kernel(unsigned long long seed, long long n,
                                   unsigned long long *bad) {
  unsigned long long nd = 0, ns = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const unsigned long long h0 = mix64(seed ^ (unsigned long long)i);
    const unsigned long long h1 = mix64(h0), h2 = mix64(h1), h3 = mix64(h2);
    const int cls = (int)(h3 & 7u);
    double a, b, x;
    if (cls < 3) {                             // the whole valid range
      b = with_exp(h1, (int)(h2 % 601) - 300);
      a = with_exp(h0, (int)((h2 >> 16) % 1201) - 600);
      x = with_exp(h3 >> 3, (int)((h2 >> 32) % 601) - 300);
    } else if (cls < 6) {                      // the force loops' ranges
      const double r2 = 0.5 + uniform01(h1) * (cls == 3 ? 20.0 : 1.0e5);
      const double p = cls == 4 ? r2 * r2 * r2 : (cls == 5 ? r2 * r2 * sqrt(r2) : r2);
      b = p;
      a = (uniform01(h0) - 0.5) * (cls == 5 ? 2.0 : 3.0e3);
      x = r2;
    } else {                                   // mantissa edge cases
      const int e = (int)(h2 % 201) - 100;
      const unsigned sel = (unsigned)(h3 >> 3) & 3u;
      b = sel == 0 ? with_exp(0, e) : (sel == 1 ? with_exp(~0ull, e) : with_exp(h1, e));
      a = sel == 2 ? 0.0 : ((h0 & 1) ? -1.0 : 1.0) * with_exp(sel == 3 ? ~0ull : h0, -e / 2);
      x = sel == 0 ? with_exp(0, e) : with_exp(sel == 1 ? ~0ull : h3, e);
    }
    if (__double_as_longlong(div_rn_pos(a, b)) != __double_as_longlong(a / b)) nd++;
    if (__double_as_longlong(sqrt_rn(x)) != __double_as_longlong(sqrt(x))) ns++;
  }
  if (nd) atomicAdd(bad, nd);
  if (ns) atomicAdd(bad + 1, ns);
}

}  // namespace
}  // namespace cosims

using namespace cosims;

extern "C" cosims_status cosims_check_exact_arith(int32_t device, uint64_t seed, int64_t n,
                                                  int64_t *div_mismatches,
                                                  int64_t *sqrt_mismatches) {
  if (n < 0 || !div_mismatches || !sqrt_mismatches)
    return fail(COSIMS_ERR_INVALID, "n >= 0 and both outputs are required");
  int sm = 0, smem = 0;
  cosims_status st = check_device(device, &sm, &smem);
  if (st != COSIMS_OK) return st;
  DeviceGuard g(device);
  unsigned long long *d = nullptr;
  cudaError_t e = cudaMalloc((void **)&d, 2 * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemset(d, 0, 2 * sizeof(unsigned long long));
  if (e == cudaSuccess) {
    arith_check_kernel<<<sm * 8, 256>>>(seed, n, d);
    e = cudaGetLastError();
  }
  unsigned long long h[2] = {0, 0};
  if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof h, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return cuda_fail(e, "arithmetic self-check");
  *div_mismatches = (int64_t)h[0];
  *sqrt_mismatches = (int64_t)h[1];
  return COSIMS_OK;
}
