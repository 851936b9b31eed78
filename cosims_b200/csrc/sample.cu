// sample.cu -- start states on their own: the Philox sampler and the
// ellipsoid projection of monteTraj::setUpTraj (monteTraj.cpp:174-278) for a
// range of trajectory indices.  The trajectory kernels call the same device
// functions inline; this entry point exists so that a caller (or a test) can
// inspect the sampled inputs and start states.
#include <cuda_runtime.h>
#include "device_util.cuh"

namespace cosims {

__global__ void sample_kernel(const DevParams p, uint64_t seed, int64_t first, int64_t n,
                              cosims_traj_in *inputs, double *pos0, double *vel0, int32_t *hit) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  cosims_traj_in in = sample_inputs(p, seed, (uint64_t)(first + i));
  double ps[3] = {0, 0, 0}, vs[3] = {0, 0, 0};
  const bool h = start_state(p, in, ps, vs);
  inputs[i] = in;
  for (int k = 0; k < 3; k++) { pos0[3 * i + k] = ps[k]; vel0[3 * i + k] = vs[k]; }
  hit[i] = h ? 1 : 0;
}

int sample_launch(const DevParams &par, uint64_t seed, int64_t first, int64_t n,
                  cosims_traj_in *inputs, double *pos0, double *vel0, int32_t *hit,
                  void *stream) {
  if (n <= 0) return 0;
  const int block = 256;
  const int64_t grid = (n + block - 1) / block;
  sample_kernel<<<(unsigned)grid, block, 0, (cudaStream_t)stream>>>(par, seed, first, n, inputs,
                                                                    pos0, vel0, hit);
  return (int)cudaGetLastError();
}

}  // namespace cosims

namespace cosims {

// ---- longest-first work order ---------------------------------------------------
// Integration steps grow roughly as 1/g (the He crosses the ellipsoid at its
// start speed), so handing out slow trajectories first keeps the last groups
// of a launch from idling behind a few long trajectories.  A counting sort on
// kOrderBuckets speed buckets, slowest first, misses last.  The order within
// a bucket is not fixed (atomics), which does not matter: each trajectory's
// result depends only on its own start state.

__device__ __forceinline__ int speed_bucket(const DevParams &p, const double *vel0,
                                            const int32_t *hit, int64_t i) {
  if (hit && !hit[i]) return kOrderBuckets;   // misses last
  const double vx = vel0[3 * i], vy = vel0[3 * i + 1], vz = vel0[3 * i + 2];
  const double g = sqrt(vx * vx + vy * vy + vz * vz);
  const double span = p.g_max - p.g_min;
  int b = span > 0 ? (int)((g - p.g_min) / span * kOrderBuckets) : 0;
  return b < 0 ? 0 : (b >= kOrderBuckets ? kOrderBuckets - 1 : b);
}

__global__ void order_hist(const DevParams p, const double *vel0, const int32_t *hit, int64_t n,
                           int32_t *hist) {
  __shared__ int32_t h[kOrderBuckets + 1];
  for (int i = threadIdx.x; i <= kOrderBuckets; i += blockDim.x) h[i] = 0;
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(&h[speed_bucket(p, vel0, hit, i)], 1);
  __syncthreads();
  for (int i = threadIdx.x; i <= kOrderBuckets; i += blockDim.x)
    if (h[i]) atomicAdd(&hist[i], h[i]);
}

__global__ void order_scan(const int32_t *hist, int32_t *offset) {
  if (threadIdx.x == 0) {
    int32_t run = 0;
    for (int i = 0; i <= kOrderBuckets; i++) {
      offset[i] = run;
      run += hist[i];
    }
  }
}

__global__ void order_scatter(const DevParams p, const double *vel0, const int32_t *hit,
                              int64_t n, int32_t *offset, int32_t *order) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int b = speed_bucket(p, vel0, hit, i);
    const int32_t slot = atomicAdd(&offset[b], 1);
    order[slot] = (int32_t)i;
  }
}

int order_launch(const DevParams &par, const double *vel0, const int32_t *hit, int64_t n,
                 int32_t *order, int32_t *scratch, void *stream) {
  if (n <= 0) return 0;
  cudaStream_t s = (cudaStream_t)stream;
  int32_t *hist = scratch, *offset = scratch + (kOrderBuckets + 1);
  cudaError_t e = cudaMemsetAsync(hist, 0, sizeof(int32_t) * (kOrderBuckets + 1), s);
  if (e != cudaSuccess) return (int)e;
  const int block = 256;
  int64_t grid = (n + block - 1) / block;
  if (grid > 1184) grid = 1184;
  order_hist<<<(unsigned)grid, block, 0, s>>>(par, vel0, hit, n, hist);
  order_scan<<<1, 32, 0, s>>>(hist, offset);
  order_scatter<<<(unsigned)grid, block, 0, s>>>(par, vel0, hit, n, offset, order);
  return (int)cudaGetLastError();
}

}  // namespace cosims

namespace cosims {

// ---- batched sampling ---------------------------------------------------------------
// Slot i of the batch belongs to the molecule whose [base, base + n_traj)
// holds it (molecules sorted by base); its start values are those of
// trajectory first_index + (i - base) of that molecule's stream, exactly as
// the single-molecule sampler draws them.
__global__ void batch_sample_kernel(const BatchMol *mols, int n_mols, int64_t total, double *pos0,
                                    double *vel0, int32_t *hit) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    int lo = 0, hi = n_mols - 1;
    while (lo < hi) {                       // last molecule with base <= i
      const int mid = (lo + hi + 1) >> 1;
      if (mols[mid].base <= i) lo = mid; else hi = mid - 1;
    }
    const BatchMol &bm = mols[lo];
    const int64_t t = i - bm.base;
    double ps[3] = {0, 0, 0}, vs[3] = {0, 0, 0};
    bool h = false;
    if (t < bm.n_traj) {
      cosims_traj_in in = sample_inputs(bm.par, bm.seed, (uint64_t)(bm.first_index + t));
      h = start_state(bm.par, in, ps, vs);
    }
    for (int k = 0; k < 3; k++) { pos0[3 * i + k] = ps[k]; vel0[3 * i + k] = vs[k]; }
    hit[i] = h ? 1 : 0;
  }
}

int batch_sample_launch(const BatchMol *mols, int n_mols, int64_t total, double *pos0,
                        double *vel0, int32_t *hit, void *stream) {
  if (total <= 0 || n_mols <= 0) return 0;
  batch_sample_kernel<<<1184, 256, 0, (cudaStream_t)stream>>>(mols, n_mols, total, pos0, vel0,
                                                              hit);
  return (int)cudaGetLastError();
}

}  // namespace cosims
