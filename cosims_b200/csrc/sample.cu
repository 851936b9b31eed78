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
