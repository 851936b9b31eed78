// traj_mixed_t1.cu -- mixed-form kernels of force variant 1 (one unit per
// variant, so the instantiations compile in parallel).
#include "mixed_impl.cuh"

namespace cosims {
int mixed_launch_t1(const TrajArgs &a, int block, int grid, size_t smem, void *stream) {
  return mixed::launch_type<1>(a, block, grid, smem, stream);
}
int mixed_occupancy_t1(int use_smem, int group_lanes, int block, size_t smem, int *per_sm) {
  return mixed::occupancy_type<1>(use_smem, group_lanes, block, smem, per_sm);
}
}  // namespace cosims
