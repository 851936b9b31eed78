// traj_mixed_t3.cu -- mixed-form kernels of force variant 3 (one unit per
// variant, so the instantiations compile in parallel).
#include "mixed_impl.cuh"

namespace cosims {
int mixed_launch_t3(const TrajArgs &a, int block, int grid, size_t smem, void *stream) {
  return mixed::launch_type<3>(a, block, grid, smem, stream);
}
int mixed_occupancy_t3(int use_smem, int group_lanes, int block, size_t smem, int *per_sm) {
  return mixed::occupancy_type<3>(use_smem, group_lanes, block, smem, per_sm);
}
}  // namespace cosims
