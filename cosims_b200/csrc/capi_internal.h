// capi_internal.h -- host-side state behind the C ABI handles.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>
#include "engine.h"

namespace cosims {

struct HostImage {
  MolImage img;
  std::vector<unsigned char> bytes;
};

struct LaunchShape {
  int block = 0, grid = 0, use_smem = 0, mode_stride = 0;
  int wide_lanes = 0;   // mixed form: threads of a hand-off wide group (0: no wide phase)
  size_t smem = 0;
};

cosims_status fail(cosims_status s, const char *fmt, ...);
cosims_status cuda_fail(cudaError_t e, const char *what);
cosims_status validate(const cosims_molecule *mol, const cosims_params *par);
DevParams make_dev_params(const cosims_params *p);
void build_images(const cosims_molecule *m, const cosims_params *p, HostImage &h64,
                  HostImage &h32);
int mode_stride_for(const MolImage &img, int force_type);
size_t batch_mol_smem(BatchMol &bm, int block, int budget, uint32_t img_cap);
void balanced_items(const std::vector<int64_t> &n_traj, const std::vector<int> &n_atoms,
                    const std::vector<int> &group_lanes, int block, int grid,
                    std::vector<BatchItem> &items);
cosims_status shape_for(bool plain, const MolImage &img, int G, int block_threads,
                        int wide_lanes, int force_type, int sm_count, int max_smem, int64_t n,
                        LaunchShape &ls);
cosims_status check_device(int device, int *sm_count, int *max_smem);

struct DeviceGuard {
  int prev = 0;
  explicit DeviceGuard(int dev);
  ~DeviceGuard();
};

int plain_occupancy(int force_type, int block, size_t smem, int *per_sm);
int mixed_occupancy(int force_type, int use_smem, int group_lanes, int block, size_t smem,
                    int *per_sm);

// Lanes per trajectory before any tuning: enough lanes that a 32-lane warp
// still holds several trajectories for small molecules, a full warp for large.
inline int default_group_lanes(int n_atoms) {
  if (n_atoms <= 160) return 4;
  if (n_atoms <= 700) return 8;
  if (n_atoms <= 2000) return 16;
  return 32;
}

}  // namespace cosims

struct cosims_ctx {
  int device = 0;
  int precision = 0;
  int sm_count = 0;
  int max_smem = 0;
  int n_atoms = 0;
  int group_lanes = 1;
  int block_threads = 256;
  cosims::DevParams par{};
  cosims::HostImage h64, h32;
  cosims::MolImage img64{}, img32{};
  unsigned char *d_img64 = nullptr, *d_img32 = nullptr;
  unsigned long long *d_queue = nullptr, *d_counters = nullptr;
  cosims_ccs_sums *d_sums = nullptr;
  cosims_ccs_sums *d_sums_many = nullptr;              // cosims_run_integrals: records + work
  int64_t sums_cap = 0;
  cosims_traj_out *d_out = nullptr;
  int64_t out_cap = 0;
  cosims_traj_in *d_in = nullptr;
  int64_t in_cap = 0;
  double *d_pos0 = nullptr, *d_vel0 = nullptr;
  int64_t list_cap = 0, vel_cap = 0;
  int32_t *d_hit = nullptr;
  int64_t hit_cap = 0;
  double *d_red = nullptr;
  int64_t red_cap = 0;
  int32_t *d_order = nullptr;
  int64_t order_cap = 0;
  int32_t *d_order_scratch = nullptr;
  int64_t order_scratch_cap = 0;
  // long-trajectory hand-off (mixed form)
  int64_t ho_budget = cosims::kDefaultHandoffBudget;   // <= 0: off
  int ho_wide = 0;                                     // 0: default for the molecule
  cosims::TrajState *d_ho_states = nullptr;
  uint32_t *d_ho_ready = nullptr;
  int64_t ho_cap = 0;
  unsigned long long *d_ho_ctrl = nullptr;             // reserve, taken
  int64_t ho_last_parked = 0;
  // tests of the error path (cosims_ctx_set_wait_test)
  uint32_t test_flags = 0;
  uint32_t test_spin_limit = 0;
  cosims::LaunchShape last_shape{};
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;   // around the last trajectory kernel
  bool timed = false;
};
