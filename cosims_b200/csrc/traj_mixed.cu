// traj_mixed.cu -- the batched mixed-form kernel and the dispatch of the
// single-molecule kernels (compiled per force variant in traj_mixed_t<N>.cu).
#include "mixed_impl.cuh"

namespace cosims {
namespace mixed {

// ---- batched form: one persistent launch over many molecules ------------------
// CTAs take work items (a molecule and a range of its trajectories) from a
// device queue.  When an item's molecule differs from the one staged, the CTA
// waits for its groups, then bulk-copies the new image into shared memory
// (molecules over the launch's shared-memory budget are read through L1/L2).
// Groups then take the item's trajectories from a shared-memory counter.
// One work item of the batched kernel.  Not inlined: each (variant, staging)
// pair gets its own register allocation instead of the union of all six.
template <int TYPE, bool SMEM>
__device__ __noinline__ void batch_item(const BatchMol &bm, unsigned char *smem,
                                        const BatchArgs &a, const BatchItem &it,
                                        unsigned long long *q) {
  const unsigned char *base = SMEM ? smem : bm.img32.gbase;
  const View m = make_view(base, bm.img32);
  const View64 m64 = make_view64(bm.img64);
  const int G = bm.group_lanes;
  GroupState *S;
  uint8_t *modes;
  narrow_scratch(smem, SMEM ? bm.img32.bytes : 0u, G, bm.mode_stride, S, modes);
  NarrowLanes ln;
  ln.G = G;
  ln.lane = threadIdx.x & (G - 1);
  ln.gmask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << ((threadIdx.x & 31) & ~(G - 1)));
  if (ln.lane == 0) {
    S->s.phase = P_ACQUIRE;
    group_counters_clear(*S);
    if (Traits<TYPE>::kClusters) modes[m.nc] = 0;
  }
  __syncwarp();
  const long long b = bm.base + it.t0;
  MainSource src;
  src.pos0 = a.pos0 + 3 * b; src.vel0 = a.vel0 + 3 * b; src.hit = a.hit + b;
  src.order = nullptr; src.n = it.t1 - it.t0;
  src.out = a.out + b; src.queue = q; src.counters = nullptr;
  src.ho = Handoff{};
  Tally tl;
  group_loop<TYPE>(m, m64, bm.par, ln, modes, *S, src, tl);
  fold_tally<TYPE>(*S, tl);
  __syncwarp();
  if (ln.lane == 0) flush_group<TYPE>(*S, m64.n, a.counters);
}

template <int TYPE>
__device__ __forceinline__ void batch_item_s(const BatchMol &bm, unsigned char *smem,
                                             const BatchArgs &a, const BatchItem &it,
                                             unsigned long long *q) {
  if (bm.use_smem) batch_item<TYPE, true>(bm, smem, a, it, q);
  else batch_item<TYPE, false>(bm, smem, a, it, q);
}

__global__ void __launch_bounds__(kBatchMaxBlock, 1) batch_mixed_kernel(const BatchArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ uint64_t bar;
  __shared__ BatchMol cur;
  __shared__ int s_item, s_mol;
  __shared__ unsigned long long s_queue;
  if (threadIdx.x == 0) {
    s_mol = -1;
    mark_first(a.counters, C_T_START_INV);
  }
  uint32_t stagings = 0;
  for (;;) {
    if (threadIdx.x == 0) s_item = (int)atomicAdd(a.item_queue, 1ull);
    __syncthreads();
    const int item = s_item;
    if (item >= a.n_items) {
      if (threadIdx.x == 0 && item == a.n_items) mark_first(a.counters, C_T_DRAIN_INV);
      break;
    }
    const BatchItem it = a.items[item];
    if (it.mol != s_mol) {
      __syncthreads();
      if (threadIdx.x == 0) {
        cur = a.mols[it.mol];
        s_mol = it.mol;
      }
      __syncthreads();
      if (cur.use_smem) {
        if (!stage_to_smem(smem, cur.img32.gbase, cur.img32.bytes, &bar, stagings & 1u,
                           stagings == 0)) {
          if (threadIdx.x == 0) atomicOr(a.counters + C_ERROR, 1ull);
          return;
        }
        stagings++;
      }
    }
    if (threadIdx.x == 0) s_queue = 0ull;
    __syncthreads();
    switch (cur.type) {
      case 1: batch_item_s<1>(cur, smem, a, it, &s_queue); break;
      case 2: batch_item_s<2>(cur, smem, a, it, &s_queue); break;
      case 3: batch_item_s<3>(cur, smem, a, it, &s_queue); break;
      case 4: batch_item_s<4>(cur, smem, a, it, &s_queue); break;
      case 5: batch_item_s<5>(cur, smem, a, it, &s_queue); break;
      default: batch_item_s<6>(cur, smem, a, it, &s_queue); break;
    }
    __syncthreads();   // every group is done with the item before a restage
  }
  if (threadIdx.x == 0) mark_last(a.counters, C_T_END);
}

}  // namespace mixed

int mixed_launch_t1(const TrajArgs &, int, int, size_t, void *);
int mixed_launch_t2(const TrajArgs &, int, int, size_t, void *);
int mixed_launch_t3(const TrajArgs &, int, int, size_t, void *);
int mixed_launch_t4(const TrajArgs &, int, int, size_t, void *);
int mixed_launch_t5(const TrajArgs &, int, int, size_t, void *);
int mixed_launch_t6(const TrajArgs &, int, int, size_t, void *);
int mixed_occupancy_t1(int, int, int, size_t, int *);
int mixed_occupancy_t2(int, int, int, size_t, int *);
int mixed_occupancy_t3(int, int, int, size_t, int *);
int mixed_occupancy_t4(int, int, int, size_t, int *);
int mixed_occupancy_t5(int, int, int, size_t, int *);
int mixed_occupancy_t6(int, int, int, size_t, int *);

int batch_launch(const BatchArgs &a, int block, int grid, size_t smem, void *stream) {
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(mixed::batch_mixed_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
  }
  mixed::batch_mixed_kernel<<<grid, block, smem, (cudaStream_t)stream>>>(a);
  return (int)cudaGetLastError();
}

int batch_occupancy(int block, size_t smem, int *per_sm) {
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(mixed::batch_mixed_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
  }
  return (int)cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, mixed::batch_mixed_kernel,
                                                            block, smem);
}

int mixed_launch(const TrajArgs &a, int block, int grid, size_t smem, void *stream) {
  switch (a.par.force_type) {
    case 1: return mixed_launch_t1(a, block, grid, smem, stream);
    case 2: return mixed_launch_t2(a, block, grid, smem, stream);
    case 3: return mixed_launch_t3(a, block, grid, smem, stream);
    case 4: return mixed_launch_t4(a, block, grid, smem, stream);
    case 5: return mixed_launch_t5(a, block, grid, smem, stream);
    default: return mixed_launch_t6(a, block, grid, smem, stream);
  }
}

int mixed_occupancy(int force_type, int use_smem, int group_lanes, int block, size_t smem,
                    int *per_sm) {
  switch (force_type) {
    case 1: return mixed_occupancy_t1(use_smem, group_lanes, block, smem, per_sm);
    case 2: return mixed_occupancy_t2(use_smem, group_lanes, block, smem, per_sm);
    case 3: return mixed_occupancy_t3(use_smem, group_lanes, block, smem, per_sm);
    case 4: return mixed_occupancy_t4(use_smem, group_lanes, block, smem, per_sm);
    case 5: return mixed_occupancy_t5(use_smem, group_lanes, block, smem, per_sm);
    default: return mixed_occupancy_t6(use_smem, group_lanes, block, smem, per_sm);
  }
}

}  // namespace cosims
