// traj_mixed.cu -- the batched mixed-form kernel and the dispatch of the
// single-molecule kernels (compiled per force variant in traj_mixed_t<N>.cu).
#include "mixed_impl.cuh"

namespace cosims {
namespace mixed {

// ---- batched form: one persistent launch over many molecules ------------------
// CTAs take work items (a molecule and a range of its trajectories) from a
// device queue.  A CTA keeps one molecule staged in shared memory (molecules
// over the launch's shared-memory budget are read through L1/L2) and its
// groups draw trajectories from the current item; the group that finds the
// item used up fetches the next one.  While the next item is of the same
// molecule the groups go straight on; only an item of another molecule makes
// the CTA wait for its groups and restage.  Items of one molecule are adjacent
// in the queue (sorted by cost), so a CTA rarely restages.

// CTA-shared state of the current molecule.
struct BatchShared {
  unsigned long long state;   // (item << 32) | next trajectory of the item; kNoItem: none
  int fetch_lock;             // held by the group fetching the next item
  int pending;                // item of another molecule to stage next, -1: none
  int staged;                 // molecule in shared memory, -1: none
};
constexpr unsigned long long kNoItem = 0xffffffffull << 32;

struct BatchSource {
  const BatchArgs *a;
  BatchShared *sh;
  int mol;                    // the staged molecule
  long long base;             // its first slot in the batch arrays
};
// 640-thread CTAs at 96 registers: room for the packed far-field pass
template <> struct PackedFar<BatchSource> { static constexpr bool value = true; };
__device__ __forceinline__ cosims_traj_out *out_of(const BatchSource &s) { return s.a->out; }
__device__ __forceinline__ long long budget_of(const BatchSource &) { return 0; }
__device__ __forceinline__ bool park(const BatchSource &, NarrowLanes &, GroupState &) {
  return false;
}

// Next trajectory of the staged molecule for a group; false when the
// molecule has no more items (the CTA then restages or stops).
__device__ __forceinline__ bool acquire(const BatchSource &src, const DevParams &p,
                                        NarrowLanes &ln, GroupState &GS) {
  const BatchArgs &A = *src.a;
  BatchShared &sh = *src.sh;
  for (;;) {
    long long slot = -1;
    if (ln.lane == 0) {
      bool gave_up = true;
      for (uint32_t spin = 0; spin < kHandoffSpinLimit; ++spin) {
        const unsigned long long w = atomicAdd(&sh.state, 0ull);
        if (w == kNoItem) { gave_up = false; break; }
        const int item = (int)(w >> 32);
        const long long t = (long long)(uint32_t)w;
        const BatchItem it = A.items[item];
        if (t < it.t1 - it.t0) {
          if (atomicCAS(&sh.state, w, w + 1) == w) {
            slot = src.base + it.t0 + t;
            gave_up = false;
            break;
          }
          continue;
        }
        // the item is used up: one group fetches the next, the others retry
        if (atomicCAS(&sh.fetch_lock, 0, 1) == 0) {
          if (atomicAdd(&sh.state, 0ull) == w) {
            const unsigned long long nxt = atomicAdd(A.item_queue, 1ull);
            if (nxt < (unsigned long long)A.n_items && A.items[nxt].mol == src.mol) {
              atomicExch(&sh.state, nxt << 32);
            } else {
              if (nxt == (unsigned long long)A.n_items) mark_first(A.counters, C_T_DRAIN_INV);
              sh.pending = nxt < (unsigned long long)A.n_items ? (int)nxt : -1;
              __threadfence_block();
              atomicExch(&sh.state, kNoItem);
            }
          }
          atomicExch(&sh.fetch_lock, 0);
        }
      }
      if (gave_up) atomicOr(A.counters + C_ERROR, 2ull);
    }
    slot = __shfl_sync(ln.gmask, slot, 0, ln.G);
    if (slot < 0) return false;
    if (!A.hit[slot]) {                       // ellipsoid miss: chi = 0
      if (ln.lane == 0) {
        cosims_traj_out o = {0.0, 0.0, 0, 0u};
        A.out[slot] = o;
      }
      continue;
    }
    traj_begin(GS.s, slot, A.pos0 + 3 * slot, A.vel0 + 3 * slot, p.dt, false);
    return true;
  }
}

// The groups of a CTA on one staged molecule until its items run out.  Not
// inlined: each (variant, staging) pair gets its own register allocation
// instead of the union of all six.
template <int TYPE, bool SMEM, int GT>
__device__ __noinline__ void batch_session(const BatchMol &bm, unsigned char *smem,
                                           const BatchArgs &a, BatchShared *sh, int mol) {
  const unsigned char *base = SMEM ? smem : bm.img32.gbase;
  const View m = make_view(base, bm.img32);
  const View64 m64 = make_view64(bm.img64);
  const int G = GT > 0 ? GT : bm.group_lanes;
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
  const BatchSource src{&a, sh, mol, bm.base};
  Tally tl;
  group_loop<TYPE>(m, m64, bm.par, ln, modes, *S, src, tl);
  fold_tally<TYPE>(*S, tl);
  flush_nolj(tl, a.counters);
  __syncwarp();
  if (ln.lane == 0) flush_group<TYPE>(*S, m64.n, a.counters);
}

// lanes per trajectory fixed at compile time for 8, 16 and 32 (as the
// single-molecule kernels); other counts at run time
template <int TYPE, bool SMEM>
__device__ __forceinline__ void batch_session_g(const BatchMol &bm, unsigned char *smem,
                                                const BatchArgs &a, BatchShared *sh, int mol) {
  switch (bm.group_lanes) {
    case 8: batch_session<TYPE, SMEM, 8>(bm, smem, a, sh, mol); break;
    case 16: batch_session<TYPE, SMEM, 16>(bm, smem, a, sh, mol); break;
    case 32: batch_session<TYPE, SMEM, 32>(bm, smem, a, sh, mol); break;
    default: batch_session<TYPE, SMEM, 0>(bm, smem, a, sh, mol); break;
  }
}

template <int TYPE>
__device__ __forceinline__ void batch_session_s(const BatchMol &bm, unsigned char *smem,
                                                const BatchArgs &a, BatchShared *sh, int mol) {
  if (bm.use_smem) batch_session_g<TYPE, true>(bm, smem, a, sh, mol);
  else batch_session_g<TYPE, false>(bm, smem, a, sh, mol);
}

__global__ void __launch_bounds__(kBatchMaxBlock, 1) batch_mixed_kernel(const BatchArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ uint64_t bar;
  __shared__ BatchMol cur;
  __shared__ BatchShared sh;
  if (threadIdx.x == 0) {
    mark_first(a.counters, C_T_START_INV);
    const unsigned long long first = atomicAdd(a.item_queue, 1ull);
    if (first == (unsigned long long)a.n_items) mark_first(a.counters, C_T_DRAIN_INV);
    sh.pending = first < (unsigned long long)a.n_items ? (int)first : -1;
    sh.staged = -1;
  }
  uint32_t stagings = 0;
  for (;;) {
    __syncthreads();
    const int item = sh.pending;
    if (item < 0) break;
    const int mol = a.items[item].mol;
    if (mol != sh.staged) {
      __syncthreads();
      if (threadIdx.x == 0) {
        cur = a.mols[mol];
        sh.staged = mol;
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
    if (threadIdx.x == 0) {
      sh.state = (unsigned long long)item << 32;
      sh.fetch_lock = 0;
      sh.pending = -1;
    }
    __syncthreads();
    switch (cur.type) {
      case 1: batch_session_s<1>(cur, smem, a, &sh, mol); break;
      case 2: batch_session_s<2>(cur, smem, a, &sh, mol); break;
      case 3: batch_session_s<3>(cur, smem, a, &sh, mol); break;
      case 4: batch_session_s<4>(cur, smem, a, &sh, mol); break;
      case 5: batch_session_s<5>(cur, smem, a, &sh, mol); break;
      default: batch_session_s<6>(cur, smem, a, &sh, mol); break;
    }
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
