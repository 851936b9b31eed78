// device_util.cuh -- device helpers shared by the trajectory kernels:
// shared-memory staging with bulk copies, the Philox4x32-10 generator, the
// start-state sampler and warp/group utilities.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "engine.h"

namespace cosims {

#ifndef COSIMS_PI
#define COSIMS_PI 3.14159265358979323846    // vector3D.h:24
#define COSIMS_PI_2 1.57079632679489661923  // vector3D.h:25
#endif

// ---- shared-memory staging ------------------------------------------------
// One thread arms an mbarrier with the byte count and issues non-multicast
// global->shared bulk copies (cp.async.bulk ... mbarrier::complete_tx); every
// thread then waits on the barrier's phase 0.  Waits are bounded: after
// kStageSpinLimit polls the thread records an error and continues, so a copy
// that never lands cannot hang the GPU.

constexpr uint32_t kBulkChunk = 32768;        // bytes per bulk copy
constexpr long long kDefaultMaxSteps = 1ll << 18;   // far above any physical trajectory

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, uint32_t bytes,
                                              uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Stage `bytes` (multiple of 16, both addresses 16-byte aligned, at most
// 2^20 - 1 bytes: the mbarrier transaction-count range) from global to shared
// memory.  Call from all threads of the CTA.  Returns false, in every thread,
// when the wait gave up after `limit` polls (the caller flags an error and
// returns); before it returns, every thread waits again, at most
// kStageSpinLimit polls, for the copies still in flight into this CTA's shared
// memory, so the CTA does not leave while they land.
// `init`: the first staging through this barrier (initialises it); later
// stagings pass init = false and the parity of their phase (0, 1, 0, ...).
__device__ __forceinline__ bool stage_to_smem(void *dst, const void *src, uint32_t bytes,
                                              uint64_t *bar, uint32_t parity, bool init,
                                              uint32_t limit = kStageSpinLimit) {
  if (threadIdx.x == 0 && init) {
    mbar_init(bar, 1);
    fence_barrier_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    // order earlier generic-proxy reads/writes of this shared memory before
    // the async-proxy writes of the bulk copies
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_arrive_expect_tx(bar, bytes);
    for (uint32_t o = 0; o < bytes; o += kBulkChunk) {
      uint32_t n = bytes - o < kBulkChunk ? bytes - o : kBulkChunk;
      bulk_copy_g2s(static_cast<unsigned char *>(dst) + o,
                    static_cast<const unsigned char *>(src) + o, n, bar);
    }
  }
  bool done = false;
  for (uint32_t spin = 0; spin < limit; ++spin) {
    if (mbar_try_wait(bar, parity)) { done = true; break; }
  }
  // one decision for the whole CTA, so no thread leaves while others go on
  const bool ok = __syncthreads_and(done ? 1 : 0) != 0;
  if (!ok) {
    for (uint32_t spin = 0; !done && spin < kStageSpinLimit; ++spin) done = mbar_try_wait(bar, parity);
    __syncthreads();
  }
  return ok;
}

// ---- Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) ----------------------
struct U4 { uint32_t x, y, z, w; };

__device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
    uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
    U4 n;
    n.x = hi1 ^ c.y ^ k0;
    n.y = lo1;
    n.z = hi0 ^ c.w ^ k1;
    n.w = lo0;
    c = n;
    k0 += W0;
    k1 += W1;
  }
  return c;
}

// 53-bit uniform in [0, 1) from two 32-bit words.
__device__ __forceinline__ double u01(uint32_t hi, uint32_t lo) {
  return ((double)(hi >> 5) * 67108864.0 + (double)(lo >> 6)) * (1.0 / 9007199254740992.0);
}

// Start values of trajectory `t` of the stream keyed by `seed`.  The counter
// block (t_lo, t_hi, draw, 0x43435331) makes every value a pure function of
// (seed, t): results do not depend on batching, launch shape or order.
// Distributions follow monteTraj::setUpTraj (monteTraj.cpp:203-231):
//   phi, gamma ~ U(0, 2 pi); theta ~ sin(theta) on [0, pi] (inverse CDF);
//   b ~ b on [0, b_max] (inverse CDF); g ~ g^5 exp(-a g^2) on [g_min, g_max]
//   by accept/reject against the density at the mode (as the reference).
__device__ __forceinline__ cosims_traj_in sample_inputs(const DevParams &p, uint64_t seed,
                                                        uint64_t t) {
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  U4 c = {(uint32_t)t, (uint32_t)(t >> 32), 0u, 0x43435331u};
  U4 r0 = philox4x32_10(c, k0, k1);
  c.z = 1u;
  U4 r1 = philox4x32_10(c, k0, k1);
  cosims_traj_in in;
  in.phi = u01(r0.x, r0.y) * 2.0 * COSIMS_PI;
  in.gamma = u01(r0.z, r0.w) * 2.0 * COSIMS_PI;
  in.theta = acos(1.0 - 2.0 * u01(r1.x, r1.y));
  in.b = p.b_max * sqrt(u01(r1.z, r1.w));
  double g = p.g_min;
  for (uint32_t draw = 2; draw < 2 + 4096; ++draw) {   // acceptance ~0.4: never reached
    c.z = draw;
    U4 r = philox4x32_10(c, k0, k1);
    g = u01(r.x, r.y) * (p.g_max - p.g_min) + p.g_min;
    double check = u01(r.z, r.w) * p.vdist_max;
    double g2 = g * g;
    double dens = g2 * g2 * g * exp(-p.vdist_a * g2) * p.vdist_norm;
    if (check <= dens) break;
  }
  in.g = g;
  return in;
}

// Start state and ellipsoid projection (monteTraj.cpp:235-269).  Returns
// false on a miss.
__device__ __forceinline__ bool start_state(const DevParams &p, const cosims_traj_in &in,
                                            double pos[3], double vel[3]) {
  double sg, cg, sp, cp, st, ct;
  sincos(in.gamma, &sg, &cg);
  sincos(in.phi, &sp, &cp);
  sincos(in.theta, &st, &ct);
  const double b = in.b, g = in.g, md = p.start_dist;
  pos[0] = b * cg * cp * ct - b * sg * sp + md * cp * st;
  pos[1] = b * cg * sp * ct + b * sg * cp + md * sp * st;
  pos[2] = md * ct - b * cg * st;
  vel[0] = -g * cp * st;
  vel[1] = -g * sp * st;
  vel[2] = -g * ct;
  if (p.projection) {
    double v0 = vel[0] / p.ell_a, v1 = vel[1] / p.ell_b, v2 = vel[2] / p.ell_c;
    double p0 = pos[0] / p.ell_a, p1 = pos[1] / p.ell_b, p2 = pos[2] / p.ell_c;
    double c0 = p1 * v2 - p2 * v1, c1 = p2 * v0 - p0 * v2, c2 = p0 * v1 - p1 * v0;
    double vv = v0 * v0 + v1 * v1 + v2 * v2;
    double discrim = -(c0 * c0 + c1 * c1 + c2 * c2) + vv;
    if (discrim < 0) return false;
    double t = -((p0 * v0 + p1 * v1 + p2 * v2) / vv) - sqrt(discrim) / vv;
    pos[0] += vel[0] * t;
    pos[1] += vel[1] * t;
    pos[2] += vel[2] * t;
  }
  return true;
}

// ---- group helpers ------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T group_sum(T v, int G) {
  for (int o = G >> 1; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ void count_add(unsigned long long *c, int k, long long v) {
  if (v) atomicAdd(c + k, (unsigned long long)v);
}

// ---- kernel timeline (globaltimer, ns) -----------------------------------------
// Counters start at 0, so the earliest-time marks keep the complement under
// atomicMax.
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mark_first(unsigned long long *c, int k) {
  atomicMax(c + k, ~global_ns());
}
__device__ __forceinline__ void mark_last(unsigned long long *c, int k) {
  atomicMax(c + k, global_ns());
}

}  // namespace cosims
