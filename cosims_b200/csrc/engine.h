// engine.h -- definitions shared by the host side of the C ABI and the kernels.
//
// Device image of one molecule.  The image is one contiguous blob in global
// memory whose sections start on 16-byte boundaries; a CTA copies the whole
// blob into shared memory with bulk copies (cp.async.bulk) and then reads it
// through the same byte offsets.  Records are array-of-structs, so a kernel
// keeps one base address per section and reaches each field by an immediate
// offset.  Two layouts exist:
//
//   F64 image (plain form, and the FP64 energy check of the mixed form):
//     AtomF64 records in "force order" -- cluster by cluster in the
//     reference's member order for the cluster force variants (1, 2, 3, 5),
//     file order otherwise; perm[i] = force-order slot of file atom i
//     (getPotential walks atoms in file order); ClusterF64 records; the event
//     slots of the exact wide phase, int2 {atom (force order) or -1 for a
//     cluster's far-field event, cluster}: cluster by cluster, a far-field
//     slot before each cluster's atoms for variants 1 and 2.
//   F32 image (mixed form), variants 1, 2 and 5: in force order, two float4
//     arrays, (x, y, z, q)
//     and (sigma^6, 24 eps/mu, cluster id as integer bits, 1 for an atom and
//     0 for padding), so lanes reading consecutive atoms hit consecutive
//     banks; ClusterF32 records (FP64 centre and squared radii, so the
//     near/far tests stay FP64; FP32 multipole moments, the dipole 0 for a
//     replaced cluster), then one all-zero record centred 1e4 Angstrom away
//     on each axis (the null cluster, whose far-field terms are exactly 0:
//     the partner of an unpaired far cluster in the packed far-field pass).  The layout is
//     cluster-blocked: each cluster's atoms start a block of kClusterBlock
//     slots and fill whole blocks, so the listed-cluster loop reads a
//     cluster's blocks with no bounds test; the image ends with at least one
//     block of padding and is padded to n_slots, a multiple of kSlotQuantum.
//     Padding is inert atoms (far away, q = sigma^6 = eps = 0, cluster id
//     n_clusters, whose mode is always 0): every pair term of a pad atom is
//     exactly zero.
//     Variants 3, 4 and 6 (no far field, no cluster lists) hold the same
//     values pair-interleaved instead, slots 2j and 2j+1 side by side, as four
//     arrays over j: (x0, x1, y0, y1), (z0, z1, q0, q1), (sigma^6 0, sigma^6 1,
//     24 eps/mu 0, 24 eps/mu 1) and the two cluster ids.  A lane's float4 load
//     then yields the register pairs that Blackwell's packed FP32 instructions
//     (FFMA2 and kin) take, with no moves to assemble them.
//     Variants 1 and 2 also hold the far-field table (S_FAR): clusters 2j and
//     2j+1 side by side in six float4 arrays over j, for the packed far pass:
//     the negated centre as an FP32 hi/lo pair (-x_hi, -y_hi, -z_hi, then
//     -x_lo, -y_lo, -z_lo), the squared multipole and dispersion radii in FP32,
//     the charge and the dipole (0 for a replaced cluster).  Pairs past the
//     last cluster are null entries (zero moments, radii -1: far, never in the
//     dispersion radius); the table has a multiple of kMaxGroupLanes pairs.
#pragma once
#include <cstdint>
#include "cosims_cuda.h"

namespace cosims {

constexpr int kMaxAtoms = 16384;
constexpr int kMaxClusters = 65535;
constexpr int kMaxGroupLanes = 32;
constexpr int kSlotQuantum = 2 * kMaxGroupLanes;   // pair loop: two atoms per lane per pass
constexpr int kClusterBlock = 16;   // blocked F32 layout: a cluster's slots, in whole blocks
// variants whose F32 image is cluster-blocked: each cluster's atoms start a
// block of kClusterBlock slots and fill whole blocks (inert padding), and the
// image ends with at least one block of inert slots
__host__ __device__ constexpr bool blocked_layout(int force_type) {
  return force_type == 1 || force_type == 2 || force_type == 5;
}
constexpr float kPadCoord = 1.0e6f;                // pad atoms sit this far out (Angstrom)
constexpr int kMixedMaxBlock = 768;                // threads per CTA of the mixed kernels (80 registers)
constexpr int kMixedFarBlock = 640;                // variants 1, 2: 96 registers, 20 warps a CTA
constexpr int kBatchMaxBlock = 640;                // threads per CTA of the batched kernel (96 registers)
constexpr int kTrajStateBytes = 200;               // one trajectory's integrator state
constexpr int kGroupStateBytes = 240;              // TrajState + a group's counters (shared memory)
constexpr int kWideSlotFloats = 24;                // per-warp reduction slot of a wide group

enum ImageSection : int { S_ATOMS = 0, S_PERM, S_CLUSTERS, S_LJ, S_SLOTS, S_PAIRS, S_FAR, S_COUNT };
// far-field table of variants 1 and 2: pairs of clusters, six float4 per pair
__host__ __device__ constexpr int far_table_pairs(int n_clusters) {
  return ((n_clusters + 1) / 2 + kMaxGroupLanes - 1) / kMaxGroupLanes * kMaxGroupLanes;
}
constexpr int kFarTableArrays = 6;
// variants whose F32 image is pair-interleaved (S_PAIRS instead of S_ATOMS / S_LJ)
__host__ __device__ constexpr bool paired_layout(int force_type) {
  return force_type == 3 || force_type == 4 || force_type == 6;
}

struct AtomF64 {            // 56 bytes
  double x, y, z, q, sig6, eps24m, eps4;
};

struct ClusterF64 {         // 176 bytes
  double cx, cy, cz;
  double mpr2;              // (r_mp + R)^2    (forceAccel.cpp:253-254)
  double dr2;               // (r_disp + R)^2  (forceAccel.cpp:255-256)
  double q;
  double dip[3];
  double quad[9];           // quad[3*i+j] = quadPole[i][j]
  double qsig6, qeps;       // sigma^6, eps24/mu of atom index n (forceAccel.cpp:353-355)
  int32_t a0, a1;           // member range in force order
  int32_t replaced;
  int32_t pad;
};

// 120 bytes: an odd number of 8-byte words, so that lanes reading consecutive
// clusters' FP64 fields (the near/far pass, one cluster per lane) spread over
// all shared-memory banks (a 112-byte stride put four lanes on each bank).
struct ClusterF32 {
  double cx, cy, cz, mpr2, dr2;
  float q;
  float dip[3];
  float quad[9];
  float qsig6, qeps;
  int32_t replaced;
  int32_t a0, a1;           // slot range (blocked layout: padded to whole blocks)
  int32_t n_atoms;          // atoms of the cluster (a1 - a0 less the padding)
  int32_t pad;
};

static_assert(sizeof(AtomF64) == 56, "AtomF64 layout");
static_assert(sizeof(ClusterF64) == 176, "ClusterF64 layout");
static_assert(sizeof(ClusterF32) == 120, "ClusterF32 layout");

struct MolImage {
  const unsigned char *gbase;   // image in global memory
  uint32_t bytes;               // image size, multiple of 16
  int32_t n_atoms;
  int32_t n_clusters;
  int32_t uses_clusters;        // force variant walks clusters (1, 2, 3, 5)
  int32_t n_slots;              // F32 image: padded atom count (F64 image: n_atoms)
  uint32_t off[S_COUNT];        // byte offsets of the sections (0 = absent)
};

// Device copy of the path scalars (cosims_params plus derived values).
struct DevParams {
  int32_t force_type;
  int32_t multipole_order;
  int32_t projection;
  int32_t charged;
  double dt, mu, dipole_scalar, r_disp, r_mp;
  double ell_a, ell_b, ell_c, max_rad;
  double inv_ell_a, inv_ell_b, inv_ell_c;   // mixed form: 1 / axis (exit test by products)
  double b_max, start_dist, g_min, g_max, vdist_a, vdist_norm, vdist_max;
  double ccs_const;
  int64_t max_steps;
};

// Device-side counters of one run (all 64-bit, summed with atomics).
enum Counter : int {
  C_STEPS = 0,      // integration steps, all attempts
  C_FORCE_EVALS,    // acceleration evaluations
  C_POT_EVALS,      // potential evaluations
  C_PAIR_LJ,        // LJ-only pair terms
  C_PAIR_ES,        // electrostatic (+LJ) pair terms
  C_PAIR_POT,       // potential pair terms
  C_FAR,            // far-field cluster terms
  C_PAIR_ESNL,      // electrostatic pair terms outside the LJ cut-off (no LJ term)
  C_ERROR,          // error flags (bit 0: staging wait gave up; bit 1: hand-off wait gave up)
  C_T_START_INV,    // ~(earliest CTA start), globaltimer ns (max of complements)
  C_T_DRAIN_INV,    // ~(first time a group found the work queue empty)
  C_T_END,          // last group exit, globaltimer ns
  C_WIDE_STEPS,     // steps integrated by wide (hand-off) groups
  C_WIDE_NS,        // time wide groups spent integrating, summed over groups (ns)
  C_COUNT
};

// Integrator state of one mixed-form trajectory: in shared memory while a
// group works on it, in global memory while it waits for a wide group.
struct TrajState {
  double pos[3], vel[3], acc[3], p0[3], v0[3];
  double E0, dt, tries, max_tries, rdot;
  int64_t t, total;
  int32_t orbits, step, phase, etries, otries, may_handoff;
};
static_assert(sizeof(TrajState) == kTrajStateBytes, "TrajState layout");

// Hand-off of long trajectories (mixed form).  A narrow group (<= 32 lanes)
// that has integrated `budget` steps of a trajectory parks its state in
// `states` and takes new work; once a CTA's narrow groups have run out of
// work, the CTA splits into wide groups of `wide_lanes` threads that finish
// the parked trajectories.  Every choice is a function of the trajectory, so
// results do not depend on timing; they do depend on budget and wide_lanes
// (the order of the FP32 sums changes with the lane count).
struct Handoff {
  TrajState *states;               // cap records
  uint32_t *ready;                 // cap flags, 0 before the launch
  unsigned long long *reserve;     // records reserved, 0 before the launch
  unsigned long long *taken;       // records taken by wide groups, 0 before the launch
  int64_t cap;
  int64_t budget;                  // steps before a hand-off; 0 = never
  int32_t wide_lanes;              // threads of a wide group (multiple of 32)
  uint32_t spin_limit;             // polls of a wide group's wait for a record's flag
  uint32_t withhold_first;         // test of the error path: record 0 is never published
  uint32_t pad;
};
constexpr uint32_t kHandoffSpinLimit = 1u << 22;   // polls of a hand-off record's flag
constexpr uint32_t kStageSpinLimit = 1u << 22;     // polls of a shared-memory staging wait

// Shared-memory bytes of one wide group: cluster modes for two steps, then
// per-warp reduction slots for two steps (2 x warps x 24 floats, 2 x warps x
// 4 doubles) and a broadcast word.  The wide group's trajectory state lives in
// registers.
__host__ __device__ inline uint32_t wide_group_bytes(int wide_lanes, int mode_stride) {
  const uint32_t warps = (uint32_t)wide_lanes / 32u;
  uint32_t b = (2u * (uint32_t)mode_stride + 15u) & ~15u;
  b += 2u * warps * kWideSlotFloats * 4u;
  b += 2u * warps * 4u * 8u;
  b += 16u;
  return b;
}
constexpr int64_t kDefaultHandoffBudget = 2048;   // steps before a trajectory goes wide

// Plain form: a parked trajectory is finished by a whole CTA (kPlainBlock
// threads): warps 1..3 evaluate the terms of kExactChunk event slots at a time
// while warp 0 adds the previous chunk in the reference's order, one
// accumulator per lane.  Shared memory of that phase: cluster flags, two chunk
// buffers of [K][kExactRow] doubles (a row padded to an odd count of doubles so
// that the adding lanes read different banks), K accumulators and a broadcast
// word.
constexpr int kPlainBlock = 128;
constexpr int kExactProducers = kPlainBlock - 32;
#ifndef COSIMS_EXACT_PER_THREAD
#define COSIMS_EXACT_PER_THREAD 1
#endif
constexpr int kExactPerThread = COSIMS_EXACT_PER_THREAD;
constexpr int kExactChunk = kExactProducers * kExactPerThread;
constexpr int kExactRow = kExactChunk + 1;
// Plain form's default step budget: a CTA finishes a parked trajectory at
// about 28x one thread's speed but with 128 threads, so the budget trades the
// tail against wide-phase work.  Measured on B200 (single integrals and calls
// of three): 256 is best for the 128-atom molecule, 512 for the 512-atom ion
// and the 3000-atom protein.
constexpr int64_t kDefaultPlainHandoffBudget = 256;
inline int64_t default_plain_budget(int n_atoms) {
  return n_atoms > 256 ? 512 : kDefaultPlainHandoffBudget;
}
__host__ __device__ inline int exact_accumulators(int force_type) {
  return (force_type == 1 || force_type == 2) ? 15 : (force_type == 3 || force_type == 4) ? 12 : 4;
}
__host__ __device__ inline uint32_t exact_scratch_bytes(int force_type, int n_clusters) {
  const uint32_t K = (uint32_t)exact_accumulators(force_type);
  uint32_t b = ((uint32_t)n_clusters + 15u) & ~15u;                  // cluster flags
  b += 2u * K * (uint32_t)kExactRow * 8u;                            // chunk buffers
  b += 16u * 8u + 16u;                                               // accumulators, broadcast
  return b;
}
// 128 threads for every molecule: on the 3000-atom protein (400 000 trajectories,
// 32 lanes) 256-thread wide groups gave 436 k trajectories/s and 128-thread
// ones 466 k, the same as a budget of 8192 steps (469 k).
inline int default_wide_lanes(int n_atoms) { (void)n_atoms; return 128; }

struct TrajArgs {
  MolImage img;          // the image staged into shared memory
  MolImage img64;        // F64 image (global) used for the energy check
  DevParams par;
  int32_t group_lanes;   // lanes per trajectory (power of two, <= 32)
  int32_t use_smem;      // image staged in shared memory (else read from global)
  int32_t mode_stride;   // bytes of per-group cluster-mode scratch in shared memory
  uint32_t stage_limit;  // polls of the shared-memory staging wait
  const double *pos0;    // 3n start positions
  const double *vel0;    // 3n start velocities
  const int32_t *hit;    // n ellipsoid hits (NULL: every start state is a hit)
  const int32_t *order;  // work order: queue slot -> trajectory (NULL: identity)
  int64_t n;
  cosims_traj_out *out;  // n records
  unsigned long long *queue;     // work counter (reset to 0 before launch)
  unsigned long long *counters;  // C_COUNT counters
  Handoff ho;            // long-trajectory hand-off (budget 0: off)
  // plain form, per-step trace (cosims_trace_list): position and velocity
  // after every integration step of trajectory t go to
  // trace[(t * trace_cap + k) * 6 ..], k < trace_cap; trace_n[t] counts steps
  double *trace;
  int32_t *trace_n;
  int32_t trace_cap;
  int32_t pad1;
};

// ---- batched form ---------------------------------------------------------------
// One molecule of a batch (device-resident; copied to shared memory per item).
struct BatchMol {
  MolImage img32;        // F32 image in the batch arena
  MolImage img64;        // F64 image in the batch arena (energy check)
  DevParams par;
  int32_t type;          // force variant
  int32_t group_lanes;   // lanes per trajectory
  int32_t mode_stride;   // bytes of cluster-mode scratch per group
  int32_t use_smem;      // stage the F32 image in shared memory
  int64_t base;          // first slot of this molecule in the batch arrays
  int64_t n_traj;        // trajectories this run
  uint64_t seed;         // Philox key
  int64_t first_index;   // first trajectory index of the stream
};

// A work item: trajectories [t0, t1) of one molecule (molecule-local indices).
struct BatchItem {
  int32_t mol, pad;
  int64_t t0, t1;
};

struct BatchArgs {
  const BatchMol *mols;
  const BatchItem *items;
  int32_t n_items;
  int32_t n_mols;
  uint32_t smem_bytes;   // dynamic shared memory of the launch
  uint32_t pad;
  const double *pos0;    // batch-wide start states (3 per slot)
  const double *vel0;
  const int32_t *hit;
  cosims_traj_out *out;  // batch-wide records
  unsigned long long *item_queue;
  unsigned long long *counters;
};

int batch_launch(const BatchArgs &a, int block, int grid, size_t smem, void *stream);
int batch_occupancy(int block, size_t smem, int *per_sm);
int batch_sample_launch(const BatchMol *mols, int n_mols, int64_t total, double *pos0,
                        double *vel0, int32_t *hit, void *stream);
int batch_reduce_launch(const BatchMol *mols, int n_mols, const cosims_traj_out *recs,
                        int64_t update_every, cosims_ccs_sums *sums, void *stream);

// Host helpers implemented in the .cu files.
int plain_launch(const TrajArgs &a, int block, int grid, size_t smem, void *stream);
int mixed_launch(const TrajArgs &a, int block, int grid, size_t smem, void *stream);
int plain_max_smem_per_block();
int sample_launch(const DevParams &par, uint64_t seed, int64_t first, int64_t n,
                  cosims_traj_in *inputs, double *pos0, double *vel0, int32_t *hit,
                  void *stream);
// Longest-first work order: trajectories bucketed by start speed, slowest
// first, misses last.  scratch: order_scratch_len() int32.
constexpr int kOrderBuckets = 256;
inline int64_t order_scratch_len() { return 2 * (kOrderBuckets + 1) + 8; }
int order_launch(const DevParams &par, const double *vel0, const int32_t *hit, int64_t n,
                 int32_t *order, int32_t *scratch, void *stream);

// Reduction of per-trajectory records into a cosims_ccs_sums (device).
int reduce_launch(const cosims_traj_out *recs, int64_t n, double ccs_const,
                  int half_angle, int64_t update_every, const unsigned long long *counters,
                  cosims_ccs_sums *d_sums, double *scratch, int64_t scratch_len,
                  void *stream);
int64_t reduce_scratch_len(int64_t n);
// Adds a launch's work counters into d_work (zero_first: clear it first).
int add_work_launch(const unsigned long long *counters, cosims_ccs_sums *d_work, int zero_first,
                    void *stream);

}  // namespace cosims
