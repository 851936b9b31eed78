/*
 * cosims_cuda.h -- C ABI of the B200 trajectory-method CCS engine.
 *
 * The reference (CoSIMS) has no plugin or operator API: its seam is the
 * in-process loop body of monteTraj::runTraj, which samples a start state
 * (monteTraj::setUpTraj, monteTraj.cpp:174-278), integrates it
 * (diffEqSolver::verletVel, diffEqSolver.cpp:81-211, forces from
 * forceAccel::getReducedVec / getPotential, forceAccel.cpp:887-982) and
 * accumulates pi*b_max^2*P*(1-cos chi) (monteTraj::runThreads,
 * monteTraj.cpp:456-502).  One call of this ABI replaces that whole OpenMP
 * loop (monteTraj.cpp:352-369) for a batch of trajectories.
 *
 * Conventions
 *   - Plain C types only; no C++ or CUDA types cross the boundary.  Streams are
 *     passed as `void*` (a cudaStream_t, NULL = the legacy default stream).
 *   - Every entry point returns a cosims_status; cosims_last_error() returns a
 *     thread-local message for the last failure on the calling thread.
 *   - The caller owns every host array.  A context copies the molecule to the
 *     device at creation and owns that copy, its scratch buffers and graphs.
 *   - A context is re-entrant per stream: calls on one context must be
 *     serialised by the caller (one host thread per context, or a lock).
 *   - Units are the reference's: Angstrom, picosecond, unified atomic mass
 *     unit, Kelvin, elementary charge (molecule2.h:69-72, maxBoltz.h:29).
 */
#ifndef COSIMS_CUDA_H
#define COSIMS_CUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define COSIMS_ABI_VERSION 2

typedef enum cosims_status {
    COSIMS_OK = 0,
    COSIMS_ERR_INVALID = 1,     /* bad argument or inconsistent molecule/params */
    COSIMS_ERR_CUDA = 2,        /* a CUDA runtime call failed */
    COSIMS_ERR_NOMEM = 3,       /* device or host allocation failed */
    COSIMS_ERR_IO = 4,          /* file could not be read or parsed */
    COSIMS_ERR_TIMEOUT = 5,     /* a bounded device wait gave up */
    COSIMS_ERR_UNSUPPORTED = 6, /* no sm_100 device, or a size beyond a limit */
    COSIMS_ERR_BUSY = 7         /* serving queue full */
} cosims_status;

/* Force variants, numbered as forceAccel::setClusters selects them
 * (forceAccel.cpp:125-140). */
typedef enum cosims_force_type {
    COSIMS_FORCE_MULTIPOLE_CUTOFF = 1,   /* multipoleCutoff   forceAccel.cpp:221-445 */
    COSIMS_FORCE_MULTIPOLE_ONLY = 2,     /* multipoleOnly     forceAccel.cpp:447-633 */
    COSIMS_FORCE_DISPERSION_ONLY = 3,    /* dispersionOnly    forceAccel.cpp:635-749 */
    COSIMS_FORCE_CHARGE_DIPOLE_LJ = 4,   /* chargeDipoleLJ    forceAccel.cpp:751-805 */
    COSIMS_FORCE_DISPERSION_NOCHARGE = 5,/* dispersionNoCharge forceAccel.cpp:807-854 */
    COSIMS_FORCE_DISPERSION_FULL = 6     /* dispersionFull    forceAccel.cpp:856-884 */
} cosims_force_type;

typedef enum cosims_precision {
    /* The reference method in FP64, one thread per trajectory, the
     * reference's operation order (bit-for-bit the same force sums). */
    COSIMS_PRECISION_PLAIN_F64 = 0,
    /* Pair forces in FP32 on molecule-centred coordinates; positions,
     * velocities, the energy check, 1-cos(chi) and the CCS sums in FP64. */
    COSIMS_PRECISION_MIXED = 1
} cosims_precision;

/* One molecule after the reference's setup: COM-centred and rotated into its
 * inertia frame (molecule2::setInertia, molecule2.cpp:1131-1308), with the
 * force-field terms of molecule2::setMolProperties (molecule2.cpp:770-903)
 * and the PCM clusters of forceAccel::setClusters (forceAccel.cpp:53-141).
 * All arrays are host memory, file order unless stated. */
typedef struct cosims_molecule {
    int32_t n_atoms;
    const double *x, *y, *z;      /* coordinates, Angstrom                     */
    const double *charge;         /* partial charges, e                         */
    const double *sig6;           /* sigma^6 (dataList::sigAvg6)                */
    const double *eps24m;         /* 24 eps'/mu (dataList::eps24_mass; atom 0 is
                                     not divided by mu, molecule2.cpp:862-863)  */
    const double *eps4;           /* 4 eps' (dataList::eps4)                    */
    /* PCM clusters; n_clusters = 0 when neither cut-off scheme is on. */
    int32_t n_clusters;
    const int32_t *cluster_offset;   /* n_clusters + 1 prefix offsets           */
    const int32_t *cluster_atoms;    /* member atom indices, reference order    */
    const double *cluster_pos;       /* 3 * n_clusters: centre used by forces   */
    const double *cluster_radius;    /* max member distance from the centre     */
    const double *cluster_charge;    /* total charge                            */
    const double *cluster_dipole;    /* 3 * n_clusters                          */
    const double *cluster_quad;      /* 9 * n_clusters, row-major               */
    const int32_t *cluster_replaced; /* centre replaced by centre of charge     */
} cosims_molecule;

/* Scalars of the trajectory path, as the reference computes them in
 * monteTraj::monteTraj (monteTraj.cpp:26-142) and fileParams defaults. */
typedef struct cosims_params {
    int32_t force_type;       /* cosims_force_type                              */
    int32_t multipole_order;  /* multipole_order_ext (0, 1 or 2)                */
    int32_t projection;       /* projection_ext: ellipsoid start/stop surface   */
    int32_t charged;          /* charge_ext: induced-dipole energy term on      */
    double dt;                /* dt_ext, ps                                      */
    double mu;                /* mass_ext: He-molecule reduced mass, u          */
    double dipole_scalar;     /* 28276.01363 / mu (forceAccel.cpp:35)           */
    double r_disp;            /* dispersion_radius_ext                          */
    double r_mp;              /* multipole_radius_ext                           */
    double ell_a, ell_b, ell_c; /* enlarged ellipsoid axes (impactParam a,b,c)  */
    double b_max;             /* impactParam::getMax()                          */
    double start_dist;        /* float(b_max): monteTraj::maxDist is a float    */
    double g_min, g_max;      /* velocity window (monteTraj.cpp:54-55)          */
    double vdist_a;           /* beta / 2 = mu / (2 k T)                        */
    double vdist_norm;        /* renormalised g^5 exp(-a g^2) normalisation     */
    double vdist_max;         /* density at the mode (maxVelDistr)              */
    double ccs_const;         /* const1 * const2 (monteTraj.cpp:91-94, :472)    */
    int64_t max_steps;        /* hard cap on integration steps per trajectory
                                 (0 = default 2^18); the reference has none.  A
                                 capped or non-finite trajectory is a failure
                                 with COSIMS_TRAJ_STEPCAP set                   */
} cosims_params;

/* Per-trajectory status bits. */
#define COSIMS_TRAJ_HIT       0x1u  /* start state reached the ellipsoid        */
#define COSIMS_TRAJ_SUCCESS   0x2u  /* verletVel returned true                  */
#define COSIMS_TRAJ_STEPCAP   0x4u  /* stopped by max_steps or a non-finite state */
#define COSIMS_TRAJ_ETRIES_SHIFT 8  /* bits 8..15: energy-check retries         */
#define COSIMS_TRAJ_OTRIES_SHIFT 16 /* bits 16..23: orbit-detector dt shrinks   */

/* One trajectory's result.  chi follows the reference's conventions: the
 * scattering angle on success, pi/2 on failure (diffEqSolver.cpp:208), 0 on
 * an ellipsoid miss (monteTraj.cpp:366-367). */
typedef struct cosims_traj_out {
    double chi;
    double de_pct;   /* energy deviation in % at the accepted exit, else 0      */
    int32_t steps;   /* localThreadParams::stepCount as the reference sets it   */
    uint32_t status; /* COSIMS_TRAJ_* bits                                      */
} cosims_traj_out;

/* Sampled start values of one trajectory (monteTraj.cpp:203-253). */
typedef struct cosims_traj_in {
    double b, phi, theta, gamma, g;
} cosims_traj_in;

/* Sums of one CCS integral, reduced in a fixed order (deterministic). */
typedef struct cosims_ccs_sums {
    double sum;           /* sum of ccs_const * (1 - cos|chi|)                   */
    double sum2;          /* sum of squares                                      */
    double max_de_pct;    /* max energy deviation over successes                 */
    int64_t n;            /* trajectories processed (misses included)            */
    int64_t n_hit;        /* start states that reached the ellipsoid             */
    int64_t n_success;    /* verletVel successes                                 */
    int64_t n_eff;        /* the reference's success count for Omega = sum/n_eff:
                             n minus the failures its one-thread bookkeeping
                             still holds at the end (monteTraj.cpp:380-381,
                             504-521); see cosims_run_sampled                   */
    int64_t steps;        /* integration steps, all attempts                     */
    /* Work done, for the roofline: acceleration and potential evaluations and
     * the pair terms they summed, by kind. */
    int64_t force_evals;
    int64_t pot_evals;
    int64_t pair_lj;      /* Lennard-Jones-only pair terms                       */
    int64_t pair_es;      /* pair terms with the charge field (+ LJ if in range) */
    int64_t pair_pot;     /* potential pair terms (energy check)                 */
    int64_t far_terms;    /* cluster multipole far-field terms                   */
    int64_t pair_es_nolj; /* of pair_es, those outside the LJ cut-off: the charge
                             field and its gradient only (force variants 1-3)   */
} cosims_ccs_sums;

typedef struct cosims_ctx cosims_ctx;

/* ---- library ------------------------------------------------------------ */
int32_t cosims_abi_version(void);
const char *cosims_last_error(void);
/* Number of usable CUDA devices (0 when none).  Never initialises a context. */
int32_t cosims_device_count(void);

/* ---- one molecule on the device ---------------------------------------- */
/* Copies mol and par to `device` and prepares the shared-memory image.
 * precision: cosims_precision.  Replaces monteTraj's per-molecule state
 * (gasAtom.setMol -> forceAccel::setMol/setClusters, monteTraj.cpp:88). */
cosims_status cosims_ctx_create(const cosims_molecule *mol, const cosims_params *par,
                                int32_t precision, int32_t device, cosims_ctx **out);
void cosims_ctx_destroy(cosims_ctx *ctx);

/* Launch shape: lanes per trajectory (1,2,4,...,32; the plain form accepts 1
 * only) and threads per CTA (plain: up to 128; mixed: up to 768, or 640 for
 * force variants 1 and 2; by default chosen per run for the most resident
 * threads).  0 keeps the current choice.
 * get_launch reports the CTA size of the last run when it was chosen. */
cosims_status cosims_ctx_set_launch(cosims_ctx *ctx, int32_t group_lanes,
                                    int32_t block_threads);
cosims_status cosims_ctx_get_launch(const cosims_ctx *ctx, int32_t *group_lanes,
                                    int32_t *block_threads);

/* Long-trajectory hand-off.  A trajectory still running after step_budget
 * integration steps (all attempts) is parked and finished by a wide group
 * once its CTA runs out of other work, so the few very long trajectories no
 * longer set the run time.
 * Mixed form: the wide group is wide_lanes threads (0 = default: 128; else a
 * multiple of 32 up to 512); results depend only
 * on the trajectory, group_lanes, step_budget and wide_lanes, not on timing.
 * Default step_budget 2048.
 * Plain form: the wide group is the whole 128-thread CTA (wide_lanes 0 or
 * 128), which evaluates a step's terms in parallel and adds them in the
 * reference's order: results are bitwise those without hand-off, whatever
 * the budget.  Default step_budget 256 up to 256 atoms, 512 above.
 * step_budget: 0 = default, < 0 = off.  The context keeps a 200-byte record
 * per trajectory of a call for this; calls of more than 2^22 trajectories run
 * without hand-off. */
cosims_status cosims_ctx_set_handoff(cosims_ctx *ctx, int64_t step_budget, int32_t wide_lanes);
/* Current settings and, for the last run: trajectories parked, steps the
 * wide groups integrated, and the time they spent on it summed over wide
 * groups (ms); wide_ms / wide_steps is the wide groups' time per step. */
cosims_status cosims_ctx_get_handoff(cosims_ctx *ctx, int64_t *step_budget, int32_t *wide_lanes,
                                     int64_t *parked, int64_t *wide_steps, double *wide_ms);

/* Tests of the error path.  Every device wait of the trajectory kernels is
 * bounded: a wait that gives up sets an error flag, the kernel returns, and
 * the call returns COSIMS_ERR_TIMEOUT with the context still usable.  This
 * makes the waits give up on purpose, without any fault: with
 * COSIMS_WAIT_TEST_STAGING every CTA's wait for its shared-memory copy of the
 * molecule gives up at once (each CTA then waits for its copies in flight to
 * land and leaves); with COSIMS_WAIT_TEST_HANDOFF the first trajectory parked
 * for the long-trajectory hand-off is never published, so the wide group that
 * takes it waits on a flag that nothing sets and gives up after spin_limit
 * polls (0: the default, 2^22), and that trajectory's record is not written.
 * flags 0 restores normal runs.  No counterpart in the reference. */
#define COSIMS_WAIT_TEST_STAGING 0x1u
#define COSIMS_WAIT_TEST_HANDOFF 0x2u
cosims_status cosims_ctx_set_wait_test(cosims_ctx *ctx, uint32_t flags, uint32_t spin_limit);

/* Fixed-list form: integrate n given start states (pos0, vel0: 3n doubles each,
 * host memory) and write n results to out (host).  Replaces, per trajectory,
 * diffEqSolver::verletVel (diffEqSolver.cpp:81-211) as monteTraj.cpp:362-364
 * calls it.  Blocks until the results are on the host. */
cosims_status cosims_run_list(cosims_ctx *ctx, const double *pos0, const double *vel0,
                              int64_t n, cosims_traj_out *out, void *stream);
/* Per-step trajectory dumps, the reference's print_traj debugging keys
 * (monteTraj::storeTraj / printTraj, monteTraj.cpp:545-586): integrate n
 * given start states in the plain FP64 form and record the He position and
 * velocity after every integration step (all attempts, in order) into frames
 * (host, [n][max_frames][6]: x, y, z, vx, vy, vz).  nframes[i] receives the
 * steps trajectory i integrated; frames holds the first min(nframes[i],
 * max_frames).  Results are cosims_run_list's bit for bit (the trace runs
 * without the hand-off).  Plain contexts only; n * max_frames * 48 bytes at
 * most 4 GiB.  Blocks until the results are on the host. */
cosims_status cosims_trace_list(cosims_ctx *ctx, const double *pos0, const double *vel0,
                                int64_t n, int32_t max_frames, double *frames,
                                int32_t *nframes, cosims_traj_out *out, void *stream);
/* Same with device pointers; stream-ordered, returns without synchronising. */
cosims_status cosims_run_list_device(cosims_ctx *ctx, const double *d_pos0,
                                     const double *d_vel0, int64_t n,
                                     cosims_traj_out *d_out, void *stream);

/* Sampled form: trajectories first_index .. first_index+n-1 of the stream
 * keyed by seed.  Start values come from counter-based Philox4x32-10 on the
 * device (one counter block per trajectory and attempt), with the
 * reference's distributions (monteTraj.cpp:203-253): g ~ g^5 exp(-a g^2) on
 * [g_min, g_max], theta ~ sin(theta), b ~ b on [0, b_max], phi and gamma
 * uniform.  Replaces one CCS integral of monteTraj::runTraj
 * (monteTraj.cpp:301-388).  update_every is the reference's progress
 * interval ceil(print_rate / threads) (monteTraj.cpp:340); n_eff reproduces
 * its one-thread success count.  sums: host; inputs/outs: optional host
 * arrays of n entries (NULL to skip).  Blocks until done. */
cosims_status cosims_run_sampled(cosims_ctx *ctx, uint64_t seed, int64_t first_index,
                                 int64_t n, int64_t update_every, cosims_ccs_sums *sums,
                                 cosims_traj_in *inputs, cosims_traj_out *outs,
                                 void *stream);
/* Same with a device-resident sums record; stream-ordered, no host sync. */
cosims_status cosims_run_sampled_device(cosims_ctx *ctx, uint64_t seed,
                                        int64_t first_index, int64_t n,
                                        int64_t update_every,
                                        cosims_ccs_sums *d_sums, void *stream);
/* Several CCS integrals of one molecule, as monteTraj::runTraj runs its
 * `iter` integrals of `traj` trajectories (monteTraj.cpp:294-388), in as few
 * trajectory-kernel launches as possible: integral k is trajectories
 * first_index + k*n_per .. first_index + (k+1)*n_per - 1 of the seed's
 * stream, and its sums are bit for bit those of cosims_run_sampled on that
 * range (every trajectory runs as it would alone; each integral is reduced on
 * its own records).  One launch holds as many whole integrals as the
 * hand-off's 2^22 records allow, so the long trajectories that end one
 * integral overlap the next integrals' work instead of leaving SMs idle.
 * sums: n_integrals records (host); work: optional host record that receives
 * the call's work counters (steps .. far_terms; the CCS fields are 0), which
 * the per-integral records leave at 0.  Blocks until done. */
cosims_status cosims_run_integrals(cosims_ctx *ctx, uint64_t seed, int64_t first_index,
                                   int64_t n_per, int32_t n_integrals, int64_t update_every,
                                   cosims_ccs_sums *sums, cosims_ccs_sums *work, void *stream);
/* Same with device-resident records (d_sums: n_integrals; d_work may be
 * NULL); stream-ordered, no host sync. */
cosims_status cosims_run_integrals_device(cosims_ctx *ctx, uint64_t seed, int64_t first_index,
                                          int64_t n_per, int32_t n_integrals,
                                          int64_t update_every, cosims_ccs_sums *d_sums,
                                          cosims_ccs_sums *d_work, void *stream);
/* Allocate now what later calls of up to n_traj trajectories (and up to
 * n_integrals integrals in one cosims_run_integrals call) need: start states,
 * records, work order, hand-off records.  Calls otherwise grow these buffers
 * on first use, with cudaMalloc/cudaFree inside the call (cudaFree waits for
 * the device); a caller that times or captures its calls reserves first. */
cosims_status cosims_ctx_reserve(cosims_ctx *ctx, int64_t n_traj, int32_t n_integrals);
/* Start states only: the sampler and the ellipsoid projection
 * (monteTraj.cpp:235-277) for trajectories first_index..first_index+n-1.
 * Host outputs; pos0/vel0 are 3n doubles; hit is n int32. */
cosims_status cosims_sample_inputs(cosims_ctx *ctx, uint64_t seed, int64_t first_index,
                                   int64_t n, cosims_traj_in *inputs, double *pos0,
                                   double *vel0, int32_t *hit, void *stream);

/* Device time (ms) of this context's last trajectory-kernel launch, from CUDA
 * events recorded around the launch on its stream; waits for the launch to
 * finish.  No counterpart in the reference: it exists for measurement. */
cosims_status cosims_ctx_kernel_ms(cosims_ctx *ctx, float *ms);
/* Timeline of the last trajectory kernel of the context (device clock):
 * drain_ms = from the first CTA's start until a group first found the work
 * queue empty; end_ms = until the last group exited.  end_ms - drain_ms is the
 * tail in which some SMs run out of trajectories.  Synchronises. */
cosims_status cosims_ctx_kernel_timeline(cosims_ctx *ctx, double *drain_ms, double *end_ms);

/* Measured FMA throughput (TFLOP/s, FMA = 2 flops) of the FP32 and FP64
 * vector pipes of `device`; either output may be NULL.  No counterpart in the
 * reference: the roofline denominator for the trajectory kernels, which are
 * bound by these pipes rather than by HBM or the tensor cores. */
cosims_status cosims_probe_peaks(int32_t device, double *fp32_tflops, double *fp64_tflops);

/* ---- no device allocation ------------------------------------------------ */
/* No counterpart in the reference.  For callers that cannot let this library
 * allocate device memory -- a host program that owns the GPU's memory through
 * its own pool or arena, or one that forbids cudaMalloc (which synchronises
 * the device and can fail mid-run) on its hot path.  It runs the list form
 * (as cosims_run_list_device) without a context and allocates nothing: the
 * caller passes the molecule and scalars (host), device buffers d_pos0 /
 * d_vel0 (3n doubles each) and d_out (n records); the molecule image, work
 * queue, work order and counters live in one static 12 MiB device array that
 * every GPU loading this library holds until the process exits.  Limits: at
 * most 2,096,128 trajectories per call and molecule images of at most 4 MiB
 * (about 100 bytes per atom and at most 850 per cluster: every molecule within
 * the 16384-atom limit fits with up to 3000 clusters); larger requests return
 * COSIMS_ERR_UNSUPPORTED before any device work.  The first call on a device
 * looks up its array (cudaGetSymbolAddress, with that device current; the
 * device's primary context, the CUDA runtime's, is the one supported) and
 * should come before any stream capture.  Calls share the array: calls that
 * overlap on the GPU (other streams or host threads) race; run them in turn.
 * The run has no long-trajectory hand-off: mixed-form results equal a
 * context's with cosims_ctx_set_handoff(ctx, -1, 0), and plain-form results
 * are bit for bit the context's but its longest trajectories run on one
 * thread each (about 5x the time of a context call on a 1e5-trajectory list).
 * The molecule images are copied from pageable host memory, so the call may
 * wait for that copy; otherwise it is stream-ordered and returns without
 * synchronising.  group_lanes: lanes per trajectory of the mixed form
 * (ignored by the plain form). */
cosims_status cosims_run_list_noalloc(const cosims_molecule *mol, const cosims_params *par,
                                      int32_t precision, int32_t group_lanes,
                                      const double *d_pos0, const double *d_vel0, int64_t n,
                                      cosims_traj_out *d_out, void *stream);

/* ---- batched: many molecules, one persistent launch -------------------- */
typedef struct cosims_batch cosims_batch;

/* mols/pars: n_mol entries.  Molecules are packed into one device arena and
 * staged per CTA with bulk copies when a work item switches molecule. */
cosims_status cosims_batch_create(const cosims_molecule *mols, const cosims_params *pars,
                                  int32_t n_mol, int32_t precision, int32_t device,
                                  cosims_batch **out);
void cosims_batch_destroy(cosims_batch *b);
/* Picks lanes-per-trajectory per molecule and the work-item size by timing
 * short trial launches (results cached by atom count and force type). */
cosims_status cosims_batch_autotune(cosims_batch *b, void *stream);
/* Runs n_traj[i] sampled trajectories of molecule i (seed[i], first_index[i])
 * through one persistent kernel fed by a device work queue; the launch is
 * captured in a CUDA graph on first use and replayed.  sums: n_mol records
 * (host).  Blocks until done. */
cosims_status cosims_batch_run(cosims_batch *b, const uint64_t *seed,
                               const int64_t *first_index, const int64_t *n_traj,
                               cosims_ccs_sums *sums, void *stream);
/* Device-resident form of cosims_batch_run: seeds/first/n and sums stay on
 * the device (host arrays are copied once at the call); no host sync. */
cosims_status cosims_batch_run_async(cosims_batch *b, const uint64_t *seed,
                                     const int64_t *first_index, const int64_t *n_traj,
                                     cosims_ccs_sums *d_sums, void *stream);
/* Lanes per trajectory of molecule mol, and the trajectories in its first
 * work item of the last run (items are cut to about equal cost, about three
 * per CTA; 0 before a run). */
cosims_status cosims_batch_get_launch(const cosims_batch *b, int32_t mol,
                                      int32_t *group_lanes, int32_t *item_traj);
/* Progress interval for the per-molecule n_eff bookkeeping (as update_every
 * of cosims_run_sampled; default 0). */
cosims_status cosims_batch_set_update_every(cosims_batch *b, int64_t update_every);
/* Work of the last run summed over all molecules (steps, evaluations, pair
 * terms; the CCS fields are 0) and its device time in ms (CUDA events around
 * the graph launch; ms may be NULL).  Waits for the run.  For measurement. */
cosims_status cosims_batch_counters(cosims_batch *b, cosims_ccs_sums *work, float *ms);

/* ---- serving: continuous batching of CCS jobs ---------------------------- */
/* No counterpart in the reference (it computes one molecule per process).
 * Jobs are admitted while their device footprint fits the HBM budget and a
 * slot is free; each job's molecule and running sums stay on the device (the
 * molecule in an image arena allocated at creation: admission allocates no
 * device memory and waits for no kernel).  A round integrates the next chunk
 * of every runnable job that fits the server's max_jobs * round_traj
 * trajectory slots (submission order) in one persistent launch, and retires
 * jobs whose relative standard error reached their target (or that reached
 * max_traj).  Up to three rounds are in flight at once on the server's own
 * streams; a job is in at most one of them, so jobs that arrive, or finish a
 * chunk, while rounds run start in the next round without waiting for the
 * others.  A job's first chunk is round_traj trajectories (or min_traj);
 * later chunks are what its running error says it still needs (+5 %, in
 * multiples of round_traj, at most 64 round_traj by default, see
 * cosims_serve_set_max_chunk).  Chunks are the next
 * trajectories of the job's own stream and their sizes follow from the job
 * alone, so its result does not depend on the other jobs or on timing.
 * The HBM budget covers the round buffers (3 * max_jobs * round_traj * 76
 * bytes) and the image arena (the rest, at most 4 GiB).  Calls on one server
 * must be serialised by the caller. */
typedef struct cosims_server cosims_server;

#define COSIMS_JOB_RUNNING 1
#define COSIMS_JOB_DONE 2

typedef struct cosims_job_status {
    int64_t job_id;
    int32_t state;            /* COSIMS_JOB_*                                     */
    int32_t rounds;           /* rounds integrated                                */
    double omega, se, rel_se; /* running CCS (Omega = sum / n_eff) and its error  */
    double device_ms;         /* submit -> retirement, host clock (done jobs)     */
    cosims_ccs_sums sums;     /* running sums                                     */
} cosims_job_status;

cosims_status cosims_serve_create(int32_t device, int64_t hbm_budget_bytes, int32_t max_jobs,
                                  int64_t round_traj, cosims_server **out);
void cosims_serve_destroy(cosims_server *s);
/* Admits a job, or returns COSIMS_ERR_BUSY when it does not fit now. */
cosims_status cosims_serve_submit(cosims_server *s, const cosims_molecule *mol,
                                  const cosims_params *par, uint64_t seed, double target_rel_se,
                                  int64_t min_traj, int64_t max_traj, int64_t *job_id);
/* Advances the server: takes the results of every round that has completed
 * (retiring jobs), then launches a round of the runnable jobs when a round
 * buffer is free; when it could do neither, waits up to 5 ms for a round to
 * complete.  Rounds are ordered after the work queued on `stream` at the call
 * (NULL: no ordering).  n_finished: jobs retired by this call. */
cosims_status cosims_serve_step(cosims_server *s, void *stream, int32_t *n_finished);
cosims_status cosims_serve_poll(cosims_server *s, int64_t job_id, cosims_job_status *out);
/* Frees a job's device resources (its slot and footprint return to the pool). */
cosims_status cosims_serve_release(cosims_server *s, int64_t job_id);
cosims_status cosims_serve_info(const cosims_server *s, int32_t *active, int64_t *bytes_in_use);
/* The most trajectories one job integrates in one round (0: the default, 64
 * round_traj; at least round_traj).  Larger chunks let jobs that need many
 * trajectories finish in fewer rounds, at the cost of longer rounds for the
 * jobs that share them.  Applies to chunks sized after this call. */
cosims_status cosims_serve_set_max_chunk(cosims_server *s, int64_t max_chunk_traj);

#ifdef __cplusplus
}
#endif
#endif /* COSIMS_CUDA_H */
