/*
 * cosims_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the CoSIMS trajectory path, used by tests/, the smoke
 * check and bench.py's cpu_baseline leg as the checker.  It is never linked
 * into, loaded by, or called from the product (cosims_b200/).  Parity is
 * pinned against the reference itself (oracle/_ref, built from the reference
 * sources by oracle/Makefile) through tests/golden fixtures.
 */
#ifndef COSIMS_ORACLE_H
#define COSIMS_ORACLE_H
#include "cosims_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

/* forceAccel::getReducedVec (forceAccel.cpp:887-908): acceleration on He. */
void oracle_force(const cosims_molecule *mol, const cosims_params *par,
                  const double pos[3], double acc[3]);
/* forceAccel::getPotential (forceAccel.cpp:943-982). */
double oracle_potential(const cosims_molecule *mol, const cosims_params *par,
                        const double pos[3]);
/* diffEqSolver::verletVel (diffEqSolver.cpp:81-211) on one start state. */
void oracle_verlet(const cosims_molecule *mol, const cosims_params *par,
                   const double pos0[3], const double vel0[3], cosims_traj_out *out);
/* oracle_verlet that also records position and velocity after every
 * integration step (all attempts) into frames[cap][6]; *nframes = steps. */
void oracle_verlet_trace(const cosims_molecule *mol, const cosims_params *par,
                         const double pos0[3], const double vel0[3], cosims_traj_out *out,
                         double *frames, int32_t cap, int32_t *nframes);
/* Start state geometry and ellipsoid projection of monteTraj::setUpTraj
 * (monteTraj.cpp:235-277).  Returns 1 on a hit, 0 on a miss. */
int oracle_start_state(const cosims_params *par, const cosims_traj_in *in,
                       double pos0[3], double vel0[3]);
/* verletVel over a list, in order. */
void oracle_run_list(const cosims_molecule *mol, const cosims_params *par, int64_t n,
                     const double *pos0, const double *vel0, cosims_traj_out *out);
/* Start states from sampled values, then verletVel; misses get chi = 0. */
void oracle_run_inputs(const cosims_molecule *mol, const cosims_params *par, int64_t n,
                       const cosims_traj_in *in, cosims_traj_out *out);
/* monteTraj::runThreads / updateCounts / runTraj accumulation
 * (monteTraj.cpp:456-521, :380-387) over results in trajectory order, with
 * the reference's one-thread bookkeeping (update_every = progress interval). */
void oracle_reduce(const cosims_params *par, int64_t n, const cosims_traj_out *out,
                   int64_t update_every, cosims_ccs_sums *sums);
/* Omega and its standard error from one integral's sums (monteTraj.cpp:381-387). */
void oracle_omega(const cosims_ccs_sums *s, double *omega, double *err);

#ifdef __cplusplus
}
#endif
#endif
