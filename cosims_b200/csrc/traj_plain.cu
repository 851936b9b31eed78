// traj_plain.cu -- the plain FP64 form: the reference method, one thread per
// trajectory, the reference's operation order in every sum.
//
// Compiled with --fmad=false (no FMA contraction) and IEEE division and square
// root, so each force and potential sum is the same sequence of IEEE double
// operations as the reference's forceAccel (forceAccel.cpp:221-982) compiled
// for x86-64: trajectories agree with the reference bit for bit except for the
// final acos of the scattering angle.
//
// Threads of a warp run different trajectories in lockstep: every loop
// iteration evaluates one acceleration per thread (at the start state or after
// a position update) and, when any thread of the warp needs it, one potential.
// A thread whose trajectory ends takes the next one from a device work queue
// at once, so a warp never waits on its slowest trajectory.
#include <cuda_runtime.h>
#include "device_util.cuh"

namespace cosims {
namespace plain {

struct View {
  const AtomF64 *at;
  const int32_t *perm;
  const ClusterF64 *cl;
  int n, nc, uses_clusters;
};

__device__ __forceinline__ View make_view(const unsigned char *base, const MolImage &img) {
  View v;
  v.at = reinterpret_cast<const AtomF64 *>(base + img.off[S_ATOMS]);
  v.perm = reinterpret_cast<const int32_t *>(base + img.off[S_PERM]);
  v.cl = reinterpret_cast<const ClusterF64 *>(base + img.off[S_CLUSTERS]);
  v.n = img.n_atoms; v.nc = img.n_clusters; v.uses_clusters = img.uses_clusters;
  return v;
}

struct Work {          // per-thread work counters, flushed when a trajectory ends
  uint32_t lj, es, pot, far;
};

// multipoleCutoff (type 1, forceAccel.cpp:221-445) / multipoleOnly (type 2,
// forceAccel.cpp:447-633): identical far-field block; in far clusters type 1
// applies the dispersion cut-off with the parameters of atom index n (the
// cluster index, forceAccel.cpp:353-355), type 2 uses each atom's own.
__device__ void force_multipole(const View &m, const DevParams &p, const double pos[3],
                                double acc[3], bool cutoff, Work &w) {
  double fieldX = 0, fieldY = 0, fieldZ = 0;
  double sMatXY = 0, sMatXZ = 0, sMatYZ = 0, aMatXY = 0, aMatXZ = 0, aMatYZ = 0;
  double diagMatXX = 0, diagMatYY = 0, diagMatZZ = 0;
  double sumX = 0, sumY = 0, sumZ = 0;
  const int order = p.multipole_order;
  for (int n = 0; n < m.nc; n++) {
    double dx0 = pos[0] - m.cl[n].cx, dx1 = pos[1] - m.cl[n].cy, dx2 = pos[2] - m.cl[n].cz;
    double xx = dx0 * dx0, yy = dx1 * dx1, zz = dx2 * dx2;
    double r2 = xx + yy + zz;
    const double multiPlusRad = m.cl[n].mpr2, dispPlusRad = m.cl[n].dr2;
    const int a0 = m.cl[n].a0, a1 = m.cl[n].a1;
    if (r2 > multiPlusRad) {
      const double *D = m.cl[n].dip;
      const double *Q = m.cl[n].quad;
      const bool dipole = order >= 1 && !m.cl[n].replaced;
      double r_2 = 1.0 / r2;
      double r_1 = 1.0 / sqrt(r2);
      double r_3 = r_2 * r_1;
      double r_5 = r_3 * r_2;
      double r_7 = 0, const1 = 0, const2 = 0, t0 = 0, t1 = 0, t2 = 0;
      double xy = dx0 * dx1, xz = dx0 * dx2, yz = dx1 * dx2;
      double chargeR_5 = m.cl[n].q * r_5;
      double chargeR_3 = chargeR_5 * r2;
      if (dipole) {
        r_7 = r_5 * r_2;
        const1 = 3 * (D[0] * dx0 + D[1] * dx1 + D[2] * dx2);
      }
      if (order >= 2) {
        r_7 = r_5 * r_2;
        t0 = (Q[0] * dx0 + Q[3] * dx1 + Q[6] * dx2) * r_7;
        t1 = (Q[1] * dx0 + Q[4] * dx1 + Q[7] * dx2) * r_7;
        t2 = (Q[2] * dx0 + Q[5] * dx1 + Q[8] * dx2) * r_7;
        const2 = 5 * (t0 * dx0 + t1 * dx1 + t2 * dx2) * r_2 * 0.5;
      }
      fieldX += chargeR_3 * dx0;
      fieldY += chargeR_3 * dx1;
      fieldZ += chargeR_3 * dx2;
      diagMatXX += (r2 - 3 * xx) * chargeR_5;
      diagMatYY += (r2 - 3 * yy) * chargeR_5;
      diagMatZZ += (r2 - 3 * zz) * chargeR_5;
      sMatXY -= 3 * xy * chargeR_5;
      sMatXZ -= 3 * xz * chargeR_5;
      sMatYZ -= 3 * yz * chargeR_5;
      if (dipole) {
        fieldX += (const1 * dx0 - r2 * D[0]) * r_5;
        fieldY += (const1 * dx1 - r2 * D[1]) * r_5;
        fieldZ += (const1 * dx2 - r2 * D[2]) * r_5;
        diagMatXX += (r2 - 5 * xx) * r_7 * const1;
        diagMatYY += (r2 - 5 * yy) * r_7 * const1;
        diagMatZZ += (r2 - 5 * zz) * r_7 * const1;
        sMatXY -= 5 * xy * r_7 * const1;
        sMatXZ -= 5 * xz * r_7 * const1;
        sMatYZ -= 5 * yz * r_7 * const1;
        aMatXY += 3 * (D[1] * dx0 - D[0] * dx1) * r_5;
        aMatXZ += 3 * (D[2] * dx0 - D[0] * dx2) * r_5;
        aMatYZ += 3 * (D[2] * dx1 - D[1] * dx2) * r_5;
      }
      if (order >= 2) {
        fieldX += (const2 * dx0 - t0) * r2;
        fieldY += (const2 * dx1 - t1) * r2;
        fieldZ += (const2 * dx2 - t2) * r2;
        diagMatXX += ((r2 - 7 * xx) * const2 - Q[0] * r_5);
        diagMatYY += ((r2 - 7 * yy) * const2 - Q[4] * r_5);
        diagMatZZ += ((r2 - 7 * zz) * const2 - Q[8] * r_5);
        sMatXY -= (7 * xy * const2 + Q[1] * r_5);
        sMatXZ -= (7 * xz * const2 + Q[2] * r_5);
        sMatYZ -= (7 * yz * const2 + Q[5] * r_5);
        aMatXY += 5 * (t1 * dx0 - t0 * dx1);
        aMatXZ += 5 * (t2 * dx0 - t0 * dx2);
        aMatYZ += 5 * (t2 * dx1 - t1 * dx2);
      }
      w.far++;
      if (!cutoff || !(r2 > dispPlusRad)) {
        const double s6 = cutoff ? m.cl[n].qsig6 : 0.0, e24 = cutoff ? m.cl[n].qeps : 0.0;
        for (int k = a0; k < a1; k++) {
          double ex0 = pos[0] - m.at[k].x, ex1 = pos[1] - m.at[k].y, ex2 = pos[2] - m.at[k].z;
          double rr2 = ex0 * ex0 + ex1 * ex1 + ex2 * ex2;
          double r6 = rr2 * rr2 * rr2;
          double term2 = (cutoff ? s6 : m.at[k].sig6) / r6;
          double term1 = 2 * term2 * term2;
          double scalarComp = (cutoff ? e24 : m.at[k].eps24m) * (term1 - term2) / rr2;
          sumX += scalarComp * ex0;
          sumY += scalarComp * ex1;
          sumZ += scalarComp * ex2;
        }
        w.lj += a1 - a0;
      }
    } else {
      const bool lj = !cutoff || !(r2 > dispPlusRad);
      for (int k = a0; k < a1; k++) {
        double charge = m.at[k].q;
        double ex0 = pos[0] - m.at[k].x, ex1 = pos[1] - m.at[k].y, ex2 = pos[2] - m.at[k].z;
        double rr2 = ex0 * ex0 + ex1 * ex1 + ex2 * ex2;
        double r_5 = 1.0 / (rr2 * rr2 * sqrt(rr2));
        double r_3 = r_5 * rr2;
        r_3 *= charge;
        r_5 *= charge;
        fieldX += ex0 * r_3;
        fieldY += ex1 * r_3;
        fieldZ += ex2 * r_3;
        diagMatXX += (rr2 - 3 * ex0 * ex0) * r_5;
        diagMatYY += (rr2 - 3 * ex1 * ex1) * r_5;
        diagMatZZ += (rr2 - 3 * ex2 * ex2) * r_5;
        sMatXY -= 3 * ex0 * ex1 * r_5;
        sMatXZ -= 3 * ex0 * ex2 * r_5;
        sMatYZ -= 3 * ex1 * ex2 * r_5;
        if (lj) {
          double r6 = rr2 * rr2 * rr2;
          double term2 = m.at[k].sig6 / r6;
          double term1 = 2 * term2 * term2;
          double scalarComp = m.at[k].eps24m * (term1 - term2) / rr2;
          sumX += scalarComp * ex0;
          sumY += scalarComp * ex1;
          sumZ += scalarComp * ex2;
        }
      }
      w.es += a1 - a0;
    }
  }
  const double ds = p.dipole_scalar;
  sumX += ds * (diagMatXX * fieldX + (sMatXY + aMatXY) * fieldY + (sMatXZ + aMatXZ) * fieldZ);
  sumY += ds * ((sMatXY - aMatXY) * fieldX + diagMatYY * fieldY + (sMatYZ + aMatYZ) * fieldZ);
  sumZ += ds * ((sMatXZ - aMatXZ) * fieldX + (sMatYZ - aMatYZ) * fieldY + diagMatZZ * fieldZ);
  acc[0] = sumX; acc[1] = sumY; acc[2] = sumZ;
}

// dispersionOnly (type 3, forceAccel.cpp:635-749).
__device__ void force_dispersion_only(const View &m, const DevParams &p, const double pos[3],
                                      double acc[3], Work &w) {
  double fieldX = 0, fieldY = 0, fieldZ = 0;
  double sMatXY = 0, sMatXZ = 0, sMatYZ = 0;
  double diagMatXX = 0, diagMatYY = 0, diagMatZZ = 0;
  double sumX = 0, sumY = 0, sumZ = 0;
  for (int n = 0; n < m.nc; n++) {
    double dx0 = pos[0] - m.cl[n].cx, dx1 = pos[1] - m.cl[n].cy, dx2 = pos[2] - m.cl[n].cz;
    double xx = dx0 * dx0, yy = dx1 * dx1, zz = dx2 * dx2;
    double r2 = xx + yy + zz;
    const bool lj = !(r2 > m.cl[n].dr2);
    const int a0 = m.cl[n].a0, a1 = m.cl[n].a1;
    for (int k = a0; k < a1; k++) {
      double charge = m.at[k].q;
      double ex0 = pos[0] - m.at[k].x, ex1 = pos[1] - m.at[k].y, ex2 = pos[2] - m.at[k].z;
      double rr2 = ex0 * ex0 + ex1 * ex1 + ex2 * ex2;
      double r_5 = 1.0 / (rr2 * rr2 * sqrt(rr2));
      double r_3 = r_5 * rr2;
      r_3 *= charge;
      r_5 *= charge;
      fieldX += ex0 * r_3;
      fieldY += ex1 * r_3;
      fieldZ += ex2 * r_3;
      diagMatXX += (rr2 - 3 * ex0 * ex0) * r_5;
      diagMatYY += (rr2 - 3 * ex1 * ex1) * r_5;
      diagMatZZ += (rr2 - 3 * ex2 * ex2) * r_5;
      sMatXY -= 3 * ex0 * ex1 * r_5;
      sMatXZ -= 3 * ex0 * ex2 * r_5;
      sMatYZ -= 3 * ex1 * ex2 * r_5;
      if (lj) {
        double r6 = rr2 * rr2 * rr2;
        double term2 = m.at[k].sig6 / r6;
        double term1 = 2 * term2 * term2;
        double scalarComp = m.at[k].eps24m * (term1 - term2) / rr2;
        sumX += scalarComp * ex0;
        sumY += scalarComp * ex1;
        sumZ += scalarComp * ex2;
      }
    }
    w.es += a1 - a0;
  }
  const double ds = p.dipole_scalar;
  sumX += ds * (diagMatXX * fieldX + sMatXY * fieldY + sMatXZ * fieldZ);
  sumY += ds * (sMatXY * fieldX + diagMatYY * fieldY + sMatYZ * fieldZ);
  sumZ += ds * (sMatXZ * fieldX + sMatYZ * fieldY + diagMatZZ * fieldZ);
  acc[0] = sumX; acc[1] = sumY; acc[2] = sumZ;
}

// chargeDipoleLJ (type 4, forceAccel.cpp:751-805).
__device__ void force_charge_dipole_lj(const View &m, const DevParams &p, const double pos[3],
                                       double acc[3], Work &w) {
  double sumXX = 0, sumYY = 0, sumZZ = 0, sumXY = 0, sumXZ = 0, sumYZ = 0;
  double dipX = 0, dipY = 0, dipZ = 0, tempx = 0, tempy = 0, tempz = 0;
  for (int n = 0; n < m.n; n++) {
    double xDiff = pos[0] - m.at[n].x, yDiff = pos[1] - m.at[n].y, zDiff = pos[2] - m.at[n].z;
    double xDiff2 = xDiff * xDiff, yDiff2 = yDiff * yDiff, zDiff2 = zDiff * zDiff;
    double r2 = xDiff2 + yDiff2 + zDiff2;
    double r = sqrt(r2);
    double r3 = r2 * r;
    double r_3 = 1.0 / r3;
    double r_5 = r_3 / r2;
    double r6 = r2 * r2 * r2;
    const double qn = m.at[n].q;
    r_3 *= qn;
    r_5 *= qn;
    double term2 = m.at[n].sig6 / r6;
    double term1 = 2 * term2 * term2;
    double scalarComp = m.at[n].eps24m * (term1 - term2) / r2;
    tempx += scalarComp * xDiff;
    tempy += scalarComp * yDiff;
    tempz += scalarComp * zDiff;
    dipX += xDiff * r_3;
    dipY += yDiff * r_3;
    dipZ += zDiff * r_3;
    sumXX += (3.0 * xDiff2 - r2) * r_5;
    sumYY += (3.0 * yDiff2 - r2) * r_5;
    sumZZ += (3.0 * zDiff2 - r2) * r_5;
    sumXY += 3 * xDiff * yDiff * r_5;
    sumXZ += 3 * xDiff * zDiff * r_5;
    sumYZ += 3 * yDiff * zDiff * r_5;
  }
  w.es += m.n;
  const double ds = p.dipole_scalar;
  tempx -= ds * (sumXX * dipX + sumXY * dipY + sumXZ * dipZ);
  tempy -= ds * (sumXY * dipX + sumYY * dipY + sumYZ * dipZ);
  tempz -= ds * (sumXZ * dipX + sumYZ * dipY + sumZZ * dipZ);
  acc[0] = tempx; acc[1] = tempy; acc[2] = tempz;
}

// dispersionNoCharge (type 5, forceAccel.cpp:807-854).
__device__ void force_dispersion_nocharge(const View &m, const double pos[3], double acc[3],
                                          Work &w) {
  double sumX = 0, sumY = 0, sumZ = 0;
  for (int n = 0; n < m.nc; n++) {
    double dx0 = pos[0] - m.cl[n].cx, dx1 = pos[1] - m.cl[n].cy, dx2 = pos[2] - m.cl[n].cz;
    double xx = dx0 * dx0, yy = dx1 * dx1, zz = dx2 * dx2;
    double r2 = xx + yy + zz;
    if (!(r2 > m.cl[n].dr2)) {
      const int a0 = m.cl[n].a0, a1 = m.cl[n].a1;
      for (int k = a0; k < a1; k++) {
        double ex0 = pos[0] - m.at[k].x, ex1 = pos[1] - m.at[k].y, ex2 = pos[2] - m.at[k].z;
        double rr2 = ex0 * ex0 + ex1 * ex1 + ex2 * ex2;
        double r6 = rr2 * rr2 * rr2;
        double term2 = m.at[k].sig6 / r6;
        double term1 = 2 * term2 * term2;
        double scalarComp = m.at[k].eps24m * (term1 - term2) / rr2;
        sumX += scalarComp * ex0;
        sumY += scalarComp * ex1;
        sumZ += scalarComp * ex2;
      }
      w.lj += a1 - a0;
    }
  }
  acc[0] = sumX; acc[1] = sumY; acc[2] = sumZ;
}

// dispersionFull (type 6, forceAccel.cpp:856-884).
__device__ void force_dispersion_full(const View &m, const double pos[3], double acc[3],
                                      Work &w) {
  double tempx = 0, tempy = 0, tempz = 0;
  for (int n = 0; n < m.n; n++) {
    double xDiff = pos[0] - m.at[n].x, yDiff = pos[1] - m.at[n].y, zDiff = pos[2] - m.at[n].z;
    double xDiff2 = xDiff * xDiff, yDiff2 = yDiff * yDiff, zDiff2 = zDiff * zDiff;
    double r2 = xDiff2 + yDiff2 + zDiff2;
    double r6 = r2 * r2 * r2;
    double term2 = m.at[n].sig6 / r6;
    double term1 = 2 * term2 * term2;
    double scalarComp = m.at[n].eps24m * (term1 - term2) / r2;
    tempx += scalarComp * xDiff;
    tempy += scalarComp * yDiff;
    tempz += scalarComp * zDiff;
  }
  w.lj += m.n;
  acc[0] = tempx; acc[1] = tempy; acc[2] = tempz;
}

__device__ __forceinline__ void force(const View &m, const DevParams &p, const double pos[3],
                                      double acc[3], Work &w) {
  switch (p.force_type) {
    case 1: force_multipole(m, p, pos, acc, true, w); break;
    case 2: force_multipole(m, p, pos, acc, false, w); break;
    case 3: force_dispersion_only(m, p, pos, acc, w); break;
    case 4: force_charge_dipole_lj(m, p, pos, acc, w); break;
    case 5: force_dispersion_nocharge(m, pos, acc, w); break;
    default: force_dispersion_full(m, pos, acc, w); break;
  }
}

// getPotential (forceAccel.cpp:943-982), atoms in file order.
__device__ double potential(const View &m, const DevParams &p, const double pos[3]) {
  double total = 0, sumX = 0, sumY = 0, sumZ = 0;
  for (int i = 0; i < m.n; i++) {
    const int k = m.uses_clusters ? m.perm[i] : i;
    double xDiff = pos[0] - m.at[k].x, yDiff = pos[1] - m.at[k].y, zDiff = pos[2] - m.at[k].z;
    double r2 = xDiff * xDiff + yDiff * yDiff + zDiff * zDiff;
    double r6 = r2 * r2 * r2;
    double term2 = m.at[k].sig6 / r6;
    double term1 = term2 * term2;
    total += m.at[k].eps4 * (term1 - term2);
    if (p.charged) {
      double r_3 = m.at[k].q / (r2 * sqrt(r2));
      sumX += xDiff * r_3;
      sumY += yDiff * r_3;
      sumZ += zDiff * r_3;
    }
  }
  if (p.charged) total -= p.dipole_scalar * 0.5 * (sumX * sumX + sumY * sumY + sumZ * sumZ);
  return total;
}

__device__ __forceinline__ double dot3(const double a[3], const double b[3]) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

// vector3D::Angle (vector3D.h:134-143).
__device__ __forceinline__ double angle3(const double a[3], const double b[3]) {
  double term1 = dot3(a, b);
  double term2 = sqrt(dot3(a, a)) * sqrt(dot3(b, b));
  double term3 = term1 / term2;
  if (term3 > 1) return 0;
  if (term3 < -1) return COSIMS_PI;
  return acos(term1 / term2);
}

enum Phase : int { P_ACQUIRE = 0, P_INIT_FIRST, P_INIT_RETRY, P_STEP, P_DONE };

__global__ void __launch_bounds__(128) traj_plain_kernel(const TrajArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ uint64_t bar;
  const unsigned char *base = a.img.gbase;
  if (a.use_smem) {
    if (!stage_to_smem(smem, a.img.gbase, a.img.bytes, &bar, 0, true)) {
      if (threadIdx.x == 0) atomicOr(a.counters + C_ERROR, 1ull);
      return;
    }
    base = smem;
  }
  if (threadIdx.x == 0) mark_first(a.counters, C_T_START_INV);
  const View m = make_view(base, a.img);
  const DevParams &p = a.par;
  const long long cap = p.max_steps > 0 ? p.max_steps : kDefaultMaxSteps;

  double p0[3], v0[3], pos[3] = {0, 0, 0}, vel[3] = {0, 0, 0}, acc[3] = {0, 0, 0};
  double E0 = 0, dt = p.dt, tries = 0, maxTries = 8, rdot = 0;
  int orbits = 0, step = 0, phase = P_ACQUIRE;
  long long total = 0, t = 0;
  unsigned etries = 0, otries = 0;
  Work w = {0, 0, 0, 0};
  uint32_t nforce = 0, npot = 0;
  unsigned long long nsteps = 0;

  auto finish = [&](double chi, double de, int steps, uint32_t status) {
    cosims_traj_out o;
    o.chi = chi; o.de_pct = de; o.steps = steps;
    o.status = status | (etries << COSIMS_TRAJ_ETRIES_SHIFT) | (otries << COSIMS_TRAJ_OTRIES_SHIFT);
    a.out[t] = o;
    phase = P_ACQUIRE;
  };

  while (true) {
    if (phase == P_ACQUIRE) {
      for (;;) {
        t = (long long)atomicAdd(a.queue, 1ull);
        if (t >= a.n) {
          if (t == a.n) mark_first(a.counters, C_T_DRAIN_INV);   // first to find it empty
          phase = P_DONE;
          break;
        }
        if (a.order) t = a.order[t];
        if (a.hit && !a.hit[t]) {                 // ellipsoid miss: chi = 0
          cosims_traj_out o = {0.0, 0.0, 0, 0u};
          a.out[t] = o;
          continue;
        }
        for (int i = 0; i < 3; i++) { p0[i] = a.pos0[3 * t + i]; v0[i] = a.vel0[3 * t + i]; }
        phase = P_INIT_FIRST;
        break;
      }
      if (phase == P_INIT_FIRST) {
        tries = 0; maxTries = 8; dt = p.dt; step = 0; total = 0; etries = 0; otries = 0;
      }
    }
    if (__all_sync(0xffffffffu, phase == P_DONE)) break;

    double ep[3];
    bool needU = false, outside = false;
    if (phase == P_INIT_FIRST || phase == P_INIT_RETRY) {
      ep[0] = p0[0]; ep[1] = p0[1]; ep[2] = p0[2];
      needU = phase == P_INIT_FIRST;
    } else if (phase == P_STEP) {
      for (int i = 0; i < 3; i++) {
        pos[i] = pos[i] + vel[i] * dt + acc[i] * dt * dt * 0.5;
        vel[i] = vel[i] + acc[i] * dt * 0.5;
      }
      ep[0] = pos[0]; ep[1] = pos[1]; ep[2] = pos[2];
      double t0 = pos[0] / p.ell_a, t1 = pos[1] / p.ell_b, t2 = pos[2] / p.ell_c;
      double mag2 = t0 * t0 + t1 * t1 + t2 * t2;
      outside = (mag2 > 1 && p.projection) || (mag2 > p.max_rad && !p.projection);
      needU = outside && step + 1 > 10;
    } else {
      ep[0] = 1.0e4; ep[1] = 0.0; ep[2] = 0.0;   // idle thread: result unused
    }

    double an[3];
    Work wi = {0, 0, 0, 0};
    force(m, p, ep, an, wi);
    double U = 0;
    if (__any_sync(0xffffffffu, needU)) U = potential(m, p, ep);
    if (phase == P_DONE) continue;
    nforce++;
    w.lj += wi.lj; w.es += wi.es; w.far += wi.far;
    if (needU) { npot++; w.pot += m.n; }

    if (phase == P_INIT_FIRST || phase == P_INIT_RETRY) {
      if (phase == P_INIT_FIRST) E0 = U + 0.5 * p.mu * dot3(v0, v0);
      for (int i = 0; i < 3; i++) { acc[i] = an[i]; pos[i] = p0[i]; vel[i] = v0[i]; }
      orbits = 0;
      rdot = dot3(pos, vel);
      phase = P_STEP;
      continue;
    }

    for (int i = 0; i < 3; i++) { vel[i] = vel[i] + an[i] * dt * 0.5; acc[i] = an[i]; }
    step++;
    total++;
    nsteps++;
    bool track = true;
    const double rold = rdot;
    rdot = dot3(pos, vel);
    const double product = rdot * rold;
    if (step > 2 && product < 0 && !(rdot > rold)) {
      orbits++;
      if (orbits > 8) track = false;          // maxOrbits = 8 (diffEqSolver.cpp:40)
    }
    if (!track) {
      tries++;
      otries++;
      dt = p.dt / ((tries + 1));
    } else if (outside && step > 10) {
      double endE = U + 0.5 * p.mu * dot3(vel, vel);
      double dE = 100 * fabs(E0 - endE) / E0;
      double chi = angle3(v0, vel);
      if (dE > 0.5) {
        tries++;
        maxTries++;
        etries++;
        dt = p.dt / ((tries + 1));
        step = 0;
      } else {
        finish(chi, dE, step, COSIMS_TRAJ_HIT | COSIMS_TRAJ_SUCCESS);
      }
    }
    if (phase == P_STEP) {
      // the step cap, or a state gone non-finite (the reference would loop)
      if (total >= cap || !isfinite(rdot))
        finish(COSIMS_PI_2, 0.0, step, COSIMS_TRAJ_HIT | COSIMS_TRAJ_STEPCAP);
      else if (!(tries < maxTries && maxTries < 10)) finish(COSIMS_PI_2, 0.0, step, COSIMS_TRAJ_HIT);
      else if (step == 0) phase = P_INIT_RETRY;
    }
  }
  unsigned long long *c = a.counters;
  count_add(c, C_STEPS, (long long)nsteps);
  count_add(c, C_FORCE_EVALS, nforce);
  count_add(c, C_POT_EVALS, npot);
  count_add(c, C_PAIR_LJ, w.lj);
  count_add(c, C_PAIR_ES, w.es);
  count_add(c, C_PAIR_POT, w.pot);
  count_add(c, C_FAR, w.far);
  if ((threadIdx.x & 31) == 0) mark_last(c, C_T_END);
}

}  // namespace plain

int plain_max_smem_per_block() {
  int dev = 0, v = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  return v - 1024;   // leave room for the static barrier word
}

int plain_launch(const TrajArgs &a, int block, int grid, size_t smem, void *stream) {
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(plain::traj_plain_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
  }
  plain::traj_plain_kernel<<<grid, block, smem, (cudaStream_t)stream>>>(a);
  return (int)cudaGetLastError();
}

}  // namespace cosims

namespace cosims {
int plain_occupancy(int block, size_t smem, int *per_sm) {
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(plain::traj_plain_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
  }
  return (int)cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, plain::traj_plain_kernel,
                                                            block, smem);
}
}  // namespace cosims
