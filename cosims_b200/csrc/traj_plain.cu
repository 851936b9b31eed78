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
  const int2 *slot;          // exact-phase events {atom or -1, cluster}
  int n, nc, uses_clusters, nslot;
};

__device__ __forceinline__ View make_view(const unsigned char *base, const MolImage &img) {
  View v;
  v.at = reinterpret_cast<const AtomF64 *>(base + img.off[S_ATOMS]);
  v.perm = reinterpret_cast<const int32_t *>(base + img.off[S_PERM]);
  v.cl = reinterpret_cast<const ClusterF64 *>(base + img.off[S_CLUSTERS]);
  v.slot = reinterpret_cast<const int2 *>(base + img.off[S_SLOTS]);
  v.n = img.n_atoms; v.nc = img.n_clusters; v.uses_clusters = img.uses_clusters;
  v.nslot = img.n_slots;
  return v;
}

struct Work {          // per-thread work counters, flushed when a trajectory ends
  uint32_t lj, es, pot, far;
  uint32_t nl;         // of es: outside the LJ cut-off (charge field only)
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
      if (!lj) w.nl += a1 - a0;
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
    if (!lj) w.nl += a1 - a0;
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

template <int TYPE>
__device__ __forceinline__ void force(const View &m, const DevParams &p, const double pos[3],
                                      double acc[3], Work &w) {
  switch (TYPE) {
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

// ---- exact wide phase: long trajectories finished by a whole CTA ------------------
// A trajectory still running after the hand-off budget is parked, and once a
// CTA's threads run out of work the CTA finishes parked trajectories one at a
// time.  Each evaluation walks the event slots (atoms, and the three parts of a
// cluster's far field) in the serial loops' order, in chunks of kExactChunk:
// warps 1..3 evaluate the terms of chunk c+1 with the serial code's own
// expressions while lane k of warp 0 adds the terms of accumulator k of chunk c
// in slot order.  A slot that adds nothing to an accumulator holds that sum's
// neutral element (-0.0 for a sum, +0.0 for a difference: x + -0.0 == x and
// x - +0.0 == x for every x, signed zeros included), so every chunk is a fixed
// run of additions.  The additions are the serial sums', in their order, so the
// forces, the potential and hence the trajectory are bitwise those of the
// one-thread loop; only the work of one step is spread.
struct Exact {
  uint8_t *cflag;     // per cluster: bit 0 far (r2 > mpr2), bit 1 in the LJ cut-off
  double *terms;      // two chunk buffers of [K][kExactRow] doubles
  double *accs;       // [16]
  long long *bcast;
  int K;
};

__device__ __forceinline__ Exact exact_scratch(unsigned char *smem, uint32_t img_bytes,
                                               int force_type, int nc) {
  Exact x;
  unsigned char *q = smem + ((img_bytes + 15u) & ~15u);
  x.K = exact_accumulators(force_type);
  x.cflag = q;
  q += ((uint32_t)nc + 15u) & ~15u;
  x.terms = reinterpret_cast<double *>(q);
  q += 2u * (uint32_t)(x.K * kExactRow) * 8u;
  x.accs = reinterpret_cast<double *>(q);
  q += 16u * 8u;
  x.bcast = reinterpret_cast<long long *>(q);
  return x;
}

// The terms column of one event slot in a chunk buffer.  `part` selects which
// of a far-field cluster's three consecutive slots this is; the other events
// have one part.
struct Col {
  double *T;
  int j, part;
  __device__ __forceinline__ void put(int k, int pt, double v) const {
    if (pt == part) T[k * kExactRow + j] = v;
  }
};

// sum_k over nitems slots, for k < K: warps 1..3 produce chunk c+1 (neutral
// fill, then produce(col, slot)), lane k of warp 0 adds chunk c.  Bit k of
// `minus` marks the accumulators the serial code decrements.  Every thread
// passes the same __syncthreads sequence; lane k < K of warp 0 returns sum k.
template <class Produce>
__device__ __forceinline__ double exact_sum(const Exact &x, int nitems, int K, uint32_t minus,
                                            Produce produce) {
  double acc = 0;
  const int nch = (nitems + kExactChunk - 1) / kExactChunk;
  const int buf = K * kExactRow;
  const bool sub = (minus >> (threadIdx.x & 15)) & 1u;
  for (int c = 0; c <= nch; c++) {
    if (threadIdx.x >= 32) {
      if (c < nch) {
        double *T = x.terms + (c & 1) * buf;
#pragma unroll
        for (int s = 0; s < kExactPerThread; s++) {
          const int j = (int)threadIdx.x - 32 + s * kExactProducers;
          for (int k = 0; k < K; k++) T[k * kExactRow + j] = ((minus >> k) & 1u) ? 0.0 : -0.0;
          const int e = c * kExactChunk + j;
          if (e < nitems) produce(T, j, e);
        }
      }
    } else if (c > 0 && (int)threadIdx.x < K) {
      const double *T = x.terms + ((c - 1) & 1) * buf + threadIdx.x * kExactRow;
      if (sub) {
#pragma unroll 16
        for (int j = 0; j < kExactChunk; j++) acc = acc - T[j];
      } else {
#pragma unroll 16
        for (int j = 0; j < kExactChunk; j++) acc = acc + T[j];
      }
    }
    __syncthreads();
  }
  return acc;
}

// One event's terms for the force variants, as the serial loops of the
// force_* functions above compute them.
template <int TYPE>
__device__ __forceinline__ void event_terms(const View &m, const DevParams &p, const double pos[3],
                                            const Exact &x, double *T, int j, int e, Work &w) {
  const int2 sl = m.slot[e];
  const Col o{T, j, sl.x < 0 ? -1 - sl.x : 0};
  constexpr int type = TYPE;
  if (type == 4 || type == 6) {
    const int n = sl.x;
    double xDiff = pos[0] - m.at[n].x, yDiff = pos[1] - m.at[n].y, zDiff = pos[2] - m.at[n].z;
    double xDiff2 = xDiff * xDiff, yDiff2 = yDiff * yDiff, zDiff2 = zDiff * zDiff;
    double r2 = xDiff2 + yDiff2 + zDiff2;
    double r6 = r2 * r2 * r2;
    double term2 = m.at[n].sig6 / r6;
    double term1 = 2 * term2 * term2;
    double scalarComp = m.at[n].eps24m * (term1 - term2) / r2;
    o.put(0, 0, scalarComp * xDiff);
    o.put(1, 0, scalarComp * yDiff);
    o.put(2, 0, scalarComp * zDiff);
    if (type == 4) {
      double r = sqrt(r2);
      double r3 = r2 * r;
      double r_3 = 1.0 / r3;
      double r_5 = r_3 / r2;
      const double qn = m.at[n].q;
      r_3 *= qn;
      r_5 *= qn;
      o.put(3, 0, xDiff * r_3);
      o.put(4, 0, yDiff * r_3);
      o.put(5, 0, zDiff * r_3);
      o.put(6, 0, (3.0 * xDiff2 - r2) * r_5);
      o.put(7, 0, (3.0 * yDiff2 - r2) * r_5);
      o.put(8, 0, (3.0 * zDiff2 - r2) * r_5);
      o.put(9, 0, 3 * xDiff * yDiff * r_5);
      o.put(10, 0, 3 * xDiff * zDiff * r_5);
      o.put(11, 0, 3 * yDiff * zDiff * r_5);
      w.es++;
    } else {
      w.lj++;
    }
    return;
  }
  const int c = sl.y;
  const uint8_t flag = x.cflag[c];
  const bool far = flag & 1u, in_lj = (flag & 2u) != 0;
  if (type == 5) {
    if (!in_lj) return;
    const int k = sl.x;
    double ex0 = pos[0] - m.at[k].x, ex1 = pos[1] - m.at[k].y, ex2 = pos[2] - m.at[k].z;
    double rr2 = ex0 * ex0 + ex1 * ex1 + ex2 * ex2;
    double r6 = rr2 * rr2 * rr2;
    double term2 = m.at[k].sig6 / r6;
    double term1 = 2 * term2 * term2;
    double scalarComp = m.at[k].eps24m * (term1 - term2) / rr2;
    o.put(0, 0, scalarComp * ex0);
    o.put(1, 0, scalarComp * ex1);
    o.put(2, 0, scalarComp * ex2);
    w.lj++;
    return;
  }
  // variants 1, 2, 3: accumulators fieldXYZ 0-2, diagMat 3-5, sMat 6-8 (minus),
  // aMat 9-11 (variants 1, 2), LJ sums 9-11 (variant 3) or 12-14 (1, 2)
  const bool cutoff = type == 1;
  const int ljk = type == 3 ? 9 : 12;
  if (sl.x < 0) {                       // far field of cluster c (variants 1, 2)
    if (!far) return;
    const ClusterF64 &C = m.cl[c];
    double dx0 = pos[0] - C.cx, dx1 = pos[1] - C.cy, dx2 = pos[2] - C.cz;
    double xx = dx0 * dx0, yy = dx1 * dx1, zz = dx2 * dx2;
    double r2 = xx + yy + zz;
    const double *D = C.dip;
    const double *Q = C.quad;
    const int order = p.multipole_order;
    const bool dipole = order >= 1 && !C.replaced;
    double r_2 = 1.0 / r2;
    double r_1 = 1.0 / sqrt(r2);
    double r_3 = r_2 * r_1;
    double r_5 = r_3 * r_2;
    double r_7 = 0, const1 = 0, const2 = 0, t0 = 0, t1 = 0, t2 = 0;
    double xy = dx0 * dx1, xz = dx0 * dx2, yz = dx1 * dx2;
    double chargeR_5 = C.q * r_5;
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
    o.put(0, 0, chargeR_3 * dx0);
    o.put(1, 0, chargeR_3 * dx1);
    o.put(2, 0, chargeR_3 * dx2);
    o.put(3, 0, (r2 - 3 * xx) * chargeR_5);
    o.put(4, 0, (r2 - 3 * yy) * chargeR_5);
    o.put(5, 0, (r2 - 3 * zz) * chargeR_5);
    o.put(6, 0, 3 * xy * chargeR_5);
    o.put(7, 0, 3 * xz * chargeR_5);
    o.put(8, 0, 3 * yz * chargeR_5);
    int pa = 0;
    if (dipole) {
      o.put(0, 1, (const1 * dx0 - r2 * D[0]) * r_5);
      o.put(1, 1, (const1 * dx1 - r2 * D[1]) * r_5);
      o.put(2, 1, (const1 * dx2 - r2 * D[2]) * r_5);
      o.put(3, 1, (r2 - 5 * xx) * r_7 * const1);
      o.put(4, 1, (r2 - 5 * yy) * r_7 * const1);
      o.put(5, 1, (r2 - 5 * zz) * r_7 * const1);
      o.put(6, 1, 5 * xy * r_7 * const1);
      o.put(7, 1, 5 * xz * r_7 * const1);
      o.put(8, 1, 5 * yz * r_7 * const1);
      o.put(9, 0, 3 * (D[1] * dx0 - D[0] * dx1) * r_5);
      o.put(10, 0, 3 * (D[2] * dx0 - D[0] * dx2) * r_5);
      o.put(11, 0, 3 * (D[2] * dx1 - D[1] * dx2) * r_5);
      pa = 1;
    }
    if (order >= 2) {
      const int pf = dipole ? 2 : 1;
      o.put(0, pf, (const2 * dx0 - t0) * r2);
      o.put(1, pf, (const2 * dx1 - t1) * r2);
      o.put(2, pf, (const2 * dx2 - t2) * r2);
      o.put(3, pf, ((r2 - 7 * xx) * const2 - Q[0] * r_5));
      o.put(4, pf, ((r2 - 7 * yy) * const2 - Q[4] * r_5));
      o.put(5, pf, ((r2 - 7 * zz) * const2 - Q[8] * r_5));
      o.put(6, pf, (7 * xy * const2 + Q[1] * r_5));
      o.put(7, pf, (7 * xz * const2 + Q[2] * r_5));
      o.put(8, pf, (7 * yz * const2 + Q[5] * r_5));
      o.put(9, pa, 5 * (t1 * dx0 - t0 * dx1));
      o.put(10, pa, 5 * (t2 * dx0 - t0 * dx2));
      o.put(11, pa, 5 * (t2 * dx1 - t1 * dx2));
    }
    if (o.part == 0) w.far++;
    return;
  }
  const int k = sl.x;
  if (type != 3 && far) {               // far cluster: the LJ band only
    if (cutoff && !in_lj) return;
    const ClusterF64 &C = m.cl[c];
    const double s6 = cutoff ? C.qsig6 : 0.0, e24 = cutoff ? C.qeps : 0.0;
    double ex0 = pos[0] - m.at[k].x, ex1 = pos[1] - m.at[k].y, ex2 = pos[2] - m.at[k].z;
    double rr2 = ex0 * ex0 + ex1 * ex1 + ex2 * ex2;
    double r6 = rr2 * rr2 * rr2;
    double term2 = (cutoff ? s6 : m.at[k].sig6) / r6;
    double term1 = 2 * term2 * term2;
    double scalarComp = (cutoff ? e24 : m.at[k].eps24m) * (term1 - term2) / rr2;
    o.put(ljk, 0, scalarComp * ex0);
    o.put(ljk + 1, 0, scalarComp * ex1);
    o.put(ljk + 2, 0, scalarComp * ex2);
    w.lj++;
    return;
  }
  // a near cluster (or any cluster of variant 3): charge field, and LJ inside the cut-off
  const bool lj = type == 2 || in_lj;
  double charge = m.at[k].q;
  double ex0 = pos[0] - m.at[k].x, ex1 = pos[1] - m.at[k].y, ex2 = pos[2] - m.at[k].z;
  double rr2 = ex0 * ex0 + ex1 * ex1 + ex2 * ex2;
  double r_5 = 1.0 / (rr2 * rr2 * sqrt(rr2));
  double r_3 = r_5 * rr2;
  r_3 *= charge;
  r_5 *= charge;
  o.put(0, 0, ex0 * r_3);
  o.put(1, 0, ex1 * r_3);
  o.put(2, 0, ex2 * r_3);
  o.put(3, 0, (rr2 - 3 * ex0 * ex0) * r_5);
  o.put(4, 0, (rr2 - 3 * ex1 * ex1) * r_5);
  o.put(5, 0, (rr2 - 3 * ex2 * ex2) * r_5);
  o.put(6, 0, 3 * ex0 * ex1 * r_5);
  o.put(7, 0, 3 * ex0 * ex2 * r_5);
  o.put(8, 0, 3 * ex1 * ex2 * r_5);
  if (lj) {
    double r6 = rr2 * rr2 * rr2;
    double term2 = m.at[k].sig6 / r6;
    double term1 = 2 * term2 * term2;
    double scalarComp = m.at[k].eps24m * (term1 - term2) / rr2;
    o.put(ljk, 0, scalarComp * ex0);
    o.put(ljk + 1, 0, scalarComp * ex1);
    o.put(ljk + 2, 0, scalarComp * ex2);
  }
  w.es++;
  if (!lj) w.nl++;
}

// The acceleration of the serial force functions, by the whole CTA.
template <int TYPE>
__device__ void exact_force(const View &m, const DevParams &p, const double pos[3],
                            double acc[3], const Exact &x, Work &w) {
  constexpr int type = TYPE;
  if (m.uses_clusters) {
    for (int c = threadIdx.x; c < m.nc; c += blockDim.x) {
      double dx0 = pos[0] - m.cl[c].cx, dx1 = pos[1] - m.cl[c].cy, dx2 = pos[2] - m.cl[c].cz;
      double xx = dx0 * dx0, yy = dx1 * dx1, zz = dx2 * dx2;
      double r2 = xx + yy + zz;
      x.cflag[c] = (uint8_t)((r2 > m.cl[c].mpr2 ? 1u : 0u) | (!(r2 > m.cl[c].dr2) ? 2u : 0u));
    }
  }
  __syncthreads();
  // sMat (accumulators 6-8) is decremented by variants 1, 2 and 3
  const uint32_t minus = (type == 1 || type == 2 || type == 3) ? 0x1c0u : 0u;
  const double a = exact_sum(x, m.nslot, x.K, minus, [&](double *T, int j, int e) {
    event_terms<TYPE>(m, p, pos, x, T, j, e, w);
  });
  if (threadIdx.x < x.K) x.accs[threadIdx.x] = a;
  __syncthreads();
  const double *A = x.accs;
  const double ds = p.dipole_scalar;
  if (type == 1 || type == 2) {
    double sumX = A[12], sumY = A[13], sumZ = A[14];
    sumX += ds * (A[3] * A[0] + (A[6] + A[9]) * A[1] + (A[7] + A[10]) * A[2]);
    sumY += ds * ((A[6] - A[9]) * A[0] + A[4] * A[1] + (A[8] + A[11]) * A[2]);
    sumZ += ds * ((A[7] - A[10]) * A[0] + (A[8] - A[11]) * A[1] + A[5] * A[2]);
    acc[0] = sumX; acc[1] = sumY; acc[2] = sumZ;
  } else if (type == 3) {
    double sumX = A[9], sumY = A[10], sumZ = A[11];
    sumX += ds * (A[3] * A[0] + A[6] * A[1] + A[7] * A[2]);
    sumY += ds * (A[6] * A[0] + A[4] * A[1] + A[8] * A[2]);
    sumZ += ds * (A[7] * A[0] + A[8] * A[1] + A[5] * A[2]);
    acc[0] = sumX; acc[1] = sumY; acc[2] = sumZ;
  } else if (type == 4) {
    double tempx = A[0], tempy = A[1], tempz = A[2];
    tempx -= ds * (A[6] * A[3] + A[9] * A[4] + A[10] * A[5]);
    tempy -= ds * (A[9] * A[3] + A[7] * A[4] + A[11] * A[5]);
    tempz -= ds * (A[10] * A[3] + A[11] * A[4] + A[8] * A[5]);
    acc[0] = tempx; acc[1] = tempy; acc[2] = tempz;
  } else {
    acc[0] = A[0]; acc[1] = A[1]; acc[2] = A[2];
  }
  __syncthreads();   // accs are rewritten by the next evaluation
}

// getPotential by the whole CTA: atoms in file order, the serial sums' order.
__device__ double exact_potential(const View &m, const DevParams &p, const double pos[3],
                                  const Exact &x, Work &w) {
  const int K = p.charged ? 4 : 1;
  const double a = exact_sum(x, m.n, K, 0u, [&](double *T, int j, int i) {
    const Col o{T, j, 0};
    const int k = m.uses_clusters ? m.perm[i] : i;
    double xDiff = pos[0] - m.at[k].x, yDiff = pos[1] - m.at[k].y, zDiff = pos[2] - m.at[k].z;
    double r2 = xDiff * xDiff + yDiff * yDiff + zDiff * zDiff;
    double r6 = r2 * r2 * r2;
    double term2 = m.at[k].sig6 / r6;
    double term1 = term2 * term2;
    o.put(0, 0, m.at[k].eps4 * (term1 - term2));
    if (p.charged) {
      double r_3 = m.at[k].q / (r2 * sqrt(r2));
      o.put(1, 0, xDiff * r_3);
      o.put(2, 0, yDiff * r_3);
      o.put(3, 0, zDiff * r_3);
    }
  });
  if (threadIdx.x < K) x.accs[threadIdx.x] = a;
  __syncthreads();
  double total = x.accs[0];
  if (p.charged) {
    const double sumX = x.accs[1], sumY = x.accs[2], sumZ = x.accs[3];
    total -= p.dipole_scalar * 0.5 * (sumX * sumX + sumY * sumY + sumZ * sumZ);
  }
  __syncthreads();
  w.pot += m.n;
  return total;
}

// Take the next parked record; -1 when none is left (the same in every thread).
__device__ __forceinline__ long long exact_take(const Exact &x, const Handoff &ho,
                                                unsigned long long *counters) {
  if (threadIdx.x == 0) {
    long long got = -1;
    unsigned long long tk = atomicAdd(ho.taken, 0ull);
    for (uint32_t it = 0; it < 4096u; ++it) {
      const unsigned long long avail = atomicAdd(ho.reserve, 0ull);
      const unsigned long long lim = avail < (unsigned long long)ho.cap
                                         ? avail : (unsigned long long)ho.cap;
      if (tk >= lim) break;
      const unsigned long long prev = atomicCAS(ho.taken, tk, tk + 1);
      if (prev == tk) { got = (long long)tk; break; }
      tk = prev;
    }
    if (got >= 0) {
      bool ok = false;
      for (uint32_t spin = 0; spin < ho.spin_limit; ++spin) {
        if (atomicAdd(ho.ready + got, 0u) != 0u) { ok = true; break; }
      }
      if (!ok) {
        atomicOr(counters + C_ERROR, 2ull);
        got = -1;
      }
      __threadfence();
    }
    *x.bcast = got;
  }
  __syncthreads();
  const long long idx = *x.bcast;
  __syncthreads();
  return idx;
}

// The CTA finishes parked trajectories: diffEqSolver::verletVel's control
// flow (diffEqSolver.cpp:81-211) from where the thread stopped, with the
// state in every thread's registers (all threads compute the same values).
template <int TYPE>
__device__ void exact_phase(const View &m, const TrajArgs &a, const Exact &x) {
  const DevParams &p = a.par;
  const Handoff &ho = a.ho;
  const long long cap = p.max_steps > 0 ? p.max_steps : kDefaultMaxSteps;
  Work w = {0, 0, 0, 0, 0};
  uint32_t nforce = 0, npot = 0;
  unsigned long long nsteps = 0;
  const unsigned long long t0 = global_ns();
  for (;;) {
    const long long idx = exact_take(x, ho, a.counters);
    if (idx < 0) break;
    const TrajState *R = ho.states + idx;
    double pos[3], vel[3], acc[3], p0[3], v0[3];
    for (int i = 0; i < 3; i++) {
      pos[i] = __ldcg(&R->pos[i]); vel[i] = __ldcg(&R->vel[i]); acc[i] = __ldcg(&R->acc[i]);
      p0[i] = __ldcg(&R->p0[i]); v0[i] = __ldcg(&R->v0[i]);
    }
    double E0 = __ldcg(&R->E0), dt = __ldcg(&R->dt), rdot = __ldcg(&R->rdot);
    double tries = __ldcg(&R->tries), maxTries = __ldcg(&R->max_tries);
    const long long t = __ldcg(&R->t);
    long long total = __ldcg(&R->total);
    int step = __ldcg(&R->step), orbits = __ldcg(&R->orbits), phase = __ldcg(&R->phase);
    unsigned etries = (unsigned)__ldcg(&R->etries), otries = (unsigned)__ldcg(&R->otries);
    for (;;) {
      double ep[3];
      bool needU = false, outside = false;
      if (phase == P_INIT_RETRY) {
        ep[0] = p0[0]; ep[1] = p0[1]; ep[2] = p0[2];
      } else {
        for (int i = 0; i < 3; i++) {
          pos[i] = pos[i] + vel[i] * dt + acc[i] * dt * dt * 0.5;
          vel[i] = vel[i] + acc[i] * dt * 0.5;
        }
        ep[0] = pos[0]; ep[1] = pos[1]; ep[2] = pos[2];
        double t0 = pos[0] / p.ell_a, t1 = pos[1] / p.ell_b, t2 = pos[2] / p.ell_c;
        double mag2 = t0 * t0 + t1 * t1 + t2 * t2;
        outside = (mag2 > 1 && p.projection) || (mag2 > p.max_rad && !p.projection);
        needU = outside && step + 1 > 10;
      }
      double an[3];
      exact_force<TYPE>(m, p, ep, an, x, w);
      double U = 0;
      if (needU) U = exact_potential(m, p, ep, x, w);
      nforce++;
      if (needU) npot++;
      if (phase == P_INIT_RETRY) {
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
        if (orbits > 8) track = false;
      }
      bool finished = false;
      double chi = COSIMS_PI_2, dE = 0.0;
      uint32_t status = COSIMS_TRAJ_HIT;
      if (!track) {
        tries++;
        otries++;
        dt = p.dt / ((tries + 1));
      } else if (outside && step > 10) {
        double endE = U + 0.5 * p.mu * dot3(vel, vel);
        double de = 100 * fabs(E0 - endE) / E0;
        double c = angle3(v0, vel);
        if (de > 0.5) {
          tries++;
          maxTries++;
          etries++;
          dt = p.dt / ((tries + 1));
          step = 0;
        } else {
          chi = c; dE = de;
          status |= COSIMS_TRAJ_SUCCESS;
          finished = true;
        }
      }
      if (!finished) {
        if (total >= cap || !isfinite(rdot)) {
          status |= COSIMS_TRAJ_STEPCAP;
          finished = true;
        } else if (!(tries < maxTries && maxTries < 10)) {
          finished = true;
        } else if (step == 0) {
          phase = P_INIT_RETRY;
        }
      }
      if (finished) {
        if (threadIdx.x == 0) {
          cosims_traj_out o;
          o.chi = chi; o.de_pct = dE; o.steps = step;
          o.status = status | (etries << COSIMS_TRAJ_ETRIES_SHIFT) |
                     (otries << COSIMS_TRAJ_OTRIES_SHIFT);
          a.out[t] = o;
        }
        break;
      }
    }
  }
  unsigned long long *c = a.counters;
  count_add(c, C_PAIR_LJ, w.lj);
  count_add(c, C_PAIR_ES, w.es);
  count_add(c, C_FAR, w.far);
  count_add(c, C_PAIR_ESNL, w.nl);
  if (threadIdx.x == 0) {
    count_add(c, C_STEPS, (long long)nsteps);
    count_add(c, C_FORCE_EVALS, nforce);
    count_add(c, C_POT_EVALS, npot);
    count_add(c, C_PAIR_POT, (long long)npot * m.n);
    count_add(c, C_WIDE_STEPS, (long long)nsteps);
    count_add(c, C_WIDE_NS, (long long)(global_ns() - t0));
  }
}

// CTAs per SM the register allocation is sized for: four 128-thread CTAs
// (128 registers a thread) for the variants whose state and sums fit without
// spills in the pair loop; three for variants 1 and 2 (15 running sums plus
// the far-field terms).  With four CTAs the molecule image is read through L1
// when four staged copies would not fit in shared memory.
template <int TYPE>
struct PlainShape {
#ifdef COSIMS_PLAIN_MIN_BLOCKS
  static constexpr int kMinBlocks = COSIMS_PLAIN_MIN_BLOCKS;
#else
  static constexpr int kMinBlocks = (TYPE == 1 || TYPE == 2) ? 3 : 4;
#endif
};

template <bool TRACE, int TYPE>
__global__ void __launch_bounds__(kPlainBlock, PlainShape<TYPE>::kMinBlocks)
    traj_plain_kernel(const TrajArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ uint64_t bar;
  const unsigned char *base = a.img.gbase;
  if (a.use_smem) {
    if (!stage_to_smem(smem, a.img.gbase, a.img.bytes, &bar, 0, true, a.stage_limit)) {
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
  Work w = {0, 0, 0, 0, 0};
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
    Work wi = {0, 0, 0, 0, 0};
    force<TYPE>(m, p, ep, an, wi);
    double U = 0;
    if (__any_sync(0xffffffffu, needU)) U = potential(m, p, ep);
    if (phase == P_DONE) continue;
    nforce++;
    w.lj += wi.lj; w.es += wi.es; w.far += wi.far; w.nl += wi.nl;
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
    if (TRACE) {                       // only this thread writes trajectory t's frames
      const int32_t k = a.trace_n[t];
      if (k < a.trace_cap) {
        double *f = a.trace + ((size_t)t * (size_t)a.trace_cap + (size_t)k) * 6;
        f[0] = pos[0]; f[1] = pos[1]; f[2] = pos[2];
        f[3] = vel[0]; f[4] = vel[1]; f[5] = vel[2];
      }
      a.trace_n[t] = k + 1;
    }
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
    // a long trajectory goes to the CTA's exact wide phase (a function of the
    // trajectory alone: its own step count; a record per trajectory exists)
    if (!TRACE && (phase == P_STEP || phase == P_INIT_RETRY) && a.ho.budget > 0 &&
        total >= a.ho.budget) {
      const unsigned long long r = atomicAdd(a.ho.reserve, 1ull);
      if (r < (unsigned long long)a.ho.cap) {
        TrajState &R = a.ho.states[r];
        for (int i = 0; i < 3; i++) {
          R.pos[i] = pos[i]; R.vel[i] = vel[i]; R.acc[i] = acc[i]; R.p0[i] = p0[i]; R.v0[i] = v0[i];
        }
        R.E0 = E0; R.dt = dt; R.tries = tries; R.max_tries = maxTries; R.rdot = rdot;
        R.t = t; R.total = total; R.orbits = orbits; R.step = step; R.phase = phase;
        R.etries = (int32_t)etries; R.otries = (int32_t)otries; R.may_handoff = 0;
        __threadfence();
        if (!(a.ho.withhold_first && r == 0)) atomicExch(a.ho.ready + r, 1u);
        phase = P_ACQUIRE;
      }
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
  count_add(c, C_PAIR_ESNL, w.nl);
  if (!TRACE && a.ho.budget > 0) {
    __syncthreads();                    // every thread done: the CTA goes wide
    const Exact x = exact_scratch(smem, a.use_smem ? a.img.bytes : 0u, TYPE, m.nc);
    exact_phase<TYPE>(m, a, x);
  }
  if ((threadIdx.x & 31) == 0) mark_last(c, C_T_END);
}

}  // namespace plain

int plain_max_smem_per_block() {
  int dev = 0, v = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  return v - 1024;   // leave room for the static barrier word
}

template <bool TRACE, int TYPE>
static int plain_launch_t(const TrajArgs &a, int block, int grid, size_t smem, void *stream) {
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(plain::traj_plain_kernel<TRACE, TYPE>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
  }
  plain::traj_plain_kernel<TRACE, TYPE><<<grid, block, smem, (cudaStream_t)stream>>>(a);
  return (int)cudaGetLastError();
}

template <bool TRACE>
static int plain_launch_v(const TrajArgs &a, int block, int grid, size_t smem, void *stream) {
  switch (a.par.force_type) {
    case 1: return plain_launch_t<TRACE, 1>(a, block, grid, smem, stream);
    case 2: return plain_launch_t<TRACE, 2>(a, block, grid, smem, stream);
    case 3: return plain_launch_t<TRACE, 3>(a, block, grid, smem, stream);
    case 4: return plain_launch_t<TRACE, 4>(a, block, grid, smem, stream);
    case 5: return plain_launch_t<TRACE, 5>(a, block, grid, smem, stream);
    default: return plain_launch_t<TRACE, 6>(a, block, grid, smem, stream);
  }
}

int plain_launch(const TrajArgs &a, int block, int grid, size_t smem, void *stream) {
  return a.trace ? plain_launch_v<true>(a, block, grid, smem, stream)
                 : plain_launch_v<false>(a, block, grid, smem, stream);
}

template <int TYPE>
static int plain_occupancy_t(int block, size_t smem, int *per_sm) {
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(plain::traj_plain_kernel<false, TYPE>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
  }
  return (int)cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      per_sm, plain::traj_plain_kernel<false, TYPE>, block, smem);
}

int plain_occupancy(int force_type, int block, size_t smem, int *per_sm) {
  switch (force_type) {
    case 1: return plain_occupancy_t<1>(block, smem, per_sm);
    case 2: return plain_occupancy_t<2>(block, smem, per_sm);
    case 3: return plain_occupancy_t<3>(block, smem, per_sm);
    case 4: return plain_occupancy_t<4>(block, smem, per_sm);
    case 5: return plain_occupancy_t<5>(block, smem, per_sm);
    default: return plain_occupancy_t<6>(block, smem, per_sm);
  }
}

}  // namespace cosims
