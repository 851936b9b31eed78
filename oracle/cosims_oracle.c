/*
 * cosims_oracle.c -- TEST INFRASTRUCTURE ONLY: the oracle.
 *
 * A plain-C restatement of the CoSIMS trajectory path.  Every function cites
 * the reference lines it follows.  Arithmetic is IEEE double, no FMA
 * contraction (-ffp-contract=off), and each expression keeps the reference's
 * evaluation order, so that for the same inputs the results agree bit for bit
 * with the reference compiled by g++ on x86-64 (SSE2, no FMA).  That claim is
 * checked against oracle/_ref (the reference's own code) by
 * tests/test_oracle_golden.py through the tests/golden fixtures.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use
 * this file, as the checker.  The product never calls it.
 */
#include <math.h>
#include <string.h>
#include "cosims_oracle.h"

#define ORACLE_PI 3.14159265358979323846      /* vector3D.h:24 */
#define ORACLE_PI_2 1.57079632679489661923    /* vector3D.h:25 */

/* ---- forces ------------------------------------------------------------ */

/* multipoleCutoff (type 1, forceAccel.cpp:221-445) and multipoleOnly
 * (type 2, forceAccel.cpp:447-633).  They share the far-field block; they
 * differ in the atom loop of far clusters: type 1 applies the dispersion
 * cut-off and takes sigma^6 / eps from atom index n (the cluster index,
 * forceAccel.cpp:353-355), type 2 uses each atom's own parameters for every
 * atom (forceAccel.cpp:563-582). */
static void force_multipole(const cosims_molecule *m, const cosims_params *p,
                            const double pos[3], double acc[3], int cutoff)
{
    double fieldX = 0, fieldY = 0, fieldZ = 0;
    double sMatXY = 0, sMatXZ = 0, sMatYZ = 0, aMatXY = 0, aMatXZ = 0, aMatYZ = 0;
    double diagMatXX = 0, diagMatYY = 0, diagMatZZ = 0;
    double sumX = 0, sumY = 0, sumZ = 0;
    const int order = p->multipole_order;
    for (int n = 0; n < m->n_clusters; n++) {
        const double *cp = m->cluster_pos + 3 * n;
        double dx[3];
        dx[0] = pos[0] - cp[0];
        dx[1] = pos[1] - cp[1];
        dx[2] = pos[2] - cp[2];
        double xx = dx[0] * dx[0], yy = dx[1] * dx[1], zz = dx[2] * dx[2];
        double r2 = xx + yy + zz;
        double multiPlusRad = p->r_mp + m->cluster_radius[n];
        multiPlusRad *= multiPlusRad;
        double dispPlusRad = p->r_disp + m->cluster_radius[n];
        dispPlusRad *= dispPlusRad;
        const int a0 = m->cluster_offset[n], a1 = m->cluster_offset[n + 1];
        const int replaced = m->cluster_replaced[n];
        const double *D = m->cluster_dipole + 3 * n;
        const double *Q = m->cluster_quad + 9 * n; /* Q[3*i+j] = quadPole[n][i][j] */

        if (r2 > multiPlusRad) {
            double r_2 = 1.0 / r2;
            double r_1 = 1.0 / sqrt(r2);
            double r_3 = r_2 * r_1;
            double r_5 = r_3 * r_2;
            double r_7 = 0, const1 = 0, const2 = 0, tMat2[3] = {0, 0, 0};
            double xy = dx[0] * dx[1], xz = dx[0] * dx[2], yz = dx[1] * dx[2];
            double chargeR_5 = m->cluster_charge[n] * r_5;
            double chargeR_3 = chargeR_5 * r2;
            if (order >= 1 && !replaced) {
                r_7 = r_5 * r_2;
                const1 = 3 * (D[0] * dx[0] + D[1] * dx[1] + D[2] * dx[2]);
            }
            if (order >= 2) {
                r_7 = r_5 * r_2;
                tMat2[0] = (Q[0] * dx[0] + Q[3] * dx[1] + Q[6] * dx[2]) * r_7;
                tMat2[1] = (Q[1] * dx[0] + Q[4] * dx[1] + Q[7] * dx[2]) * r_7;
                tMat2[2] = (Q[2] * dx[0] + Q[5] * dx[1] + Q[8] * dx[2]) * r_7;
                const2 = 5 * (tMat2[0] * dx[0] + tMat2[1] * dx[1] + tMat2[2] * dx[2]) * r_2 * 0.5;
            }
            fieldX += chargeR_3 * dx[0];
            fieldY += chargeR_3 * dx[1];
            fieldZ += chargeR_3 * dx[2];
            diagMatXX += (r2 - 3 * xx) * chargeR_5;
            diagMatYY += (r2 - 3 * yy) * chargeR_5;
            diagMatZZ += (r2 - 3 * zz) * chargeR_5;
            sMatXY -= 3 * xy * chargeR_5;
            sMatXZ -= 3 * xz * chargeR_5;
            sMatYZ -= 3 * yz * chargeR_5;
            if (order >= 1 && !replaced) {
                fieldX += (const1 * dx[0] - r2 * D[0]) * r_5;
                fieldY += (const1 * dx[1] - r2 * D[1]) * r_5;
                fieldZ += (const1 * dx[2] - r2 * D[2]) * r_5;
                diagMatXX += (r2 - 5 * xx) * r_7 * const1;
                diagMatYY += (r2 - 5 * yy) * r_7 * const1;
                diagMatZZ += (r2 - 5 * zz) * r_7 * const1;
                sMatXY -= 5 * xy * r_7 * const1;
                sMatXZ -= 5 * xz * r_7 * const1;
                sMatYZ -= 5 * yz * r_7 * const1;
                aMatXY += 3 * (D[1] * dx[0] - D[0] * dx[1]) * r_5;
                aMatXZ += 3 * (D[2] * dx[0] - D[0] * dx[2]) * r_5;
                aMatYZ += 3 * (D[2] * dx[1] - D[1] * dx[2]) * r_5;
            }
            if (order >= 2) {
                fieldX += (const2 * dx[0] - tMat2[0]) * r2;
                fieldY += (const2 * dx[1] - tMat2[1]) * r2;
                fieldZ += (const2 * dx[2] - tMat2[2]) * r2;
                diagMatXX += ((r2 - 7 * xx) * const2 - Q[0] * r_5);
                diagMatYY += ((r2 - 7 * yy) * const2 - Q[4] * r_5);
                diagMatZZ += ((r2 - 7 * zz) * const2 - Q[8] * r_5);
                sMatXY -= (7 * xy * const2 + Q[1] * r_5);
                sMatXZ -= (7 * xz * const2 + Q[2] * r_5);
                sMatYZ -= (7 * yz * const2 + Q[5] * r_5);
                aMatXY += 5 * (tMat2[1] * dx[0] - tMat2[0] * dx[1]);
                aMatXZ += 5 * (tMat2[2] * dx[0] - tMat2[0] * dx[2]);
                aMatYZ += 5 * (tMat2[2] * dx[1] - tMat2[1] * dx[2]);
            }
            if (!cutoff || !(r2 > dispPlusRad)) {
                /* type 1: parameters of atom n (the cluster index); type 2: own */
                for (int k = a0; k < a1; k++) {
                    int index = m->cluster_atoms[k];
                    int pi = cutoff ? n : index;
                    dx[0] = pos[0] - m->x[index];
                    dx[1] = pos[1] - m->y[index];
                    dx[2] = pos[2] - m->z[index];
                    double rr2 = dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2];
                    double r6 = rr2 * rr2 * rr2;
                    double term2 = m->sig6[pi] / r6;
                    double term1 = 2 * term2 * term2;
                    double scalarComp = m->eps24m[pi] * (term1 - term2) / rr2;
                    sumX += scalarComp * dx[0];
                    sumY += scalarComp * dx[1];
                    sumZ += scalarComp * dx[2];
                }
            }
        } else {
            const int lj = (!cutoff) || !(r2 > dispPlusRad);
            for (int k = a0; k < a1; k++) {
                int index = m->cluster_atoms[k];
                double charge = m->charge[index];
                dx[0] = pos[0] - m->x[index];
                dx[1] = pos[1] - m->y[index];
                dx[2] = pos[2] - m->z[index];
                double rr2 = dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2];
                double r_5 = 1.0 / (rr2 * rr2 * sqrt(rr2));
                double r_3 = r_5 * rr2;
                r_3 *= charge;
                r_5 *= charge;
                fieldX += dx[0] * r_3;
                fieldY += dx[1] * r_3;
                fieldZ += dx[2] * r_3;
                diagMatXX += (rr2 - 3 * dx[0] * dx[0]) * r_5;
                diagMatYY += (rr2 - 3 * dx[1] * dx[1]) * r_5;
                diagMatZZ += (rr2 - 3 * dx[2] * dx[2]) * r_5;
                sMatXY -= 3 * dx[0] * dx[1] * r_5;
                sMatXZ -= 3 * dx[0] * dx[2] * r_5;
                sMatYZ -= 3 * dx[1] * dx[2] * r_5;
                if (lj) {
                    double r6 = rr2 * rr2 * rr2;
                    double term2 = m->sig6[index] / r6;
                    double term1 = 2 * term2 * term2;
                    double scalarComp = m->eps24m[index] * (term1 - term2) / rr2;
                    sumX += scalarComp * dx[0];
                    sumY += scalarComp * dx[1];
                    sumZ += scalarComp * dx[2];
                }
            }
        }
    }
    const double ds = p->dipole_scalar;
    sumX += ds * (diagMatXX * fieldX + (sMatXY + aMatXY) * fieldY + (sMatXZ + aMatXZ) * fieldZ);
    sumY += ds * ((sMatXY - aMatXY) * fieldX + diagMatYY * fieldY + (sMatYZ + aMatYZ) * fieldZ);
    sumZ += ds * ((sMatXZ - aMatXZ) * fieldX + (sMatYZ - aMatYZ) * fieldY + diagMatZZ * fieldZ);
    acc[0] = sumX; acc[1] = sumY; acc[2] = sumZ;
}

/* dispersionOnly (type 3, forceAccel.cpp:635-749): exact electrostatics for
 * every atom, LJ only inside the cluster cut-off. */
static void force_dispersion_only(const cosims_molecule *m, const cosims_params *p,
                                  const double pos[3], double acc[3])
{
    double fieldX = 0, fieldY = 0, fieldZ = 0;
    double sMatXY = 0, sMatXZ = 0, sMatYZ = 0;
    double diagMatXX = 0, diagMatYY = 0, diagMatZZ = 0;
    double sumX = 0, sumY = 0, sumZ = 0;
    for (int n = 0; n < m->n_clusters; n++) {
        const double *cp = m->cluster_pos + 3 * n;
        double dx[3];
        dx[0] = pos[0] - cp[0];
        dx[1] = pos[1] - cp[1];
        dx[2] = pos[2] - cp[2];
        double xx = dx[0] * dx[0], yy = dx[1] * dx[1], zz = dx[2] * dx[2];
        double r2 = xx + yy + zz;
        double dispPlusRad = p->r_disp + m->cluster_radius[n];
        dispPlusRad *= dispPlusRad;
        const int lj = !(r2 > dispPlusRad);
        for (int k = m->cluster_offset[n]; k < m->cluster_offset[n + 1]; k++) {
            int index = m->cluster_atoms[k];
            double charge = m->charge[index];
            dx[0] = pos[0] - m->x[index];
            dx[1] = pos[1] - m->y[index];
            dx[2] = pos[2] - m->z[index];
            double rr2 = dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2];
            double r_5 = 1.0 / (rr2 * rr2 * sqrt(rr2));
            double r_3 = r_5 * rr2;
            r_3 *= charge;
            r_5 *= charge;
            fieldX += dx[0] * r_3;
            fieldY += dx[1] * r_3;
            fieldZ += dx[2] * r_3;
            diagMatXX += (rr2 - 3 * dx[0] * dx[0]) * r_5;
            diagMatYY += (rr2 - 3 * dx[1] * dx[1]) * r_5;
            diagMatZZ += (rr2 - 3 * dx[2] * dx[2]) * r_5;
            sMatXY -= 3 * dx[0] * dx[1] * r_5;
            sMatXZ -= 3 * dx[0] * dx[2] * r_5;
            sMatYZ -= 3 * dx[1] * dx[2] * r_5;
            if (lj) {
                double r6 = rr2 * rr2 * rr2;
                double term2 = m->sig6[index] / r6;
                double term1 = 2 * term2 * term2;
                double scalarComp = m->eps24m[index] * (term1 - term2) / rr2;
                sumX += scalarComp * dx[0];
                sumY += scalarComp * dx[1];
                sumZ += scalarComp * dx[2];
            }
        }
    }
    const double ds = p->dipole_scalar;
    sumX += ds * (diagMatXX * fieldX + sMatXY * fieldY + sMatXZ * fieldZ);
    sumY += ds * (sMatXY * fieldX + diagMatYY * fieldY + sMatYZ * fieldZ);
    sumZ += ds * (sMatXZ * fieldX + sMatYZ * fieldY + diagMatZZ * fieldZ);
    acc[0] = sumX; acc[1] = sumY; acc[2] = sumZ;
}

/* chargeDipoleLJ (type 4, forceAccel.cpp:751-805). */
static void force_charge_dipole_lj(const cosims_molecule *m, const cosims_params *p,
                                   const double pos[3], double acc[3])
{
    double sumXX = 0, sumYY = 0, sumZZ = 0, sumXY = 0, sumXZ = 0, sumYZ = 0;
    double dipX = 0, dipY = 0, dipZ = 0, tempx = 0, tempy = 0, tempz = 0;
    for (int n = 0; n < m->n_atoms; n++) {
        double xDiff = pos[0] - m->x[n];
        double yDiff = pos[1] - m->y[n];
        double zDiff = pos[2] - m->z[n];
        double xDiff2 = xDiff * xDiff, yDiff2 = yDiff * yDiff, zDiff2 = zDiff * zDiff;
        double r2 = xDiff2 + yDiff2 + zDiff2;
        double r = sqrt(r2);
        double r3 = r2 * r;
        double r_3 = 1.0 / r3;
        double r_5 = r_3 / r2;
        double r6 = r2 * r2 * r2;
        r_3 *= m->charge[n];
        r_5 *= m->charge[n];
        double term2 = m->sig6[n] / r6;
        double term1 = 2 * term2 * term2;
        double scalarComp = m->eps24m[n] * (term1 - term2) / r2;
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
    const double ds = p->dipole_scalar;
    tempx -= ds * (sumXX * dipX + sumXY * dipY + sumXZ * dipZ);
    tempy -= ds * (sumXY * dipX + sumYY * dipY + sumYZ * dipZ);
    tempz -= ds * (sumXZ * dipX + sumYZ * dipY + sumZZ * dipZ);
    acc[0] = tempx; acc[1] = tempy; acc[2] = tempz;
}

/* dispersionNoCharge (type 5, forceAccel.cpp:807-854). */
static void force_dispersion_nocharge(const cosims_molecule *m, const cosims_params *p,
                                      const double pos[3], double acc[3])
{
    double sumX = 0, sumY = 0, sumZ = 0;
    for (int n = 0; n < m->n_clusters; n++) {
        const double *cp = m->cluster_pos + 3 * n;
        double dx[3];
        dx[0] = pos[0] - cp[0];
        dx[1] = pos[1] - cp[1];
        dx[2] = pos[2] - cp[2];
        double xx = dx[0] * dx[0], yy = dx[1] * dx[1], zz = dx[2] * dx[2];
        double r2 = xx + yy + zz;
        double dispPlusRad = p->r_disp + m->cluster_radius[n];
        dispPlusRad *= dispPlusRad;
        if (!(r2 > dispPlusRad)) {
            for (int k = m->cluster_offset[n]; k < m->cluster_offset[n + 1]; k++) {
                int index = m->cluster_atoms[k];
                dx[0] = pos[0] - m->x[index];
                dx[1] = pos[1] - m->y[index];
                dx[2] = pos[2] - m->z[index];
                double rr2 = dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2];
                double r6 = rr2 * rr2 * rr2;
                double term2 = m->sig6[index] / r6;
                double term1 = 2 * term2 * term2;
                double scalarComp = m->eps24m[index] * (term1 - term2) / rr2;
                sumX += scalarComp * dx[0];
                sumY += scalarComp * dx[1];
                sumZ += scalarComp * dx[2];
            }
        }
    }
    acc[0] = sumX; acc[1] = sumY; acc[2] = sumZ;
}

/* dispersionFull (type 6, forceAccel.cpp:856-884). */
static void force_dispersion_full(const cosims_molecule *m, const double pos[3],
                                  double acc[3])
{
    double tempx = 0, tempy = 0, tempz = 0;
    for (int n = 0; n < m->n_atoms; n++) {
        double xDiff = pos[0] - m->x[n];
        double yDiff = pos[1] - m->y[n];
        double zDiff = pos[2] - m->z[n];
        double xDiff2 = xDiff * xDiff, yDiff2 = yDiff * yDiff, zDiff2 = zDiff * zDiff;
        double r2 = xDiff2 + yDiff2 + zDiff2;
        double r6 = r2 * r2 * r2;
        double term2 = m->sig6[n] / r6;
        double term1 = 2 * term2 * term2;
        double scalarComp = m->eps24m[n] * (term1 - term2) / r2;
        tempx += scalarComp * xDiff;
        tempy += scalarComp * yDiff;
        tempz += scalarComp * zDiff;
    }
    acc[0] = tempx; acc[1] = tempy; acc[2] = tempz;
}

/* getReducedVec dispatch (forceAccel.cpp:887-908). */
void oracle_force(const cosims_molecule *mol, const cosims_params *par,
                  const double pos[3], double acc[3])
{
    switch (par->force_type) {
    case 1: force_multipole(mol, par, pos, acc, 1); break;
    case 2: force_multipole(mol, par, pos, acc, 0); break;
    case 3: force_dispersion_only(mol, par, pos, acc); break;
    case 4: force_charge_dipole_lj(mol, par, pos, acc); break;
    case 5: force_dispersion_nocharge(mol, par, pos, acc); break;
    default: force_dispersion_full(mol, pos, acc); break;
    }
}

/* getPotential (forceAccel.cpp:943-982).  The induced-dipole term uses
 * dipoleScalar, which already carries 1/mu (forceAccel.cpp:35, :977). */
double oracle_potential(const cosims_molecule *m, const cosims_params *p,
                        const double pos[3])
{
    double total = 0, sumX = 0, sumY = 0, sumZ = 0;
    for (int n = 0; n < m->n_atoms; n++) {
        double xDiff = pos[0] - m->x[n];
        double yDiff = pos[1] - m->y[n];
        double zDiff = pos[2] - m->z[n];
        double r2 = xDiff * xDiff + yDiff * yDiff + zDiff * zDiff;
        double r6 = r2 * r2 * r2;
        double term2 = m->sig6[n] / r6;
        double term1 = term2 * term2;
        total += m->eps4[n] * (term1 - term2);
        if (p->charged) {
            double r_3 = m->charge[n] / (r2 * sqrt(r2));
            sumX += xDiff * r_3;
            sumY += yDiff * r_3;
            sumZ += zDiff * r_3;
        }
    }
    if (p->charged) total -= p->dipole_scalar * 0.5 * (sumX * sumX + sumY * sumY + sumZ * sumZ);
    return total;
}

/* ---- integrator -------------------------------------------------------- */

static double dot3(const double a[3], const double b[3])
{
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];       /* vector3D.h:168-171 */
}

/* vector3D::Angle (vector3D.h:134-143). */
static double angle3(const double a[3], const double b[3])
{
    double term1 = dot3(a, b);
    double term2 = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]) *
                   sqrt(b[0] * b[0] + b[1] * b[1] + b[2] * b[2]);
    double term3 = term1 / term2;
    if (term3 > 1) return 0;
    else if (term3 < -1) return ORACLE_PI;
    return acos(term1 / term2);
}

/* diffEqSolver::verletVel (diffEqSolver.cpp:81-211).  Besides chi, the
 * return value and stepCount it reports the retry counts and stops at
 * par->max_steps (default 2^18) or when the state turns non-finite; the
 * reference has neither stop (it would loop), and no trajectory it finishes
 * comes near the cap. */
static void verlet(const cosims_molecule *mol, const cosims_params *par,
                   const double initPos[3], const double initVel[3],
                   cosims_traj_out *out, double *frames, int32_t fcap, int32_t *nframes)
{
    const double a = par->ell_a, b = par->ell_b, c = par->ell_c;
    const double maxRad = fmax(a, fmax(b, c));
    const double time = par->dt;
    const int64_t cap = par->max_steps > 0 ? par->max_steps : ((int64_t)1 << 18);
    double maxTries = 8, trajTries = 0;
    double dt = time;
    double rDot_new = 0, rDot_old = 0, orbits = 0;
    double pos[3], vel[3], acc[3];
    int stepCount = 0;
    int64_t total_steps = 0;
    unsigned etries = 0, otries = 0;
    double startEnergy = oracle_potential(mol, par, initPos) + 0.5 * par->mu * dot3(initVel, initVel);
    out->de_pct = 0;
    while (trajTries < maxTries && maxTries < 10) {
        if (stepCount == 0) {
            oracle_force(mol, par, initPos, acc);
            memcpy(pos, initPos, sizeof pos);
            memcpy(vel, initVel, sizeof vel);
            rDot_old = 0;
            rDot_new = 0;
            orbits = 0;
            rDot_new = dot3(pos, vel);
        }
        for (int i = 0; i < 3; i++) {
            pos[i] = pos[i] + vel[i] * dt + acc[i] * dt * dt * 0.5;
            vel[i] = vel[i] + acc[i] * dt * 0.5;
        }
        oracle_force(mol, par, pos, acc);
        for (int i = 0; i < 3; i++) vel[i] = vel[i] + acc[i] * dt * 0.5;
        stepCount++;
        total_steps++;
        if (nframes) {                 /* per-step record of position and velocity */
            if (*nframes < fcap) {
                double *f = frames + (size_t)*nframes * 6;
                for (int i = 0; i < 3; i++) { f[i] = pos[i]; f[3 + i] = vel[i]; }
            }
            (*nframes)++;
        }

        int track = 1;
        rDot_old = rDot_new;
        rDot_new = dot3(pos, vel);
        double product = rDot_new * rDot_old;
        if (stepCount > 2 && product < 0 && !(rDot_new > rDot_old)) {
            orbits++;
            if (orbits > 8) track = 0;   /* maxOrbits = 8, diffEqSolver.cpp:40 */
        }
        if (!track) {
            trajTries++;
            otries++;
            dt = time / ((trajTries + 1));
        } else {
            double t0 = pos[0] / a, t1 = pos[1] / b, t2 = pos[2] / c;
            double mag2 = t0 * t0 + t1 * t1 + t2 * t2;
            if (((mag2 > 1 && par->projection) || (mag2 > maxRad && !par->projection)) &&
                stepCount > 10) {
                double endEnergy = oracle_potential(mol, par, pos) + 0.5 * par->mu * dot3(vel, vel);
                double energyPctDiff = 100 * fabs(startEnergy - endEnergy) / startEnergy;
                out->chi = angle3(initVel, vel);
                out->steps = stepCount;
                if (energyPctDiff > 0.5) {
                    trajTries++;
                    maxTries++;
                    etries++;
                    dt = time / ((trajTries + 1));
                    stepCount = 0;
                } else {
                    out->de_pct = energyPctDiff;
                    out->status = COSIMS_TRAJ_HIT | COSIMS_TRAJ_SUCCESS |
                                  (etries << COSIMS_TRAJ_ETRIES_SHIFT) |
                                  (otries << COSIMS_TRAJ_OTRIES_SHIFT);
                    return;
                }
            }
        }
        if (total_steps >= cap || !isfinite(rDot_new)) {
            out->chi = ORACLE_PI_2;
            out->steps = stepCount;
            out->status = COSIMS_TRAJ_HIT | COSIMS_TRAJ_STEPCAP |
                          (etries << COSIMS_TRAJ_ETRIES_SHIFT) |
                          (otries << COSIMS_TRAJ_OTRIES_SHIFT);
            return;
        }
    }
    out->chi = ORACLE_PI_2;
    out->steps = stepCount;
    out->status = COSIMS_TRAJ_HIT | (etries << COSIMS_TRAJ_ETRIES_SHIFT) |
                  (otries << COSIMS_TRAJ_OTRIES_SHIFT);
}

void oracle_verlet(const cosims_molecule *mol, const cosims_params *par,
                   const double initPos[3], const double initVel[3], cosims_traj_out *out)
{
    verlet(mol, par, initPos, initVel, out, NULL, 0, NULL);
}

void oracle_verlet_trace(const cosims_molecule *mol, const cosims_params *par,
                         const double initPos[3], const double initVel[3],
                         cosims_traj_out *out, double *frames, int32_t fcap, int32_t *nframes)
{
    *nframes = 0;
    verlet(mol, par, initPos, initVel, out, frames, fcap, nframes);
}

/* ---- start states and accumulation ------------------------------------- */

/* monteTraj::setUpTraj geometry (monteTraj.cpp:235-242) and ellipsoid
 * projection (monteTraj.cpp:254-269); start_dist is the float maxDist. */
int oracle_start_state(const cosims_params *par, const cosims_traj_in *in,
                       double pos0[3], double vel0[3])
{
    const double b = in->b, phi = in->phi, theta = in->theta, gamma = in->gamma, g = in->g;
    const double maxDist = par->start_dist;
    double tp[3], tv[3];
    tp[0] = b * cos(gamma) * cos(phi) * cos(theta) - b * sin(gamma) * sin(phi) + maxDist * cos(phi) * sin(theta);
    tp[1] = b * cos(gamma) * sin(phi) * cos(theta) + b * sin(gamma) * cos(phi) + maxDist * sin(phi) * sin(theta);
    tp[2] = maxDist * cos(theta) - b * cos(gamma) * sin(theta);
    tv[0] = -g * cos(phi) * sin(theta);
    tv[1] = -g * sin(phi) * sin(theta);
    tv[2] = -g * cos(theta);
    if (par->projection) {
        double v[3] = {tv[0] / par->ell_a, tv[1] / par->ell_b, tv[2] / par->ell_c};
        double p[3] = {tp[0] / par->ell_a, tp[1] / par->ell_b, tp[2] / par->ell_c};
        double cr[3];
        cr[0] = (p[1] * v[2]) - (p[2] * v[1]);
        cr[1] = (p[2] * v[0]) - (p[0] * v[2]);
        cr[2] = (p[0] * v[1]) - (p[1] * v[0]);
        double discrim = -dot3(cr, cr) + dot3(v, v);
        if (discrim < 0) return 0;
        double positParam = -(dot3(p, v) / (dot3(v, v))) - sqrt(discrim) / dot3(v, v);
        for (int i = 0; i < 3; i++) tp[i] = tp[i] + tv[i] * positParam;
    }
    memcpy(pos0, tp, sizeof tp);
    memcpy(vel0, tv, sizeof tv);
    return 1;
}

void oracle_run_list(const cosims_molecule *mol, const cosims_params *par, int64_t n,
                     const double *pos0, const double *vel0, cosims_traj_out *out)
{
    for (int64_t i = 0; i < n; i++) {
        memset(&out[i], 0, sizeof out[i]);
        oracle_verlet(mol, par, pos0 + 3 * i, vel0 + 3 * i, &out[i]);
    }
}

void oracle_run_inputs(const cosims_molecule *mol, const cosims_params *par, int64_t n,
                       const cosims_traj_in *in, cosims_traj_out *out)
{
    for (int64_t i = 0; i < n; i++) {
        double p0[3], v0[3];
        memset(&out[i], 0, sizeof out[i]);
        if (oracle_start_state(par, &in[i], p0, v0))
            oracle_verlet(mol, par, p0, v0, &out[i]);
        else
            out[i].chi = 0;   /* monteTraj.cpp:366-367 */
    }
}

/* runThreads (monteTraj.cpp:456-502) + updateCounts (:504-521) with one
 * thread: succTraj keeps its previous value on an ellipsoid miss
 * (monteTraj.cpp:326-367), and the final success count only subtracts the
 * failures since the last progress update (monteTraj.cpp:380, :511). */
void oracle_reduce(const cosims_params *par, int64_t n, const cosims_traj_out *out,
                   int64_t update_every, cosims_ccs_sums *s)
{
    memset(s, 0, sizeof *s);
    int succTraj = 0;
    int64_t orbitCount = 0;
    for (int64_t i = 0; i < n; i++) {
        double chi;
        if (out[i].status & COSIMS_TRAJ_HIT) {
            succTraj = (out[i].status & COSIMS_TRAJ_SUCCESS) ? 1 : 0;
            chi = out[i].chi;
            s->n_hit++;
            if (succTraj) {
                s->n_success++;
                if (out[i].de_pct > s->max_de_pct) s->max_de_pct = out[i].de_pct;
            }
        } else {
            chi = 0;
        }
        if (!succTraj) orbitCount++;
        double dOmega = 1.0 * (1 - cos(fabs(chi)));     /* pow(g, 5 - 5) = 1 */
        double tmpTotal = par->ccs_const * dOmega;
        s->sum += tmpTotal;
        s->sum2 += tmpTotal * tmpTotal;
        if (update_every > 0 && (i + 1) % update_every == 0) orbitCount = 0;
    }
    s->n = n;
    s->n_eff = n - orbitCount;
}

void oracle_omega(const cosims_ccs_sums *s, double *omega, double *err)
{
    double total = s->sum, total2 = s->sum2, currSuccTraj = (double)s->n_eff;
    *omega = total / currSuccTraj;
    *err = sqrt((total2 / currSuccTraj - (total / currSuccTraj) * (total / currSuccTraj)) /
                currSuccTraj);
}
