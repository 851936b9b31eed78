// traj_mixed.cu -- the mixed-precision form.
//
// Pair forces (Lennard-Jones and the ion-induced-dipole field and field
// gradient) are FP32 on molecule-centred coordinates; the He position enters
// as an FP32 hi/lo pair, so dx = (x_hi - x_atom) + x_lo keeps the separation
// accurate to FP32 precision of dx itself at close approach.  FP64 is kept for
// the position/velocity accumulators of the Verlet step, the cluster near/far
// tests, the energy-conservation check (exact potential, FP64) and the
// scattering angle; the CCS sum uses 2 sin^2(chi/2) for 1 - cos(chi).
//
// G lanes (1..32) work on one trajectory: they split the atoms, reduce the
// accumulators with xor-butterfly shuffles (bitwise identical in every lane),
// and run the integrator redundantly, so the group needs no broadcast.  The
// physics is the reference's (forceAccel.cpp:221-884), including its
// multipoleCutoff far band that takes sigma^6/eps of atom index n
// (forceAccel.cpp:353-355); only the arithmetic precision and the order of the
// sums differ from the plain form.
#include <cuda_runtime.h>
#include "device_util.cuh"

namespace cosims {
namespace mixed {

enum ModeBits : uint8_t { M_ES = 1, M_LJ = 2, M_LJQ = 4 };

struct View {
  const float4 *a4;        // x, y, z, q
  const float2 *lj;        // sigma^6, 24 eps/mu
  const uint16_t *cid;     // cluster of each atom
  const ClusterF32 *cl;
  int n, nc;
};

struct View64 {   // FP64 image in global memory, for the energy check
  const AtomF64 *at;
  int n;
};

__device__ __forceinline__ View make_view(const unsigned char *b, const MolImage &img) {
  View v;
  v.a4 = reinterpret_cast<const float4 *>(b + img.off[S_ATOMS]);
  v.lj = reinterpret_cast<const float2 *>(b + img.off[S_LJ]);
  v.cid = reinterpret_cast<const uint16_t *>(b + img.off[S_CID]);
  v.cl = reinterpret_cast<const ClusterF32 *>(b + img.off[S_CLUSTERS]);
  v.n = img.n_atoms;
  v.nc = img.n_clusters;
  return v;
}

__device__ __forceinline__ View64 make_view64(const MolImage &img) {
  View64 v;
  v.at = reinterpret_cast<const AtomF64 *>(img.gbase + img.off[S_ATOMS]);
  v.n = img.n_atoms;
  return v;
}

struct Acc {
  float Fx, Fy, Fz;                 // Lennard-Jones force sum
  float Ex, Ey, Ez;                 // charge field
  float Pxx, Pxy, Pxz, Pyy, Pyz, Pzz, Q3;   // sum q d d^T / r^5, sum q / r^3
  float Mdx, Mdy, Mdz, Msxy, Msxz, Msyz, Maxy, Maxz, Mayz;  // far-field gradient
};

template <int TYPE>
struct Traits {
  static constexpr bool kClusters = TYPE == 1 || TYPE == 2 || TYPE == 3 || TYPE == 5;
  static constexpr bool kCharge = TYPE <= 4;
  static constexpr bool kFar = TYPE == 1 || TYPE == 2;
  // every atom carries the charge field (types 3, 4): no per-pair branch
  static constexpr bool kEsAlways = TYPE == 3 || TYPE == 4;
};

// Far-field monopole + dipole (+ quadrupole) terms of one cluster, in FP32,
// the reference's far block (forceAccel.cpp:258-337).
__device__ __forceinline__ void far_terms(const View &m, int n, int order, float dx0, float dx1,
                                          float dx2, Acc &s) {
  const float xx = dx0 * dx0, yy = dx1 * dx1, zz = dx2 * dx2;
  const float r2 = xx + yy + zz;
  const float r_2 = 1.0f / r2;
  const float r_1 = rsqrtf(r2);
  const float r_3 = r_2 * r_1;
  const float r_5 = r_3 * r_2;
  const float xy = dx0 * dx1, xz = dx0 * dx2, yz = dx1 * dx2;
  const ClusterF32 &C = m.cl[n];
  const float cR5 = C.q * r_5;
  const float cR3 = cR5 * r2;
  s.Ex += cR3 * dx0; s.Ey += cR3 * dx1; s.Ez += cR3 * dx2;
  s.Mdx += (r2 - 3.f * xx) * cR5; s.Mdy += (r2 - 3.f * yy) * cR5; s.Mdz += (r2 - 3.f * zz) * cR5;
  s.Msxy -= 3.f * xy * cR5; s.Msxz -= 3.f * xz * cR5; s.Msyz -= 3.f * yz * cR5;
  if (order >= 1 && !C.replaced) {
    const float *D = C.dip;
    const float r_7 = r_5 * r_2;
    const float c1 = 3.f * (D[0] * dx0 + D[1] * dx1 + D[2] * dx2);
    s.Ex += (c1 * dx0 - r2 * D[0]) * r_5;
    s.Ey += (c1 * dx1 - r2 * D[1]) * r_5;
    s.Ez += (c1 * dx2 - r2 * D[2]) * r_5;
    s.Mdx += (r2 - 5.f * xx) * r_7 * c1;
    s.Mdy += (r2 - 5.f * yy) * r_7 * c1;
    s.Mdz += (r2 - 5.f * zz) * r_7 * c1;
    s.Msxy -= 5.f * xy * r_7 * c1; s.Msxz -= 5.f * xz * r_7 * c1; s.Msyz -= 5.f * yz * r_7 * c1;
    s.Maxy += 3.f * (D[1] * dx0 - D[0] * dx1) * r_5;
    s.Maxz += 3.f * (D[2] * dx0 - D[0] * dx2) * r_5;
    s.Mayz += 3.f * (D[2] * dx1 - D[1] * dx2) * r_5;
  }
  if (order >= 2) {
    const float *Q = C.quad;
    const float r_7 = r_5 * r_2;
    const float t0 = (Q[0] * dx0 + Q[3] * dx1 + Q[6] * dx2) * r_7;
    const float t1 = (Q[1] * dx0 + Q[4] * dx1 + Q[7] * dx2) * r_7;
    const float t2 = (Q[2] * dx0 + Q[5] * dx1 + Q[8] * dx2) * r_7;
    const float c2 = 5.f * (t0 * dx0 + t1 * dx1 + t2 * dx2) * r_2 * 0.5f;
    s.Ex += (c2 * dx0 - t0) * r2; s.Ey += (c2 * dx1 - t1) * r2; s.Ez += (c2 * dx2 - t2) * r2;
    s.Mdx += (r2 - 7.f * xx) * c2 - Q[0] * r_5;
    s.Mdy += (r2 - 7.f * yy) * c2 - Q[4] * r_5;
    s.Mdz += (r2 - 7.f * zz) * c2 - Q[8] * r_5;
    s.Msxy -= 7.f * xy * c2 + Q[1] * r_5;
    s.Msxz -= 7.f * xz * c2 + Q[2] * r_5;
    s.Msyz -= 7.f * yz * c2 + Q[5] * r_5;
    s.Maxy += 5.f * (t1 * dx0 - t0 * dx1);
    s.Maxz += 5.f * (t2 * dx0 - t0 * dx2);
    s.Mayz += 5.f * (t2 * dx1 - t1 * dx2);
  }
}

// One atom pair, FP32.  mode selects the field terms and which LJ parameters;
// mode 0 (an idle lane or an atom outside every cut-off) contributes nothing.
// The LJ term is branch-free (a zero prefactor switches it off), so two calls
// in a row interleave; the field terms branch only for the multipole variants.
template <int TYPE>
__device__ __forceinline__ void pair(const View &m, int k, uint32_t mode, float hx, float hy,
                                     float hz, float lx, float ly, float lz, Acc &s) {
  const bool act = mode != 0u;
  const int kk = act ? k : 0;
  const float4 a = m.a4[kk];
  float2 lj = m.lj[kk];
  if (TYPE == 1 && (mode & M_LJQ)) {
    const ClusterF32 &C = m.cl[m.cid[kk]];
    lj = make_float2(C.qsig6, C.qeps);
  }
  const float eps = (mode & (M_LJ | M_LJQ)) ? lj.y : 0.0f;
  const float dx = act ? (hx - a.x) + lx : 1.0e3f;
  const float dy = act ? (hy - a.y) + ly : 1.0e3f;
  const float dz = act ? (hz - a.z) + lz : 1.0e3f;
  const float r2 = dx * dx + dy * dy + dz * dz;
  const float ir = rsqrtf(r2);
  const float ir2 = ir * ir;
  const float s6 = lj.x * (ir2 * ir2 * ir2);
  const float f = eps * ir2 * s6 * (2.0f * s6 - 1.0f);
  s.Fx += f * dx; s.Fy += f * dy; s.Fz += f * dz;
  if (Traits<TYPE>::kCharge && (Traits<TYPE>::kEsAlways || (mode & M_ES))) {
    const float q = (Traits<TYPE>::kEsAlways && !(mode & M_ES)) ? 0.0f : a.w;
    const float q3 = q * ir * ir2;
    const float q5 = q3 * ir2;
    s.Ex += q3 * dx; s.Ey += q3 * dy; s.Ez += q3 * dz;
    s.Q3 += q3;
    const float wx = q5 * dx, wy = q5 * dy;
    s.Pxx += wx * dx; s.Pxy += wx * dy; s.Pxz += wx * dz;
    s.Pyy += wy * dy; s.Pyz += wy * dz; s.Pzz += q5 * dz * dz;
  }
}

struct WorkM { uint32_t lj, es, far; };

// Acceleration at pos (FP64 in, FP64 out) for one group of G lanes.
template <int TYPE>
__device__ void force(const View &m, const DevParams &p, const double pos[3], double acc[3],
                      int G, int lane, uint8_t *modes, WorkM &w) {
  Acc s = {};
  const float hx = (float)pos[0], hy = (float)pos[1], hz = (float)pos[2];
  const float lx = (float)(pos[0] - (double)hx), ly = (float)(pos[1] - (double)hy),
              lz = (float)(pos[2] - (double)hz);
  if (Traits<TYPE>::kClusters) {
    // pass 1: near/far decision per cluster (FP64), far-field terms
    for (int c = lane; c < m.nc; c += G) {
      const ClusterF32 &C = m.cl[c];
      const double d0 = pos[0] - C.cx, d1 = pos[1] - C.cy, d2 = pos[2] - C.cz;
      const double r2 = d0 * d0 + d1 * d1 + d2 * d2;
      const bool in_disp = !(r2 > C.dr2);
      uint8_t mode;
      if (TYPE == 5) {
        mode = in_disp ? M_LJ : 0;
      } else if (TYPE == 3) {
        mode = M_ES | (in_disp ? M_LJ : 0);
      } else {
        if (r2 > C.mpr2) {
          far_terms(m, c, p.multipole_order, (float)d0, (float)d1, (float)d2, s);
          w.far++;
          mode = TYPE == 2 ? M_LJ : (in_disp ? M_LJQ : 0);
        } else {
          mode = M_ES | ((TYPE == 2 || in_disp) ? M_LJ : 0);
        }
      }
      modes[c] = mode;
    }
    __syncwarp();
    // pass 2: atoms, 2G at a time (two independent pairs per lane); the trip
    // count is the same for every lane of the warp
    for (int base = 0; base < m.n; base += 2 * G) {
      const int k0 = base + lane, k1 = k0 + G;
      const uint32_t m0 = k0 < m.n ? modes[m.cid[k0]] : 0u;
      const uint32_t m1 = k1 < m.n ? modes[m.cid[k1]] : 0u;
      pair<TYPE>(m, k0, m0, hx, hy, hz, lx, ly, lz, s);
      pair<TYPE>(m, k1, m1, hx, hy, hz, lx, ly, lz, s);
      w.es += ((m0 & M_ES) != 0) + ((m1 & M_ES) != 0);
      w.lj += (m0 && !(m0 & M_ES)) + (m1 && !(m1 & M_ES));
    }
    __syncwarp();
  } else {
    constexpr uint32_t mode = TYPE == 4 ? (M_ES | M_LJ) : M_LJ;
    for (int base = 0; base < m.n; base += 2 * G) {
      const int k0 = base + lane, k1 = k0 + G;
      pair<TYPE>(m, k0, k0 < m.n ? mode : 0u, hx, hy, hz, lx, ly, lz, s);
      pair<TYPE>(m, k1, k1 < m.n ? mode : 0u, hx, hy, hz, lx, ly, lz, s);
    }
    const uint32_t mine = lane < m.n ? (uint32_t)((m.n - 1 - lane) / G + 1) : 0u;
    if (TYPE == 4) w.es += mine; else w.lj += mine;
  }
  // group reduction (identical result in every lane of the group)
  s.Fx = group_sum(s.Fx, G); s.Fy = group_sum(s.Fy, G); s.Fz = group_sum(s.Fz, G);
  acc[0] = s.Fx; acc[1] = s.Fy; acc[2] = s.Fz;
  if (Traits<TYPE>::kCharge) {
    s.Ex = group_sum(s.Ex, G); s.Ey = group_sum(s.Ey, G); s.Ez = group_sum(s.Ez, G);
    s.Pxx = group_sum(s.Pxx, G); s.Pxy = group_sum(s.Pxy, G); s.Pxz = group_sum(s.Pxz, G);
    s.Pyy = group_sum(s.Pyy, G); s.Pyz = group_sum(s.Pyz, G); s.Pzz = group_sum(s.Pzz, G);
    s.Q3 = group_sum(s.Q3, G);
    double Mxx = (double)s.Q3 - 3.0 * s.Pxx, Myy = (double)s.Q3 - 3.0 * s.Pyy,
           Mzz = (double)s.Q3 - 3.0 * s.Pzz;
    double Sxy = -3.0 * s.Pxy, Sxz = -3.0 * s.Pxz, Syz = -3.0 * s.Pyz;
    double Axy = 0, Axz = 0, Ayz = 0;
    if (Traits<TYPE>::kFar) {
      s.Mdx = group_sum(s.Mdx, G); s.Mdy = group_sum(s.Mdy, G); s.Mdz = group_sum(s.Mdz, G);
      s.Msxy = group_sum(s.Msxy, G); s.Msxz = group_sum(s.Msxz, G); s.Msyz = group_sum(s.Msyz, G);
      s.Maxy = group_sum(s.Maxy, G); s.Maxz = group_sum(s.Maxz, G); s.Mayz = group_sum(s.Mayz, G);
      Mxx += s.Mdx; Myy += s.Mdy; Mzz += s.Mdz;
      Sxy += s.Msxy; Sxz += s.Msxz; Syz += s.Msyz;
      Axy = s.Maxy; Axz = s.Maxz; Ayz = s.Mayz;
    }
    const double Ex = s.Ex, Ey = s.Ey, Ez = s.Ez, ds = p.dipole_scalar;
    acc[0] += ds * (Mxx * Ex + (Sxy + Axy) * Ey + (Sxz + Axz) * Ez);
    acc[1] += ds * ((Sxy - Axy) * Ex + Myy * Ey + (Syz + Ayz) * Ez);
    acc[2] += ds * ((Sxz - Axz) * Ex + (Syz - Ayz) * Ey + Mzz * Ez);
  }
}

// Exact potential in FP64 (forceAccel.cpp:943-982), lanes split the atoms.
__device__ double potential(const View64 &m, const DevParams &p, const double pos[3], int G,
                            int lane) {
  double total = 0, sX = 0, sY = 0, sZ = 0;
  for (int k = lane; k < m.n; k += G) {
    const double *A = reinterpret_cast<const double *>(m.at + k);
    const double dx = pos[0] - __ldg(A + 0), dy = pos[1] - __ldg(A + 1),
                 dz = pos[2] - __ldg(A + 2);
    const double r2 = dx * dx + dy * dy + dz * dz;
    const double r6 = r2 * r2 * r2;
    const double term2 = __ldg(A + 4) / r6;
    total += __ldg(A + 6) * (term2 * term2 - term2);
    if (p.charged) {
      const double r_3 = __ldg(A + 3) / (r2 * sqrt(r2));
      sX += dx * r_3; sY += dy * r_3; sZ += dz * r_3;
    }
  }
  total = group_sum(total, G);
  if (p.charged) {
    sX = group_sum(sX, G); sY = group_sum(sY, G); sZ = group_sum(sZ, G);
    total -= p.dipole_scalar * 0.5 * (sX * sX + sY * sY + sZ * sZ);
  }
  return total;
}

__device__ __forceinline__ double dot3(const double a[3], const double b[3]) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

__device__ __forceinline__ double angle3(const double a[3], const double b[3]) {
  double term1 = dot3(a, b);
  double term2 = sqrt(dot3(a, a)) * sqrt(dot3(b, b));
  double term3 = term1 / term2;
  if (term3 > 1) return 0;
  if (term3 < -1) return COSIMS_PI;
  return acos(term3);
}

enum Phase : int { P_ACQUIRE = 0, P_INIT_FIRST, P_INIT_RETRY, P_STEP, P_DONE };

// Work counters of one thread, flushed to the device counters at kernel end.
struct Tally {
  uint32_t lj = 0, es = 0, far = 0, nforce = 0, npot = 0, npotpairs = 0;
  unsigned long long nsteps = 0;
};

// Pair counters are per lane; step and evaluation counters are kept by each
// group's lane 0 only, so a plain sum over threads is right for any G.
__device__ __forceinline__ void flush_tally(const Tally &tl, unsigned long long *c) {
  count_add(c, C_PAIR_LJ, tl.lj);
  count_add(c, C_PAIR_ES, tl.es);
  count_add(c, C_FAR, tl.far);
  count_add(c, C_STEPS, (long long)tl.nsteps);
  count_add(c, C_FORCE_EVALS, tl.nforce);
  count_add(c, C_POT_EVALS, tl.npot);
  count_add(c, C_PAIR_POT, tl.npotpairs);
}

// The trajectory loop of one group of G lanes (every warp of the CTA calls it
// together).  Groups take queue slots 0..n-1 from `queue` (global or shared
// memory); slot k integrates trajectory order[k] (k without an order), whose
// start state is pos0/vel0[3t..3t+2] and whose record goes to out[t]; a
// trajectory with hit[t] == 0 is an ellipsoid miss.  Every iteration
// evaluates one acceleration per group (at the start state or after a
// position update) and, when any group of the warp needs it, one potential;
// a group whose trajectory ends takes the next slot at once.
template <int TYPE>
__device__ __forceinline__ void group_loop(const View &m, const View64 &m64, const DevParams &p,
                                           int G, uint8_t *modes, const double *pos0,
                                           const double *vel0, const int32_t *hit,
                                           const int32_t *order, long long n,
                                           cosims_traj_out *out, unsigned long long *queue,
                                           Tally &tl) {
  const int lane = threadIdx.x & (G - 1);
  const unsigned gmask = G == 32 ? 0xffffffffu
                                 : (((1u << G) - 1u) << ((threadIdx.x & 31) & ~(G - 1)));
  const long long cap = p.max_steps > 0 ? p.max_steps : kDefaultMaxSteps;

  double p0[3] = {0, 0, 0}, v0[3] = {0, 0, 0}, pos[3] = {0, 0, 0}, vel[3] = {0, 0, 0},
         acc[3] = {0, 0, 0};
  double E0 = 0, dt = p.dt, tries = 0, maxTries = 8, rdot = 0;
  int orbits = 0, step = 0, phase = P_ACQUIRE;
  long long total = 0, t = 0;
  unsigned etries = 0, otries = 0;

  auto finish = [&](double chi, double de, int steps, uint32_t status) {
    if (lane == 0) {
      cosims_traj_out o;
      o.chi = chi; o.de_pct = de; o.steps = steps;
      o.status = status | (etries << COSIMS_TRAJ_ETRIES_SHIFT) |
                 (otries << COSIMS_TRAJ_OTRIES_SHIFT);
      out[t] = o;
    }
    phase = P_ACQUIRE;
  };

  while (true) {
    if (phase == P_ACQUIRE) {
      for (;;) {
        long long tk = 0;
        if (lane == 0) tk = (long long)atomicAdd(queue, 1ull);
        t = __shfl_sync(gmask, tk, 0, G);
        if (t >= n) { phase = P_DONE; break; }
        if (order) t = order[t];
        if (hit && !hit[t]) {                 // ellipsoid miss: chi = 0
          if (lane == 0) {
            cosims_traj_out o = {0.0, 0.0, 0, 0u};
            out[t] = o;
          }
          continue;
        }
        for (int i = 0; i < 3; i++) { p0[i] = pos0[3 * t + i]; v0[i] = vel0[3 * t + i]; }
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
      const double t0 = pos[0] / p.ell_a, t1 = pos[1] / p.ell_b, t2 = pos[2] / p.ell_c;
      const double mag2 = t0 * t0 + t1 * t1 + t2 * t2;
      outside = (mag2 > 1 && p.projection) || (mag2 > p.max_rad && !p.projection);
      needU = outside && step + 1 > 10;
    } else {
      ep[0] = 1.0e4; ep[1] = 0.0; ep[2] = 0.0;
    }

    double an[3];
    WorkM wi = {0, 0, 0};
    force<TYPE>(m, p, ep, an, G, lane, modes, wi);
    double U = 0;
    if (__any_sync(0xffffffffu, needU)) U = potential(m64, p, ep, G, lane);
    if (phase == P_DONE) continue;
    const uint32_t lead = lane == 0 ? 1u : 0u;
    tl.nforce += lead;
    tl.lj += wi.lj; tl.es += wi.es; tl.far += wi.far;
    if (needU) { tl.npot += lead; tl.npotpairs += lead * (uint32_t)m64.n; }

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
    tl.nsteps += lead;
    bool track = true;
    const double rold = rdot;
    rdot = dot3(pos, vel);
    if (step > 2 && rdot * rold < 0 && !(rdot > rold)) {
      orbits++;
      if (orbits > 8) track = false;
    }
    if (!track) {
      tries++;
      otries++;
      dt = p.dt / (tries + 1);
    } else if (outside && step > 10) {
      const double endE = U + 0.5 * p.mu * dot3(vel, vel);
      const double dE = 100 * fabs(E0 - endE) / E0;
      const double chi = angle3(v0, vel);
      if (dE > 0.5) {
        tries++;
        maxTries++;
        etries++;
        dt = p.dt / (tries + 1);
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
}

template <int TYPE>
__global__ void __launch_bounds__(256) traj_mixed_kernel(const TrajArgs a) {
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
  const View m = make_view(base, a.img);
  const View64 m64 = make_view64(a.img64);
  const int G = a.group_lanes;
  uint8_t *modes =
      smem + (a.use_smem ? a.img.bytes : 0) + (size_t)(threadIdx.x / G) * a.mode_stride;
  Tally tl;
  group_loop<TYPE>(m, m64, a.par, G, modes, a.pos0, a.vel0, a.hit, a.order, a.n, a.out,
                   a.queue, tl);
  flush_tally(tl, a.counters);
}

// ---- batched form: one persistent launch over many molecules ------------------
// CTAs take work items (a molecule and a range of its trajectories) from a
// device queue.  When an item's molecule differs from the one staged, the CTA
// waits for its groups, then bulk-copies the new image into shared memory
// (molecules over the launch's shared-memory budget are read through L1/L2).
// Groups then take the item's trajectories from a shared-memory counter.
template <int TYPE>
__device__ __forceinline__ void batch_item(const BatchMol &bm, const unsigned char *base,
                                           uint8_t *modes_base, const BatchArgs &a,
                                           const BatchItem &it, unsigned long long *q,
                                           Tally &tl) {
  const View m = make_view(base, bm.img32);
  const View64 m64 = make_view64(bm.img64);
  const int G = bm.group_lanes;
  uint8_t *modes = modes_base + (size_t)(threadIdx.x / G) * bm.mode_stride;
  const long long b = bm.base + it.t0;
  group_loop<TYPE>(m, m64, bm.par, G, modes, a.pos0 + 3 * b, a.vel0 + 3 * b, a.hit + b,
                   nullptr, it.t1 - it.t0, a.out + b, q, tl);
}

__global__ void __launch_bounds__(256) batch_mixed_kernel(const BatchArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ uint64_t bar;
  __shared__ BatchMol cur;
  __shared__ int s_item, s_mol;
  __shared__ unsigned long long s_queue;
  if (threadIdx.x == 0) s_mol = -1;
  uint32_t stagings = 0;
  Tally tl;
  for (;;) {
    if (threadIdx.x == 0) s_item = (int)atomicAdd(a.item_queue, 1ull);
    __syncthreads();
    const int item = s_item;
    if (item >= a.n_items) break;
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
    const unsigned char *base = cur.use_smem ? smem : cur.img32.gbase;
    uint8_t *modes = smem + (cur.use_smem ? cur.img32.bytes : 0);
    switch (cur.type) {
      case 1: batch_item<1>(cur, base, modes, a, it, &s_queue, tl); break;
      case 2: batch_item<2>(cur, base, modes, a, it, &s_queue, tl); break;
      case 3: batch_item<3>(cur, base, modes, a, it, &s_queue, tl); break;
      case 4: batch_item<4>(cur, base, modes, a, it, &s_queue, tl); break;
      case 5: batch_item<5>(cur, base, modes, a, it, &s_queue, tl); break;
      default: batch_item<6>(cur, base, modes, a, it, &s_queue, tl); break;
    }
    __syncthreads();   // every group is done with the item before a restage
  }
  flush_tally(tl, a.counters);
}

template <int TYPE>
int launch_t(const TrajArgs &a, int block, int grid, size_t smem, void *stream) {
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(traj_mixed_kernel<TYPE>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
  }
  traj_mixed_kernel<TYPE><<<grid, block, smem, (cudaStream_t)stream>>>(a);
  return (int)cudaGetLastError();
}

}  // namespace mixed

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
    case 1: return mixed::launch_t<1>(a, block, grid, smem, stream);
    case 2: return mixed::launch_t<2>(a, block, grid, smem, stream);
    case 3: return mixed::launch_t<3>(a, block, grid, smem, stream);
    case 4: return mixed::launch_t<4>(a, block, grid, smem, stream);
    case 5: return mixed::launch_t<5>(a, block, grid, smem, stream);
    default: return mixed::launch_t<6>(a, block, grid, smem, stream);
  }
}

}  // namespace cosims

namespace cosims {
namespace mixed {
template <int TYPE>
int occupancy_t(int block, size_t smem, int *per_sm) {
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(traj_mixed_kernel<TYPE>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
  }
  return (int)cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, traj_mixed_kernel<TYPE>,
                                                            block, smem);
}
}  // namespace mixed

int mixed_occupancy(int force_type, int block, size_t smem, int *per_sm) {
  switch (force_type) {
    case 1: return mixed::occupancy_t<1>(block, smem, per_sm);
    case 2: return mixed::occupancy_t<2>(block, smem, per_sm);
    case 3: return mixed::occupancy_t<3>(block, smem, per_sm);
    case 4: return mixed::occupancy_t<4>(block, smem, per_sm);
    case 5: return mixed::occupancy_t<5>(block, smem, per_sm);
    default: return mixed::occupancy_t<6>(block, smem, per_sm);
  }
}
}  // namespace cosims
