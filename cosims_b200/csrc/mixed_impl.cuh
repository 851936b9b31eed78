// mixed_impl.cuh -- the mixed-precision form (device code shared by the
// per-variant compilation units traj_mixed_t<N>.cu and traj_mixed.cu).
//
// Pair forces (Lennard-Jones and the ion-induced-dipole field and field
// gradient) are FP32 on molecule-centred coordinates; the He position enters
// as an FP32 hi/lo pair, so dx = (x_hi - x_atom) + x_lo keeps the separation
// accurate to FP32 precision of dx itself at close approach.  FP64 is kept for
// the position/velocity accumulators of the Verlet step, the cluster near/far
// tests, the energy-conservation check (the potential in FP64) and the
// scattering angle; the CCS sum uses 2 sin^2(chi/2) for 1 - cos(chi).
//
// G lanes (1..32) work on one trajectory: they split the atoms, two pairs per
// packed FP32 instruction, reduce the accumulators with shuffles
// (reduce-scatter plus broadcast for 16 and 32 lanes, xor butterfly
// otherwise; bitwise identical in every lane), and run the integrator
// redundantly, so the group needs no further broadcast.  The
// physics is the reference's (forceAccel.cpp:221-884), including its
// multipoleCutoff far band that takes sigma^6/eps of atom index n
// (forceAccel.cpp:353-355); only the arithmetic precision and the order of the
// sums differ from the plain form.
#pragma once
#include <cuda_runtime.h>
#include "device_util.cuh"

namespace cosims {
namespace mixed {

enum ModeBits : uint8_t { M_ES = 1, M_LJ = 2, M_LJQ = 4 };

struct View {
  const float4 *a4;        // x, y, z, q
  const float4 *b4;        // sigma^6, 24 eps/mu, cluster id (integer bits), 0
  // pair-interleaved layout (variants 3, 4, 6): slot pair j = atoms 2j, 2j+1
  const float4 *px;        // x0, x1, y0, y1
  const float4 *pz;        // z0, z1, q0, q1
  const float4 *pl;        // sigma^6 0, sigma^6 1, 24 eps/mu 0, 24 eps/mu 1
  const uint2 *pc;         // cluster ids
  const ClusterF32 *cl;
  const float4 *ft;        // far-field table (variants 1, 2): clusters 2j, 2j+1 per entry j
  int n, nc, nslots;        // atoms, clusters, padded atom slots
  int nfp;                  // far-field table pairs (a multiple of 32)
};

struct View64 {   // FP64 image in global memory, for the energy check
  const AtomF64 *at;
  int n;
};

__device__ __forceinline__ View make_view(const unsigned char *b, const MolImage &img) {
  View v;
  v.a4 = reinterpret_cast<const float4 *>(b + img.off[S_ATOMS]);
  v.b4 = reinterpret_cast<const float4 *>(b + img.off[S_LJ]);
  const int np = img.n_slots / 2;
  v.px = reinterpret_cast<const float4 *>(b + img.off[S_PAIRS]);
  v.pz = v.px + np;
  v.pl = v.pz + np;
  v.pc = reinterpret_cast<const uint2 *>(v.pl + np);
  v.cl = reinterpret_cast<const ClusterF32 *>(b + img.off[S_CLUSTERS]);
  v.ft = reinterpret_cast<const float4 *>(b + img.off[S_FAR]);
  v.n = img.n_atoms;
  v.nc = img.n_clusters;
  v.nslots = img.n_slots;
  v.nfp = far_table_pairs(img.n_clusters);
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
  // pair terms per evaluation depend on the position (far clusters, cut-off
  // without a charge field); for 3, 4 and 6 they are n_atoms every time
  static constexpr bool kVaryingPairs = TYPE == 1 || TYPE == 2 || TYPE == 5;
  // the per-cluster decision is one bit (the LJ cut-off) and every atom adds
  // a charge field, so all slots are evaluated with a register cut-off mask
  static constexpr bool kMaskable = TYPE == 3;
  // clusters with nothing to add are common (far field, cut-off): pass 2
  // walks a list of the clusters that add something
  static constexpr bool kListed = TYPE == 1 || TYPE == 2 || TYPE == 5;
  static constexpr bool kCharge = TYPE <= 4;
  static constexpr bool kFar = TYPE == 1 || TYPE == 2;
  // every atom carries the charge field (types 3, 4): no per-pair branch
  static constexpr bool kEsAlways = TYPE == 3 || TYPE == 4;
};

// rsqrt.approx without the denormal handling of rsqrtf(): a pair distance is
// never below an Angstrom squared, and pad atoms sit at 1e6 Angstrom.
__device__ __forceinline__ float rsqrt_ftz(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Far-field monopole + dipole (+ quadrupole) terms of one cluster, in FP32,
// the reference's far block (forceAccel.cpp:258-337).
__device__ __forceinline__ void far_terms(const View &m, int n, int order, float dx0, float dx1,
                                          float dx2, Acc &s) {
  const float xx = dx0 * dx0, yy = dx1 * dx1, zz = dx2 * dx2;
  const float r2 = xx + yy + zz;
  // far clusters lie beyond the multipole radius: r2 is large and normal
  const float r_1 = rsqrt_ftz(r2);
  const float r_2 = r_1 * r_1;
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


__device__ __forceinline__ uint32_t cluster_of(const float4 &b) { return __float_as_uint(b.z); }

// One atom pair, FP32, from the atom's two records.  mode selects the field
// terms and which LJ parameters; mode 0 (a pad atom, or an atom outside every
// cut-off) adds nothing to the LJ sum.  Pad atoms are inert (q = sigma^6 =
// eps = 0), so every slot is evaluated without a bounds test.  The LJ term is
// branch-free (a zero prefactor switches it off), so two calls in a row
// interleave; the field terms branch only for the multipole variants.
template <int TYPE>
__device__ __forceinline__ void pair(const View &m, const float4 &a, const float4 &b,
                                     uint32_t mode, float hx, float hy, float hz, float lx,
                                     float ly, float lz, Acc &s,
                                     const ClusterF32 *own = nullptr) {
  // own: the slot's cluster when the caller has it (its band parameters then
  // load once per cluster rather than per pair)
  float sig6 = b.x, eps24 = b.y;
  if (TYPE == 1 && (mode & M_LJQ)) {
    const ClusterF32 &C = own ? *own : m.cl[cluster_of(b)];
    sig6 = C.qsig6;
    eps24 = C.qeps;
  }
  const float eps = (TYPE == 4 || TYPE == 6 || (mode & (M_LJ | M_LJQ))) ? eps24 : 0.0f;
  const float dx = (hx - a.x) + lx;
  const float dy = (hy - a.y) + ly;
  const float dz = (hz - a.z) + lz;
  const float r2 = dx * dx + dy * dy + dz * dz;
  const float ir = rsqrt_ftz(r2);
  const float ir2 = ir * ir;
  const float s6 = sig6 * (ir2 * ir2 * ir2);
  const float f = eps * ir2 * s6 * (2.0f * s6 - 1.0f);
  s.Fx += f * dx; s.Fy += f * dy; s.Fz += f * dz;
  if (Traits<TYPE>::kCharge && (Traits<TYPE>::kEsAlways || (mode & M_ES))) {
    const float q3 = a.w * ir * ir2;
    const float q5 = q3 * ir2;
    s.Ex += q3 * dx; s.Ey += q3 * dy; s.Ez += q3 * dz;
    s.Q3 += q3;
    const float wx = q5 * dx, wy = q5 * dy;
    s.Pxx += wx * dx; s.Pxy += wx * dy; s.Pxz += wx * dz;
    s.Pyy += wy * dy; s.Pyz += wy * dz; s.Pzz += q5 * dz * dz;
  }
}

// Two atom pairs at once in Blackwell's packed FP32 instructions (FADD2,
// FMUL2, FFMA2: one issue slot for two FP32 operations): component .x is the
// first pair, .y the second, each summed into its own half of the packed
// accumulators (folded at the end of the evaluation).  The caller passes the
// LJ parameters (sigma^6 and the prefactor, 0 outside the cut-off) and whether
// the pairs add the charge field (the same for both).
struct Acc2 {
  float2 Fx, Fy, Fz, Ex, Ey, Ez, Pxx, Pxy, Pxz, Pyy, Pyz, Pzz, Q3;
};

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

template <int TYPE>
__device__ __forceinline__ void pair2v(const float2 &ax, const float2 &ay, const float2 &az,
                                       const float2 &aq, const float2 &sig6, const float2 &eps,
                                       bool es, const float2 &hx, const float2 &hy,
                                       const float2 &hz, const float2 &lx, const float2 &ly,
                                       const float2 &lz, Acc2 &s) {
  const float2 neg = f2(-1.0f, -1.0f);
  // (h - a) + l: the FMA with -1 is the exact difference rounded once
  const float2 dx = __fadd2_rn(__ffma2_rn(ax, neg, hx), lx);
  const float2 dy = __fadd2_rn(__ffma2_rn(ay, neg, hy), ly);
  const float2 dz = __fadd2_rn(__ffma2_rn(az, neg, hz), lz);
  const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
  const float2 ir = f2(rsqrt_ftz(r2.x), rsqrt_ftz(r2.y));
  const float2 ir2 = __fmul2_rn(ir, ir);
  const float2 s6 = __fmul2_rn(sig6, __fmul2_rn(__fmul2_rn(ir2, ir2), ir2));
  const float2 f = __fmul2_rn(__fmul2_rn(eps, ir2),
                              __fmul2_rn(s6, __ffma2_rn(f2(2.0f, 2.0f), s6, neg)));
  s.Fx = __ffma2_rn(f, dx, s.Fx);
  s.Fy = __ffma2_rn(f, dy, s.Fy);
  s.Fz = __ffma2_rn(f, dz, s.Fz);
  if (Traits<TYPE>::kCharge && (Traits<TYPE>::kEsAlways || es)) {
    const float2 q3 = __fmul2_rn(__fmul2_rn(aq, ir), ir2);
    const float2 q5 = __fmul2_rn(q3, ir2);
    s.Ex = __ffma2_rn(q3, dx, s.Ex);
    s.Ey = __ffma2_rn(q3, dy, s.Ey);
    s.Ez = __ffma2_rn(q3, dz, s.Ez);
    s.Q3 = __fadd2_rn(s.Q3, q3);
    const float2 wx = __fmul2_rn(q5, dx), wy = __fmul2_rn(q5, dy), wz = __fmul2_rn(q5, dz);
    s.Pxx = __ffma2_rn(wx, dx, s.Pxx);
    s.Pxy = __ffma2_rn(wx, dy, s.Pxy);
    s.Pxz = __ffma2_rn(wx, dz, s.Pxz);
    s.Pyy = __ffma2_rn(wy, dy, s.Pyy);
    s.Pyz = __ffma2_rn(wy, dz, s.Pyz);
    s.Pzz = __ffma2_rn(wz, dz, s.Pzz);
  }
}

// Two slots from the (x, y, z, q) records of the a4 layout.
template <int TYPE>
__device__ __forceinline__ void pair2(const float4 &a0, const float4 &a1, const float2 &sig6,
                                      const float2 &eps, bool es, const float2 &hx,
                                      const float2 &hy, const float2 &hz, const float2 &lx,
                                      const float2 &ly, const float2 &lz, Acc2 &s) {
  pair2v<TYPE>(f2(a0.x, a1.x), f2(a0.y, a1.y), f2(a0.z, a1.z), f2(a0.w, a1.w), sig6, eps, es,
               hx, hy, hz, lx, ly, lz, s);
}

// Slot pair j of the pair-interleaved layout; eps holds the prefactors the
// cut-off leaves (0 outside it).
template <int TYPE>
__device__ __forceinline__ void pair2j(const View &m, int j, const float2 &eps, bool es,
                                       const float2 &hx, const float2 &hy, const float2 &hz,
                                       const float2 &lx, const float2 &ly, const float2 &lz,
                                       Acc2 &s) {
  const float4 X = m.px[j], Z = m.pz[j], L = m.pl[j];
  pair2v<TYPE>(f2(X.x, X.y), f2(X.z, X.w), f2(Z.x, Z.y), f2(Z.z, Z.w), f2(L.x, L.y), eps, es,
               hx, hy, hz, lx, ly, lz, s);
}

// LJ parameters of a slot under its cluster mode (pair's selection): the
// band parameters of the cluster for variant 1's M_LJQ, 0 outside every cut-off.
template <int TYPE>
__device__ __forceinline__ float2 lj_params(const View &m, const float4 &b, uint32_t mode) {
  if (TYPE == 1 && (mode & M_LJQ)) {
    const ClusterF32 &C = m.cl[cluster_of(b)];
    return f2(C.qsig6, C.qeps);
  }
  return f2(b.x, (TYPE == 4 || TYPE == 6 || (mode & (M_LJ | M_LJQ))) ? b.y : 0.0f);
}

// Fold the packed halves into the scalar accumulators.
template <int TYPE>
__device__ __forceinline__ void fold(const Acc2 &t, Acc &s) {
  s.Fx += t.Fx.x + t.Fx.y; s.Fy += t.Fy.x + t.Fy.y; s.Fz += t.Fz.x + t.Fz.y;
  if (Traits<TYPE>::kCharge) {
    s.Ex += t.Ex.x + t.Ex.y; s.Ey += t.Ey.x + t.Ey.y; s.Ez += t.Ez.x + t.Ez.y;
    s.Pxx += t.Pxx.x + t.Pxx.y; s.Pxy += t.Pxy.x + t.Pxy.y; s.Pxz += t.Pxz.x + t.Pxz.y;
    s.Pyy += t.Pyy.x + t.Pyy.y; s.Pyz += t.Pyz.x + t.Pyz.y; s.Pzz += t.Pzz.x + t.Pzz.y;
    s.Q3 += t.Q3.x + t.Q3.y;
  }
}

// Far-field sums of the packed far pass (one cluster per half).
struct Far2 {
  float2 Ex, Ey, Ez, Mdx, Mdy, Mdz, Msxy, Msxz, Msyz, Maxy, Maxz, Mayz;
};

__device__ __forceinline__ float2 neg2(const float2 &a) { return f2(-a.x, -a.y); }
// far_terms for two clusters at once, one per half of the packed
// instructions (forceAccel.cpp:258-337), from the two clusters' separations,
// their squares, r2 and 1/r, charges, dipoles and (order 2) quadrupoles.
// Replaced clusters carry a zero dipole.  Every term carries a power of 1/r,
// so a half whose 1/r is 0 adds exactly 0 (with finite separations), and a
// null entry (zero moments) adds exactly 0 at any finite distance.
__device__ __forceinline__ void far2_core(int order, const float2 &dx, const float2 &dy,
                                          const float2 &dz, const float2 &xx, const float2 &yy,
                                          const float2 &zz, const float2 &r2, const float2 &r_1,
                                          const float2 &q, const float2 &D0, const float2 &D1,
                                          const float2 &D2, const float *QA, const float *QB,
                                          Far2 &s) {
  const float2 r_2 = __fmul2_rn(r_1, r_1);
  const float2 r_3 = __fmul2_rn(r_2, r_1);
  const float2 r_5 = __fmul2_rn(r_3, r_2);
  const float2 xy = __fmul2_rn(dx, dy), xz = __fmul2_rn(dx, dz), yz = __fmul2_rn(dy, dz);
  const float2 cR5 = __fmul2_rn(q, r_5);
  const float2 cR3 = __fmul2_rn(cR5, r2);
  const float2 m3 = f2(-3.0f, -3.0f);
  s.Ex = __ffma2_rn(cR3, dx, s.Ex);
  s.Ey = __ffma2_rn(cR3, dy, s.Ey);
  s.Ez = __ffma2_rn(cR3, dz, s.Ez);
  s.Mdx = __ffma2_rn(__ffma2_rn(m3, xx, r2), cR5, s.Mdx);
  s.Mdy = __ffma2_rn(__ffma2_rn(m3, yy, r2), cR5, s.Mdy);
  s.Mdz = __ffma2_rn(__ffma2_rn(m3, zz, r2), cR5, s.Mdz);
  s.Msxy = __ffma2_rn(__fmul2_rn(m3, xy), cR5, s.Msxy);
  s.Msxz = __ffma2_rn(__fmul2_rn(m3, xz), cR5, s.Msxz);
  s.Msyz = __ffma2_rn(__fmul2_rn(m3, yz), cR5, s.Msyz);
  if (order >= 1) {
    const float2 r_7 = __fmul2_rn(r_5, r_2);
    const float2 c1 = __fmul2_rn(f2(3.0f, 3.0f),
                                 __ffma2_rn(D2, dz, __ffma2_rn(D1, dy, __fmul2_rn(D0, dx))));
    const float2 nr2 = neg2(r2);
    s.Ex = __ffma2_rn(__ffma2_rn(c1, dx, __fmul2_rn(nr2, D0)), r_5, s.Ex);
    s.Ey = __ffma2_rn(__ffma2_rn(c1, dy, __fmul2_rn(nr2, D1)), r_5, s.Ey);
    s.Ez = __ffma2_rn(__ffma2_rn(c1, dz, __fmul2_rn(nr2, D2)), r_5, s.Ez);
    const float2 r7c1 = __fmul2_rn(r_7, c1);
    const float2 m5 = f2(-5.0f, -5.0f);
    s.Mdx = __ffma2_rn(__ffma2_rn(m5, xx, r2), r7c1, s.Mdx);
    s.Mdy = __ffma2_rn(__ffma2_rn(m5, yy, r2), r7c1, s.Mdy);
    s.Mdz = __ffma2_rn(__ffma2_rn(m5, zz, r2), r7c1, s.Mdz);
    s.Msxy = __ffma2_rn(__fmul2_rn(m5, xy), r7c1, s.Msxy);
    s.Msxz = __ffma2_rn(__fmul2_rn(m5, xz), r7c1, s.Msxz);
    s.Msyz = __ffma2_rn(__fmul2_rn(m5, yz), r7c1, s.Msyz);
    const float2 r5_3 = __fmul2_rn(f2(3.0f, 3.0f), r_5);
    s.Maxy = __ffma2_rn(__ffma2_rn(D1, dx, __fmul2_rn(neg2(D0), dy)), r5_3, s.Maxy);
    s.Maxz = __ffma2_rn(__ffma2_rn(D2, dx, __fmul2_rn(neg2(D0), dz)), r5_3, s.Maxz);
    s.Mayz = __ffma2_rn(__ffma2_rn(D2, dy, __fmul2_rn(neg2(D1), dz)), r5_3, s.Mayz);
  }
  if (order >= 2) {
    const float2 r_7 = __fmul2_rn(r_5, r_2);
    const float2 t0 = __fmul2_rn(__ffma2_rn(f2(QA[6], QB[6]), dz,
                                  __ffma2_rn(f2(QA[3], QB[3]), dy, __fmul2_rn(f2(QA[0], QB[0]), dx))), r_7);
    const float2 t1 = __fmul2_rn(__ffma2_rn(f2(QA[7], QB[7]), dz,
                                  __ffma2_rn(f2(QA[4], QB[4]), dy, __fmul2_rn(f2(QA[1], QB[1]), dx))), r_7);
    const float2 t2 = __fmul2_rn(__ffma2_rn(f2(QA[8], QB[8]), dz,
                                  __ffma2_rn(f2(QA[5], QB[5]), dy, __fmul2_rn(f2(QA[2], QB[2]), dx))), r_7);
    const float2 c2 = __fmul2_rn(__fmul2_rn(f2(2.5f, 2.5f),
                                            __ffma2_rn(t2, dz, __ffma2_rn(t1, dy, __fmul2_rn(t0, dx)))),
                                 r_2);
    s.Ex = __ffma2_rn(__ffma2_rn(c2, dx, neg2(t0)), r2, s.Ex);
    s.Ey = __ffma2_rn(__ffma2_rn(c2, dy, neg2(t1)), r2, s.Ey);
    s.Ez = __ffma2_rn(__ffma2_rn(c2, dz, neg2(t2)), r2, s.Ez);
    const float2 m7 = f2(-7.0f, -7.0f);
    s.Mdx = __ffma2_rn(__ffma2_rn(m7, xx, r2), c2, __ffma2_rn(neg2(f2(QA[0], QB[0])), r_5, s.Mdx));
    s.Mdy = __ffma2_rn(__ffma2_rn(m7, yy, r2), c2, __ffma2_rn(neg2(f2(QA[4], QB[4])), r_5, s.Mdy));
    s.Mdz = __ffma2_rn(__ffma2_rn(m7, zz, r2), c2, __ffma2_rn(neg2(f2(QA[8], QB[8])), r_5, s.Mdz));
    s.Msxy = __ffma2_rn(__fmul2_rn(m7, xy), c2, __ffma2_rn(neg2(f2(QA[1], QB[1])), r_5, s.Msxy));
    s.Msxz = __ffma2_rn(__fmul2_rn(m7, xz), c2, __ffma2_rn(neg2(f2(QA[2], QB[2])), r_5, s.Msxz));
    s.Msyz = __ffma2_rn(__fmul2_rn(m7, yz), c2, __ffma2_rn(neg2(f2(QA[5], QB[5])), r_5, s.Msyz));
    const float2 p5 = f2(5.0f, 5.0f);
    s.Maxy = __ffma2_rn(p5, __ffma2_rn(t1, dx, __fmul2_rn(neg2(t0), dy)), s.Maxy);
    s.Maxz = __ffma2_rn(p5, __ffma2_rn(t2, dx, __fmul2_rn(neg2(t0), dz)), s.Maxz);
    s.Mayz = __ffma2_rn(p5, __ffma2_rn(t2, dy, __fmul2_rn(neg2(t1), dz)), s.Mayz);
  }
}

// The 12 far-field sums of a lane (both halves added), in the order of the
// group reduction: E (3), then the nine far-field gradient terms.
__device__ __forceinline__ void far_values(const Far2 &t, float (&v)[12]) {
  v[0] = t.Ex.x + t.Ex.y; v[1] = t.Ey.x + t.Ey.y; v[2] = t.Ez.x + t.Ez.y;
  v[3] = t.Mdx.x + t.Mdx.y; v[4] = t.Mdy.x + t.Mdy.y; v[5] = t.Mdz.x + t.Mdz.y;
  v[6] = t.Msxy.x + t.Msxy.y; v[7] = t.Msxz.x + t.Msxz.y; v[8] = t.Msyz.x + t.Msyz.y;
  v[9] = t.Maxy.x + t.Maxy.y; v[10] = t.Maxz.x + t.Maxz.y; v[11] = t.Mayz.x + t.Mayz.y;
}

// Pair counters of one evaluation: LJ-only, charge-field (+ LJ inside the
// cut-off) and far-field terms, and nl: charge-field pairs outside the LJ
// cut-off (no LJ term, fewer flops).
struct WorkM { uint32_t lj, es, far, nl; };

// Reduce-scatter of K values over a group of G lanes (G a power of two <= 32,
// aligned in the warp) by recursive halving: at each level a lane keeps half
// of the values it still holds and receives its partner's partial sums of
// that half, so the group spends P/2 + P/4 + ... shuffles (P = K rounded up to
// a power of two, P <= G) instead of log2(G) per value.  Lane l of the group
// ends with the group sum of value idx; after the halving levels a plain
// butterfly over the remaining lane bits makes the G/P lanes holding one index
// agree bitwise (IEEE addition commutes).  The lanes holding value k are
// k * (G / P) + j, j < G / P.
template <int K>
struct PowTwo {
  static constexpr int P = K <= 1 ? 1 : K <= 2 ? 2 : K <= 4 ? 4 : K <= 8 ? 8 : K <= 16 ? 16 : 32;
};

template <int K>
__device__ __forceinline__ float reduce_scatter(const float (&in)[K], int G, int lane, int &idx) {
  constexpr int P = PowTwo<K>::P;
  float v[P];
#pragma unroll
  for (int i = 0; i < P; i++) v[i] = i < K ? in[i] : 0.0f;
  idx = 0;
  int o = G >> 1;
#pragma unroll
  for (int c = P; c > 1; c >>= 1) {
    const int half = c >> 1;
    const bool up = (lane & o) != 0;
#pragma unroll
    for (int i = 0; i < half; i++) {
      const float send = up ? v[i] : v[i + half];
      const float keep = up ? v[i + half] : v[i];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
    }
    if (up) idx += half;
    o >>= 1;
  }
  for (; o > 0; o >>= 1) v[0] += __shfl_xor_sync(0xffffffffu, v[0], o);
  return v[0];
}

// ---- lanes of one trajectory ------------------------------------------------------
// A narrow group is G <= 32 lanes of one warp: shuffles reduce (bitwise the
// same sums in every lane), __syncwarp orders the group's shared-memory state.
struct NarrowLanes {
  int G, lane;
  unsigned gmask;
  __device__ __forceinline__ void sync() const { __syncwarp(gmask); }
  // the predicate over the whole warp: every group of the warp takes the same
  // branch, so the full-warp shuffles inside it stay convergent
  __device__ __forceinline__ bool any(bool p) const { return __any_sync(0xffffffffu, p); }
  __device__ __forceinline__ bool all(bool p) const { return __all_sync(0xffffffffu, p); }
  template <typename T, int K>
  __device__ __forceinline__ void sum(T (&v)[K]) {
#pragma unroll
    for (int k = 0; k < K; k++) v[k] = group_sum(v[k], G);
  }
  // float sums of 16- and 32-lane groups: reduce-scatter, then each lane
  // fetches every value from a lane that holds it (P/2 + ... + K shuffles
  // instead of K log2(G); the 22 sums of the far-field variants on 32 lanes:
  // 31 + 22 instead of 110); other widths use the butterfly
  template <int K>
  __device__ __forceinline__ void sum(float (&v)[K]) {
    constexpr int P = PowTwo<K>::P;
    if (K > 2 && P <= G && (G == 16 || G == 32)) {
      int idx;
      const float r = reduce_scatter<K>(v, G, lane, idx);
      const int gbase = (threadIdx.x & 31) & ~(G - 1);
      const int stride = G / P;
#pragma unroll
      for (int k = 0; k < K; k++) v[k] = __shfl_sync(0xffffffffu, r, gbase + k * stride);
    } else {
#pragma unroll
      for (int k = 0; k < K; k++) v[k] = group_sum(v[k], G);
    }
  }
};

// Acceleration at pos (FP64 in, FP64 out) for one group.  Pair counts are
// taken per cluster in pass 1 (or per evaluation), not per pair.
// PACKED_FAR: the far field of variants 1 and 2 in packed instructions, for
// kernels with the registers for it (the single-molecule kernel of those
// variants and the batched kernel run 640-thread CTAs at 96 registers).
template <int TYPE, bool PACKED_FAR, class L>
__device__ __forceinline__ void force(const View &m, const DevParams &p, const double pos[3],
                                      double acc[3], L &ln, uint8_t *modes, WorkM &w) {
  const int G = ln.G, lane = ln.lane;
  Acc s = {};
  // far-field sums already reduced over the group (listed variants 1 and 2
  // with G >= 16): this lane's share of the 12, see the far pass
  float far_share = 0.0f;
  bool far_reduced = false;
  const float hx = (float)pos[0], hy = (float)pos[1], hz = (float)pos[2];
  const float lx = (float)(pos[0] - (double)hx), ly = (float)(pos[1] - (double)hy),
              lz = (float)(pos[2] - (double)hz);
  if (Traits<TYPE>::kMaskable && m.nc < 64) {
    // variant 3 with fewer than 64 clusters: the cut-off decision of every
    // cluster in one register (ballot per round of G clusters) and, for the
    // pair loop, as a factor 1 or 0 per cluster in the group's scratch (one
    // shared load and a packed multiply per slot pair instead of 64-bit bit
    // tests and selects)
    unsigned long long in_mask = 0;
    float *fac = reinterpret_cast<float *>(modes);
    const int gbase = (threadIdx.x & 31) & ~(G - 1);
    const unsigned gbits = G == 32 ? 0xffffffffu : ((1u << G) - 1u);
    for (int c0 = 0; c0 < m.nc; c0 += G) {
      const int c = c0 + lane;
      bool in = false;
      if (c < m.nc) {
        const ClusterF32 &C = m.cl[c];
        const double d0 = pos[0] - C.cx, d1 = pos[1] - C.cy, d2 = pos[2] - C.cz;
        in = !(d0 * d0 + d1 * d1 + d2 * d2 > C.dr2);
        if (TYPE == 5 && in) w.lj += (uint32_t)C.n_atoms;
        if (TYPE == 3 && !in) w.nl += (uint32_t)C.n_atoms;
        fac[c] = in ? 1.0f : 0.0f;
      }
      const unsigned b = __ballot_sync(0xffffffffu, in);
      in_mask |= (unsigned long long)((b >> gbase) & gbits) << c0;
    }
    if (lane == 0) fac[m.nc] = 0.0f;                   // the pad atoms' cluster
    Acc2 t = {};
    const float2 hx2 = f2(hx, hx), hy2 = f2(hy, hy), hz2 = f2(hz, hz);
    const float2 lx2 = f2(lx, lx), ly2 = f2(ly, ly), lz2 = f2(lz, lz);
    // slot pairs j = jb + lane (pair-interleaved layout; slots come in multiples
    // of 64, so the n_slots / 2 pairs are a multiple of G).  When every
    // cluster of every group in the warp is inside the cut-off (the usual case
    // near the molecule) the prefactors are taken as stored, with no per-slot
    // mask test; pad atoms carry a zero prefactor either way.
    const unsigned long long all = m.nc == 64 ? ~0ull : ((1ull << m.nc) - 1ull);
    if (ln.all(in_mask == all)) {
      for (int jb = 0; jb < (m.nslots >> 1); jb += G) {
        const int j = jb + lane;
        pair2j<TYPE>(m, j, f2(m.pl[j].z, m.pl[j].w), true, hx2, hy2, hz2, lx2, ly2, lz2, t);
      }
    } else {
      ln.sync();
      for (int jb = 0; jb < (m.nslots >> 1); jb += G) {
        const int j = jb + lane;
        const uint2 c = m.pc[j];
        const float2 eps = __fmul2_rn(f2(m.pl[j].z, m.pl[j].w), f2(fac[c.x], fac[c.y]));
        pair2j<TYPE>(m, j, eps, true, hx2, hy2, hz2, lx2, ly2, lz2, t);
      }
    }
    fold<TYPE>(t, s);
  } else if (Traits<TYPE>::kListed) {
    // pass 1: near/far decision per cluster (FP64).  The clusters that add
    // pair terms go into the group's list (cluster << 8 | mode), compacted by
    // ballot: those with the charge field from the front, the LJ-only ones
    // from the back, so pass 2 skips the rest as the reference does
    // (forceAccel.cpp:221-633, 807-854) and packs pairs of one kind.
    uint32_t *list = reinterpret_cast<uint32_t *>(modes);
    const int gbase = (threadIdx.x & 31) & ~(G - 1);
    const unsigned gbits = G == 32 ? 0xffffffffu : ((1u << G) - 1u);
    const unsigned below = (1u << lane) - 1u;
    int n_es = 0, n_lj = 0;
    // the far-table pass leaves the pair counts of the listed clusters to pass 2
    bool count_listed = false;
    // one round: the clusters c0 + lane (FP64 tests, list entries, counters)
    auto classify = [&](int c0) {
      const int c = c0 + lane;
      uint32_t mode = 0;
      if (c < m.nc) {
        const ClusterF32 &C = m.cl[c];
        const double d0 = pos[0] - C.cx, d1 = pos[1] - C.cy, d2 = pos[2] - C.cz;
        const double r2 = d0 * d0 + d1 * d1 + d2 * d2;
        const bool in_disp = !(r2 > C.dr2);
        if (TYPE == 5) {
          mode = in_disp ? M_LJ : 0;
        } else if (r2 > C.mpr2) {
          w.far++;
          mode = TYPE == 2 ? M_LJ : (in_disp ? M_LJQ : 0);
        } else {
          mode = M_ES | ((TYPE == 2 || in_disp) ? M_LJ : 0);
        }
        const uint32_t cnt = (uint32_t)C.n_atoms;
        if (mode & M_ES) w.es += cnt;
        else if (mode) w.lj += cnt;
        if ((mode & M_ES) && !(mode & M_LJ)) w.nl += cnt;
      }
      const bool es = (mode & M_ES) != 0, ljo = mode != 0 && !es;
      const unsigned m_es = (__ballot_sync(0xffffffffu, es) >> gbase) & gbits;
      const unsigned m_lj = (__ballot_sync(0xffffffffu, ljo) >> gbase) & gbits;
      const uint32_t e = ((uint32_t)c << 8) | mode;
      if (es) list[n_es + __popc(m_es & below)] = e;
      if (ljo) list[m.nc - 1 - n_lj - __popc(m_lj & below)] = e;
      n_es += __popc(m_es);
      n_lj += __popc(m_lj);
    };
    if (Traits<TYPE>::kFar && PACKED_FAR && G >= 16) {
      // far field in the same pass (variants 1 and 2, G >= 16), from the
      // far-field table: lane j of a round takes clusters 2j and 2j+1, one per
      // half of the packed instructions.  The separations come from the FP32
      // hi/lo centres and the He position (as accurate as the FP64 difference
      // rounded to FP32), and the near/far and dispersion tests run on them;
      // a squared distance within 2^-16 (relative) of a radius is tested again
      // in FP64 from the cluster record, so every decision is the FP64 test's
      // (the FP32 value is within about 1e-6 of it).  A near half gets 1/r = 0
      // and adds exactly 0.  The 12 sums are reduced over the group at once
      // (reduce-scatter: one value per lane), so the pair loop below runs with
      // one extra register instead of 24.
      Far2 f = {};
      const float4 *T = m.ft;
      const int nfp = m.nfp;
      const float2 hx2 = f2(hx, hx), hy2 = f2(hy, hy), hz2 = f2(hz, hz);
      const float2 lx2 = f2(lx, lx), ly2 = f2(ly, ly), lz2 = f2(lz, lz);
      constexpr float kMargin = 1.0f / 65536.0f;
      for (int jb = 0; jb < nfp; jb += G) {
        const int j = jb + lane;
        const float4 t0 = T[j], t1 = T[nfp + j], t2 = T[2 * nfp + j], t3 = T[3 * nfp + j];
        const float4 t4 = T[4 * nfp + j], t5 = T[5 * nfp + j];
        const float2 dx = __fadd2_rn(__fadd2_rn(hx2, f2(t0.x, t0.y)), __fadd2_rn(lx2, f2(t1.z, t1.w)));
        const float2 dy = __fadd2_rn(__fadd2_rn(hy2, f2(t0.z, t0.w)), __fadd2_rn(ly2, f2(t2.x, t2.y)));
        const float2 dz = __fadd2_rn(__fadd2_rn(hz2, f2(t1.x, t1.y)), __fadd2_rn(lz2, f2(t2.z, t2.w)));
        const float2 xx = __fmul2_rn(dx, dx), yy = __fmul2_rn(dy, dy), zz = __fmul2_rn(dz, dz);
        const float2 r2 = __fadd2_rn(__fadd2_rn(xx, yy), zz);
        bool far_a = r2.x > t3.x, far_b = r2.y > t3.y;
        bool in_a = !(r2.x > t3.z), in_b = !(r2.y > t3.w);
        const bool amb = fabsf(r2.x - t3.x) <= kMargin * t3.x ||
                         fabsf(r2.y - t3.y) <= kMargin * t3.y ||
                         fabsf(r2.x - t3.z) <= kMargin * t3.z ||
                         fabsf(r2.y - t3.w) <= kMargin * t3.w;
        const int ca = 2 * j, cb = 2 * j + 1;
        if (ln.any(amb) && amb) {
          // the FP64 tests of both clusters (null entries are never ambiguous:
          // their radii are -1)
          const ClusterF32 &A = m.cl[ca];
          double d0 = pos[0] - A.cx, d1 = pos[1] - A.cy, d2 = pos[2] - A.cz;
          double q2 = d0 * d0 + d1 * d1 + d2 * d2;
          far_a = q2 > A.mpr2;
          in_a = !(q2 > A.dr2);
          if (cb < m.nc) {
            const ClusterF32 &B = m.cl[cb];
            d0 = pos[0] - B.cx; d1 = pos[1] - B.cy; d2 = pos[2] - B.cz;
            q2 = d0 * d0 + d1 * d1 + d2 * d2;
            far_b = q2 > B.mpr2;
            in_b = !(q2 > B.dr2);
          }
        }
        const float2 r_1 = f2(far_a ? rsqrt_ftz(r2.x) : 0.0f, far_b ? rsqrt_ftz(r2.y) : 0.0f);
        const int qa = ca < m.nc ? ca : m.nc, qb = cb < m.nc ? cb : m.nc;
        far2_core(p.multipole_order, dx, dy, dz, xx, yy, zz, r2, r_1, f2(t4.x, t4.y),
                  f2(t4.z, t4.w), f2(t5.x, t5.y), f2(t5.z, t5.w), m.cl[qa].quad, m.cl[qb].quad, f);
        // the clusters that add pair terms: a near one (charge field), or a
        // far one inside the dispersion radius (variant 1: band LJ) or, for
        // variant 2, every far one; null entries (far, never inside) only
        // need the bound for variant 2
        const bool es_a = !far_a, es_b = !far_b;
        const bool lj_a = far_a && (TYPE == 2 ? ca < m.nc : in_a);
        const bool lj_b = far_b && (TYPE == 2 ? cb < m.nc : in_b);
        const uint32_t mode_a = es_a ? (M_ES | ((TYPE == 2 || in_a) ? M_LJ : 0))
                                     : (TYPE == 2 ? M_LJ : M_LJQ);
        const uint32_t mode_b = es_b ? (M_ES | ((TYPE == 2 || in_b) ? M_LJ : 0))
                                     : (TYPE == 2 ? M_LJ : M_LJQ);
        const unsigned e_a = (__ballot_sync(0xffffffffu, es_a) >> gbase) & gbits;
        const unsigned e_b = (__ballot_sync(0xffffffffu, es_b) >> gbase) & gbits;
        const unsigned l_a = (__ballot_sync(0xffffffffu, lj_a) >> gbase) & gbits;
        const unsigned l_b = (__ballot_sync(0xffffffffu, lj_b) >> gbase) & gbits;
        // lane order, a before b: charge-field clusters from the front, the
        // LJ-only ones from the back
        const int pe = n_es + __popc(e_a & below) + __popc(e_b & below);
        const int pl = m.nc - 1 - n_lj - __popc(l_a & below) - __popc(l_b & below);
        if (es_a) list[pe] = ((uint32_t)ca << 8) | mode_a;
        if (es_b) list[pe + (es_a ? 1 : 0)] = ((uint32_t)cb << 8) | mode_b;
        if (lj_a) list[pl] = ((uint32_t)ca << 8) | mode_a;
        if (lj_b) list[pl - (lj_a ? 1 : 0)] = ((uint32_t)cb << 8) | mode_b;
        n_es += __popc(e_a) + __popc(e_b);
        n_lj += __popc(l_a) + __popc(l_b);
      }
      // every cluster that adds no charge field is far (variants 1, 2)
      if (lane == 0) w.far += (uint32_t)(m.nc - n_es);
      count_listed = true;
      float fv[12];
      far_values(f, fv);
      int idx;
      far_share = reduce_scatter<12>(fv, G, lane, idx);
      far_reduced = true;
    } else {
      for (int c0 = 0; c0 < m.nc; c0 += G) classify(c0);
    }
    ln.sync();
    // pass 2: the listed clusters, two at a time per (half-)group in the two
    // halves of the packed instructions.  The image is cluster-blocked: a
    // cluster fills whole blocks of kClusterBlock slots, padded with inert
    // atoms (whose prefactor flag b.w is 0), so lane `sub` walks both
    // clusters' blocks with no bounds test; a cluster without a partner is
    // paired with the image's last block, which is all padding
    const int split = G == 32 ? 16 : G;
    const int sub = lane & (split - 1), half = G == 32 ? (lane >> 4) : 0;
    const int step = G == 32 ? 2 : 1;
    const int inert0 = m.nslots - kClusterBlock;
    Acc2 t = {};
    const float2 hx2 = f2(hx, hx), hy2 = f2(hy, hy), hz2 = f2(hz, hz);
    const float2 lx2 = f2(lx, lx), ly2 = f2(ly, ly), lz2 = f2(lz, lz);
    auto params = [&](const ClusterF32 &C, const float4 &b, uint32_t mode) {
      if (TYPE == 1 && (mode & M_LJQ)) return f2(C.qsig6, C.qeps * b.w);
      return f2(b.x, (mode & (M_LJ | M_LJQ)) ? b.y : 0.0f);
    };
    auto run_pairs = [&](int lo, int hi, bool es) {
      for (int i = lo + 2 * half; i < hi; i += 2 * step) {
        const uint32_t ea = list[i];
        const bool has_b = i + 1 < hi;
        const uint32_t eb = has_b ? list[i + 1] : ea;
        const ClusterF32 &CA = m.cl[ea >> 8];
        const ClusterF32 &CB = m.cl[eb >> 8];
        const int na = CA.a1 - CA.a0, nb = has_b ? CB.a1 - CB.a0 : 0;
        if (count_listed && sub == 0) {
          // one lane per listed cluster: its pair terms by kind
          const uint32_t ca_n = (uint32_t)CA.n_atoms, cb_n = has_b ? (uint32_t)CB.n_atoms : 0u;
          if (es) {
            w.es += ca_n + cb_n;
            if (!(ea & M_LJ)) w.nl += ca_n;
            if (!(eb & M_LJ)) w.nl += cb_n;
          } else {
            w.lj += ca_n + cb_n;
          }
        }
        const int nmax = na > nb ? na : nb;
        if (TYPE == 1 && !es) {
          // variant 1's LJ-only clusters are far ones inside the dispersion
          // radius: every atom takes the cluster's band parameters, so the
          // per-atom LJ records are not read.  The prefactor is the cluster's
          // for its atoms (the first n_atoms slots of its blocks) and 0 for
          // padding, as the records' atom flag gives it.
          const float2 sig = f2(CA.qsig6, CB.qsig6);
          const int ra = CA.n_atoms, rb = has_b ? CB.n_atoms : 0;
          for (int k = sub; k < nmax; k += split) {
            const int ka = k < na ? CA.a0 + k : inert0 + (k & (kClusterBlock - 1));
            const int kb = k < nb ? CB.a0 + k : inert0 + (k & (kClusterBlock - 1));
            const float2 eps = f2(k < ra ? CA.qeps : 0.0f, k < rb ? CB.qeps : 0.0f);
            pair2<TYPE>(m.a4[ka], m.a4[kb], sig, eps, false, hx2, hy2, hz2, lx2, ly2, lz2, t);
          }
          continue;
        }
        for (int k = sub; k < nmax; k += split) {
          const int ka = k < na ? CA.a0 + k : inert0 + (k & (kClusterBlock - 1));
          const int kb = k < nb ? CB.a0 + k : inert0 + (k & (kClusterBlock - 1));
          const float4 a0 = m.a4[ka], b0 = m.b4[ka], a1 = m.a4[kb], b1 = m.b4[kb];
          const float2 p0 = params(CA, b0, ea & 0xffu), p1 = params(CB, b1, eb & 0xffu);
          pair2<TYPE>(a0, a1, f2(p0.x, p1.x), f2(p0.y, p1.y), es, hx2, hy2, hz2, lx2, ly2, lz2,
                      t);
        }
      }
    };
    if (Traits<TYPE>::kCharge) run_pairs(0, n_es, true);
    run_pairs(m.nc - n_lj, m.nc, false);
    fold<TYPE>(t, s);
    // pass 3 (G < 16): the far field of the far clusters, after the pair
    // sums are folded, so the pair loop keeps its registers for them
    if (Traits<TYPE>::kFar && !far_reduced) {
      for (int c = lane; c < m.nc; c += G) {
        const ClusterF32 &C = m.cl[c];
        const double d0 = pos[0] - C.cx, d1 = pos[1] - C.cy, d2 = pos[2] - C.cz;
        const double r2 = d0 * d0 + d1 * d1 + d2 * d2;
        if (r2 > C.mpr2) far_terms(m, c, p.multipole_order, (float)d0, (float)d1, (float)d2, s);
      }
    }
    ln.sync();
  } else if (Traits<TYPE>::kClusters) {
    // pass 1: near/far decision per cluster (FP64), far-field terms
    for (int c = lane; c < m.nc; c += G) {
      const ClusterF32 &C = m.cl[c];
      const double d0 = pos[0] - C.cx, d1 = pos[1] - C.cy, d2 = pos[2] - C.cz;
      const double r2 = d0 * d0 + d1 * d1 + d2 * d2;
      const bool in_disp = !(r2 > C.dr2);
      uint32_t mode;
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
      modes[c] = (uint8_t)mode;
      if (Traits<TYPE>::kVaryingPairs) {
        const uint32_t cnt = (uint32_t)C.n_atoms;
        if (mode & M_ES) w.es += cnt;
        else if (mode) w.lj += cnt;
      }
      if ((mode & M_ES) && !(mode & M_LJ)) w.nl += (uint32_t)C.n_atoms;
    }
    ln.sync();
    // pass 2: atom slots, two per lane per pass (G <= 32 and slots come in
    // multiples of 64, so both are in range)
    Acc2 t = {};
    const float2 hx2 = f2(hx, hx), hy2 = f2(hy, hy), hz2 = f2(hz, hz);
    const float2 lx2 = f2(lx, lx), ly2 = f2(ly, ly), lz2 = f2(lz, lz);
    if (paired_layout(TYPE)) {
      // variant 3: every slot adds the charge field, the mode only switches LJ
      for (int jb = 0; jb < (m.nslots >> 1); jb += G) {
        const int j = jb + lane;
        const uint2 c = m.pc[j];
        const float2 e = f2(m.pl[j].z, m.pl[j].w);
        const float2 eps = f2((modes[c.x] & M_LJ) ? e.x : 0.0f, (modes[c.y] & M_LJ) ? e.y : 0.0f);
        pair2j<TYPE>(m, j, eps, true, hx2, hy2, hz2, lx2, ly2, lz2, t);
      }
    } else {
      for (int base = 0; base < m.nslots; base += 2 * G) {
        const int k0 = base + lane, k1 = k0 + G;
        const float4 a0 = m.a4[k0], b0 = m.b4[k0], a1 = m.a4[k1], b1 = m.b4[k1];
        const uint32_t m0 = modes[cluster_of(b0)];
        const uint32_t m1 = modes[cluster_of(b1)];
        if (Traits<TYPE>::kEsAlways || TYPE == 5 || ((m0 ^ m1) & M_ES) == 0) {
          const float2 p0 = lj_params<TYPE>(m, b0, m0), p1 = lj_params<TYPE>(m, b1, m1);
          pair2<TYPE>(a0, a1, f2(p0.x, p1.x), f2(p0.y, p1.y), (m0 & M_ES) != 0, hx2, hy2, hz2,
                      lx2, ly2, lz2, t);
        } else {
          pair<TYPE>(m, a0, b0, m0, hx, hy, hz, lx, ly, lz, s);
          pair<TYPE>(m, a1, b1, m1, hx, hy, hz, lx, ly, lz, s);
        }
      }
    }
    fold<TYPE>(t, s);
    ln.sync();
  } else {
    Acc2 t = {};
    const float2 hx2 = f2(hx, hx), hy2 = f2(hy, hy), hz2 = f2(hz, hz);
    const float2 lx2 = f2(lx, lx), ly2 = f2(ly, ly), lz2 = f2(lz, lz);
    for (int jb = 0; jb < (m.nslots >> 1); jb += G) {
      const int j = jb + lane;
      pair2j<TYPE>(m, j, f2(m.pl[j].z, m.pl[j].w), TYPE == 4, hx2, hy2, hz2, lx2, ly2, lz2, t);
    }
    fold<TYPE>(t, s);
  }
  // group reduction (identical result in every lane of the group)
  if (Traits<TYPE>::kFar && far_reduced) {
    // the 13 pair sums, then the far sums from the lanes that hold them
    float v[13];
    v[0] = s.Fx; v[1] = s.Fy; v[2] = s.Fz;
    v[3] = s.Ex; v[4] = s.Ey; v[5] = s.Ez;
    v[6] = s.Pxx; v[7] = s.Pxy; v[8] = s.Pxz; v[9] = s.Pyy; v[10] = s.Pyz; v[11] = s.Pzz;
    v[12] = s.Q3;
    ln.sum(v);
    float fv[12];
    const int gbase = (threadIdx.x & 31) & ~(G - 1);
    const int stride = G / 16;
#pragma unroll
    for (int k = 0; k < 12; k++) fv[k] = __shfl_sync(0xffffffffu, far_share, gbase + k * stride);
    acc[0] = v[0]; acc[1] = v[1]; acc[2] = v[2];
    const double Mxx = (double)v[12] - 3.0 * v[6] + fv[3], Myy = (double)v[12] - 3.0 * v[9] + fv[4],
                 Mzz = (double)v[12] - 3.0 * v[11] + fv[5];
    const double Sxy = -3.0 * v[7] + fv[6], Sxz = -3.0 * v[8] + fv[7], Syz = -3.0 * v[10] + fv[8];
    const double Axy = fv[9], Axz = fv[10], Ayz = fv[11];
    const double Ex = (double)v[3] + fv[0], Ey = (double)v[4] + fv[1], Ez = (double)v[5] + fv[2];
    const double ds = p.dipole_scalar;
    acc[0] += ds * (Mxx * Ex + (Sxy + Axy) * Ey + (Sxz + Axz) * Ez);
    acc[1] += ds * ((Sxy - Axy) * Ex + Myy * Ey + (Syz + Ayz) * Ez);
    acc[2] += ds * ((Sxz - Axz) * Ex + (Syz - Ayz) * Ey + Mzz * Ez);
    return;
  }
  constexpr int K = Traits<TYPE>::kFar ? 22 : (Traits<TYPE>::kCharge ? 13 : 3);
  float v[K];
  v[0] = s.Fx; v[1] = s.Fy; v[2] = s.Fz;
  if (Traits<TYPE>::kCharge) {
    v[3] = s.Ex; v[4] = s.Ey; v[5] = s.Ez;
    v[6] = s.Pxx; v[7] = s.Pxy; v[8] = s.Pxz; v[9] = s.Pyy; v[10] = s.Pyz; v[11] = s.Pzz;
    v[12] = s.Q3;
  }
  if (Traits<TYPE>::kFar) {
    v[13] = s.Mdx; v[14] = s.Mdy; v[15] = s.Mdz; v[16] = s.Msxy; v[17] = s.Msxz;
    v[18] = s.Msyz; v[19] = s.Maxy; v[20] = s.Maxz; v[21] = s.Mayz;
  }
  ln.sum(v);
  acc[0] = v[0]; acc[1] = v[1]; acc[2] = v[2];
  if (Traits<TYPE>::kCharge) {
    double Mxx = (double)v[12] - 3.0 * v[6], Myy = (double)v[12] - 3.0 * v[9],
           Mzz = (double)v[12] - 3.0 * v[11];
    double Sxy = -3.0 * v[7], Sxz = -3.0 * v[8], Syz = -3.0 * v[10];
    double Axy = 0, Axz = 0, Ayz = 0;
    if (Traits<TYPE>::kFar) {
      Mxx += v[13]; Myy += v[14]; Mzz += v[15];
      Sxy += v[16]; Sxz += v[17]; Syz += v[18];
      Axy = v[19]; Axz = v[20]; Ayz = v[21];
    }
    const double Ex = v[3], Ey = v[4], Ez = v[5], ds = p.dipole_scalar;
    acc[0] += ds * (Mxx * Ex + (Sxy + Axy) * Ey + (Sxz + Axz) * Ez);
    acc[1] += ds * ((Sxy - Axy) * Ex + Myy * Ey + (Syz + Ayz) * Ez);
    acc[2] += ds * ((Sxz - Axz) * Ex + (Syz - Ayz) * Ey + Mzz * Ez);
  }
}

// 1/sqrt(x) in FP64: the hardware approximation and two Newton steps
// y <- y (3/2 - x y^2 / 2), each doubling the correct bits (to within a few
// ulps; no division or square-root sequence).
__device__ __forceinline__ double rsqrt_f64(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  const double h = 0.5 * x;
  y = y * fma(-h * y, y, 1.5);
  y = y * fma(-h * y, y, 1.5);
  return y;
}

// The potential in FP64 (forceAccel.cpp:943-982), lanes split the atoms.  The
// mixed form's energy check needs FP64 accuracy, not the reference's rounding:
// the powers of 1/r come from one reciprocal square root instead of two IEEE
// divisions and a square root per atom.
template <class L>
__device__ double potential(const View64 &m, const DevParams &p, const double pos[3], L &ln) {
  double v[4] = {0, 0, 0, 0};
  for (int k = ln.lane; k < m.n; k += ln.G) {
    const double *A = reinterpret_cast<const double *>(m.at + k);
    const double dx = pos[0] - __ldg(A + 0), dy = pos[1] - __ldg(A + 1),
                 dz = pos[2] - __ldg(A + 2);
    const double r2 = dx * dx + dy * dy + dz * dz;
    const double ir = rsqrt_f64(r2), ir2 = ir * ir;
    const double term2 = __ldg(A + 4) * (ir2 * ir2 * ir2);
    v[0] += __ldg(A + 6) * (term2 * term2 - term2);
    if (p.charged) {
      const double r_3 = __ldg(A + 3) * (ir * ir2);
      v[1] += dx * r_3; v[2] += dy * r_3; v[3] += dz * r_3;
    }
  }
  ln.sum(v);
  double total = v[0];
  if (p.charged) total -= p.dipole_scalar * 0.5 * (v[1] * v[1] + v[2] * v[2] + v[3] * v[3]);
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

// Trajectory state of one group, in shared memory rather than registers, so
// the pair loop runs at 64 registers a thread.  Every lane of the group
// computes the same values (the group sums are bitwise identical in every
// lane); each update reads the fields it needs, synchronises the group, then
// writes, so no lane overwrites a value another lane has yet to read.  The
// group's evaluation counters are kept by its leader lane only.
struct GroupState {
  TrajState s;
  unsigned long long nsteps;
  uint32_t nforce, npot;
  unsigned long long lj, es, far;     // pair terms (shared-memory atomics of all lanes)
};
static_assert(sizeof(GroupState) == kGroupStateBytes, "GroupState layout");

// Pair counters of one lane (force variants 1, 2, 5), added to the group's
// counters once the lane is done.
struct Tally {
  uint32_t lj = 0, es = 0, far = 0, nl = 0;
};

__device__ __forceinline__ void group_counters_clear(GroupState &G) {
  G.nsteps = 0; G.nforce = 0; G.npot = 0; G.lj = 0; G.es = 0; G.far = 0;
}

// Fold a lane's pair tally into its group (shared-memory atomics, once).
// A lane's charge-only pair count goes straight to the global counter (every
// lane, once, at the end of its narrow phase).
__device__ __forceinline__ void flush_nolj(const Tally &tl, unsigned long long *c) {
  count_add(c, C_PAIR_ESNL, tl.nl);
}

template <int TYPE>
__device__ __forceinline__ void fold_tally(GroupState &G, const Tally &tl) {
  if (Traits<TYPE>::kVaryingPairs) {
    if (tl.lj) atomicAdd(&G.lj, (unsigned long long)tl.lj);
    if (tl.es) atomicAdd(&G.es, (unsigned long long)tl.es);
    if (tl.far) atomicAdd(&G.far, (unsigned long long)tl.far);
  }
}

// Group counters, once per group (leader lane) at the end of its work.  For
// the variants with a fixed pair count the pair terms are n_atoms per
// acceleration evaluation.
template <int TYPE>
__device__ __forceinline__ void flush_group(GroupState &G, int n_atoms, unsigned long long *c) {
  if (!Traits<TYPE>::kVaryingPairs) {
    if (Traits<TYPE>::kCharge) G.es = (unsigned long long)G.nforce * n_atoms;
    else G.lj = (unsigned long long)G.nforce * n_atoms;
  }
  const int n_atoms_pot = n_atoms;
  count_add(c, C_STEPS, (long long)G.nsteps);
  count_add(c, C_FORCE_EVALS, G.nforce);
  count_add(c, C_POT_EVALS, G.npot);
  count_add(c, C_PAIR_POT, (long long)G.npot * n_atoms_pot);
  count_add(c, C_PAIR_LJ, (long long)G.lj);
  count_add(c, C_PAIR_ES, (long long)G.es);
  count_add(c, C_FAR, (long long)G.far);
  group_counters_clear(G);
}

// Start a trajectory: slot t, start state p0/v0 (every lane writes the same).
__device__ __forceinline__ void traj_begin(TrajState &S, long long t, const double *p0,
                                           const double *v0, double dt, bool may_handoff) {
  S.t = t;
  for (int i = 0; i < 3; i++) { S.p0[i] = p0[i]; S.v0[i] = v0[i]; }
  S.tries = 0; S.max_tries = 8; S.dt = dt; S.step = 0; S.total = 0;
  S.etries = 0; S.otries = 0;
  S.may_handoff = may_handoff ? 1 : 0;
  S.phase = P_INIT_FIRST;
}

// Where a group's trajectories come from.  Narrow groups draw queue slots
// 0..n-1 (slot k integrates trajectory order[k]; a trajectory with hit[t] == 0
// is an ellipsoid miss, chi = 0) and may park long ones; wide groups finish
// parked trajectories.
struct MainSource {
  const double *pos0, *vel0;
  const int32_t *hit, *order;
  long long n;
  cosims_traj_out *out;
  unsigned long long *queue, *counters;
  Handoff ho;
};

// The single-molecule kernel reads the same fields straight from its
// (grid-constant) parameters, so they take no registers.
struct ArgsSource {
  const TrajArgs &a;
};

// Whether a source's kernel takes the packed far-field pass (see force).
template <class Src> struct PackedFar { static constexpr bool value = false; };
template <> struct PackedFar<ArgsSource> { static constexpr bool value = true; };

__device__ __forceinline__ cosims_traj_out *out_of(const MainSource &s) { return s.out; }
__device__ __forceinline__ cosims_traj_out *out_of(const ArgsSource &s) { return s.a.out; }
__device__ __forceinline__ long long budget_of(const MainSource &s) { return s.ho.budget; }
__device__ __forceinline__ long long budget_of(const ArgsSource &s) { return s.a.ho.budget; }

// Acquire the next trajectory into S; false when the source is exhausted.
template <class A>
__device__ __forceinline__ bool acquire_main(const A &src, const DevParams &p, NarrowLanes &ln,
                                             GroupState &GS) {
  for (;;) {
    long long tk = 0;
    if (ln.lane == 0) tk = (long long)atomicAdd(src.queue, 1ull);
    long long t = __shfl_sync(ln.gmask, tk, 0, ln.G);
    if (t >= src.n) {
      // the one group that drew slot n saw the queue empty first
      if (ln.lane == 0 && src.counters && t == src.n) mark_first(src.counters, C_T_DRAIN_INV);
      return false;
    }
    if (src.order) t = src.order[t];
    if (src.hit && !src.hit[t]) {               // ellipsoid miss: chi = 0
      if (ln.lane == 0) {
        cosims_traj_out o = {0.0, 0.0, 0, 0u};
        src.out[t] = o;
      }
      continue;
    }
    traj_begin(GS.s, t, src.pos0 + 3 * t, src.vel0 + 3 * t, p.dt, src.ho.budget > 0);
    return true;
  }
}
__device__ __forceinline__ bool acquire(const MainSource &src, const DevParams &p,
                                        NarrowLanes &ln, GroupState &GS) {
  return acquire_main(src, p, ln, GS);
}
__device__ __forceinline__ bool acquire(const ArgsSource &src, const DevParams &p,
                                        NarrowLanes &ln, GroupState &GS) {
  return acquire_main(src.a, p, ln, GS);
}

// Park the trajectory in S for a wide group; false when the record array is
// full (the group then keeps it).
__device__ __forceinline__ bool park_to(const Handoff &ho, NarrowLanes &ln, GroupState &GS) {
  long long r = 0;
  if (ln.lane == 0) r = (long long)atomicAdd(ho.reserve, 1ull);
  r = __shfl_sync(ln.gmask, r, 0, ln.G);
  if (r >= ho.cap) return false;
  const double *s = reinterpret_cast<const double *>(&GS.s);
  double *g = reinterpret_cast<double *>(ho.states + r);
  for (int k = ln.lane; k < kTrajStateBytes / 8; k += ln.G) g[k] = s[k];
  __threadfence();
  ln.sync();
  if (ln.lane == 0 && !(ho.withhold_first && r == 0)) atomicExch(ho.ready + r, 1u);
  return true;
}
__device__ __forceinline__ bool park(const MainSource &src, NarrowLanes &ln, GroupState &GS) {
  return park_to(src.ho, ln, GS);
}
__device__ __forceinline__ bool park(const ArgsSource &src, NarrowLanes &ln, GroupState &GS) {
  return park_to(src.a.ho, ln, GS);
}

// The trajectory loop of one group.  Every iteration evaluates one
// acceleration per group (at the start state or after a position update)
// and, when any group of the warp needs it, one potential; a group whose
// trajectory ends takes the next one at once.  The control flow is
// diffEqSolver::verletVel's (diffEqSolver.cpp:81-211).
template <int TYPE, class L, class Src>
__device__ __forceinline__ void group_loop(const View &m, const View64 &m64, const DevParams &p,
                                           L &ln, uint8_t *modes, GroupState &GS,
                                           const Src &src, Tally &tl) {
  TrajState &S = GS.s;
  const long long cap = p.max_steps > 0 ? p.max_steps : kDefaultMaxSteps;

  while (true) {
    int phase = S.phase;
    if (phase == P_ACQUIRE) {
      ln.sync();
      const bool got = acquire(src, p, ln, GS);
      ln.sync();
      // a new trajectory starts at INIT_FIRST, a parked one where it stopped
      phase = got ? S.phase : (int)P_DONE;
      ln.sync();
      if (!got) S.phase = P_DONE;
    }
    if (ln.all(phase == P_DONE)) break;

    double ep[3];
    bool needU = false, outside = false;
    if (phase == P_INIT_FIRST || phase == P_INIT_RETRY) {
      ep[0] = S.p0[0]; ep[1] = S.p0[1]; ep[2] = S.p0[2];
      needU = phase == P_INIT_FIRST;
    } else if (phase == P_STEP) {
      const double dt = S.dt;
      double vh[3];
      for (int i = 0; i < 3; i++) {
        const double a = S.acc[i], v = S.vel[i];
        ep[i] = S.pos[i] + v * dt + a * dt * dt * 0.5;
        vh[i] = v + a * dt * 0.5;
      }
      const int step = S.step;
      ln.sync();
      for (int i = 0; i < 3; i++) { S.pos[i] = ep[i]; S.vel[i] = vh[i]; }
      // the ellipsoid exit test by reciprocal axes (no FP64 division per step)
      const double t0 = ep[0] * p.inv_ell_a, t1 = ep[1] * p.inv_ell_b, t2 = ep[2] * p.inv_ell_c;
      const double mag2 = t0 * t0 + t1 * t1 + t2 * t2;
      outside = (mag2 > 1 && p.projection) || (mag2 > p.max_rad && !p.projection);
      needU = outside && step + 1 > 10;
    } else {
      ep[0] = 1.0e4; ep[1] = 0.0; ep[2] = 0.0;
    }
    ln.sync();

    double an[3];
    WorkM wi = {0, 0, 0, 0};
    force<TYPE, PackedFar<Src>::value>(m, p, ep, an, ln, modes, wi);
    // a group without a trajectory evaluates at a dummy point only to keep the
    // warp's shuffles convergent: its pair terms are not counted (their number
    // depends on when the other groups of the warp finish)
    if (Traits<TYPE>::kVaryingPairs && phase != P_DONE) {
      tl.lj += wi.lj; tl.es += wi.es; tl.far += wi.far;
    }
    if (Traits<TYPE>::kCharge && Traits<TYPE>::kClusters && phase != P_DONE) {
      tl.nl += wi.nl;
    }
    double U = 0;
    if (ln.any(needU)) {
      double up[3];
      if (phase == P_STEP) { up[0] = S.pos[0]; up[1] = S.pos[1]; up[2] = S.pos[2]; }
      else if (phase == P_DONE) { up[0] = 1.0e4; up[1] = 0.0; up[2] = 0.0; }
      else { up[0] = S.p0[0]; up[1] = S.p0[1]; up[2] = S.p0[2]; }
      U = potential(m64, p, up, ln);
    }
    if (phase == P_DONE) continue;
    if (ln.lane == 0) {
      GS.nforce += 1;
      if (needU) GS.npot += 1;
    }

    if (phase == P_INIT_FIRST || phase == P_INIT_RETRY) {
      double p0[3], v0[3];
      for (int i = 0; i < 3; i++) { p0[i] = S.p0[i]; v0[i] = S.v0[i]; }
      ln.sync();
      if (phase == P_INIT_FIRST) S.E0 = U + 0.5 * p.mu * dot3(v0, v0);
      for (int i = 0; i < 3; i++) { S.acc[i] = an[i]; S.pos[i] = p0[i]; S.vel[i] = v0[i]; }
      S.orbits = 0;
      S.rdot = dot3(p0, v0);
      S.phase = P_STEP;
      ln.sync();
      continue;
    }

    // read the fields this step rewrites, synchronise, then read the rest
    const double dt = S.dt, rold = S.rdot;
    double vel[3];
    for (int i = 0; i < 3; i++) vel[i] = S.vel[i] + an[i] * dt * 0.5;
    const int step = S.step + 1;
    const long long total = S.total + 1;
    int orbits = S.orbits, etries = S.etries, otries = S.otries;
    double tries = S.tries, max_tries = S.max_tries, dt_new = dt;
    ln.sync();
    double pos[3];
    for (int i = 0; i < 3; i++) pos[i] = S.pos[i];
    const double E0 = S.E0;
    const bool may_handoff = S.may_handoff != 0;
    const long long t = S.t;

    if (ln.lane == 0) GS.nsteps += 1;
    bool track = true;
    const double rdot = dot3(pos, vel);
    if (step > 2 && rdot * rold < 0 && !(rdot > rold)) {
      orbits++;
      if (orbits > 8) track = false;
    }
    int step_out = step;
    int next = P_STEP;
    double chi = COSIMS_PI_2, dE = 0.0;
    uint32_t status = 0;
    bool finished = false;
    if (!track) {
      tries++;
      otries++;
      dt_new = p.dt / (tries + 1);
    } else if (outside && step > 10) {
      const double endE = U + 0.5 * p.mu * dot3(vel, vel);
      dE = 100 * fabs(E0 - endE) / E0;
      // a non-finite energy fails the check: a pair term that overflows FP32
      // at a near collision leaves inf or NaN where FP64 holds a huge, finite
      // energy error, which fails it (diffEqSolver.cpp:188-194)
      if (!(dE <= 0.5)) {
        tries++;
        max_tries++;
        etries++;
        dt_new = p.dt / (tries + 1);
        step_out = 0;
      } else {
        const double v0[3] = {S.v0[0], S.v0[1], S.v0[2]};
        chi = angle3(v0, vel);
        status = COSIMS_TRAJ_HIT | COSIMS_TRAJ_SUCCESS;
        finished = true;
      }
    }
    if (!finished) {
      // the step cap, or a state gone non-finite (the reference would loop);
      // a step whose energy check just failed retries instead
      if (total >= cap || (!isfinite(rdot) && step_out != 0)) {
        chi = COSIMS_PI_2; dE = 0.0;
        status = COSIMS_TRAJ_HIT | COSIMS_TRAJ_STEPCAP;
        finished = true;
      } else if (!(tries < max_tries && max_tries < 10)) {
        chi = COSIMS_PI_2; dE = 0.0;
        status = COSIMS_TRAJ_HIT;
        finished = true;
      } else if (step_out == 0) {
        next = P_INIT_RETRY;
      }
    }
    if (finished) {
      if (ln.lane == 0) {
        cosims_traj_out o;
        o.chi = chi; o.de_pct = dE; o.steps = step_out;
        o.status = status | ((uint32_t)etries << COSIMS_TRAJ_ETRIES_SHIFT) |
                   ((uint32_t)otries << COSIMS_TRAJ_OTRIES_SHIFT);
        out_of(src)[t] = o;
      }
      next = P_ACQUIRE;
    }
    for (int i = 0; i < 3; i++) { S.vel[i] = vel[i]; S.acc[i] = an[i]; }
    S.rdot = rdot; S.orbits = orbits; S.etries = etries; S.otries = otries;
    S.tries = tries; S.max_tries = max_tries; S.dt = dt_new;
    S.step = step_out; S.total = total;
    S.phase = next;
    ln.sync();
    // a long trajectory moves to a wide group (deterministic: its own step count)
    if (!finished && may_handoff && total >= budget_of(src)) {
      if (park(src, ln, GS)) S.phase = P_ACQUIRE;
      else S.may_handoff = 0;
      ln.sync();
    }
  }
}

#ifndef COSIMS_MIXED_MIN_BLOCKS
#define COSIMS_MIXED_MIN_BLOCKS 1
#endif

// Dynamic shared memory of the mixed kernels: [F32 image, 16-byte padded]
// then the groups' scratch.  Narrow phase: [GroupState x groups][cluster modes
// x groups].  Wide phase (same bytes, after a CTA barrier): per wide group
// [GroupState][modes][float slots 2 x warps x 24][double slots 2 x warps x 4]
// [broadcast word].
__device__ __forceinline__ unsigned char *scratch_base(unsigned char *smem, uint32_t img_bytes) {
  return smem + ((img_bytes + 15u) & ~15u);
}

__device__ __forceinline__ void narrow_scratch(unsigned char *smem, uint32_t img_bytes, int G,
                                               int mode_stride, GroupState *&S,
                                               uint8_t *&modes) {
  const int ngroups = blockDim.x / G;
  const int g = threadIdx.x / G;
  unsigned char *p = scratch_base(smem, img_bytes);
  S = reinterpret_cast<GroupState *>(p) + g;
  modes = p + (size_t)ngroups * sizeof(GroupState) + (size_t)g * mode_stride;
}

// ---- wide groups: one trajectory per WG threads, latency first ---------------------
// A parked trajectory is finished by a wide group.  Its state stays in
// registers (every thread of the group computes the same values: the sums are
// read from shared memory in warp order by all), each thread evaluates the
// pair terms of nslots / WG atom slots, and a step costs two barriers: after
// the cluster pass, and after the per-warp partial sums.  Modes and slots are
// double-buffered by step parity, so no barrier closes a step.
struct Wide {
  int WG, lane, warp, nwarps, bar;
  uint8_t *modes;     // [2][mode_stride]
  int mode_stride;
  float *fslots;      // [2][nwarps][kWideSlotFloats]
  double *dslots;     // [2][nwarps][4]
  long long *bcast;
  __device__ __forceinline__ void sync() const {
    asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(WG) : "memory");
  }
  // sum of v over the group, the same in every thread
  template <int K>
  __device__ __forceinline__ void sum(float (&v)[K], int par) const {
    int idx;
    const float r = reduce_scatter<K>(v, 32, lane & 31, idx);
    float *slot = fslots + par * nwarps * kWideSlotFloats;
    if (idx < K) slot[warp * kWideSlotFloats + idx] = r;   // lanes of one index agree
    sync();
#pragma unroll
    for (int k = 0; k < K; k++) v[k] = slot[k];
    for (int w = 1; w < nwarps; w++) {
#pragma unroll
      for (int k = 0; k < K; k++) v[k] += slot[w * kWideSlotFloats + k];
    }
  }
  template <int K>
  __device__ __forceinline__ void sum(double (&v)[K], int par) const {
#pragma unroll
    for (int k = 0; k < K; k++) v[k] = group_sum(v[k], 32);
    double *slot = dslots + par * nwarps * 4;
    if ((lane & 31) == 0) {
#pragma unroll
      for (int k = 0; k < K; k++) slot[warp * 4 + k] = v[k];
    }
    sync();
#pragma unroll
    for (int k = 0; k < K; k++) v[k] = slot[k];
    for (int w = 1; w < nwarps; w++) {
#pragma unroll
      for (int k = 0; k < K; k++) v[k] += slot[w * 4 + k];
    }
  }
};

template <int TYPE>
__device__ __forceinline__ void wide_force(const View &m, const DevParams &p, const double pos[3],
                                           double acc[3], const Wide &wd, int par, Tally &tl) {
  Acc s = {};
  const float hx = (float)pos[0], hy = (float)pos[1], hz = (float)pos[2];
  const float lx = (float)(pos[0] - (double)hx), ly = (float)(pos[1] - (double)hy),
              lz = (float)(pos[2] - (double)hz);
  const int lane = wd.lane, WG = wd.WG;
  if (Traits<TYPE>::kClusters) {
    uint8_t *modes = wd.modes + par * wd.mode_stride;
    for (int c = lane; c < m.nc; c += WG) {
      const ClusterF32 &C = m.cl[c];
      const double d0 = pos[0] - C.cx, d1 = pos[1] - C.cy, d2 = pos[2] - C.cz;
      const double r2 = d0 * d0 + d1 * d1 + d2 * d2;
      const bool in_disp = !(r2 > C.dr2);
      uint32_t mode;
      if (TYPE == 5) {
        mode = in_disp ? M_LJ : 0;
      } else if (TYPE == 3) {
        mode = M_ES | (in_disp ? M_LJ : 0);
      } else {
        // far clusters: their far-field terms follow the pair loop
        if (r2 > C.mpr2) {
          tl.far++;
          mode = TYPE == 2 ? M_LJ : (in_disp ? M_LJQ : 0);
        } else {
          mode = M_ES | ((TYPE == 2 || in_disp) ? M_LJ : 0);
        }
      }
      modes[c] = (uint8_t)mode;
      if (Traits<TYPE>::kVaryingPairs) {
        const uint32_t cnt = (uint32_t)C.n_atoms;
        if (mode & M_ES) tl.es += cnt;
        else if (mode) tl.lj += cnt;
      }
      if ((mode & M_ES) && !(mode & M_LJ)) tl.nl += (uint32_t)C.n_atoms;
    }
    wd.sync();
    int k = lane;
    if (paired_layout(TYPE)) {
      // variant 3: slot pairs of the pair-interleaved layout, LJ by cluster mode
      Acc2 t = {};
      const float2 hx2 = f2(hx, hx), hy2 = f2(hy, hy), hz2 = f2(hz, hz);
      const float2 lx2 = f2(lx, lx), ly2 = f2(ly, ly), lz2 = f2(lz, lz);
      for (int j = lane; j < (m.nslots >> 1); j += WG) {
        const uint2 c = m.pc[j];
        const float2 e = f2(m.pl[j].z, m.pl[j].w);
        const float2 eps = f2((modes[c.x] & M_LJ) ? e.x : 0.0f, (modes[c.y] & M_LJ) ? e.y : 0.0f);
        pair2j<TYPE>(m, j, eps, true, hx2, hy2, hz2, lx2, ly2, lz2, t);
      }
      fold<TYPE>(t, s);
      k = m.nslots;
    } else if (Traits<TYPE>::kListed) {
      // cluster-blocked image (variants 1, 2, 5): a 16-lane slice takes two
      // blocks at a time, one per half of the packed instructions, and skips
      // pairs of blocks whose clusters add nothing (far field only, or beyond
      // the cut-off).  A half whose cluster adds no charge field gets charge 0,
      // so two blocks of different modes share one packed evaluation.
      Acc2 t = {};
      const float2 hx2 = f2(hx, hx), hy2 = f2(hy, hy), hz2 = f2(hz, hz);
      const float2 lx2 = f2(lx, lx), ly2 = f2(ly, ly), lz2 = f2(lz, lz);
      const int sub = lane & (kClusterBlock - 1);
      const int slices = WG / kClusterBlock;
      const int nblk = m.nslots / kClusterBlock - 1;      // the last block is padding
      for (int bA = 2 * (lane / kClusterBlock); bA < nblk; bA += 2 * slices) {
        const int bB = bA + 1 < nblk ? bA + 1 : nblk;
        const uint32_t cA = cluster_of(m.b4[bA * kClusterBlock]);
        const uint32_t cB = cluster_of(m.b4[bB * kClusterBlock]);
        const uint32_t mA = modes[cA], mB = modes[cB];
        if ((mA | mB) == 0) continue;
        const int sA = bA * kClusterBlock + sub, sB = bB * kClusterBlock + sub;
        const float4 a0 = m.a4[sA], b0 = m.b4[sA], a1 = m.a4[sB], b1 = m.b4[sB];
        float2 sg, ep;
        if (TYPE == 1 && (mA & M_LJQ)) { sg.x = m.cl[cA].qsig6; ep.x = m.cl[cA].qeps * b0.w; }
        else { sg.x = b0.x; ep.x = (mA & (M_LJ | M_LJQ)) ? b0.y : 0.0f; }
        if (TYPE == 1 && (mB & M_LJQ)) { sg.y = m.cl[cB].qsig6; ep.y = m.cl[cB].qeps * b1.w; }
        else { sg.y = b1.x; ep.y = (mB & (M_LJ | M_LJQ)) ? b1.y : 0.0f; }
        const float2 q = f2((mA & M_ES) ? a0.w : 0.0f, (mB & M_ES) ? a1.w : 0.0f);
        pair2v<TYPE>(f2(a0.x, a1.x), f2(a0.y, a1.y), f2(a0.z, a1.z), q, sg, ep,
                     ((mA | mB) & M_ES) != 0, hx2, hy2, hz2, lx2, ly2, lz2, t);
      }
      fold<TYPE>(t, s);
      k = m.nslots;
      if (Traits<TYPE>::kFar) {
        for (int c = lane; c < m.nc; c += WG) {
          if (modes[c] & M_ES) continue;               // near: pair terms above
          const ClusterF32 &C = m.cl[c];
          const double d0 = pos[0] - C.cx, d1 = pos[1] - C.cy, d2 = pos[2] - C.cz;
          far_terms(m, c, p.multipole_order, (float)d0, (float)d1, (float)d2, s);
        }
      }
    }
    for (; k < m.nslots; k += WG) {
      const float4 a = m.a4[k], b = m.b4[k];
      pair<TYPE>(m, a, b, (uint32_t)modes[cluster_of(b)], hx, hy, hz, lx, ly, lz, s);
    }
  } else {
    // variants 4, 6: slot pairs of the pair-interleaved layout, every pair in full
    Acc2 t = {};
    const float2 hx2 = f2(hx, hx), hy2 = f2(hy, hy), hz2 = f2(hz, hz);
    const float2 lx2 = f2(lx, lx), ly2 = f2(ly, ly), lz2 = f2(lz, lz);
    for (int j = lane; j < (m.nslots >> 1); j += WG)
      pair2j<TYPE>(m, j, f2(m.pl[j].z, m.pl[j].w), TYPE == 4, hx2, hy2, hz2, lx2, ly2, lz2, t);
    fold<TYPE>(t, s);
  }
  constexpr int K = Traits<TYPE>::kFar ? 22 : (Traits<TYPE>::kCharge ? 13 : 3);
  float v[K];
  v[0] = s.Fx; v[1] = s.Fy; v[2] = s.Fz;
  if (Traits<TYPE>::kCharge) {
    v[3] = s.Ex; v[4] = s.Ey; v[5] = s.Ez;
    v[6] = s.Pxx; v[7] = s.Pxy; v[8] = s.Pxz; v[9] = s.Pyy; v[10] = s.Pyz; v[11] = s.Pzz;
    v[12] = s.Q3;
  }
  if (Traits<TYPE>::kFar) {
    v[13] = s.Mdx; v[14] = s.Mdy; v[15] = s.Mdz; v[16] = s.Msxy; v[17] = s.Msxz;
    v[18] = s.Msyz; v[19] = s.Maxy; v[20] = s.Maxz; v[21] = s.Mayz;
  }
  wd.sum(v, par);
  acc[0] = v[0]; acc[1] = v[1]; acc[2] = v[2];
  if (Traits<TYPE>::kCharge) {
    double Mxx = (double)v[12] - 3.0 * v[6], Myy = (double)v[12] - 3.0 * v[9],
           Mzz = (double)v[12] - 3.0 * v[11];
    double Sxy = -3.0 * v[7], Sxz = -3.0 * v[8], Syz = -3.0 * v[10];
    double Axy = 0, Axz = 0, Ayz = 0;
    if (Traits<TYPE>::kFar) {
      Mxx += v[13]; Myy += v[14]; Mzz += v[15];
      Sxy += v[16]; Sxz += v[17]; Syz += v[18];
      Axy = v[19]; Axz = v[20]; Ayz = v[21];
    }
    const double Ex = v[3], Ey = v[4], Ez = v[5], ds = p.dipole_scalar;
    acc[0] += ds * (Mxx * Ex + (Sxy + Axy) * Ey + (Sxz + Axz) * Ez);
    acc[1] += ds * ((Sxy - Axy) * Ex + Myy * Ey + (Syz + Ayz) * Ez);
    acc[2] += ds * ((Sxz - Axz) * Ex + (Syz - Ayz) * Ey + Mzz * Ez);
  }
}

__device__ __forceinline__ double wide_potential(const View64 &m, const DevParams &p,
                                                 const double pos[3], const Wide &wd, int par) {
  double v[4] = {0, 0, 0, 0};
  for (int k = wd.lane; k < m.n; k += wd.WG) {
    const double *A = reinterpret_cast<const double *>(m.at + k);
    const double dx = pos[0] - __ldg(A + 0), dy = pos[1] - __ldg(A + 1),
                 dz = pos[2] - __ldg(A + 2);
    const double r2 = dx * dx + dy * dy + dz * dz;
    const double ir = rsqrt_f64(r2), ir2 = ir * ir;
    const double term2 = __ldg(A + 4) * (ir2 * ir2 * ir2);
    v[0] += __ldg(A + 6) * (term2 * term2 - term2);
    if (p.charged) {
      const double r_3 = __ldg(A + 3) * (ir * ir2);
      v[1] += dx * r_3; v[2] += dy * r_3; v[3] += dz * r_3;
    }
  }
  wd.sum(v, par);
  double total = v[0];
  if (p.charged) total -= p.dipole_scalar * 0.5 * (v[1] * v[1] + v[2] * v[2] + v[3] * v[3]);
  return total;
}

// Take the next parked record; -1 when none is left (the same in every thread).
__device__ __forceinline__ long long wide_take(const Wide &wd, const Handoff &ho,
                                               unsigned long long *counters) {
  if (wd.lane == 0) {
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
      // the parking group reserved the record before writing it: wait for its flag
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
    *wd.bcast = got;
  }
  wd.sync();
  return *wd.bcast;   // rewritten only after the next trajectory's barriers
}

// The trajectory loop of a wide group over parked records: the control flow
// of diffEqSolver::verletVel (diffEqSolver.cpp:81-211) from where the narrow
// group stopped.
template <int TYPE>
__device__ __forceinline__ void wide_loop(const View &m, const View64 &m64, const DevParams &p,
                                          const Wide &wd, const Handoff &ho,
                                          cosims_traj_out *out, unsigned long long *counters,
                                          Tally &tl, unsigned long long &nsteps, uint32_t &nforce,
                                          uint32_t &npot) {
  const long long cap = p.max_steps > 0 ? p.max_steps : kDefaultMaxSteps;
  int par = 0;        // step parity: which half of the modes and slots
  for (;;) {
    const long long idx = wide_take(wd, ho, counters);
    if (idx < 0) break;
    const TrajState *R = ho.states + idx;
    double pos[3], vel[3], acc[3];
    for (int i = 0; i < 3; i++) {
      pos[i] = __ldcg(&R->pos[i]); vel[i] = __ldcg(&R->vel[i]); acc[i] = __ldcg(&R->acc[i]);
    }
    double dt = __ldcg(&R->dt), rdot = __ldcg(&R->rdot);
    int tries = (int)__ldcg(&R->tries), max_tries = (int)__ldcg(&R->max_tries);
    long long total = __ldcg(&R->total);
    int step = __ldcg(&R->step), orbits = __ldcg(&R->orbits), phase = __ldcg(&R->phase);
    int etries = __ldcg(&R->etries), otries = __ldcg(&R->otries);
    for (;;) {
      // evaluation point: the start state (retry) or the Verlet position update
      bool outside = false, needU = false;
      if (phase == P_INIT_RETRY) {
        for (int i = 0; i < 3; i++) pos[i] = __ldcg(&R->p0[i]);
      } else {
        for (int i = 0; i < 3; i++) {
          pos[i] = pos[i] + vel[i] * dt + acc[i] * dt * dt * 0.5;
          vel[i] = vel[i] + acc[i] * dt * 0.5;
        }
        const double t0 = pos[0] * p.inv_ell_a, t1 = pos[1] * p.inv_ell_b,
                     t2 = pos[2] * p.inv_ell_c;
        const double mag2 = t0 * t0 + t1 * t1 + t2 * t2;
        outside = (mag2 > 1 && p.projection) || (mag2 > p.max_rad && !p.projection);
        needU = outside && step + 1 > 10;
      }
      double an[3];
      wide_force<TYPE>(m, p, pos, an, wd, par, tl);
      double U = 0;
      if (needU) U = wide_potential(m64, p, pos, wd, par);
      par ^= 1;
      if (wd.lane == 0) { nforce++; if (needU) npot++; }
      if (phase == P_INIT_RETRY) {
        for (int i = 0; i < 3; i++) { vel[i] = __ldcg(&R->v0[i]); acc[i] = an[i]; }
        orbits = 0;
        rdot = dot3(pos, vel);
        phase = P_STEP;
        continue;
      }
      for (int i = 0; i < 3; i++) { vel[i] = vel[i] + an[i] * dt * 0.5; acc[i] = an[i]; }
      step++;
      total++;
      if (wd.lane == 0) nsteps++;
      bool track = true;
      const double rold = rdot;
      rdot = dot3(pos, vel);
      if (step > 2 && rdot * rold < 0 && !(rdot > rold)) {
        orbits++;
        if (orbits > 8) track = false;
      }
      bool finished = false;
      double chi = COSIMS_PI_2, dE = 0.0;
      uint32_t status = COSIMS_TRAJ_HIT;
      if (!track) {
        tries++;
        otries++;
        dt = p.dt / ((double)tries + 1);
      } else if (outside && step > 10) {
        const double E0 = __ldcg(&R->E0);
        const double endE = U + 0.5 * p.mu * dot3(vel, vel);
        dE = 100 * fabs(E0 - endE) / E0;
        if (!(dE <= 0.5)) {                    // non-finite fails, as in the narrow loop
          tries++;
          max_tries++;
          etries++;
          dt = p.dt / ((double)tries + 1);
          step = 0;
          dE = 0.0;
        } else {
          double v0[3];
          for (int i = 0; i < 3; i++) v0[i] = __ldcg(&R->v0[i]);
          chi = angle3(v0, vel);
          status |= COSIMS_TRAJ_SUCCESS;
          finished = true;
        }
      }
      if (!finished) {
        if (total >= cap || (!isfinite(rdot) && step != 0)) {
          status |= COSIMS_TRAJ_STEPCAP;
          finished = true;
        } else if (!(tries < max_tries && max_tries < 10)) {
          finished = true;
        } else if (step == 0) {
          phase = P_INIT_RETRY;
        }
      }
      if (finished) {
        if (wd.lane == 0) {
          cosims_traj_out o;
          o.chi = chi; o.de_pct = dE; o.steps = step;
          o.status = status | ((uint32_t)etries << COSIMS_TRAJ_ETRIES_SHIFT) |
                     ((uint32_t)otries << COSIMS_TRAJ_OTRIES_SHIFT);
          out[__ldcg(&R->t)] = o;
        }
        break;
      }
    }
  }
}

// Wide phase of one CTA: groups of ho.wide_lanes threads finish parked
// trajectories.  Called by every thread of the CTA after the narrow phase.
template <int TYPE>
__device__ __noinline__ void wide_phase(unsigned char *smem, uint32_t img_bytes, const View m,
                                        const View64 m64, const DevParams &p, int mode_stride,
                                        const Handoff &ho, cosims_traj_out *out,
                                        unsigned long long *counters) {
  const int WG = ho.wide_lanes;
  const int nwide = min((int)(blockDim.x / WG), 15);   // named barriers 1..15
  const int wg = threadIdx.x / WG;
  if (wg >= nwide) return;           // threads beyond whole wide groups sit out
  unsigned char *base = scratch_base(smem, img_bytes) + (size_t)wg * wide_group_bytes(WG, mode_stride);
  Wide wd;
  wd.WG = WG;
  wd.lane = threadIdx.x - wg * WG;
  wd.warp = wd.lane >> 5;
  wd.nwarps = WG >> 5;
  wd.bar = 1 + wg;
  wd.modes = base;
  wd.mode_stride = mode_stride;
  unsigned char *q = base + ((2u * (uint32_t)mode_stride + 15u) & ~15u);
  wd.fslots = reinterpret_cast<float *>(q);
  wd.dslots = reinterpret_cast<double *>(q + 2u * wd.nwarps * kWideSlotFloats * 4u);
  wd.bcast = reinterpret_cast<long long *>(q + 2u * wd.nwarps * kWideSlotFloats * 4u +
                                           2u * wd.nwarps * 4u * 8u);
  if (Traits<TYPE>::kClusters && wd.lane == 0) {
    wd.modes[m.nc] = 0;                      // the pad atoms' cluster, both halves
    wd.modes[mode_stride + m.nc] = 0;
  }
  wd.sync();
  Tally tl;
  unsigned long long nsteps = 0;
  uint32_t nforce = 0, npot = 0;
  const unsigned long long t0 = global_ns();
  wide_loop<TYPE>(m, m64, p, wd, ho, out, counters, tl, nsteps, nforce, npot);
  if (Traits<TYPE>::kVaryingPairs) {
    count_add(counters, C_PAIR_LJ, tl.lj);
    count_add(counters, C_PAIR_ES, tl.es);
    count_add(counters, C_FAR, tl.far);
  }
  count_add(counters, C_PAIR_ESNL, tl.nl);
  if (wd.lane == 0) {
    count_add(counters, C_WIDE_STEPS, (long long)nsteps);
    count_add(counters, C_WIDE_NS, (long long)(global_ns() - t0));
    count_add(counters, C_STEPS, (long long)nsteps);
    count_add(counters, C_FORCE_EVALS, nforce);
    count_add(counters, C_POT_EVALS, npot);
    count_add(counters, C_PAIR_POT, (long long)npot * m64.n);
    if (!Traits<TYPE>::kVaryingPairs)
      count_add(counters, Traits<TYPE>::kCharge ? C_PAIR_ES : C_PAIR_LJ,
                (long long)nforce * m64.n);
  }
}

// Threads per CTA at most: 768 gives 80 registers a thread, enough for the
// wide groups' register-resident state (the narrow phase runs as fast at 24
// warps per SM as at 32).  The far-field variants 1 and 2 take 640 threads
// and 96 registers: their packed far-field pass holds 12 packed sums and
// the multipole temporaries, which spill about 200 bytes a thread at 80
// (at 96 a few dozen; 640 threads measured faster than 512 at 128).
template <int TYPE>
struct KernelShape {
  static constexpr int kMaxThreads = (TYPE == 1 || TYPE == 2) ? kMixedFarBlock : kMixedMaxBlock;
};

// SMEM: the F32 image is staged in shared memory (else read from global
// memory through L1); a separate instantiation, so the pair loop's loads are
// shared-memory loads with 32-bit addresses.
// GT: lanes per trajectory fixed at compile time (4, 8, 16, 32), or 0 for
// the launch's group_lanes (1 and 2): a constant G unrolls the group sums and
// strides the pair loop by an immediate.
template <int TYPE, bool SMEM, int GT>
__global__ void __launch_bounds__(KernelShape<TYPE>::kMaxThreads, COSIMS_MIXED_MIN_BLOCKS)
    traj_mixed_kernel(const __grid_constant__ TrajArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ uint64_t bar;
  const unsigned char *base = a.img.gbase;
  if (SMEM) {
    if (!stage_to_smem(smem, a.img.gbase, a.img.bytes, &bar, 0, true, a.stage_limit)) {
      if (threadIdx.x == 0) atomicOr(a.counters + C_ERROR, 1ull);
      return;
    }
    base = smem;
  }
  if (threadIdx.x == 0) mark_first(a.counters, C_T_START_INV);
  const View m = make_view(base, a.img);
  const View64 m64 = make_view64(a.img64);
  const int G = GT > 0 ? GT : a.group_lanes;
  const uint32_t img_bytes = SMEM ? a.img.bytes : 0u;
  GroupState *S;
  uint8_t *modes;
  narrow_scratch(smem, img_bytes, G, a.mode_stride, S, modes);
  NarrowLanes ln;
  ln.G = G;
  ln.lane = threadIdx.x & (G - 1);
  ln.gmask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << ((threadIdx.x & 31) & ~(G - 1)));
  if (ln.lane == 0) {
    S->s.phase = P_ACQUIRE;
    group_counters_clear(*S);
    if (Traits<TYPE>::kClusters) modes[m.nc] = 0;    // the pad atoms' cluster
  }
  __syncwarp();
  const ArgsSource src{a};
  Tally tl;
  group_loop<TYPE>(m, m64, a.par, ln, modes, *S, src, tl);
  fold_tally<TYPE>(*S, tl);
  flush_nolj(tl, a.counters);
  __syncwarp();
  if (ln.lane == 0) flush_group<TYPE>(*S, m64.n, a.counters);
  if (a.ho.budget > 0) {
    __syncthreads();     // the narrow groups' scratch is reused
    wide_phase<TYPE>(smem, img_bytes, m, m64, a.par, a.mode_stride, a.ho, a.out, a.counters);
  }
  if ((threadIdx.x & 31) == 0) mark_last(a.counters, C_T_END);
}

}  // namespace mixed
}  // namespace cosims

namespace cosims {
namespace mixed {

template <int TYPE, bool SMEM, int GT>
int launch_t(const TrajArgs &a, int block, int grid, size_t smem, void *stream) {
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(traj_mixed_kernel<TYPE, SMEM, GT>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
  }
  traj_mixed_kernel<TYPE, SMEM, GT><<<grid, block, smem, (cudaStream_t)stream>>>(a);
  return (int)cudaGetLastError();
}

template <int TYPE, bool SMEM>
int launch_g(const TrajArgs &a, int block, int grid, size_t smem, void *stream) {
  switch (a.group_lanes) {
    case 4: return launch_t<TYPE, SMEM, 4>(a, block, grid, smem, stream);
    case 8: return launch_t<TYPE, SMEM, 8>(a, block, grid, smem, stream);
    case 16: return launch_t<TYPE, SMEM, 16>(a, block, grid, smem, stream);
    case 32: return launch_t<TYPE, SMEM, 32>(a, block, grid, smem, stream);
    default: return launch_t<TYPE, SMEM, 0>(a, block, grid, smem, stream);
  }
}

template <int TYPE>
int launch_type(const TrajArgs &a, int block, int grid, size_t smem, void *stream) {
  return a.use_smem ? launch_g<TYPE, true>(a, block, grid, smem, stream)
                    : launch_g<TYPE, false>(a, block, grid, smem, stream);
}

// Every instantiation has the same resource use up to its lane count, so the
// occupancy query uses the one the launch will take.
template <int TYPE, bool SMEM, int GT>
int occupancy_t(int block, size_t smem, int *per_sm) {
  if (block > KernelShape<TYPE>::kMaxThreads) { *per_sm = 0; return 0; }
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(traj_mixed_kernel<TYPE, SMEM, GT>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
  }
  return (int)cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      per_sm, traj_mixed_kernel<TYPE, SMEM, GT>, block, smem);
}

template <int TYPE>
int occupancy_type(int use_smem, int group_lanes, int block, size_t smem, int *per_sm) {
  switch (group_lanes) {
    case 4: return use_smem ? occupancy_t<TYPE, true, 4>(block, smem, per_sm)
                            : occupancy_t<TYPE, false, 4>(block, smem, per_sm);
    case 8: return use_smem ? occupancy_t<TYPE, true, 8>(block, smem, per_sm)
                            : occupancy_t<TYPE, false, 8>(block, smem, per_sm);
    case 16: return use_smem ? occupancy_t<TYPE, true, 16>(block, smem, per_sm)
                             : occupancy_t<TYPE, false, 16>(block, smem, per_sm);
    case 32: return use_smem ? occupancy_t<TYPE, true, 32>(block, smem, per_sm)
                             : occupancy_t<TYPE, false, 32>(block, smem, per_sm);
    default: return use_smem ? occupancy_t<TYPE, true, 0>(block, smem, per_sm)
                             : occupancy_t<TYPE, false, 0>(block, smem, per_sm);
  }
}

}  // namespace mixed
}  // namespace cosims
