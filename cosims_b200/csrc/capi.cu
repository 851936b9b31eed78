// capi.cu -- the C ABI (include/cosims_cuda.h): contexts, device images,
// launch sizing and the list / sampled run paths.
#include <cuda_runtime.h>
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "capi_internal.h"

namespace cosims {

static thread_local std::string g_last_error;

cosims_status fail(cosims_status s, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return s;
}

cosims_status cuda_fail(cudaError_t e, const char *what) {
  return fail(COSIMS_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

const char *last_error() { return g_last_error.c_str(); }

// ---- image building ----------------------------------------------------------

namespace {

struct Builder {
  std::vector<unsigned char> buf;
  uint32_t add(const void *src, size_t bytes) {
    size_t off = (buf.size() + 15) & ~size_t(15);
    buf.resize(off + bytes);
    if (bytes) std::memcpy(buf.data() + off, src, bytes);
    return (uint32_t)off;
  }
  void finish() { buf.resize((buf.size() + 15) & ~size_t(15)); }
};

}  // namespace

cosims_status validate(const cosims_molecule *mol, const cosims_params *par) {
  if (!mol || !par) return fail(COSIMS_ERR_INVALID, "molecule and params are required");
  if (mol->n_atoms <= 0 || mol->n_atoms > kMaxAtoms)
    return fail(COSIMS_ERR_UNSUPPORTED, "n_atoms %d outside 1..%d", mol->n_atoms, kMaxAtoms);
  if (!mol->x || !mol->y || !mol->z || !mol->charge || !mol->sig6 || !mol->eps24m || !mol->eps4)
    return fail(COSIMS_ERR_INVALID, "molecule arrays must not be NULL");
  if (par->force_type < 1 || par->force_type > 6)
    return fail(COSIMS_ERR_INVALID, "force_type %d outside 1..6", par->force_type);
  const bool uses = par->force_type != 4 && par->force_type != 6;
  if (mol->n_clusters < 0 || mol->n_clusters > kMaxClusters)
    return fail(COSIMS_ERR_UNSUPPORTED, "n_clusters %d outside 0..%d", mol->n_clusters,
                kMaxClusters);
  if (uses) {
    if (mol->n_clusters == 0)
      return fail(COSIMS_ERR_INVALID, "force_type %d needs clusters", par->force_type);
    if (!mol->cluster_offset || !mol->cluster_atoms || !mol->cluster_pos ||
        !mol->cluster_radius || !mol->cluster_charge || !mol->cluster_dipole ||
        !mol->cluster_quad || !mol->cluster_replaced)
      return fail(COSIMS_ERR_INVALID, "cluster arrays must not be NULL");
    if (mol->cluster_offset[0] != 0 || mol->cluster_offset[mol->n_clusters] != mol->n_atoms)
      return fail(COSIMS_ERR_INVALID, "cluster offsets must run from 0 to n_atoms");
    std::vector<char> seen(mol->n_atoms, 0);
    for (int c = 0; c < mol->n_clusters; c++) {
      if (mol->cluster_offset[c + 1] < mol->cluster_offset[c])
        return fail(COSIMS_ERR_INVALID, "cluster offsets must not decrease");
      for (int k = mol->cluster_offset[c]; k < mol->cluster_offset[c + 1]; k++) {
        int a = mol->cluster_atoms[k];
        if (a < 0 || a >= mol->n_atoms || seen[a])
          return fail(COSIMS_ERR_INVALID, "clusters must partition the atoms");
        seen[a] = 1;
      }
    }
  }
  // non-finite atom data would make every trajectory non-finite (the
  // reference reads such input unchecked and integrates NaN)
  for (int i = 0; i < mol->n_atoms; i++) {
    if (!std::isfinite(mol->x[i]) || !std::isfinite(mol->y[i]) || !std::isfinite(mol->z[i]) ||
        !std::isfinite(mol->charge[i]) || !std::isfinite(mol->sig6[i]) ||
        !std::isfinite(mol->eps24m[i]) || !std::isfinite(mol->eps4[i]))
      return fail(COSIMS_ERR_INVALID, "atom %d has a non-finite coordinate or parameter", i);
  }
  if (uses) {
    for (int c = 0; c < mol->n_clusters; c++) {
      bool fin = std::isfinite(mol->cluster_radius[c]) && std::isfinite(mol->cluster_charge[c]);
      for (int k = 0; k < 3; k++)
        fin = fin && std::isfinite(mol->cluster_pos[3 * c + k]) &&
              std::isfinite(mol->cluster_dipole[3 * c + k]);
      for (int k = 0; k < 9; k++) fin = fin && std::isfinite(mol->cluster_quad[9 * c + k]);
      if (!fin) return fail(COSIMS_ERR_INVALID, "cluster %d has a non-finite value", c);
    }
  }
  if (!(par->dt > 0) || !(par->mu > 0) || !(par->ell_a > 0) || !(par->ell_b > 0) ||
      !(par->ell_c > 0))
    return fail(COSIMS_ERR_INVALID, "dt, mu and the ellipsoid axes must be positive");
  if (!std::isfinite(par->dt) || !std::isfinite(par->mu) || !std::isfinite(par->ell_a) ||
      !std::isfinite(par->ell_b) || !std::isfinite(par->ell_c) || !std::isfinite(par->b_max) ||
      !std::isfinite(par->g_min) || !std::isfinite(par->g_max) ||
      !std::isfinite(par->ccs_const) || !std::isfinite(par->dipole_scalar))
    return fail(COSIMS_ERR_INVALID, "the path scalars must be finite");
  if (par->multipole_order < 0 || par->multipole_order > 2)
    return fail(COSIMS_ERR_INVALID, "multipole_order must be 0, 1 or 2");
  return COSIMS_OK;
}

DevParams make_dev_params(const cosims_params *p) {
  DevParams d;
  std::memset(&d, 0, sizeof d);
  d.force_type = p->force_type;
  d.multipole_order = p->multipole_order;
  d.projection = p->projection;
  d.charged = p->charged;
  d.dt = p->dt; d.mu = p->mu; d.dipole_scalar = p->dipole_scalar;
  d.r_disp = p->r_disp; d.r_mp = p->r_mp;
  d.ell_a = p->ell_a; d.ell_b = p->ell_b; d.ell_c = p->ell_c;
  d.inv_ell_a = 1.0 / p->ell_a; d.inv_ell_b = 1.0 / p->ell_b; d.inv_ell_c = 1.0 / p->ell_c;
  d.max_rad = std::max(p->ell_a, std::max(p->ell_b, p->ell_c));   // diffEqSolver.cpp:99
  d.b_max = p->b_max; d.start_dist = p->start_dist;
  d.g_min = p->g_min; d.g_max = p->g_max;
  d.vdist_a = p->vdist_a; d.vdist_norm = p->vdist_norm; d.vdist_max = p->vdist_max;
  d.ccs_const = p->ccs_const;
  d.max_steps = p->max_steps;
  return d;
}

void build_images(const cosims_molecule *m, const cosims_params *p, HostImage &h64,
                  HostImage &h32) {
  const int n = m->n_atoms;
  const bool uses = p->force_type != 4 && p->force_type != 6;
  const int nc = uses ? m->n_clusters : 0;
  std::vector<int> order(n), perm(n), cid(n, 0), coff(nc + 1, 0);
  if (uses) {
    for (int c = 0; c < nc; c++) {
      coff[c + 1] = m->cluster_offset[c + 1];
      for (int k = m->cluster_offset[c]; k < m->cluster_offset[c + 1]; k++) {
        order[k] = m->cluster_atoms[k];
        cid[k] = c;
      }
    }
  } else {
    for (int i = 0; i < n; i++) order[i] = i;
  }
  for (int k = 0; k < n; k++) perm[order[k]] = k;

  // F32 slot of each force-order atom: in order, or cluster-blocked (each
  // cluster from a block start, whole blocks, then one block of padding)
  const bool blocked = uses && blocked_layout(p->force_type);
  std::vector<int> slot_of(n), c_slot0(nc + 1, 0);
  int used = n;
  if (blocked) {
    int sidx = 0;
    for (int c = 0; c < nc; c++) {
      c_slot0[c] = sidx;
      for (int k = coff[c]; k < coff[c + 1]; k++) slot_of[k] = sidx + (k - coff[c]);
      const int sz = coff[c + 1] - coff[c];
      sidx += (sz + kClusterBlock - 1) / kClusterBlock * kClusterBlock;
    }
    c_slot0[nc] = sidx;
    used = sidx + kClusterBlock;
  } else {
    for (int k = 0; k < n; k++) slot_of[k] = k;
  }
  // F32 arrays padded to a multiple of kSlotQuantum with inert atoms
  const int ns = (used + kSlotQuantum - 1) / kSlotQuantum * kSlotQuantum;
  std::vector<AtomF64> a64(n);
  std::vector<float4> a4(ns, make_float4(kPadCoord, kPadCoord, kPadCoord, 0.0f));
  // second record: sigma^6, 24 eps/mu, cluster id (integer bits), 0; pad atoms
  // belong to cluster nc, whose mode is always 0
  std::vector<float4> b4(ns, make_float4(0.0f, 0.0f, 0.0f, 0.0f));
  uint32_t pad_cid = (uint32_t)nc;
  float pad_cid_f;
  std::memcpy(&pad_cid_f, &pad_cid, 4);
  for (int k = 0; k < ns; k++) b4[k].z = pad_cid_f;
  for (int k = 0; k < n; k++) {
    const int i = order[k];
    AtomF64 &A = a64[k];
    A.x = m->x[i]; A.y = m->y[i]; A.z = m->z[i]; A.q = m->charge[i];
    A.sig6 = m->sig6[i]; A.eps24m = m->eps24m[i]; A.eps4 = m->eps4[i];
    const int sl = slot_of[k];
    a4[sl] = make_float4((float)A.x, (float)A.y, (float)A.z, (float)A.q);
    uint32_t ck = (uint32_t)cid[k];
    float ck_f;
    std::memcpy(&ck_f, &ck, 4);
    b4[sl] = make_float4((float)A.sig6, (float)A.eps24m, ck_f, 1.0f);
  }
  std::vector<ClusterF64> c64(nc);
  // F32 records: the clusters, then the null cluster (zero moments, centre
  // 1e4 A away on each axis: its far-field terms are exactly zero)
  std::vector<ClusterF32> c32(nc + 1);
  {
    ClusterF32 &Z = c32[nc];
    std::memset(&Z, 0, sizeof Z);
    Z.cx = Z.cy = Z.cz = 1.0e4;
  }
  for (int c = 0; c < nc; c++) {
    ClusterF64 &C = c64[c];
    std::memset(&C, 0, sizeof C);
    C.cx = m->cluster_pos[3 * c]; C.cy = m->cluster_pos[3 * c + 1];
    C.cz = m->cluster_pos[3 * c + 2];
    double a = p->r_mp + m->cluster_radius[c];      // forceAccel.cpp:253-256
    a *= a;
    double b = p->r_disp + m->cluster_radius[c];
    b *= b;
    C.mpr2 = a; C.dr2 = b;
    C.q = m->cluster_charge[c];
    for (int k = 0; k < 3; k++) C.dip[k] = m->cluster_dipole[3 * c + k];
    for (int k = 0; k < 9; k++) C.quad[k] = m->cluster_quad[9 * c + k];
    // multipoleCutoff's far band reads atom index n = the cluster index
    C.qsig6 = c < n ? m->sig6[c] : 0.0;
    C.qeps = c < n ? m->eps24m[c] : 0.0;
    C.a0 = coff[c]; C.a1 = coff[c + 1];
    C.replaced = m->cluster_replaced[c];
    ClusterF32 &F = c32[c];
    std::memset(&F, 0, sizeof F);
    F.cx = C.cx; F.cy = C.cy; F.cz = C.cz; F.mpr2 = C.mpr2; F.dr2 = C.dr2;
    F.q = (float)C.q;
    // a replaced cluster has no dipole term (forceAccel.cpp:258-337)
    for (int k = 0; k < 3; k++) F.dip[k] = C.replaced ? 0.0f : (float)C.dip[k];
    for (int k = 0; k < 9; k++) F.quad[k] = (float)C.quad[k];
    F.qsig6 = (float)C.qsig6; F.qeps = (float)C.qeps;
    F.replaced = C.replaced;
    F.a0 = blocked ? c_slot0[c] : C.a0;
    F.a1 = blocked ? c_slot0[c + 1] : C.a1;
    F.n_atoms = C.a1 - C.a0;
  }

  Builder b64;
  MolImage &i64 = h64.img;
  std::memset(&i64, 0, sizeof i64);
  i64.off[S_ATOMS] = b64.add(a64.data(), sizeof(AtomF64) * n);
  i64.off[S_PERM] = b64.add(perm.data(), 4 * n);
  i64.off[S_CLUSTERS] = b64.add(c64.data(), sizeof(ClusterF64) * nc);
  // event slots of the plain form's exact wide phase, in the serial order
  std::vector<int32_t> slots;
  const bool far_events = p->force_type == 1 || p->force_type == 2;
  if (uses) {
    for (int c = 0; c < nc; c++) {
      if (far_events)                  // the far field's three parts, in order
        for (int part = 0; part < 3; part++) { slots.push_back(-1 - part); slots.push_back(c); }
      for (int k = coff[c]; k < coff[c + 1]; k++) { slots.push_back(k); slots.push_back(c); }
    }
  } else {
    for (int k = 0; k < n; k++) { slots.push_back(k); slots.push_back(0); }
  }
  i64.off[S_SLOTS] = b64.add(slots.data(), 4 * slots.size());
  b64.finish();
  i64.bytes = (uint32_t)b64.buf.size();
  i64.n_atoms = n;
  i64.n_slots = (int)(slots.size() / 2);      // exact-phase events
  i64.n_clusters = nc;
  i64.uses_clusters = uses ? 1 : 0;
  h64.bytes = std::move(b64.buf);

  Builder b32;
  MolImage &i32 = h32.img;
  std::memset(&i32, 0, sizeof i32);
  if (paired_layout(p->force_type)) {
    // slots 2j and 2j+1 side by side: [np x (x,x,y,y)][np x (z,z,q,q)][np x (s,s,e,e)][np x cids]
    const int np = ns / 2;
    std::vector<unsigned char> pairs((size_t)np * (3 * sizeof(float4) + sizeof(uint2)));
    float4 *pa = reinterpret_cast<float4 *>(pairs.data());
    float4 *pb = pa + np, *pl = pb + np;
    uint2 *pc = reinterpret_cast<uint2 *>(pl + np);
    for (int j = 0; j < np; j++) {
      const float4 &u = a4[2 * j], &v = a4[2 * j + 1], &s = b4[2 * j], &t = b4[2 * j + 1];
      pa[j] = make_float4(u.x, v.x, u.y, v.y);
      pb[j] = make_float4(u.z, v.z, u.w, v.w);
      pl[j] = make_float4(s.x, t.x, s.y, t.y);
      uint32_t c0, c1;
      std::memcpy(&c0, &s.z, 4);
      std::memcpy(&c1, &t.z, 4);
      pc[j] = make_uint2(c0, c1);
    }
    i32.off[S_PAIRS] = b32.add(pairs.data(), pairs.size());
  } else {
    i32.off[S_ATOMS] = b32.add(a4.data(), sizeof(float4) * ns);
    i32.off[S_LJ] = b32.add(b4.data(), sizeof(float4) * ns);
  }
  i32.off[S_CLUSTERS] = b32.add(c32.data(), sizeof(ClusterF32) * (nc + 1));
  if (p->force_type == 1 || p->force_type == 2) {
    // far-field table: clusters 2j, 2j+1 side by side (see engine.h)
    const int nfp = far_table_pairs(nc);
    std::vector<float4> ft((size_t)kFarTableArrays * nfp);
    for (int j = 0; j < nfp; j++) {
      // per cluster: -x_hi, -y_hi, -z_hi, -x_lo, -y_lo, -z_lo, mpr2, dr2, q, dipole;
      // a null entry sits 1e4 A out with zero moments and radii -1
      float v[12][2];
      for (int h = 0; h < 2; h++) {
        const int c = 2 * j + h;
        float w[12] = {-1.0e4f, -1.0e4f, -1.0e4f, 0.0f, 0.0f, 0.0f, -1.0f, -1.0f,
                       0.0f, 0.0f, 0.0f, 0.0f};
        if (c < nc) {
          const ClusterF32 &F = c32[c];
          const double ctr[3] = {F.cx, F.cy, F.cz};
          for (int k = 0; k < 3; k++) {
            const float hi = (float)ctr[k];
            w[k] = -hi;
            w[3 + k] = -(float)(ctr[k] - (double)hi);
          }
          w[6] = (float)F.mpr2;
          w[7] = (float)F.dr2;
          w[8] = F.q;
          for (int k = 0; k < 3; k++) w[9 + k] = F.dip[k];
        }
        for (int k = 0; k < 12; k++) v[k][h] = w[k];
      }
      // value pairs (2a, 2a+1) of the two clusters in array a:
      // (x_hi, y_hi), (z_hi, x_lo), (y_lo, z_lo), (mpr2, dr2), (q, dip_x), (dip_y, dip_z)
      for (int a = 0; a < kFarTableArrays; a++)
        ft[(size_t)a * nfp + j] = make_float4(v[2 * a][0], v[2 * a][1], v[2 * a + 1][0],
                                              v[2 * a + 1][1]);
    }
    i32.off[S_FAR] = b32.add(ft.data(), sizeof(float4) * ft.size());
  }
  b32.finish();
  i32.bytes = (uint32_t)b32.buf.size();
  i32.n_atoms = n;
  i32.n_slots = ns;
  i32.n_clusters = nc;
  i32.uses_clusters = uses ? 1 : 0;
  h32.bytes = std::move(b32.buf);
}

// ---- device helpers ------------------------------------------------------------

cosims_status check_device(int device, int *sm_count, int *max_smem) {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0)
    return fail(COSIMS_ERR_UNSUPPORTED, "no CUDA device: %s", cudaGetErrorString(e));
  if (device < 0 || device >= count)
    return fail(COSIMS_ERR_INVALID, "device %d outside 0..%d", device, count - 1);
  cudaDeviceProp prop;
  e = cudaGetDeviceProperties(&prop, device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceProperties");
  if (prop.major != 10)
    return fail(COSIMS_ERR_UNSUPPORTED, "device %d is sm_%d%d; this build targets sm_100a",
                device, prop.major, prop.minor);
  *sm_count = prop.multiProcessorCount;
  *max_smem = (int)prop.sharedMemPerBlockOptin;
  return COSIMS_OK;
}

DeviceGuard::DeviceGuard(int dev) {
  cudaGetDevice(&prev);
  if (prev != dev) cudaSetDevice(dev);
}
DeviceGuard::~DeviceGuard() { cudaSetDevice(prev); }

template <typename T>
static cosims_status grow(T **p, int64_t *cap, int64_t need) {
  if (*cap >= need) return COSIMS_OK;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  int64_t n = std::max<int64_t>(need, 1024);
  cudaError_t e = cudaMalloc((void **)p, sizeof(T) * (size_t)n);
  if (e != cudaSuccess) return fail(COSIMS_ERR_NOMEM, "cudaMalloc of %lld bytes: %s",
                                    (long long)(sizeof(T) * n), cudaGetErrorString(e));
  *cap = n;
  return COSIMS_OK;
}

// Shared-memory bytes of one mixed-form group: its trajectory state and its
// cluster-mode scratch (n_clusters + 1 bytes: the last entry, always 0,
// belongs to the pad atoms).
int mode_stride_for(const MolImage &img, int force_type) {
  if (!img.uses_clusters) return 0;
  // variants 1, 2, 5 keep a 4-byte entry per cluster (the list of clusters
  // that add pair terms) and variant 3 a 4-byte cut-off factor per cluster;
  // the others one mode byte per cluster; plus the pad atoms' cluster
  const int per = (force_type == 1 || force_type == 2 || force_type == 3 || force_type == 5) ? 4 : 1;
  int s = ((img.n_clusters + 1) * per + 3) & ~3;
  if (((s / 4) & 1) == 0) s += 4;     // odd word count: groups hit distinct banks
  return s;
}

// Launch shape: threads per CTA, CTAs, dynamic shared memory, whether the
// image is staged, and the per-group mode scratch.  block_threads 0 (mixed
// form) picks the CTA size (256, 512 or 768 threads; 256, 512 or 640 for the
// far-field variants 1 and 2: the occupancy query refuses more) that keeps the
// most threads resident per SM, preferring a staged image: one staged copy of
// the molecule serves every group of a CTA.
cosims_status shape_for(bool plain, const MolImage &img, int G, int block_threads,
                        int wide_lanes, int force_type, int sm_count, int max_smem, int64_t n,
                        LaunchShape &ls) {
  const int budget = max_smem - 1024;
  const int stride = plain ? 0 : mode_stride_for(img, force_type);
  const size_t per_group = plain ? 0 : (size_t)kGroupStateBytes + (size_t)stride;
  const size_t per_wide = wide_lanes <= 0 ? 0
                         : plain ? exact_scratch_bytes(force_type, img.n_clusters)
                                 : wide_group_bytes(wide_lanes, stride);
  const size_t img_bytes = (img.bytes + 15u) & ~15u;
  int cands[4] = {block_threads, 0, 0, 0};
  int ncand = 1;
  if (!plain && block_threads == 0) {
    cands[0] = 256; cands[1] = 512; cands[2] = kMixedMaxBlock;
    ncand = 3;
    // variants 1 and 2 run at most kMixedFarBlock threads (96 registers)
    if (force_type == 1 || force_type == 2) cands[ncand++] = kMixedFarBlock;
  }
  bool found = false;
  int best_resident = -1;
  for (int ci = 0; ci < ncand; ci++) {
    for (int staged = 1; staged >= 0; staged--) {   // staged image first, then read from L2
      int block = cands[ci];
      if (block < G) continue;
      if (staged && (int)img_bytes > budget) continue;
      LaunchShape t;
      t.use_smem = staged;
      t.mode_stride = stride;
      // shrink the CTA until image + group scratch fit
      bool ok = true;
      for (;;) {
        size_t scratch = (size_t)(block / G) * per_group;
        if (plain) {
          // plain form: one exact wide group per CTA, which must be kPlainBlock threads
          t.wide_lanes = (per_wide && block == kPlainBlock) ? kPlainBlock : 0;
          if (t.wide_lanes) scratch = per_wide;
        } else {
          // wide phase: whole wide groups only, at most 15 (named barriers 1..15);
          // threads beyond them sit the phase out
          t.wide_lanes = (per_wide && block >= wide_lanes) ? wide_lanes : 0;
          if (t.wide_lanes)
            scratch = std::max(scratch, (size_t)std::min(block / wide_lanes, 15) * per_wide);
        }
        size_t smem = (t.use_smem ? img_bytes : 0) + scratch;
        if ((int)smem <= budget) { t.smem = smem; break; }
        if (block <= std::max(G, 32)) { ok = false; break; }
        block /= 2;
      }
      if (!ok) continue;
      t.block = block;
      int per_sm = 0;
      int rc = plain ? plain_occupancy(force_type, block, t.smem, &per_sm)
                     : mixed_occupancy(force_type, t.use_smem, G, block, t.smem, &per_sm);
      if (rc != 0) {
        cudaGetLastError();             // a refused shared-memory size: try the next shape
        continue;
      }
      if (per_sm <= 0) continue;        // over the kernel's thread, register or smem limit
      // mixed form: a staged image counts double (one copy serves a CTA's many
      // groups from shared memory); plain form: every lane of a warp reads the
      // same atom, a broadcast that L1 serves as well, so the most resident
      // threads win (the staged shape on a tie)
      // a shape that keeps the requested long-trajectory hand-off beats one
      // that drops it (a CTA shrunk below the wide group size has none)
      const bool keeps_wide = !per_wide || t.wide_lanes > 0;
      const int resident = per_sm * block * (t.use_smem && !plain ? 2 : 1) +
                           (keeps_wide ? (1 << 24) : 0);
      if (resident > best_resident) {
        best_resident = resident;
        t.grid = per_sm;                // CTAs per SM until the grid is sized below
        ls = t;
        found = true;
      }
      // staged works: no need to try unstaged, unless staging dropped the hand-off
      if (per_sm > 0 && !plain && keeps_wide) break;
    }
  }
  if (!found) return fail(COSIMS_ERR_UNSUPPORTED, "molecule image does not fit in shared memory");
  const int64_t groups_per_cta = ls.block / G;
  int64_t grid = (int64_t)ls.grid * sm_count;
  grid = std::min<int64_t>(grid, (n + groups_per_cta - 1) / groups_per_cta);
  ls.grid = (int)std::max<int64_t>(grid, 1);
  return COSIMS_OK;
}

int ctx_wide_lanes(const cosims_ctx *c) {
  if (c->ho_budget <= 0) return 0;
  if (c->precision == COSIMS_PRECISION_PLAIN_F64) return kPlainBlock;   // the whole CTA
  return c->ho_wide > 0 ? c->ho_wide : default_wide_lanes(c->n_atoms);
}

cosims_status launch_shape(const cosims_ctx *c, int64_t n, LaunchShape &ls) {
  const bool plain = c->precision == COSIMS_PRECISION_PLAIN_F64;
  return shape_for(plain, plain ? c->img64 : c->img32, plain ? 1 : c->group_lanes,
                   c->block_threads, ctx_wide_lanes(c), c->par.force_type, c->sm_count,
                   c->max_smem, n, ls);
}

// Hand-off buffers for n trajectories: a record for every trajectory, so a
// park never fails and which trajectories go wide depends on them alone (a
// smaller array would fill in timing order).  Above kHandoffMaxRecords
// trajectories a call runs without hand-off.  Ready flags and counters are
// cleared on the stream.
constexpr int64_t kHandoffMaxRecords = 1 << 22;    // 800 MiB of records
constexpr int64_t kTraceMaxBytes = int64_t(1) << 32;  // frames of one cosims_trace_list call

// Hand-off records for calls of up to n trajectories (allocated once, kept).
cosims_status handoff_grow(cosims_ctx *c, int64_t n) {
  const int64_t want = std::max<int64_t>(n, 256);
  if (c->ho_cap < want) {
    cudaFree(c->d_ho_states);
    cudaFree(c->d_ho_ready);
    c->d_ho_states = nullptr;
    c->d_ho_ready = nullptr;
    c->ho_cap = 0;
    cudaError_t e = cudaMalloc((void **)&c->d_ho_states, sizeof(TrajState) * (size_t)want);
    if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_ho_ready, sizeof(uint32_t) * (size_t)want);
    if (e != cudaSuccess) return fail(COSIMS_ERR_NOMEM, "hand-off buffers: %s", cudaGetErrorString(e));
    c->ho_cap = want;
  }
  if (!c->d_ho_ctrl) {
    cudaError_t e = cudaMalloc((void **)&c->d_ho_ctrl, 2 * sizeof(unsigned long long));
    if (e != cudaSuccess) return fail(COSIMS_ERR_NOMEM, "hand-off counters: %s", cudaGetErrorString(e));
  }
  return COSIMS_OK;
}

cosims_status handoff_prepare(cosims_ctx *c, int64_t n, const LaunchShape &ls, Handoff &ho,
                              cudaStream_t s) {
  std::memset(&ho, 0, sizeof ho);
  if (!ls.wide_lanes || n == 0 || n > kHandoffMaxRecords) return COSIMS_OK;
  cosims_status st = handoff_grow(c, n);
  if (st != COSIMS_OK) return st;
  cudaError_t e = cudaMemsetAsync(c->d_ho_ready, 0, sizeof(uint32_t) * (size_t)c->ho_cap, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->d_ho_ctrl, 0, 2 * sizeof(unsigned long long), s);
  if (e != cudaSuccess) return cuda_fail(e, "hand-off reset");
  ho.states = c->d_ho_states;
  ho.ready = c->d_ho_ready;
  ho.reserve = c->d_ho_ctrl;
  ho.taken = c->d_ho_ctrl + 1;
  ho.cap = c->ho_cap;
  ho.budget = c->ho_budget;
  ho.wide_lanes = ls.wide_lanes;
  ho.spin_limit = c->test_spin_limit ? c->test_spin_limit : kHandoffSpinLimit;
  ho.withhold_first = (c->test_flags & COSIMS_WAIT_TEST_HANDOFF) ? 1u : 0u;
  return COSIMS_OK;
}

cosims_status run_core(cosims_ctx *c, const double *d_pos0, const double *d_vel0,
                       const int32_t *d_hit, int64_t n, cosims_traj_out *d_out, void *stream,
                       double *d_trace = nullptr, int32_t *d_trace_n = nullptr,
                       int32_t trace_cap = 0, bool clear_error = true) {
  LaunchShape ls;
  cosims_status st = launch_shape(c, n, ls);
  if (st != COSIMS_OK) return st;
  if (n > INT32_MAX) return fail(COSIMS_ERR_UNSUPPORTED, "at most 2^31-1 trajectories per call");
  cudaStream_t s = (cudaStream_t)stream;
  // longest-first work order (slow start speeds first)
  st = grow(&c->d_order, &c->order_cap, n);
  if (st == COSIMS_OK) st = grow(&c->d_order_scratch, &c->order_scratch_cap, order_scratch_len());
  if (st != COSIMS_OK) return st;
  if (n > 0) {
    int orc = order_launch(c->par, d_vel0, d_hit, n, c->d_order, c->d_order_scratch, stream);
    if (orc != 0) return cuda_fail((cudaError_t)orc, "work-order launch");
  }
  cudaError_t e = cudaMemsetAsync(c->d_queue, 0, sizeof(unsigned long long), s);
  // the error flags stay set across the launches of one multi-launch call
  if (e == cudaSuccess)
    e = cudaMemsetAsync(c->d_counters, 0, sizeof(unsigned long long) * C_ERROR, s);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(c->d_counters + (clear_error ? C_ERROR : C_ERROR + 1), 0,
                        sizeof(unsigned long long) * (C_COUNT - C_ERROR - (clear_error ? 0 : 1)), s);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync");
  if (n == 0) return COSIMS_OK;
  TrajArgs a;
  std::memset(&a, 0, sizeof a);
  const bool plain = c->precision == COSIMS_PRECISION_PLAIN_F64;
  a.img = plain ? c->img64 : c->img32;
  a.img64 = c->img64;
  a.par = c->par;
  a.group_lanes = plain ? 1 : c->group_lanes;
  a.use_smem = ls.use_smem;
  a.mode_stride = ls.mode_stride;
  a.stage_limit = (c->test_flags & COSIMS_WAIT_TEST_STAGING) ? 0u : kStageSpinLimit;
  a.pos0 = d_pos0;
  a.vel0 = d_vel0;
  a.hit = d_hit;
  a.order = c->d_order;
  a.n = n;
  a.out = d_out;
  a.queue = c->d_queue;
  a.counters = c->d_counters;
  if (d_trace) {                    // a traced call integrates in the one-thread loop only
    a.trace = d_trace;
    a.trace_n = d_trace_n;
    a.trace_cap = trace_cap;
  } else {
    st = handoff_prepare(c, n, ls, a.ho, s);
    if (st != COSIMS_OK) return st;
  }
  if (!c->ev0) {
    e = cudaEventCreate(&c->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&c->ev1);
    if (e != cudaSuccess) return cuda_fail(e, "cudaEventCreate");
  }
  cudaEventRecord(c->ev0, s);
  int rc = plain ? plain_launch(a, ls.block, ls.grid, ls.smem, stream)
                 : mixed_launch(a, ls.block, ls.grid, ls.smem, stream);
  if (rc != 0) return cuda_fail((cudaError_t)rc, "trajectory kernel launch");
  cudaEventRecord(c->ev1, s);
  c->timed = true;
  c->last_shape = ls;
  return COSIMS_OK;
}

// Start states of trajectories first..first+n-1 into the context's buffers
// (one sampler kernel: the trajectory kernels only read them).
cosims_status sample_into(cosims_ctx *c, uint64_t seed, int64_t first, int64_t n,
                          bool keep_inputs, void *stream) {
  cosims_status st = grow(&c->d_out, &c->out_cap, n);
  if (st == COSIMS_OK) st = grow(&c->d_in, &c->in_cap, n);
  if (st == COSIMS_OK) st = grow(&c->d_pos0, &c->list_cap, 3 * n);
  if (st == COSIMS_OK) st = grow(&c->d_vel0, &c->vel_cap, 3 * n);
  if (st == COSIMS_OK) st = grow(&c->d_hit, &c->hit_cap, n);
  if (st != COSIMS_OK) return st;
  (void)keep_inputs;
  int rc = sample_launch(c->par, seed, first, n, c->d_in, c->d_pos0, c->d_vel0, c->d_hit, stream);
  if (rc != 0) return cuda_fail((cudaError_t)rc, "sampler launch");
  return COSIMS_OK;
}

cosims_status check_error_flag(cosims_ctx *c, cudaStream_t s) {
  unsigned long long flag = 0;
  cudaError_t e = cudaMemcpyAsync(&flag, c->d_counters + C_ERROR, sizeof flag,
                                  cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "trajectory run");
  if (flag)
    return fail(COSIMS_ERR_TIMEOUT, "a bounded device wait gave up:%s%s (flags %llu)",
                (flag & 1ull) ? " shared-memory staging" : "",
                (flag & 2ull) ? " long-trajectory hand-off record" : "", flag);
  return COSIMS_OK;
}

}  // namespace cosims

using namespace cosims;

extern "C" {

int32_t cosims_abi_version(void) { return COSIMS_ABI_VERSION; }

const char *cosims_last_error(void) { return cosims::last_error(); }

int32_t cosims_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
  return n;
}

cosims_status cosims_ctx_create(const cosims_molecule *mol, const cosims_params *par,
                                int32_t precision, int32_t device, cosims_ctx **out) {
  if (!out) return fail(COSIMS_ERR_INVALID, "out is NULL");
  *out = nullptr;
  if (precision != COSIMS_PRECISION_PLAIN_F64 && precision != COSIMS_PRECISION_MIXED)
    return fail(COSIMS_ERR_INVALID, "unknown precision %d", precision);
  cosims_status st = validate(mol, par);
  if (st != COSIMS_OK) return st;
  int sm = 0, smem = 0;
  st = check_device(device, &sm, &smem);
  if (st != COSIMS_OK) return st;
  DeviceGuard g(device);
  cosims_ctx *c = new cosims_ctx();
  c->device = device;
  c->precision = precision;
  c->sm_count = sm;
  c->max_smem = smem;
  c->par = make_dev_params(par);
  c->n_atoms = mol->n_atoms;
  build_images(mol, par, c->h64, c->h32);
  c->img64 = c->h64.img;
  c->img32 = c->h32.img;
  c->group_lanes = precision == COSIMS_PRECISION_PLAIN_F64 ? 1 : default_group_lanes(mol->n_atoms);
  c->block_threads = precision == COSIMS_PRECISION_PLAIN_F64 ? 128 : 0;   // 0: chosen per run
  if (precision == COSIMS_PRECISION_PLAIN_F64) c->ho_budget = default_plain_budget(mol->n_atoms);
  cudaError_t e = cudaMalloc((void **)&c->d_img64, c->img64.bytes);
  if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_img32, c->img32.bytes);
  if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_queue, sizeof(unsigned long long));
  if (e == cudaSuccess)
    e = cudaMalloc((void **)&c->d_counters, sizeof(unsigned long long) * C_COUNT);
  if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_sums, sizeof(cosims_ccs_sums));
  if (e == cudaSuccess)
    e = cudaMemcpy(c->d_img64, c->h64.bytes.data(), c->img64.bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(c->d_img32, c->h32.bytes.data(), c->img32.bytes, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cosims_ctx_destroy(c);
    return fail(COSIMS_ERR_NOMEM, "context allocation: %s", cudaGetErrorString(e));
  }
  c->img64.gbase = c->d_img64;
  c->img32.gbase = c->d_img32;
  st = grow(&c->d_red, &c->red_cap, reduce_scratch_len(0));
  if (st != COSIMS_OK) { cosims_ctx_destroy(c); return st; }
  *out = c;
  return COSIMS_OK;
}

void cosims_ctx_destroy(cosims_ctx *c) {
  if (!c) return;
  DeviceGuard g(c->device);
  cudaFree(c->d_img64);
  cudaFree(c->d_img32);
  cudaFree(c->d_queue);
  cudaFree(c->d_counters);
  cudaFree(c->d_sums);
  cudaFree(c->d_sums_many);
  cudaFree(c->d_out);
  cudaFree(c->d_in);
  cudaFree(c->d_pos0);
  cudaFree(c->d_vel0);
  cudaFree(c->d_red);
  cudaFree(c->d_hit);
  cudaFree(c->d_order);
  cudaFree(c->d_order_scratch);
  cudaFree(c->d_ho_states);
  cudaFree(c->d_ho_ready);
  cudaFree(c->d_ho_ctrl);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  delete c;
}

cosims_status cosims_ctx_kernel_ms(cosims_ctx *c, float *ms) {
  if (!c || !ms) return fail(COSIMS_ERR_INVALID, "ctx and ms are required");
  if (!c->timed) return fail(COSIMS_ERR_INVALID, "no trajectory kernel has run on this context");
  DeviceGuard g(c->device);
  cudaError_t e = cudaEventSynchronize(c->ev1);
  if (e == cudaSuccess) e = cudaEventElapsedTime(ms, c->ev0, c->ev1);
  if (e != cudaSuccess) return cuda_fail(e, "kernel timing");
  return COSIMS_OK;
}

cosims_status cosims_ctx_kernel_timeline(cosims_ctx *c, double *drain_ms, double *end_ms) {
  if (!c) return fail(COSIMS_ERR_INVALID, "ctx is NULL");
  if (!c->timed) return fail(COSIMS_ERR_INVALID, "no trajectory kernel has run on this context");
  DeviceGuard g(c->device);
  unsigned long long t[3];
  cudaError_t e = cudaEventSynchronize(c->ev1);
  if (e == cudaSuccess)
    e = cudaMemcpy(t, c->d_counters + C_T_START_INV, sizeof t, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "kernel timeline");
  const unsigned long long t0 = ~t[0], td = ~t[1], te = t[2];
  if (drain_ms) *drain_ms = t[1] ? (double)(long long)(td - t0) * 1e-6 : 0.0;
  if (end_ms) *end_ms = (double)(long long)(te - t0) * 1e-6;
  return COSIMS_OK;
}

cosims_status cosims_ctx_set_handoff(cosims_ctx *c, int64_t step_budget, int32_t wide_lanes) {
  if (!c) return fail(COSIMS_ERR_INVALID, "ctx is NULL");
  const bool plain = c->precision == COSIMS_PRECISION_PLAIN_F64;
  if (plain && wide_lanes != 0 && wide_lanes != kPlainBlock)
    return fail(COSIMS_ERR_INVALID, "the plain form's wide group is its %d-thread CTA", kPlainBlock);
  if (wide_lanes < 0 || wide_lanes > 512 || (wide_lanes & 31))
    return fail(COSIMS_ERR_INVALID, "wide_lanes must be 0 or a multiple of 32 up to 512");
  const int64_t dflt = plain ? default_plain_budget(c->n_atoms) : kDefaultHandoffBudget;
  c->ho_budget = step_budget == 0 ? dflt : (step_budget < 0 ? 0 : step_budget);
  c->ho_wide = wide_lanes;
  return COSIMS_OK;
}

cosims_status cosims_ctx_get_handoff(cosims_ctx *c, int64_t *step_budget, int32_t *wide_lanes,
                                     int64_t *parked, int64_t *wide_steps, double *wide_ms) {
  if (!c) return fail(COSIMS_ERR_INVALID, "ctx is NULL");
  if (step_budget) *step_budget = c->ho_budget;
  if (wide_lanes) *wide_lanes = c->last_shape.wide_lanes ? c->last_shape.wide_lanes : ctx_wide_lanes(c);
  unsigned long long r = 0, w[2] = {0, 0};
  if (c->d_ho_ctrl && c->timed && c->last_shape.wide_lanes) {
    DeviceGuard g(c->device);
    cudaError_t e = cudaEventSynchronize(c->ev1);
    if (e == cudaSuccess) e = cudaMemcpy(&r, c->d_ho_ctrl, sizeof r, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess)
      e = cudaMemcpy(w, c->d_counters + C_WIDE_STEPS, sizeof w, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "hand-off statistics");
  }
  if (parked) *parked = (int64_t)std::min<unsigned long long>(r, (unsigned long long)c->ho_cap);
  if (wide_steps) *wide_steps = (int64_t)w[0];
  if (wide_ms) *wide_ms = (double)w[1] * 1e-6;
  return COSIMS_OK;
}

cosims_status cosims_ctx_set_launch(cosims_ctx *c, int32_t group_lanes, int32_t block_threads) {
  if (!c) return fail(COSIMS_ERR_INVALID, "ctx is NULL");
  if (group_lanes) {
    if (group_lanes < 1 || group_lanes > 32 || (group_lanes & (group_lanes - 1)))
      return fail(COSIMS_ERR_INVALID, "group_lanes must be a power of two in 1..32");
    if (c->precision == COSIMS_PRECISION_PLAIN_F64 && group_lanes != 1)
      return fail(COSIMS_ERR_INVALID, "the plain form runs one lane per trajectory");
    c->group_lanes = group_lanes;
  }
  if (block_threads) {
    const int maxb = c->precision == COSIMS_PRECISION_PLAIN_F64 ? 128
                     : (c->par.force_type == 1 || c->par.force_type == 2) ? kMixedFarBlock
                                                                         : kMixedMaxBlock;
    if (block_threads < 32 || block_threads > maxb || (block_threads & 31))
      return fail(COSIMS_ERR_INVALID, "block_threads must be a multiple of 32 in 32..%d", maxb);
    c->block_threads = block_threads;
  }
  if (c->block_threads && c->block_threads < c->group_lanes)
    return fail(COSIMS_ERR_INVALID, "block_threads smaller than group_lanes");
  return COSIMS_OK;
}

cosims_status cosims_ctx_set_wait_test(cosims_ctx *c, uint32_t flags, uint32_t spin_limit) {
  if (!c) return fail(COSIMS_ERR_INVALID, "ctx is NULL");
  if (flags & ~(uint32_t)(COSIMS_WAIT_TEST_STAGING | COSIMS_WAIT_TEST_HANDOFF))
    return fail(COSIMS_ERR_INVALID, "unknown wait-test flags 0x%x", flags);
  c->test_flags = flags;
  c->test_spin_limit = spin_limit;
  return COSIMS_OK;
}

cosims_status cosims_ctx_get_launch(const cosims_ctx *c, int32_t *group_lanes,
                                    int32_t *block_threads) {
  if (!c) return fail(COSIMS_ERR_INVALID, "ctx is NULL");
  if (group_lanes) *group_lanes = c->precision == COSIMS_PRECISION_PLAIN_F64 ? 1 : c->group_lanes;
  if (block_threads)
    *block_threads = c->block_threads ? c->block_threads : c->last_shape.block;
  return COSIMS_OK;
}

cosims_status cosims_run_list_device(cosims_ctx *c, const double *d_pos0, const double *d_vel0,
                                     int64_t n, cosims_traj_out *d_out, void *stream) {
  if (!c) return fail(COSIMS_ERR_INVALID, "ctx is NULL");
  if (n < 0) return fail(COSIMS_ERR_INVALID, "n must be >= 0");
  if (n > 0 && (!d_pos0 || !d_vel0 || !d_out))
    return fail(COSIMS_ERR_INVALID, "pos0, vel0 and out are required");
  DeviceGuard g(c->device);
  return run_core(c, d_pos0, d_vel0, nullptr, n, d_out, stream);
}

cosims_status cosims_run_list(cosims_ctx *c, const double *pos0, const double *vel0, int64_t n,
                              cosims_traj_out *out, void *stream) {
  if (!c) return fail(COSIMS_ERR_INVALID, "ctx is NULL");
  if (n < 0) return fail(COSIMS_ERR_INVALID, "n must be >= 0");
  if (n == 0) return COSIMS_OK;
  if (!pos0 || !vel0 || !out) return fail(COSIMS_ERR_INVALID, "pos0, vel0 and out are required");
  DeviceGuard g(c->device);
  cosims_status st = grow(&c->d_pos0, &c->list_cap, 3 * n);
  if (st == COSIMS_OK) st = grow(&c->d_vel0, &c->vel_cap, 3 * n);
  if (st == COSIMS_OK) st = grow(&c->d_out, &c->out_cap, n);
  if (st != COSIMS_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = cudaMemcpyAsync(c->d_pos0, pos0, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(c->d_vel0, vel0, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return cuda_fail(e, "copy of start states");
  st = run_core(c, c->d_pos0, c->d_vel0, nullptr, n, c->d_out, stream);
  if (st != COSIMS_OK) return st;
  e = cudaMemcpyAsync(out, c->d_out, sizeof(cosims_traj_out) * n, cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) return cuda_fail(e, "copy of results");
  return check_error_flag(c, s);
}

cosims_status cosims_trace_list(cosims_ctx *c, const double *pos0, const double *vel0,
                                int64_t n, int32_t max_frames, double *frames, int32_t *nframes,
                                cosims_traj_out *out, void *stream) {
  if (!c) return fail(COSIMS_ERR_INVALID, "ctx is NULL");
  if (c->precision != COSIMS_PRECISION_PLAIN_F64)
    return fail(COSIMS_ERR_UNSUPPORTED, "trajectory traces come from the plain FP64 form");
  if (n < 0 || max_frames < 0) return fail(COSIMS_ERR_INVALID, "n and max_frames must be >= 0");
  if (n == 0) return COSIMS_OK;
  if (!pos0 || !vel0 || !out || !nframes || (max_frames > 0 && !frames))
    return fail(COSIMS_ERR_INVALID, "pos0, vel0, out, nframes (and frames) are required");
  const int64_t frame_bytes = n * (int64_t)max_frames * 6 * (int64_t)sizeof(double);
  if (frame_bytes > (int64_t)kTraceMaxBytes)
    return fail(COSIMS_ERR_INVALID, "n * max_frames * 48 bytes exceeds %lld",
                (long long)kTraceMaxBytes);
  DeviceGuard g(c->device);
  cosims_status st = grow(&c->d_pos0, &c->list_cap, 3 * n);
  if (st == COSIMS_OK) st = grow(&c->d_vel0, &c->vel_cap, 3 * n);
  if (st == COSIMS_OK) st = grow(&c->d_out, &c->out_cap, n);
  if (st != COSIMS_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  double *d_frames = nullptr;
  int32_t *d_n = nullptr;
  cudaError_t e = cudaMalloc((void **)&d_n, sizeof(int32_t) * (size_t)n);
  if (e == cudaSuccess && frame_bytes > 0) e = cudaMalloc((void **)&d_frames, (size_t)frame_bytes);
  if (e != cudaSuccess) {
    cudaFree(d_n);
    return fail(COSIMS_ERR_NOMEM, "trace buffers: %s", cudaGetErrorString(e));
  }
  e = cudaMemsetAsync(d_n, 0, sizeof(int32_t) * (size_t)n, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(c->d_pos0, pos0, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(c->d_vel0, vel0, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) {
    // with max_frames 0 no frame is written; the counts buffer stands in as the
    // (non-null) frame pointer that selects the traced kernel
    st = run_core(c, c->d_pos0, c->d_vel0, nullptr, n, c->d_out, stream,
                  d_frames ? d_frames : reinterpret_cast<double *>(d_n), d_n, max_frames);
    if (st == COSIMS_OK) {
      e = cudaMemcpyAsync(out, c->d_out, sizeof(cosims_traj_out) * n, cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(nframes, d_n, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess && frame_bytes > 0)
        e = cudaMemcpyAsync(frames, d_frames, (size_t)frame_bytes, cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) st = cuda_fail(e, "trace copies");
    }
  } else {
    st = cuda_fail(e, "trace inputs");
  }
  cudaFree(d_frames);
  cudaFree(d_n);
  if (st != COSIMS_OK) return st;
  return check_error_flag(c, s);
}

cosims_status cosims_run_sampled_device(cosims_ctx *c, uint64_t seed, int64_t first, int64_t n,
                                        int64_t update_every, cosims_ccs_sums *d_sums,
                                        void *stream) {
  if (!c) return fail(COSIMS_ERR_INVALID, "ctx is NULL");
  if (n < 0 || first < 0) return fail(COSIMS_ERR_INVALID, "n and first_index must be >= 0");
  if (!d_sums) return fail(COSIMS_ERR_INVALID, "sums is NULL");
  DeviceGuard g(c->device);
  cosims_status st = sample_into(c, seed, first, n, false, stream);
  if (st != COSIMS_OK) return st;
  st = run_core(c, c->d_pos0, c->d_vel0, c->d_hit, n, c->d_out, stream);
  if (st != COSIMS_OK) return st;
  int rc = reduce_launch(c->d_out, n, c->par.ccs_const,
                         c->precision == COSIMS_PRECISION_MIXED ? 1 : 0, update_every,
                         c->d_counters, d_sums, c->d_red, c->red_cap, stream);
  if (rc != 0) return cuda_fail((cudaError_t)rc, "reduction launch");
  return COSIMS_OK;
}

cosims_status cosims_run_sampled(cosims_ctx *c, uint64_t seed, int64_t first, int64_t n,
                                 int64_t update_every, cosims_ccs_sums *sums,
                                 cosims_traj_in *inputs, cosims_traj_out *outs, void *stream) {
  if (!c) return fail(COSIMS_ERR_INVALID, "ctx is NULL");
  if (!sums) return fail(COSIMS_ERR_INVALID, "sums is NULL");
  if (n < 0 || first < 0) return fail(COSIMS_ERR_INVALID, "n and first_index must be >= 0");
  DeviceGuard g(c->device);
  cosims_status st = sample_into(c, seed, first, n, true, stream);
  if (st != COSIMS_OK) return st;
  st = run_core(c, c->d_pos0, c->d_vel0, c->d_hit, n, c->d_out, stream);
  if (st != COSIMS_OK) return st;
  int rc = reduce_launch(c->d_out, n, c->par.ccs_const,
                         c->precision == COSIMS_PRECISION_MIXED ? 1 : 0, update_every,
                         c->d_counters, c->d_sums, c->d_red, c->red_cap, stream);
  if (rc != 0) return cuda_fail((cudaError_t)rc, "reduction launch");
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = cudaMemcpyAsync(sums, c->d_sums, sizeof(cosims_ccs_sums), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && outs && n)
    e = cudaMemcpyAsync(outs, c->d_out, sizeof(cosims_traj_out) * n, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && inputs && n)
    e = cudaMemcpyAsync(inputs, c->d_in, sizeof(cosims_traj_in) * n, cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) return cuda_fail(e, "copy of results");
  return check_error_flag(c, s);
}

cosims_status cosims_run_integrals_device(cosims_ctx *c, uint64_t seed, int64_t first,
                                          int64_t n_per, int32_t n_integrals,
                                          int64_t update_every, cosims_ccs_sums *d_sums,
                                          cosims_ccs_sums *d_work, void *stream) {
  if (!c) return fail(COSIMS_ERR_INVALID, "ctx is NULL");
  if (n_per < 0 || first < 0 || n_integrals < 0)
    return fail(COSIMS_ERR_INVALID, "n_per, n_integrals and first_index must be >= 0");
  if (n_integrals > 0 && !d_sums) return fail(COSIMS_ERR_INVALID, "sums is NULL");
  const int64_t total = n_per * (int64_t)n_integrals;
  if (n_per > 0 && total / n_per != n_integrals) return fail(COSIMS_ERR_INVALID, "count overflow");
  DeviceGuard g(c->device);
  cosims_status st = sample_into(c, seed, first, total, false, stream);
  if (st != COSIMS_OK) return st;
  // whole integrals per launch, at most the hand-off's record count, so every
  // trajectory runs as it would in a call of its integral alone
  const int64_t per_launch =
      n_per > 0 ? std::max<int64_t>(1, kHandoffMaxRecords / n_per) : (int64_t)n_integrals;
  for (int64_t k0 = 0; k0 < n_integrals || (k0 == 0 && d_work); k0 += per_launch) {
    const int64_t k1 = std::min<int64_t>(n_integrals, k0 + per_launch);
    const int64_t off = k0 * n_per, m = (k1 - k0) * n_per;
    st = run_core(c, c->d_pos0 + 3 * off, c->d_vel0 + 3 * off, c->d_hit + off, m,
                  c->d_out + off, stream, nullptr, nullptr, 0, k0 == 0);
    if (st != COSIMS_OK) return st;
    if (d_work) {
      const int rc = add_work_launch(c->d_counters, d_work, k0 == 0 ? 1 : 0, stream);
      if (rc != 0) return cuda_fail((cudaError_t)rc, "work counters");
    }
    for (int64_t k = k0; k < k1; k++) {
      const int rc = reduce_launch(c->d_out + k * n_per, n_per, c->par.ccs_const,
                                   c->precision == COSIMS_PRECISION_MIXED ? 1 : 0, update_every,
                                   nullptr, d_sums + k, c->d_red, c->red_cap, stream);
      if (rc != 0) return cuda_fail((cudaError_t)rc, "reduction launch");
    }
    if (n_integrals == 0) break;
  }
  return COSIMS_OK;
}

cosims_status cosims_run_integrals(cosims_ctx *c, uint64_t seed, int64_t first, int64_t n_per,
                                   int32_t n_integrals, int64_t update_every,
                                   cosims_ccs_sums *sums, cosims_ccs_sums *work, void *stream) {
  if (!c) return fail(COSIMS_ERR_INVALID, "ctx is NULL");
  if (n_integrals > 0 && !sums) return fail(COSIMS_ERR_INVALID, "sums is NULL");
  if (n_integrals < 0) return fail(COSIMS_ERR_INVALID, "n_integrals must be >= 0");
  DeviceGuard g(c->device);
  cosims_status st = grow(&c->d_sums_many, &c->sums_cap, (int64_t)n_integrals + 1);
  if (st != COSIMS_OK) return st;
  cosims_ccs_sums *d_work = c->d_sums_many + n_integrals;
  st = cosims_run_integrals_device(c, seed, first, n_per, n_integrals, update_every,
                                   c->d_sums_many, d_work, stream);
  if (st != COSIMS_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = cudaSuccess;
  if (n_integrals > 0)
    e = cudaMemcpyAsync(sums, c->d_sums_many, sizeof(cosims_ccs_sums) * (size_t)n_integrals,
                        cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && work)
    e = cudaMemcpyAsync(work, d_work, sizeof(cosims_ccs_sums), cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) return cuda_fail(e, "copy of results");
  return check_error_flag(c, s);
}

cosims_status cosims_ctx_reserve(cosims_ctx *c, int64_t n_traj, int32_t n_integrals) {
  if (!c) return fail(COSIMS_ERR_INVALID, "ctx is NULL");
  if (n_traj < 0 || n_integrals < 0)
    return fail(COSIMS_ERR_INVALID, "n_traj and n_integrals must be >= 0");
  if (n_traj > INT32_MAX) return fail(COSIMS_ERR_UNSUPPORTED, "at most 2^31-1 trajectories per call");
  DeviceGuard g(c->device);
  cosims_status st = grow(&c->d_out, &c->out_cap, n_traj);
  if (st == COSIMS_OK) st = grow(&c->d_in, &c->in_cap, n_traj);
  if (st == COSIMS_OK) st = grow(&c->d_pos0, &c->list_cap, 3 * n_traj);
  if (st == COSIMS_OK) st = grow(&c->d_vel0, &c->vel_cap, 3 * n_traj);
  if (st == COSIMS_OK) st = grow(&c->d_hit, &c->hit_cap, n_traj);
  if (st == COSIMS_OK) st = grow(&c->d_order, &c->order_cap, n_traj);
  if (st == COSIMS_OK) st = grow(&c->d_order_scratch, &c->order_scratch_cap, order_scratch_len());
  if (st == COSIMS_OK) st = grow(&c->d_sums_many, &c->sums_cap, (int64_t)n_integrals + 1);
  // hand-off records for the largest single launch the calls make
  if (st == COSIMS_OK && c->ho_budget > 0 && n_traj > 0)
    st = handoff_grow(c, std::min<int64_t>(n_traj, kHandoffMaxRecords));
  return st;
}

cosims_status cosims_sample_inputs(cosims_ctx *c, uint64_t seed, int64_t first, int64_t n,
                                   cosims_traj_in *inputs, double *pos0, double *vel0,
                                   int32_t *hit, void *stream) {
  if (!c) return fail(COSIMS_ERR_INVALID, "ctx is NULL");
  if (n < 0 || first < 0) return fail(COSIMS_ERR_INVALID, "n and first_index must be >= 0");
  if (n == 0) return COSIMS_OK;
  if (!inputs || !pos0 || !vel0 || !hit)
    return fail(COSIMS_ERR_INVALID, "inputs, pos0, vel0 and hit are required");
  DeviceGuard g(c->device);
  cosims_status st = sample_into(c, seed, first, n, true, stream);
  if (st != COSIMS_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = cudaMemcpyAsync(inputs, c->d_in, sizeof(cosims_traj_in) * n, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(pos0, c->d_pos0, 24 * n, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(vel0, c->d_vel0, 24 * n, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(hit, c->d_hit, 4 * n, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "sampler");
  return COSIMS_OK;
}

}  // extern "C"
