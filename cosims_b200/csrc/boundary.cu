// boundary.cu -- the ray march of the potential-energy boundary on the GPU.
//
// impactParam::setBoundry (impactParam.cpp:663-721) marches 20 rays per z
// level inward in 0.1 Angstrom steps until the potential reaches -1 % of the
// slowest kinetic energy.  Each ray is independent: one warp per ray here,
// each lane one step of the ray, with the potential summed in file order in
// IEEE double (this file is compiled with --fmad=false), so every boundary
// point equals the host's bit for bit.  Ray starts and directions are the host's (libm cos/sin).  A ray
// that runs past kMaxSteps stops and flags an error instead of looping.
#include <cuda_runtime.h>
#include <cstdio>
#include <vector>

namespace cosims {

constexpr long long kMaxSteps = 40000000;

struct RayAtoms {
  const double *x, *y, *z, *q, *sig6, *eps4;
  int n;
};

// forceAccel::getPotential (forceAccel.cpp:943-982), file order
__device__ double ray_potential(const RayAtoms &m, int charged, double ds, double px, double py,
                                double pz) {
  double total = 0, sumX = 0, sumY = 0, sumZ = 0;
  for (int k = 0; k < m.n; k++) {
    double xDiff = px - __ldg(m.x + k), yDiff = py - __ldg(m.y + k), zDiff = pz - __ldg(m.z + k);
    double r2 = xDiff * xDiff + yDiff * yDiff + zDiff * zDiff;
    double r6 = r2 * r2 * r2;
    double term2 = __ldg(m.sig6 + k) / r6;
    double term1 = term2 * term2;
    total += __ldg(m.eps4 + k) * (term1 - term2);
    if (charged) {
      double r_3 = __ldg(m.q + k) / (r2 * sqrt(r2));
      sumX += xDiff * r_3;
      sumY += yDiff * r_3;
      sumZ += zDiff * r_3;
    }
  }
  if (charged) total -= ds * 0.5 * (sumX * sumX + sumY * sumY + sumZ * sumZ);
  return total;
}

__device__ __forceinline__ double mag3(double x, double y, double z) {
  return sqrt((x * x) + (y * y) + (z * z));
}

// One warp per ray.  The march is sequential only in its stopping point, so
// the warp evaluates 32 consecutive steps at once, one per lane, and stops at
// the first lane whose step meets a stop condition.  Lane l's position is the
// chunk's base position plus l additions of the step vector: the same
// sequence of roundings as the serial march (px = px + vx each step), so the
// positions, potentials and the boundary point are the host's bit for bit.
// The steps after the stopping one are evaluated and discarded.
__global__ void boundary_rays(const RayAtoms m, int charged, double ds, double minKin, double zMax,
                              double zInc, int levels, int rotations, const double *sx,
                              const double *sy, const double *vx, const double *vy, double *out,
                              int *err) {
  const int r = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (r >= levels * rotations) return;           // whole warps: r is warp-uniform
  const int i = r / rotations, n = r % rotations;
  const double zPos = -zMax + i * zInc;
  const double startX = sx[n], startY = sy[n];
  double vxs = vx[n], vys = vy[n], vzs = 0.0;
  double sl = 1;
  const double e0 = ray_potential(m, charged, ds, startX, startY, zPos);
  if (e0 + minKin < 0) sl = -1;
  vxs = vxs * sl; vys = vys * sl; vzs = vzs * sl;
  double bx = startX, by = startY, bz = zPos;       // position of the chunk's first step
  double qx = 0, qy = 0, qz = 0;                    // position of the step before it
  double ox = 0, oy = 0, oz = 0;
  for (long long s0 = 0;; s0 += 32) {
    double px = bx, py = by, pz = bz;
    for (int k = 0; k < lane; k++) { px = px + vxs; py = py + vys; pz = pz + vzs; }
    const double e = ray_potential(m, charged, ds, px, py, pz);
    const bool stop_e = (e + minKin) * sl < 0;
    const bool stop_axis = (startX == 0 && startY / py <= 0) ||
                           (startY == 0 && startX / px <= 0) ||
                           (startX / px <= 0 && startY / py <= 0);
    // prevPos of each lane's step: the lane below, or the previous chunk's last
    double rx = __shfl_up_sync(0xffffffffu, px, 1), ry = __shfl_up_sync(0xffffffffu, py, 1),
           rz = __shfl_up_sync(0xffffffffu, pz, 1);
    if (lane == 0) { rx = qx; ry = qy; rz = qz; }
    const unsigned stops = __ballot_sync(0xffffffffu, stop_e || stop_axis);
    if (stops) {
      const int f = __ffs(stops) - 1;               // the serial march's stopping step
      if (lane == f && stop_e) {
        if (mag3(rx, ry, rz) > mag3(px, py, pz)) { ox = rx; oy = ry; oz = rz; }
        else { ox = px; oy = py; oz = pz; }
      }
      ox = __shfl_sync(0xffffffffu, ox, f);
      oy = __shfl_sync(0xffffffffu, oy, f);
      oz = __shfl_sync(0xffffffffu, oz, f);
      break;
    }
    qx = __shfl_sync(0xffffffffu, px, 31);
    qy = __shfl_sync(0xffffffffu, py, 31);
    qz = __shfl_sync(0xffffffffu, pz, 31);
    bx = qx + vxs; by = qy + vys; bz = qz + vzs;
    if (s0 > kMaxSteps) {
      if (lane == 0) atomicExch(err, 1);
      break;
    }
  }
  if (lane == 0) {
    out[3 * r] = ox;
    out[3 * r + 1] = oy;
    out[3 * r + 2] = oz;
  }
}

namespace host {
int boundary_march_gpu(int device, int n_atoms, const double *x, const double *y, const double *z,
                       const double *q, const double *sig6, const double *eps4, int charged,
                       double dipole_scalar, double min_kin, double z_max, double z_inc,
                       int levels, int rotations, const double *start_x, const double *start_y,
                       const double *vel_x, const double *vel_y, double *out_xyz, char *err,
                       int err_cap) {
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(device);
  const size_t na = (size_t)n_atoms, nr = (size_t)levels * rotations;
  std::vector<double> atoms(6 * na);
  for (size_t k = 0; k < na; k++) {
    atoms[k] = x[k]; atoms[na + k] = y[k]; atoms[2 * na + k] = z[k];
    atoms[3 * na + k] = q[k]; atoms[4 * na + k] = sig6[k]; atoms[5 * na + k] = eps4[k];
  }
  std::vector<double> dirs(4 * (size_t)rotations);
  for (int k = 0; k < rotations; k++) {
    dirs[k] = start_x[k]; dirs[rotations + k] = start_y[k];
    dirs[2 * rotations + k] = vel_x[k]; dirs[3 * rotations + k] = vel_y[k];
  }
  double *d_atoms = nullptr, *d_dirs = nullptr, *d_out = nullptr;
  int *d_err = nullptr, h_err = 0;
  cudaError_t e = cudaMalloc((void **)&d_atoms, sizeof(double) * atoms.size());
  if (e == cudaSuccess) e = cudaMalloc((void **)&d_dirs, sizeof(double) * dirs.size());
  if (e == cudaSuccess) e = cudaMalloc((void **)&d_out, sizeof(double) * 3 * nr);
  if (e == cudaSuccess) e = cudaMalloc((void **)&d_err, sizeof(int));
  if (e == cudaSuccess)
    e = cudaMemcpy(d_atoms, atoms.data(), sizeof(double) * atoms.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(d_dirs, dirs.data(), sizeof(double) * dirs.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(d_err, 0, sizeof(int));
  if (e == cudaSuccess) {
    RayAtoms m{d_atoms, d_atoms + na, d_atoms + 2 * na, d_atoms + 3 * na, d_atoms + 4 * na,
               d_atoms + 5 * na, n_atoms};
    const int block = 64;  // two rays (warps) per CTA: the rays spread over all SMs
    const int grid = (int)((nr * 32 + block - 1) / block);
    boundary_rays<<<grid, block>>>(m, charged, dipole_scalar, min_kin, z_max, z_inc, levels,
                                   rotations, d_dirs, d_dirs + rotations, d_dirs + 2 * rotations,
                                   d_dirs + 3 * rotations, d_out, d_err);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpy(out_xyz, d_out, sizeof(double) * 3 * nr, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(d_atoms); cudaFree(d_dirs); cudaFree(d_out); cudaFree(d_err);
  cudaSetDevice(prev);
  if (e != cudaSuccess) {
    snprintf(err, err_cap, "%s", cudaGetErrorString(e));
    return 1;
  }
  if (h_err) {
    snprintf(err, err_cap, "a boundary ray did not terminate");
    return 1;
  }
  return 0;
}
}  // namespace host

}  // namespace cosims
