// host_internal.h -- types of the host-side setup (not part of the ABI).
#pragma once
#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include "cosims_host.h"

namespace cosims {
namespace host {

struct Log {
  std::string text;
  void printf(const char *fmt, ...);
  void copy_to(char *dst, int64_t cap) const;
};

struct FFEntry {            // molecule2::forceField (molecule2.h:40-49)
  std::string name, symbol;
  double mass = 0, sigma = 0, epsilon = 0;
  int atomCount = 0, intMass = 0;
};

struct RawAtom {
  std::string type, line;
  double x = 0, y = 0, z = 0, charge = 0;
  bool has_charge = false;
};

struct RawMolecule {
  std::string name;
  std::vector<RawAtom> atoms;
};

struct MolFlags {           // charge_ext / totalCharge_ext as the readers set them
  bool charged = false;
  double total_charge = 0;
};

struct Atom {
  std::string symbol;
  double x = 0, y = 0, z = 0;
  double mass = 0, sigma = 0, epsilon = 0, charge = 0;
  double sig6 = 0, eps24m = 0, eps4 = 0;
};

struct Molecule {
  std::vector<Atom> atoms;
  double totalMass = 0, mu = 0;
  double center[3] = {0, 0, 0};
  double inertia[9] = {0}, rotation[9] = {0}, dipole[3] = {0}, quad[9] = {0};
  double maxX = 0, maxY = 0, maxZ = 0, radius_gyration = 0;
};

struct Ellipsoid {
  double a = 0, b = 0, c = 0, unc[3] = {0, 0, 0}, rmsd = 0, avg_axes = 0, avg_axes_unc = 0;
  double surf_area = 0, surf_area_unc = 0, enlarge = 0, cov[9] = {0};
};

struct Clusters {
  std::vector<int32_t> offset, atoms, replaced;
  std::vector<double> pos, radius, charge, dipole, quad;
  int n_replaced = 0;
  double avg_size = 0, avg_radius = 0;
};

// vector3D<double> (vector3D.h): the operations the setup uses.
struct V3 {
  double X = 0, Y = 0, Z = 0;
  V3() {}
  V3(double x, double y, double z) : X(x), Y(y), Z(z) {}
  double mag() const { return std::sqrt((X * X) + (Y * Y) + (Z * Z)); }
  double mag2() const { return (X * X) + (Y * Y) + (Z * Z); }
  double dot(const V3 &v) const { return ((X * v.X) + (Y * v.Y) + (Z * v.Z)); }
  V3 operator+(const V3 &v) const { return V3(X + v.X, Y + v.Y, Z + v.Z); }
  V3 operator-(const V3 &v) const { return V3(X - v.X, Y - v.Y, Z - v.Z); }
  V3 operator*(double s) const { return V3(X * s, Y * s, Z * s); }
  V3 operator/(double s) const { return V3(X / s, Y / s, Z / s); }
  double at(int i) const { return i == 0 ? X : (i == 1 ? Y : Z); }
};


std::vector<FFEntry> default_force_field();
bool read_atom_file(const std::string &path, std::vector<FFEntry> &ff, Log &log);
// Coordinate sets in a molecule file: the MFJ header's count (at least 1), or
// the PDB file's MODEL records (1 without them).  -1 when it cannot be read.
int count_structures(const std::string &path, bool pdb);
// structure < 0: the reference's reader (every record is one molecule);
// structure >= 0: coordinate set `structure` of a multi-structure file.
bool read_mfj(const std::string &path, const std::vector<FFEntry> &ff, RawMolecule &raw,
              MolFlags &fl, Log &log, int structure = -1);
bool read_pdb(const std::string &path, RawMolecule &raw, Log &log, int structure = -1);
bool set_properties(const RawMolecule &raw, std::vector<FFEntry> &ff, const MolFlags &fl,
                    Molecule &m, double &r_disp, double &r_mp, bool dispersion_cutoff,
                    bool multipole, Log &log);
void rotate_to_inertia_frame(Molecule &m, Log &log);
double vd_norm(int n, double a);
double vd_mean(int n, double a);
double vd_mode(int n, double a);
double vd_variance(int n, double a);
double vd_std(int n, double a);
double vd_cdf(int n, double a, double x);
void fit_ellipsoid(const std::vector<V3> &pts, Ellipsoid &e);
void enlarge_ellipsoid(const std::vector<V3> &pts, Ellipsoid &e);
bool form_clusters(const Molecule &m, int maxClusterSize, Clusters &cl, Log &log);
double potential(const Molecule &m, bool charged, double dipole_scalar, const V3 &pos);
// impactParam::setBoundry: the z-axis search on the host, the ray march on
// host threads (device < 0) or on the GPU (boundary_march_gpu).
bool boundary_scan(const Molecule &m, bool charged, double dipole_scalar, double minKin,
                   int threads, int device, std::vector<V3> &out, Log &log);

constexpr long kMaxRaySteps = 40000000;   // 4e6 Angstrom of 0.1 A steps; the reference has no cap

// The ray march of impactParam::setBoundry (impactParam.cpp:663-721) on the
// GPU: one thread per (z level, rotation), the potential summed in file order
// with IEEE double and no FMA, so the boundary equals the host's bit for bit.
// Ray starts and directions come from the host (libm cos/sin).  out_xyz:
// levels * rotations points, (0,0,0) where a ray found none.  Returns 0 on
// success, else writes a message to err.
int boundary_march_gpu(int device, int n_atoms, const double *x, const double *y, const double *z,
                       const double *q, const double *sig6, const double *eps4, int charged,
                       double dipole_scalar, double min_kin, double z_max, double z_inc,
                       int levels, int rotations, const double *start_x, const double *start_y,
                       const double *vel_x, const double *vel_y, double *out_xyz, char *err,
                       int err_cap);

}  // namespace host
}  // namespace cosims
