// setup.cpp -- per-molecule setup on the host (include/cosims_host.h).
//
// The arithmetic of every step keeps the reference's expression order (and
// uses the same libm functions), because the trajectory path's parity with
// the reference depends on identical rotated coordinates, ellipsoid axes and
// clusters.  The boundary ray march runs on std::threads; each ray is
// independent, so the result does not depend on the thread count.
#include <algorithm>
#include <cctype>
#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "cosims_host.h"
#include "host_internal.h"

namespace cosims {
namespace host {

static const double kPi = 3.14159265358979323846;     // vector3D.h:24
static const double kPi2 = 1.57079632679489661923;    // vector3D.h:25
static const double kBoltzmann = 0.831446214563;      // maxBoltz.h:29, u A^2 ps^-2 K^-1
static const double kHeliumMass = 4.002602;           // monteTraj.cpp:31, molecule2.h:72
static const double kAvogadro = 6.02214199e+23;       // molecule2.h:69
static const double kCalorie = 4.184;                 // molecule2.h:70
static const double kProtonMassKg = 1.67262158e-27;   // molecule2.h:71
static const double kDipoleScalar = 28276.01363;      // forceAccel.cpp:35

// vector3D::Angle against a plain array (vector3D.h:145-157)
static double angle_to(const V3 &v, const double in[3]) {
  double term1 = v.X * in[0] + v.Y * in[1] + v.Z * in[2];
  double term2 = v.mag() * std::sqrt(in[0] * in[0] + in[1] * in[1] + in[2] * in[2]);
  double term3 = term1 / term2;
  if (term3 > 1) return 0;
  else if (term3 < -1) return kPi;
  return std::acos(term1 / term2);
}

// ---- log ---------------------------------------------------------------------

void Log::printf(const char *fmt, ...) {
  char buf[2048];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  text += buf;
}

void Log::copy_to(char *dst, int64_t cap) const {
  if (!dst || cap <= 0) return;
  size_t n = std::min<size_t>(text.size(), (size_t)cap - 1);
  std::memcpy(dst, text.data(), n);
  dst[n] = 0;
}

// ---- force field ---------------------------------------------------------------

// molecule2::assignDefaultFF (molecule2.cpp:43-129)
std::vector<FFEntry> default_force_field() {
  return {
      {"Hydrogen", "H", 1.0079, 2.38, 0.01498936, 0, 1},
      {"Carbon", "C", 12.010, 3.043, 0.03090114, 0, 12},
      {"Nitrogen", "N", 14.006, 3.043, 0.03090114, 0, 14},
      {"Oxygen", "O", 15.999, 3.043, 0.03090114, 0, 16},
      {"Sodium", "Na", 22.98977, 3.043, 0.03090114, 0, 23},
      {"Silicon", "Si", 28.086, 3.5, 0.03113175, 0, 28},
      {"Phosphorus", "P", 30.97396, 3.5, 0.03113175, 0, 31},
      {"Sulfur", "S", 32.07, 3.5, 0.03113175, 0, 32},
      {"Iron", "Fe", 55.84, 3.5, 0.03113175, 0, 56},
  };
}

// molecule2::importFile (molecule2.cpp:132-192): six whitespace-separated
// tokens per record; a record whose name starts with '#' is skipped; an entry
// with the same symbol or integer mass is overwritten, otherwise appended.
bool read_atom_file(const std::string &path, std::vector<FFEntry> &ff, Log &log) {
  std::ifstream f(path.c_str());
  if (!f) {
    log.printf("Error: cannot open atom parameter file %s\n", path.c_str());
    return false;
  }
  log.printf("\nAtom parameters are located at: \n%s\n", path.c_str());
  std::string name, symbol, mass, sigma, epsilon, intMass;
  while (f >> name >> symbol >> mass >> sigma >> epsilon >> intMass) {
    std::transform(name.begin(), name.end(), name.begin(), ::tolower);
    if (name.at(0) == '#') continue;
    size_t index = ff.size();
    for (size_t i = 0; i < ff.size(); i++)
      if (symbol.compare(ff[i].symbol) == 0 || ff[i].intMass == atoi(intMass.c_str())) {
        index = i;
        break;
      }
    if (index == ff.size()) ff.push_back(FFEntry());
    FFEntry &e = ff[index];
    e.name = name;
    e.symbol = symbol;
    e.mass = atof(mass.c_str());
    e.sigma = atof(sigma.c_str());
    e.epsilon = atof(epsilon.c_str());
    e.atomCount = 0;
    e.intMass = atoi(intMass.c_str());
  }
  return true;
}

// ---- molecule files -------------------------------------------------------------

static std::string strip_spaces(std::string s) {
  s.erase(std::remove_if(s.begin(), s.end(), ::isspace), s.end());
  return s;
}

static bool all_digits(const std::string &s, bool allow_dot, bool allow_space) {
  for (char ch : s)
    if (!(isdigit((unsigned char)ch) || (allow_dot && ch == '.') || (allow_space && ch == ' ')))
      return false;
  return true;
}

static bool numeric_token(const std::string &t) {
  if (t.empty()) return false;
  char *end = nullptr;
  std::strtod(t.c_str(), &end);
  return end && *end == 0;
}

int count_structures(const std::string &path, bool pdb) {
  std::ifstream f(path.c_str());
  if (!f) return -1;
  std::string line;
  if (pdb) {
    int models = 0;
    while (std::getline(f, line))
      if (line.compare(0, 5, "MODEL") == 0) models++;
    return models > 0 ? models : 1;
  }
  std::getline(f, line);                 // name
  if (!std::getline(f, line)) return -1;  // number of coordinate sets
  const int k = atoi(strip_spaces(line).c_str());
  return k > 1 ? k : 1;
}

// molecule2::importMFJ (molecule2.cpp:442-647).  With structure >= 0 the
// coordinate records after the header are read line by line: a line of at
// least five tokens whose first three are numbers is a record, any other line
// separates sets, and set s is records s*N .. s*N+N-1 (N from the header).
// The reference reads every record as one molecule and warns that multiple
// coordinate sets are not supported (molecule2.cpp:497-501).
bool read_mfj(const std::string &path, const std::vector<FFEntry> &ff, RawMolecule &raw,
              MolFlags &fl, Log &log, int structure) {
  std::ifstream f(path.c_str());
  if (!f) {
    log.printf("ERROR: Cannot read molecule file.\n");
    return false;
  }
  std::string line;
  std::getline(f, line);
  line = strip_spaces(line);
  if (line.empty())
    log.printf(" Warning: Project name in MFJ file is empty\n");
  else
    raw.name = line;
  std::getline(f, line);
  const int sets = std::max(1, atoi(strip_spaces(line).c_str()));
  if (sets > 1 && structure < 0)
    log.printf(" Warning: Multiple coordinate sets not yet supported.\n");
  if (structure >= sets) {
    log.printf(" Error: coordinate set %d requested, the file holds %d.\n", structure, sets);
    return false;
  }
  std::getline(f, line);
  line = strip_spaces(line);
  if (line.empty()) log.printf(" Error: Number of atoms not specified.\n");
  const int header_atoms = atoi(line.c_str());
  std::getline(f, line);
  line = strip_spaces(line);
  std::transform(line.begin(), line.end(), line.begin(), ::tolower);
  std::string unit;
  if (line.empty() || !(line == "ang" || line == "au"))
    log.printf(" Warning: Coordinate units not specified; Assuming Angstroms.\n");
  else
    unit = line;
  std::getline(f, line);
  line = strip_spaces(line);
  bool uniform = false, calc = false;
  if (line.empty()) {
    log.printf(" Warning: Charge type not specified; Assuming no charge.\n");
    fl.charged = false;
  } else if (line == "none") {
    fl.charged = false;
  } else if (line == "equal") {
    fl.charged = true;
    fl.total_charge = 1.0;
    uniform = true;
  } else if (all_digits(line, false, true)) {
    fl.charged = true;
    fl.total_charge = atoi(line.c_str());
    uniform = true;
  } else if (line == "calc") {
    calc = true;
    fl.charged = true;
  } else {
    log.printf(" Warning: Charge type incorrectly specified; Assuming no charge.\n");
    fl.charged = false;
  }
  double scale = 1.0;
  std::getline(f, line);
  line = strip_spaces(line);
  if (line.empty())
    log.printf(" Warning: Correction factor not given; assuming identity\n");
  else if (all_digits(line, false, true) || all_digits(line, true, false))
    scale = atof(line.c_str());
  else
    log.printf(" Warning: Incorrect correction factor; assuming .\n");
  const double unitConv = unit == "au" ? 0.529177210 : 1.0;
  std::string sx, sy, sz, sm, sq;
  double total = 0.0;
  // the records of the requested set (structure mode)
  std::vector<std::string> recs;
  size_t next = 0;
  if (structure >= 0) {
    if (sets > 1) log.printf(" Coordinate set %d of %d.\n", structure + 1, sets);
    int seen = 0;
    const int first = structure * header_atoms, last = first + header_atoms;
    while (std::getline(f, line) && seen < last) {
      std::istringstream ls(line);
      std::string t[5];
      int nt = 0;
      while (nt < 5 && ls >> t[nt]) nt++;
      if (nt < 5 || !numeric_token(t[0]) || !numeric_token(t[1]) || !numeric_token(t[2]))
        continue;                                   // a separator line
      if (seen >= first)
        for (int k = 0; k < 5; k++) recs.push_back(t[k]);
      seen++;
    }
    if (seen < last || header_atoms <= 0) {
      log.printf(" Error: coordinate set %d needs records %d..%d; the file has %d.\n",
                 structure + 1, first + 1, last, seen);
      return false;
    }
  }
  auto next_record = [&]() -> bool {
    if (structure < 0) return (bool)(f >> sx >> sy >> sz >> sm >> sq);
    if (next + 5 > recs.size()) return false;
    sx = recs[next]; sy = recs[next + 1]; sz = recs[next + 2];
    sm = recs[next + 3]; sq = recs[next + 4];
    next += 5;
    return true;
  };
  while (next_record()) {
    // a record whose numbers do not parse, or are not finite, is corrupt: the
    // reference reads it unchecked (atof: 0 for a word, NaN for "nan") and
    // would integrate a wrong or non-finite molecule; here it is an error
    const size_t line_no = raw.atoms.size() + 1;
    if (!numeric_token(sx) || !numeric_token(sy) || !numeric_token(sz) ||
        !numeric_token(sm) || (calc && !numeric_token(sq))) {
      log.printf("Error: MFJ atom record %zu is not five numbers (%s %s %s %s %s)\n", line_no,
                 sx.c_str(), sy.c_str(), sz.c_str(), sm.c_str(), sq.c_str());
      return false;
    }
    RawAtom a;
    a.x = atof(sx.c_str()) * scale * unitConv;
    a.y = atof(sy.c_str()) * scale * unitConv;
    a.z = atof(sz.c_str()) * scale * unitConv;
    if (!std::isfinite(a.x) || !std::isfinite(a.y) || !std::isfinite(a.z) ||
        (calc && !std::isfinite(atof(sq.c_str())))) {
      log.printf("Error: MFJ atom record %zu has a non-finite coordinate or charge\n", line_no);
      return false;
    }
    a.has_charge = true;
    if (fl.charged) {
      double q = uniform ? fl.total_charge / (double)header_atoms : atof(sq.c_str());
      a.charge = q;
      total += q;
    } else {
      a.charge = 0.0;
    }
    const int im = atoi(sm.c_str());
    for (size_t j = 0; j < ff.size(); j++)
      if (im == ff[j].intMass) { a.type = ff[j].symbol; break; }
    if (a.type.empty()) {
      log.printf("Error: no atom type with integer mass %d (MFJ line %zu)\n", im,
                 raw.atoms.size() + 1);
      return false;
    }
    raw.atoms.push_back(a);
  }
  if (calc) fl.total_charge = total;
  if (structure < 0 && header_atoms > 0 && (int)raw.atoms.size() != header_atoms)
    log.printf(" Warning: the MFJ header gives %d atoms; %zu complete atom records were read\n",
               header_atoms, raw.atoms.size());
  if (raw.atoms.empty()) log.printf("Error: MFJ file holds no atom records\n");
  return !raw.atoms.empty();
}

// molecule2::importPDB (molecule2.cpp:649-768): ATOM / HETATM records; the
// element from columns 77-78 when the line is long enough, else the first
// letter of the atom name (columns 13-17); coordinates from fixed columns.
// With structure >= 0 and MODEL records in the file, only the records of the
// structure-th MODEL (up to its ENDMDL) are read; the reference reads all.
bool read_pdb(const std::string &path, RawMolecule &raw, Log &log, int structure) {
  const int models = structure >= 0 ? count_structures(path, true) : 1;
  const bool by_model = structure >= 0 && models >= 1 && [&] {
    std::ifstream g(path.c_str());
    std::string l;
    while (std::getline(g, l))
      if (l.compare(0, 5, "MODEL") == 0) return true;
    return false;
  }();
  if (structure >= models) {
    log.printf(" Error: model %d requested, the file holds %d.\n", structure + 1, models);
    return false;
  }
  int model = -1;          // index of the MODEL block being read
  bool inside = false;
  std::ifstream f(path.c_str());
  if (!f) {
    log.printf("ERROR: Cannot read molecule file.\n");
    return false;
  }
  const int SIZE = 800;
  std::vector<char> buf(SIZE);
  f.getline(buf.data(), SIZE, '\n');
  while (!f.eof()) {
    const char *t = buf.data();
    if (by_model) {
      if (std::strncmp(t, "MODEL", 5) == 0) {
        model++;
        inside = model == structure;
      } else if (std::strncmp(t, "ENDMDL", 6) == 0) {
        inside = false;
      }
    }
    const bool atom = std::strncmp(t, "ATOM", 4) == 0;
    const bool het = std::strncmp(t, "HETATM", 6) == 0;
    if ((atom || het) && (!by_model || inside)) {
      char type[10];
      int nameLen = 1;
      if (std::strlen(t) >= 78) {
        std::memcpy(type, t + 76, 2);
        type[2] = 0;
        if (type[0] == ' ' && type[1] == ' ') {
          std::memcpy(type, t + 12, 5);
          type[5] = 0;
        } else {
          nameLen = 2;
        }
      } else {
        std::memcpy(type, t + 12, 5);
        type[5] = 0;
      }
      std::string temps;
      for (int i = 0; i < (int)std::strlen(type); i++)
        if (isalpha((unsigned char)type[i])) {
          temps.append(1, type[i]);
          if ((int)temps.length() == nameLen) break;
        }
      RawAtom a;
      a.type = temps;
      char part[9];
      std::memcpy(part, t + 30, 8); part[8] = 0; a.x = atof(part);
      std::memcpy(part, t + 38, 8); part[8] = 0; a.y = atof(part);
      std::memcpy(part, t + 46, 8); part[8] = 0; a.z = atof(part);
      a.has_charge = false;
      a.line = t;
      raw.atoms.push_back(a);
    }
    f.getline(buf.data(), SIZE, '\n');
  }
  return !raw.atoms.empty();
}

// ---- molecule properties ----------------------------------------------------------

// molecule2::setMolProperties (molecule2.cpp:770-903)
bool set_properties(const RawMolecule &raw, std::vector<FFEntry> &ff, const MolFlags &fl,
                    Molecule &m, double &r_disp, double &r_mp, bool dispersion_cutoff,
                    bool multipole, Log &log) {
  const int n = (int)raw.atoms.size();
  m.atoms.assign(n, Atom());
  m.totalMass = 0;
  double cX = 0, cY = 0, cZ = 0;
  for (int i = 0; i < n; i++) {
    const RawAtom &r = raw.atoms[i];
    Atom &a = m.atoms[i];
    bool found = false;
    for (size_t j = 0; j < ff.size(); j++) {
      if (ff[j].symbol.compare(r.type) == 0) {
        found = true;
        a.mass = ff[j].mass;
        a.sigma = ff[j].sigma;
        a.epsilon = ff[j].epsilon;
        double epsAvg = ff[j].epsilon;
        epsAvg *= kCalorie / (kAvogadro * kProtonMassKg * 10.0);
        a.sig6 = std::pow(ff[j].sigma, 6);
        a.eps24m = epsAvg * 24;
        a.eps4 = epsAvg * 4;
        if (fl.charged)
          a.charge = r.has_charge ? r.charge : fl.total_charge / (double)n;
        else
          a.charge = 0.0;
        ff[j].atomCount++;
        break;
      }
    }
    if (!found) {
      log.printf("Error: Force field does not contain atoms of type %s from molecule file "
                 "line:\n%s\n", r.type.c_str(), r.line.c_str());
      return false;
    }
    a.symbol = r.type;
    a.x = r.x; a.y = r.y; a.z = r.z;
    cX += a.mass * a.x;
    cY += a.mass * a.y;
    cZ += a.mass * a.z;
    m.totalMass += a.mass;
  }
  m.mu = (m.totalMass * kHeliumMass) / (m.totalMass + kHeliumMass);
  cX /= m.totalMass; cY /= m.totalMass; cZ /= m.totalMass;
  m.center[0] = cX; m.center[1] = cY; m.center[2] = cZ;
  // molecule2.cpp:862-863: the loop starts at atom 1, atom 0 keeps 24 eps'
  for (int k = 1; k < n; k++) m.atoms[k].eps24m /= m.mu;
  for (int k = 0; k < n; k++) {
    m.atoms[k].x -= cX;
    m.atoms[k].y -= cY;
    m.atoms[k].z -= cZ;
  }
  if ((dispersion_cutoff && r_disp == 0) || (multipole && r_mp == 0)) {
    double sigmaMax = 0;
    const double minPct = 0.5;
    for (size_t j = 0; j < ff.size(); j++)
      if (ff[j].sigma > sigmaMax) sigmaMax = ff[j].sigma;
    if (dispersion_cutoff && r_disp == 0) {
      r_disp = sigmaMax * std::pow(150.0 / minPct, 1.0 / 3.0);
      log.printf(" Dispersion cut-off radius not specified in input file: \n\tUsing a cut-off "
                 "radius of %6.2f\n\t Determined by largest VDW radius of %5.3f\n", r_disp,
                 sigmaMax);
    }
    if (multipole && r_mp == 0) r_mp = 20.0;
  }
  return true;
}

// molecule2::getEigenvalues (molecule2.cpp:1315-1358)
static void mol_eigenvalues(double A[3][3], double ev[3]) {
  double a0, a1, a2, p, q, R, Q, D, a, b, phase, mag;
  a0 = A[0][0] * A[1][1] * A[2][2] - A[0][0] * A[1][2] * A[2][1] - A[1][1] * A[0][2] * A[2][0] -
       A[2][2] * A[0][1] * A[1][0] + A[0][1] * A[1][2] * A[2][0] + A[0][2] * A[2][1] * A[1][0];
  a1 = A[0][1] * A[1][0] + A[0][2] * A[2][0] + A[1][2] * A[2][1] - A[0][0] * A[1][1] -
       A[1][1] * A[2][2] - A[2][2] * A[0][0];
  a2 = A[0][0] + A[1][1] + A[2][2];
  a0 = -a0; a1 = -a1; a2 = -a2;
  p = (3 * a1 - a2 * a2) / 3;
  q = (9 * a1 * a2 - 27 * a0 - 2 * a2 * a2 * a2) / 27;
  Q = p / 3; R = q / 2; D = Q * Q * Q + R * R;
  if (D < 0) {
    a = R; b = std::sqrt(-D);
  } else {
    a = R + std::sqrt(D);
    b = 0;
  }
  phase = std::atan2(b, a);
  mag = std::pow(a * a + b * b, 1.0 / 6.0);
  ev[0] = -(a2 / 3) + mag * 2 * std::cos(phase / 3.0);
  ev[1] = -(a2 / 3) - mag * (std::cos(phase / 3.0) + std::sqrt(3) * std::sin(phase / 3.0));
  ev[2] = -(a2 / 3) - mag * (std::cos(phase / 3.0) - std::sqrt(3) * std::sin(phase / 3.0));
}

// molecule2::getEigenvectors (molecule2.cpp:1360-1391)
static void mol_eigenvectors(double A[3][3], const double l[3], double E[3][3]) {
  double det, x, y, z, nf;
  det = l[0] * l[0] - l[0] * A[1][1] - A[1][2] * A[1][2] - l[0] * A[2][2] + A[1][1] * A[2][2];
  y = (l[0] * A[1][0] - A[2][2] * A[1][0] + A[1][2] * A[2][0]) / det;
  z = (A[2][1] * A[1][0] + l[0] * A[2][0] - A[1][1] * A[2][0]) / det;
  nf = std::sqrt(1 + y * y + z * z);
  E[0][0] = 1.0 / nf; E[0][1] = y / nf; E[0][2] = z / nf;
  det = l[1] * l[1] - l[1] * A[0][0] - A[0][2] * A[0][2] - l[1] * A[2][2] + A[0][0] * A[2][2];
  x = (l[1] * A[0][1] + A[0][2] * A[2][1] - A[0][1] * A[2][2]) / det;
  z = (A[0][1] * A[0][2] + (l[1] - A[0][0]) * A[2][1]) / det;
  nf = std::sqrt(1 + x * x + z * z);
  E[1][0] = x / nf; E[1][1] = 1 / nf; E[1][2] = z / nf;
  E[2][0] = E[0][1] * E[1][2] - E[0][2] * E[1][1];
  E[2][1] = E[0][2] * E[1][0] - E[0][0] * E[1][2];
  E[2][2] = E[0][0] * E[1][1] - E[0][1] * E[1][0];
}

static void rotate_z(Atom &a, double t) {   // vector3D::rotateZ (vector3D.h:298-303)
  double x = a.x * std::cos(t) - a.y * std::sin(t);
  double y = a.x * std::sin(t) + a.y * std::cos(t);
  a.x = x; a.y = y;
}

static void rotate_y(Atom &a, double t) {   // vector3D::rotateY (vector3D.h:291-296)
  double x = a.x * std::cos(t) + a.z * std::sin(t);
  double z = -a.x * std::sin(t) + a.z * std::cos(t);
  a.x = x; a.z = z;
}

// molecule2::setMultipole -> setDipole / setQuadpole / setInertia(true)
// (molecule2.cpp:948-1308): moments for the log, then the rotation into the
// inertia frame and the longest-extent swap.
void rotate_to_inertia_frame(Molecule &m, Log &log) {
  const int n = (int)m.atoms.size();
  for (int k = 0; k < 3; k++) m.dipole[k] = 0.0;
  for (int k = 0; k < 9; k++) m.quad[k] = 0.0;
  for (int i = 0; i < n; i++) {
    const double c[3] = {m.atoms[i].x, m.atoms[i].y, m.atoms[i].z};
    for (int k = 0; k < 3; k++) m.dipole[k] += m.atoms[i].charge * c[k];
  }
  for (int i = 0; i < n; i++) {
    const double c[3] = {m.atoms[i].x, m.atoms[i].y, m.atoms[i].z};
    const double r2 = c[0] * c[0] + c[1] * c[1] + c[2] * c[2];
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++)
        m.quad[3 * a + b] += m.atoms[i].charge * (3 * c[a] * c[b] - r2 * (a == b ? 1.0 : 0.0));
  }
  double inertia[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  for (int i = 0; i < n; i++) {
    const double c[3] = {m.atoms[i].x, m.atoms[i].y, m.atoms[i].z};
    const double r2 = c[0] * c[0] + c[1] * c[1] + c[2] * c[2];
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++)
        inertia[a][b] += m.atoms[i].mass * (r2 * (a == b ? 1.0 : 0.0) - c[a] * c[b]);
  }
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) m.inertia[3 * a + b] = inertia[a][b];
  double vals[3], vecs[3][3];
  mol_eigenvalues(inertia, vals);
  mol_eigenvectors(inertia, vals, vecs);
  V3 t1(vecs[0][0], vecs[0][1], vecs[0][2]), t2(vecs[1][0], vecs[1][1], vecs[1][2]),
      t3(vecs[2][0], vecs[2][1], vecs[2][2]);
  double dotProd = std::fabs(t1.dot(t2));
  dotProd = std::max(std::fabs(t1.dot(t3)), dotProd);
  dotProd = std::max(std::fabs(t2.dot(t3)), dotProd);
  if (dotProd > 1E-6) {
    log.printf("\nFailed to find proper eigenvectors of Inertia tensor:\nAtom with longest "
               "vector magnitude will be aligned\nwith z-axis and the atom with greatest "
               "XY-projection \nwill then be aligned along the x-axis.\n");
    double maxMag = 0;
    int maxcoord = 0;
    for (int i = 0; i < n; i++) {
      double t = V3(m.atoms[i].x, m.atoms[i].y, m.atoms[i].z).mag();
      if (t > maxMag) { maxMag = t; maxcoord = i; }
    }
    double theta = std::acos(m.atoms[maxcoord].z / maxMag);
    // molecule2.cpp:1205 reads data[i] with i == numAtoms after the loop (one
    // past the end); the last atom's x stands in for it here
    double phi = std::atan2(m.atoms[maxcoord].y, m.atoms[n - 1].x);
    for (int i = 0; i < n; i++) {
      rotate_z(m.atoms[i], -phi);
      rotate_y(m.atoms[i], -theta);
    }
    maxMag = 0;
    for (int i = 0; i < n; i++) {
      double t = std::sqrt(std::pow(m.atoms[i].x, 2) + std::pow(m.atoms[i].y, 2));
      if (t > maxMag) { maxMag = t; maxcoord = i; }
    }
    double gamma = std::acos(m.atoms[maxcoord].x / maxMag);
    for (int i = 0; i < n; i++) rotate_z(m.atoms[i], -gamma);
    for (int k = 0; k < 9; k++) m.rotation[k] = (k % 4 == 0) ? 1.0 : 0.0;
  } else {
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) m.rotation[3 * a + b] = vecs[a][b];
    for (int i = 0; i < n; i++) {   // vector3D::rotate2 (vector3D.h:250-260)
      Atom &A = m.atoms[i];
      double x = A.x, y = A.y, z = A.z;
      A.x = x * vecs[0][0] + y * vecs[0][1] + z * vecs[0][2];
      A.y = x * vecs[1][0] + y * vecs[1][1] + z * vecs[1][2];
      A.z = x * vecs[2][0] + y * vecs[2][1] + z * vecs[2][2];
    }
  }
  double maxX = 0, maxY = 0, maxZ = 0;
  for (int i = 0; i < n; i++) {
    if (std::fabs(m.atoms[i].x) > std::fabs(maxX)) maxX = std::fabs(m.atoms[i].x);
    if (std::fabs(m.atoms[i].y) > std::fabs(maxY)) maxY = std::fabs(m.atoms[i].y);
    if (std::fabs(m.atoms[i].z) > std::fabs(maxZ)) maxZ = std::fabs(m.atoms[i].z);
  }
  if (maxX > maxY && maxX > maxZ) {
    for (int i = 0; i < n; i++) {
      double t = m.atoms[i].x;
      m.atoms[i].x = -m.atoms[i].z;
      m.atoms[i].z = t;
    }
  } else if (maxY > maxX && maxY > maxZ) {
    for (int i = 0; i < n; i++) {
      double t = m.atoms[i].y;
      m.atoms[i].y = m.atoms[i].z;
      m.atoms[i].z = -t;
    }
  }
  maxX = 0; maxY = 0; maxZ = 0;
  for (int i = 0; i < n; i++) {
    if (std::fabs(m.atoms[i].x) > std::fabs(maxX)) maxX = m.atoms[i].x;
    if (std::fabs(m.atoms[i].y) > std::fabs(maxY)) maxY = m.atoms[i].y;
    if (std::fabs(m.atoms[i].z) > std::fabs(maxZ)) maxZ = m.atoms[i].z;
  }
  m.maxX = maxX; m.maxY = maxY; m.maxZ = maxZ;
  double rg = 0;
  for (int i = 0; i < n; i++) rg += V3(m.atoms[i].x, m.atoms[i].y, m.atoms[i].z).mag2();
  m.radius_gyration = std::sqrt(rg / n);
}

// ---- potential (for the boundary scan) -----------------------------------------------

// forceAccel::getPotential (forceAccel.cpp:943-982), file order.
double potential(const Molecule &m, bool charged, double dipole_scalar, const V3 &pos) {
  double total = 0, sumX = 0, sumY = 0, sumZ = 0;
  for (const Atom &a : m.atoms) {
    double xDiff = pos.X - a.x, yDiff = pos.Y - a.y, zDiff = pos.Z - a.z;
    double r2 = xDiff * xDiff + yDiff * yDiff + zDiff * zDiff;
    double r6 = r2 * r2 * r2;
    double term2 = a.sig6 / r6;
    double term1 = term2 * term2;
    total += a.eps4 * (term1 - term2);
    if (charged) {
      double r_3 = a.charge / (r2 * std::sqrt(r2));
      sumX += xDiff * r_3;
      sumY += yDiff * r_3;
      sumZ += zDiff * r_3;
    }
  }
  if (charged) total -= dipole_scalar * 0.5 * (sumX * sumX + sumY * sumY + sumZ * sumZ);
  return total;
}

// ---- velocity distribution -------------------------------------------------------------

// VelocityDistribution (VelocityDistribution.cpp:46-151) for power n.
static int factorial(int x) { return x <= 1 ? 1 : x * factorial(x - 1); }
static int d_factorial(int x) { return (x == 1 || x == 0) ? 1 : x * d_factorial(x - 2); }

double vd_norm(int n, double a) { return 2 * std::pow(a, (n + 1) / 2.0) / std::tgamma((n + 1) / 2.0); }
double vd_mean(int n, double a) {
  return std::tgamma((n + 2) / 2.0) / (std::tgamma((n + 1) / 2.0) * std::sqrt(a));
}
double vd_mode(int n, double a) { return std::sqrt(n / (2 * a)); }
double vd_variance(int n, double a) {
  return ((n + 1) / 2.0 - std::pow(std::tgamma((n + 2) / 2.0) / std::tgamma((n + 1) / 2.0), 2)) / a;
}
double vd_std(int n, double a) { return std::sqrt(vd_variance(n, a)); }
double vd_cdf(int n, double a, double x) {
  double sum = 0;
  if (n % 2 == 0) {
    for (int k = 0; k <= (n / 2.0 - 1); k++)
      sum += std::pow(2 * x * x * a, k) / (double)d_factorial(2 * k + 1);
    return std::erf(std::sqrt(a) * x) - std::sqrt(a / kPi) * std::exp(-a * x * x) * 2 * x * sum;
  }
  for (int k = 0; k <= n; k++) sum += std::pow(x * x * a, k) / (double)factorial(k);
  return 1 - std::exp(-a * x * x) * sum;
}

// ---- impact-parameter boundary ------------------------------------------------------------

// impactParam::setBoundry (impactParam.cpp:602-736): ray march of the
// potential-energy surface; a boundary point is where |U| reaches 1 % of
// the slowest kinetic energy.  Rays of one z level are independent; levels are
// spread over threads.
bool boundary_scan(const Molecule &m, bool charged, double dipole_scalar, double minKin,
                   int threads, int device, std::vector<V3> &out, Log &log) {
  const int numRotations = 20;
  const double velMag = 0.1;
  double posMag = std::fabs(std::max(std::fabs(m.maxX), std::fabs(m.maxY)));
  double zMax = 0.0, slope = 1.0;
  V3 pos(0, 0, std::fabs(m.maxZ) + 20), prev;
  double energy = potential(m, charged, dipole_scalar, pos);
  minKin = 0.01 * minKin;
  if (energy + minKin < 0) slope = -1;
  long guard = 0;
  for (;;) {
    prev = pos;
    pos.Z -= 0.5 * slope;
    energy = potential(m, charged, dipole_scalar, pos);
    if ((energy + minKin) * slope < 0) {
      zMax = std::max(pos.Z, prev.Z);
      break;
    }
    if (++guard > 4000000) {   // the reference would search forever
      log.printf("Error: the potential-energy boundary was not found along the z axis\n");
      return false;
    }
  }
  zMax *= 1.3;
  posMag += std::fabs(zMax - std::fabs(m.maxZ));
  const int maxZLevels = (int)std::ceil(std::max(25, (int)std::ceil(zMax)));
  const double zInc = 2 * zMax / (maxZLevels);
  // ray directions with the host's libm, as the reference computes them
  std::vector<double> sx(numRotations), sy(numRotations), vx(numRotations), vy(numRotations);
  for (int n = 0; n < numRotations; n++) {
    const double theta = n * 2 * kPi / ((double)numRotations);
    sx[n] = posMag * std::cos(theta);
    sy[n] = posMag * std::sin(theta);
    vx[n] = -velMag * std::cos(theta);
    vy[n] = -velMag * std::sin(theta);
  }
  std::vector<V3> tmp((size_t)(maxZLevels + 1) * numRotations, V3(0, 0, 0));
  if (device >= 0) {
    // the ray march on the GPU (one thread per ray, the same IEEE sequence)
    const int n = (int)m.atoms.size();
    std::vector<double> x(n), y(n), z(n), q(n), s6(n), e4(n);
    for (int k = 0; k < n; k++) {
      x[k] = m.atoms[k].x; y[k] = m.atoms[k].y; z[k] = m.atoms[k].z;
      q[k] = m.atoms[k].charge; s6[k] = m.atoms[k].sig6; e4[k] = m.atoms[k].eps4;
    }
    std::vector<double> xyz(tmp.size() * 3, 0.0);
    char err[256] = {0};
    if (boundary_march_gpu(device, n, x.data(), y.data(), z.data(), q.data(), s6.data(),
                           e4.data(), charged ? 1 : 0, dipole_scalar, minKin, zMax, zInc,
                           maxZLevels + 1, numRotations, sx.data(), sy.data(), vx.data(),
                           vy.data(), xyz.data(), err, sizeof err) != 0) {
      log.printf("Error: device boundary scan: %s\n", err);
      return false;
    }
    for (size_t k = 0; k < tmp.size(); k++) tmp[k] = V3(xyz[3 * k], xyz[3 * k + 1], xyz[3 * k + 2]);
  } else {
    std::vector<char> failed(maxZLevels + 1, 0);
    auto level = [&](int i) {
      const double zPos = -zMax + i * zInc;
      V3 prevPos;
      for (int n = 0; n < numRotations; n++) {
        double sl = 1;
        const double startX = sx[n], startY = sy[n];
        V3 p(startX, startY, zPos);
        V3 vel(vx[n], vy[n], 0.0);
        double e = potential(m, charged, dipole_scalar, p);
        if (e + minKin < 0) sl = -1;
        vel = vel * sl;
        for (long step = 0;; step++) {
          e = potential(m, charged, dipole_scalar, p);
          if ((e + minKin) * sl < 0) {
            tmp[(size_t)i * numRotations + n] = prevPos.mag() > p.mag() ? prevPos : p;
            break;
          } else if ((startX == 0 && startY / p.Y <= 0) || (startY == 0 && startX / p.X <= 0) ||
                     (startX / p.X <= 0 && startY / p.Y <= 0)) {
            break;
          }
          prevPos = p;
          p = p + vel;
          if (step > kMaxRaySteps) { failed[i] = 1; return; }
        }
      }
    };
    int nt = std::max(1, threads);
    nt = std::min(nt, maxZLevels + 1);
    if (nt == 1) {
      for (int i = 0; i <= maxZLevels; i++) level(i);
    } else {
      std::vector<std::thread> pool;
      for (int t = 0; t < nt; t++)
        pool.emplace_back([&, t]() {
          for (int i = t; i <= maxZLevels; i += nt) level(i);
        });
      for (auto &th : pool) th.join();
    }
    for (char f : failed)
      if (f) {
        log.printf("Error: a boundary ray did not terminate\n");
        return false;
      }
  }
  out.clear();
  for (const V3 &p : tmp)
    if (!(p.X == 0 && p.Y == 0 && p.Z == 0)) out.push_back(p);
  return !out.empty();
}

// impactParam::findEllipsoidBound (impactParam.cpp:853-939): least-squares
// axis-aligned ellipsoid through the boundary points, with uncertainties.
void fit_ellipsoid(const std::vector<V3> &pts, Ellipsoid &e) {
  double mu = 0, nu = 0, epsilon = 0, delta = 0, sigma = 0, rho = 0;
  double alpha = 0, beta = 0, gamma = 0;
  for (const V3 &p : pts) {
    double x2 = p.X * p.X, y2 = p.Y * p.Y, z2 = p.Z * p.Z;
    double x4 = x2 * x2, y4 = y2 * y2, z4 = z2 * z2;
    mu = mu + x4; nu = nu + y4; epsilon = epsilon + z4;
    delta = delta + x2 * y2; sigma = sigma + x2 * z2; rho = rho + y2 * z2;
    alpha = alpha + x2; beta = beta + y2; gamma = gamma + z2;
  }
  double det = epsilon * mu * nu - epsilon * delta * delta - mu * rho * rho +
               2 * delta * rho * sigma - nu * sigma * sigma;
  double A = (alpha * (nu * epsilon - rho * rho) + delta * (rho * gamma - beta * epsilon) +
              sigma * (beta * rho - nu * gamma)) / det;
  double B = (mu * (beta * epsilon - gamma * rho) + alpha * (rho * sigma - delta * epsilon) +
              sigma * (delta * gamma - beta * sigma)) / det;
  double C = (mu * (nu * gamma - beta * rho) + delta * (beta * sigma - delta * gamma) +
              alpha * (delta * rho - nu * sigma)) / det;
  double a = 1 / std::sqrt(A), b = 1 / std::sqrt(B), c = 1 / std::sqrt(C);
  const double np = (double)pts.size();
  double rmsd = std::sqrt((A * A * mu + B * B * nu + C * C * epsilon +
                           2 * (A * B * delta + B * C * rho + A * C * sigma - A * alpha -
                                B * beta - C * gamma) + pts.size()) / (pts.size() - 1));
  (void)np;
  double cov_aa = 2 * rmsd * rmsd * (epsilon * nu - rho * rho) * a * a / (4 * A * A * det);
  double cov_bb = 2 * rmsd * rmsd * (epsilon * mu - sigma * sigma) * b * b / (4 * B * B * det);
  double cov_cc = 2 * rmsd * rmsd * (mu * nu - delta * delta) * c * c / (4 * C * C * det);
  double cov_ab = 2 * rmsd * rmsd * (rho * sigma - delta * epsilon) * a * b / (4 * A * B * det);
  double cov_ac = 2 * rmsd * rmsd * (delta * rho - nu * sigma) * a * c / (4 * A * C * det);
  double cov_bc = 2 * rmsd * rmsd * (delta * sigma - mu * rho) * b * c / (4 * B * C * det);
  e.unc[0] = (a / A) * std::sqrt((epsilon * nu - rho * rho) * 2 / det) * rmsd / 2;
  e.unc[1] = (b / B) * std::sqrt((epsilon * mu - sigma * sigma) * 2 / det) * rmsd / 2;
  e.unc[2] = (c / C) * std::sqrt((mu * nu - delta * delta) * 2 / det) * rmsd / 2;
  e.avg_axes = (a + b + c) / 3.0;
  e.avg_axes_unc = std::sqrt(cov_aa + cov_bb + cov_cc + 2 * (cov_ab + cov_ac + cov_bc)) / 3.0;
  const double p = 1.6075;
  double f = (std::pow(a * b, p) + std::pow(a * c, p) + std::pow(b * c, p)) / 3;
  e.surf_area = 4 * kPi * std::pow(f, 1.0 / p);
  double da = e.surf_area * std::pow(a, p - 1) * (std::pow(b, p) + std::pow(c, p)) / (3 * f);
  double db = e.surf_area * std::pow(b, p - 1) * (std::pow(a, p) + std::pow(c, p)) / (3 * f);
  double dc = e.surf_area * std::pow(c, p - 1) * (std::pow(a, p) + std::pow(b, p)) / (3 * f);
  e.surf_area_unc = std::sqrt(da * da * cov_aa + db * db * cov_bb + dc * dc * cov_cc +
                              2 * (da * db * cov_ab + da * dc * cov_ac + db * dc * cov_bc));
  e.a = a; e.b = b; e.c = c;
  e.rmsd = rmsd;
  double cv[9] = {cov_aa, cov_ab, cov_ac, cov_ab, cov_bb, cov_bc, cov_ac, cov_bc, cov_cc};
  std::memcpy(e.cov, cv, sizeof cv);
}

// impactParam::enlargeEllipBoundry (impactParam.cpp:950-995): grow all axes
// by 0.01 A until every boundary point is inside (at most 3x the fit).
void enlarge_ellipsoid(const std::vector<V3> &pts, Ellipsoid &e) {
  const double aOld = e.a;
  double a = e.a, b = e.b, c = e.c;
  bool accept = false;
  do {
    for (int i = 0; i < (int)pts.size() + 1; i++) {
      if (i == (int)pts.size() || a > 3 * aOld) { accept = true; break; }
      double mag = pts[i].X * pts[i].X / (a * a) + pts[i].Y * pts[i].Y / (b * b) +
                   pts[i].Z * pts[i].Z / (c * c);
      if (mag > 1) {
        a = a + 0.01; b = b + 0.01; c = c + 0.01;
        break;
      }
    }
  } while (!accept);
  e.enlarge = a - aOld;
  e.a = a; e.b = b; e.c = c;
}

// ---- PCM clusters ------------------------------------------------------------------------

// eigen3D::getEigenvalues / getEigenvectors (eigen3D.cpp:34-113)
static void pcm_eigenvalues(double A[3][3], double ev[3]) {
  double a0, a1, a2, p, q, R, Q, D, a, b = 0, phase, mag;
  a0 = A[0][0] * A[1][1] * A[2][2] - A[0][0] * A[1][2] * A[2][1] - A[1][1] * A[0][2] * A[2][0] -
       A[2][2] * A[0][1] * A[1][0] + A[0][1] * A[1][2] * A[2][0] + A[0][2] * A[2][1] * A[1][0];
  a1 = A[0][1] * A[1][0] + A[0][2] * A[2][0] + A[1][2] * A[2][1] - A[0][0] * A[1][1] -
       A[1][1] * A[2][2] - A[2][2] * A[0][0];
  a2 = A[0][0] + A[1][1] + A[2][2];
  a0 = -a0; a1 = -a1; a2 = -a2;
  p = (3 * a1 - a2 * a2) / 3;
  q = (9 * a1 * a2 - 27 * a0 - 2 * a2 * a2 * a2) / 27;
  Q = p / 3; R = q / 2; D = Q * Q * Q + R * R;
  if (D < 0) {
    a = R; b = std::sqrt(-D);
  } else {
    a = R + std::sqrt(D);   // eigen3D.cpp:68-71 leaves b as it was; it starts at 0 here
  }
  phase = std::atan2(b, a);
  mag = std::pow(a * a + b * b, 1.0 / 6.0);
  ev[0] = -(a2 / 3) + mag * 2 * std::cos(phase / 3.0);
  ev[1] = -(a2 / 3) - mag * (std::cos(phase / 3.0) + std::sqrt(3) * std::sin(phase / 3.0));
  ev[2] = -(a2 / 3) - mag * (std::cos(phase / 3.0) - std::sqrt(3) * std::sin(phase / 3.0));
}

static void pcm_eigenvectors(double A[3][3], const double l[3], double E[3][3]) {
  double T[3][3];
  for (int n = 0; n < 3; n++) {
    double det = l[n] * A[0][2] - A[0][2] * A[1][1] + A[0][1] * A[1][2];
    double y = (A[0][2] * A[1][0] + l[n] * A[1][2] - A[0][0] * A[1][2]) / det;
    double z = (l[n] * l[n] - l[n] * (A[0][0] + A[1][1]) - A[0][1] * A[1][0] + A[0][0] * A[1][1]) / det;
    double nf = std::sqrt(1 + y * y + z * z);
    T[0][n] = 1.0 / nf; T[1][n] = y / nf; T[2][n] = z / nf;
  }
  for (int n = 0; n < 3; n++)
    for (int m = 0; m < 3; m++) E[n][m] = T[m][n];
}

struct PCM {
  std::vector<V3> coords;
  std::vector<std::vector<int>> groups;
  std::vector<V3> center, maxDist;

  // PCM_Cluster::setProperties (PCM_Cluster.cpp:163-225): geometric centre;
  // maxDist skips the first member (the reference stores it as minDist).
  bool set_properties() {
    const size_t nc = groups.size();
    center.assign(nc, V3());
    maxDist.assign(nc, V3());
    for (size_t i = 0; i < nc; i++) {
      if (groups[i].empty()) return false;
      V3 c(0, 0, 0);
      for (int j : groups[i]) c = c + coords.at(j);
      center[i] = c / (double)groups[i].size();
    }
    for (size_t i = 0; i < nc; i++) {
      bool first = true;
      for (size_t j = 0; j < groups[i].size(); j++) {
        V3 d = center[i] - coords[groups[i][j]];
        double dm = d.mag();
        if (first) first = false;
        else if (dm > maxDist[i].mag()) maxDist[i] = center[i] - coords[groups[i][j]];
      }
    }
    return true;
  }

  void cov(const std::vector<int> &ids, double M[3][3]) const {   // PCM_Cluster.cpp:134-161
    double mean[3] = {0.0, 0.0, 0.0};
    for (int i : ids)
      for (int j = 0; j < 3; j++) mean[j] += coords[i].at(j);
    for (int j = 0; j < 3; j++) mean[j] = mean[j] / ((double)ids.size());
    for (int i = 0; i < 3; i++)
      for (int j = i; j < 3; j++) {
        double sum = 0;
        for (int k : ids) sum += (coords[k].at(i) - mean[i]) * (coords[k].at(j) - mean[j]);
        M[i][j] = sum;
        if (i != j) M[j][i] = sum;
      }
  }

  // PCM_Cluster::formClusters (PCM_Cluster.cpp:38-132)
  bool form(int maxClusterSize) {
    std::vector<int> all(coords.size());
    for (size_t i = 0; i < coords.size(); i++) all[i] = (int)i;
    groups.assign(1, all);
    if (!set_properties()) return false;
    for (int pass = 0;; pass++) {
      if (pass > 100000) return false;
      const size_t size = groups.size();
      for (size_t i = 0; i < size; i++) {
        if (maxDist[i].mag() > maxClusterSize) {
          double vals[3], vecs[3][3], M[3][3];
          cov(groups[i], M);
          pcm_eigenvalues(M, vals);
          pcm_eigenvectors(M, vals, vecs);
          int imax = 0;
          for (int k = 0; k < 3; k++)
            if (std::fabs(vals[k]) > vals[imax]) imax = k;
          V3 c(0.0, 0.0, 0.0);
          for (int k : groups[i]) c = c + coords[k];
          c = c / ((double)groups[i].size());
          std::vector<int> c1, c2;
          for (int k : groups[i]) {
            double ang = angle_to(coords[k] - c, vecs[imax]);
            if (ang <= kPi2) c1.push_back(k);
            else c2.push_back(k);
          }
          groups[i].swap(c1);
          groups.push_back(c2);
        }
      }
      if (!set_properties()) return false;
      bool accept = true;
      for (size_t i = 0; i < groups.size(); i++)
        if (maxDist[i].mag() > maxClusterSize) { accept = false; break; }
      if (accept) break;
    }
    if (!set_properties()) return false;
    // orderClusters (PCM_Cluster.cpp:227-249): selection sort by centre z
    const int size = (int)groups.size();
    for (int n = 0; n < size - 1; n++) {
      int minIndex = n;
      double minValue = center[n].Z;
      for (int i = n + 1; i < size; i++)
        if (center[i].Z < minValue) { minValue = center[i].Z; minIndex = i; }
      std::swap(maxDist[n], maxDist[minIndex]);
      std::swap(center[n], center[minIndex]);
      std::swap(groups[n], groups[minIndex]);
    }
    return true;
  }
};

// forceAccel::setClusters + addMultipole + addClusterPos (forceAccel.cpp:53-210)
bool form_clusters(const Molecule &m, int maxClusterSize, Clusters &cl, Log &log) {
  PCM pcm;
  for (const Atom &a : m.atoms) pcm.coords.push_back(V3(a.x, a.y, a.z));
  if (!pcm.form(maxClusterSize)) {
    log.printf("Error: cluster formation failed (empty cluster)\n");
    return false;
  }
  const int nc = (int)pcm.groups.size();
  cl.offset.assign(1, 0);
  cl.atoms.clear();
  cl.pos.clear(); cl.radius.clear(); cl.charge.clear(); cl.dipole.clear(); cl.quad.clear();
  cl.replaced.clear();
  cl.n_replaced = 0;
  double avgRad = 0, avgSize = 0;
  for (int k = 0; k < nc; k++) {
    const std::vector<int> &g = pcm.groups[k];
    const V3 center = pcm.center[k];
    double sumCharge = 0.0;
    double dip[3] = {0, 0, 0}, quad[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int idx : g) {
      const Atom &a = m.atoms[idx];
      double charge = a.charge;
      sumCharge += charge;
      double p[3] = {a.x - center.X, a.y - center.Y, a.z - center.Z};
      double mag2 = p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
      for (int i = 0; i < 3; i++) {
        dip[i] += charge * p[i];
        for (int j = 0; j < 3; j++) quad[i][j] += charge * (3 * p[i] * p[j] - mag2 * (i == j ? 1.0 : 0.0));
      }
    }
    V3 coc(0, 0, 0);
    for (int idx : g) coc = coc + V3(m.atoms[idx].x, m.atoms[idx].y, m.atoms[idx].z) * m.atoms[idx].charge;
    coc = coc / sumCharge;
    double pct = 100 * std::fabs((coc.mag() - center.mag()) / coc.mag());
    const bool repl = pct <= 5;
    const V3 pos = repl ? coc : center;
    cl.n_replaced += repl ? 1 : 0;
    const double R = pcm.maxDist[k].mag();
    for (int idx : g) cl.atoms.push_back(idx);
    cl.offset.push_back((int)cl.atoms.size());
    cl.pos.push_back(pos.X); cl.pos.push_back(pos.Y); cl.pos.push_back(pos.Z);
    cl.radius.push_back(R);
    cl.charge.push_back(sumCharge);
    for (int i = 0; i < 3; i++) cl.dipole.push_back(dip[i]);
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) cl.quad.push_back(quad[i][j]);
    cl.replaced.push_back(repl ? 1 : 0);
    avgRad += R;
    avgSize += g.size();
  }
  cl.avg_size = avgSize / (double)nc;
  cl.avg_radius = avgRad / (double)nc;
  return true;
}

}  // namespace host
}  // namespace cosims
