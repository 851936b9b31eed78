// host_api.cpp -- C ABI of the host side (include/cosims_host.h): input-file
// parameters and the per-molecule setup sequence of monteTraj::monteTraj.
#include <algorithm>
#include <cctype>
#include <chrono>
#include <cmath>
#include <cstring>
#include <fstream>
#include <random>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "host_internal.h"

namespace cosims {
cosims_status fail(cosims_status s, const char *fmt, ...);
}

namespace cosims {
namespace host {

static const double kPi = 3.14159265358979323846;
static const double kBoltzmann = 0.831446214563;      // maxBoltz.h:29
static const double kHeliumMass = 4.002602;           // monteTraj.cpp:31
static const double kDipoleScalar = 28276.01363;      // forceAccel.cpp:35

static void copy_str(char *dst, size_t cap, const std::string &s) {
  size_t n = std::min(cap - 1, s.size());
  std::memcpy(dst, s.data(), n);
  dst[n] = 0;
}

// fileParams::setDefaultParams name rule (fileParams.cpp:212-224): the file
// name's stem up to its first '.'.
static std::string stem_of(const std::string &path) {
  std::string t;
  for (int i = (int)path.size() - 1; i >= 0; i--) {
    char ch = path[i];
    if (ch == '/' || ch == '\\') break;
    if (ch == '.') t.clear();
    else t += ch;
  }
  std::reverse(t.begin(), t.end());
  return t;
}

static bool is_int(const std::string &s) {
  for (char ch : s)
    if (!isdigit((unsigned char)ch)) return false;
  return true;
}

// fileParams::getBool (fileParams.cpp:62-76)
static bool get_bool(const std::string &v) {
  std::string s = v;
  std::transform(s.begin(), s.end(), s.begin(), ::tolower);
  if (is_int(v)) return std::strtoll(v.c_str(), nullptr, 10) != 0;
  return s == "true";
}

}  // namespace host
}  // namespace cosims

using namespace cosims;
using namespace cosims::host;

struct cosims_setup {
  cosims_config cfg;
  std::vector<FFEntry> ff;
  Molecule mol;
  MolFlags flags;
  std::vector<V3> boundary;
  Ellipsoid ell;
  Clusters cl;
  cosims_setup_info info;
  // views handed out through cosims_setup_molecule
  std::vector<double> x, y, z, q, sig6, eps24m, eps4;
  cosims_params par;
};

extern "C" {

cosims_status cosims_config_defaults(cosims_config *c, const char *mol_path) {
  if (!c) return fail(COSIMS_ERR_INVALID, "config is NULL");
  const bool keep_threads = (c->changed & COSIMS_KEY_THREADS) != 0;
  const bool keep_seed = (c->changed & COSIMS_KEY_SEED) != 0;
  const int32_t threads = c->threads;
  const int64_t seed = c->seed;
  std::memset(c, 0, sizeof *c);
  copy_str(c->name, sizeof c->name, stem_of(mol_path ? mol_path : ""));
  c->dt = 0.01;
  c->temp = 298;
  c->traj = 50000;
  c->iter = 10;
  c->threads = keep_threads ? threads : 1;
  if (keep_seed) {
    c->seed = seed;
    c->seed_set = 1;
    c->changed |= COSIMS_KEY_SEED;
  } else {
    std::random_device rd;
    c->seed = rd();
  }
  if (keep_threads) c->changed |= COSIMS_KEY_THREADS;
  c->dispersion_cutoff = 1;
  c->dispersion_radius = 0;
  c->multipole = 1;
  c->multipole_radius = 0;
  c->multipole_order = 1;
  c->print_rate = 20000;
  c->display_progress = 1;
  c->max_cluster_size = 4;
  c->charge = 0;
  c->charged = 0;
  c->gmax = 35;
  c->gmin = 5;
  c->proj = 1;
  return COSIMS_OK;
}

// fileParams::importParams (fileParams.cpp:261-510)
cosims_status cosims_config_read(cosims_config *c, const char *input_path, const char *mol_path,
                                 char *log_out, int64_t log_cap) {
  if (!c || !input_path) return fail(COSIMS_ERR_INVALID, "config and input path are required");
  Log log;
  log.printf(" Reading input file: %s\n", input_path);
  std::ifstream f(input_path);
  if (!f) {
    log.copy_to(log_out, log_cap);
    return fail(COSIMS_ERR_IO, "cannot open input file %s", input_path);
  }
  cosims_config_defaults(c, mol_path);
  uint32_t seen = 0;   // keys already given, for the repeated-key warning
  std::string line;
  int lineNum = 1;
  bool changed_print_rate = false;
  while (std::getline(f, line)) {
    std::istringstream st(line);
    if (!line.empty()) {
      std::string option, value;
      st >> option >> value;
      if (value.empty()) {
        log.printf("\t ERROR: Line number %i in %s is incomplete;\n\t This line wil be "
                   "ignored.\n\n", lineNum, input_path);
      } else if (option[0] != '#') {
        static const char *keys[] = {
            "name", "dir", "dt", "temp", "traj", "iter", "threads", "seed", "gmax", "gmin",
            "print_mol", "proj", "print_traj", "print_traj_fail", "print_data",
            "print_data_fail", "dispersion_cutoff", "dispersion_radius", "multipole_radius",
            "multipole_order", "print_rate", "multipole", "max_cluster_size", "charge"};
        int k = -1;
        for (int i = 0; i < (int)(sizeof keys / sizeof keys[0]); i++)
          if (option == keys[i]) { k = i; break; }
        if (k < 0) {
          log.printf("\tERROR: Can not interpret option '%s' on \n\tline number %i in %s;\n"
                     "\tThis line wil be ignored.\n\n", option.c_str(), lineNum, input_path);
        } else {
          if (seen & (1u << k)) {
            std::string up = option;
            std::transform(up.begin(), up.end(), up.begin(), ::toupper);
            log.printf("\tWARNING: Parameter %s already specified at line number %i;\n"
                       "\tMost recent value will be applied.\n\n", up.c_str(), lineNum);
          }
          seen |= 1u << k;
          const char *v = value.c_str();
          switch (k) {
            case 0: copy_str(c->name, sizeof c->name, value); c->changed |= COSIMS_KEY_NAME; break;
            case 1: copy_str(c->dir, sizeof c->dir, value); break;
            case 2: c->dt = atof(v); break;
            case 3: c->temp = atof(v); break;
            case 4: c->traj = (int)(atof(v) * 1000); break;
            case 5: c->iter = (int)atof(v); break;
            case 6: c->threads = (int)atof(v); c->changed |= COSIMS_KEY_THREADS; break;
            case 7: c->seed = atoll(v); c->seed_set = 1; c->changed |= COSIMS_KEY_SEED; break;
            case 8: c->gmax = atof(v); c->debugging = 1; break;
            case 9: c->gmin = atof(v); c->debugging = 1; break;
            case 10: c->print_mol = std::strtoll(v, nullptr, 10) != 0; c->debugging = 1; break;
            case 11: c->proj = (int)atof(v) != 0; c->debugging = 1; break;
            case 12: c->print_traj = get_bool(value); c->debugging = 1; break;
            case 13: c->print_traj_fail = get_bool(value); c->debugging = 1; break;
            case 14: c->print_data = get_bool(value); c->debugging = 1; break;
            case 15: c->print_data_fail = get_bool(value); c->debugging = 1; break;
            case 16: c->dispersion_cutoff = get_bool(value); break;
            case 17: c->dispersion_radius = atof(v); break;
            case 18: c->multipole_radius = atof(v); break;
            case 19: c->multipole_order = atoi(v); break;
            case 20: c->print_rate = (int)atof(v); c->display_progress = 1;
                     changed_print_rate = true; c->changed |= COSIMS_KEY_PRINT_RATE; break;
            case 21: c->multipole = get_bool(value); break;
            case 22: c->max_cluster_size = atoi(v); break;
            case 23: c->charge = atof(v); c->charged = c->charge != 0;
                     c->changed |= COSIMS_KEY_CHARGE; break;
          }
        }
      }
    }
    lineNum++;
  }
  if (!changed_print_rate) {
    c->print_rate = (int)(c->traj / 5.0);
  } else if (c->print_rate > c->traj || c->print_rate == 0) {
    c->print_rate = (int)c->traj;
    c->display_progress = 0;
  }
  std::string dir = c->dir;
  if (!dir.empty() && dir.back() != '/') {
    dir += "/";
    copy_str(c->dir, sizeof c->dir, dir);
  }
  std::string name = c->name;
  name += "_" + std::to_string((int)c->charge);
  copy_str(c->name, sizeof c->name, name);
  log.copy_to(log_out, log_cap);
  return COSIMS_OK;
}

static cosims_status setup_create(const cosims_config *cfg, const char *mol_path,
                                  const char *atom_path, int device, int structure,
                                  char *log_out, int64_t log_cap, cosims_setup **out) {
  if (!cfg || !mol_path || !out) return fail(COSIMS_ERR_INVALID, "config, molecule and out are required");
  *out = nullptr;
  // wall time of the setup phases (cosims_setup_info::setup_ms)
  double phase_ms[6] = {0, 0, 0, 0, 0, 0};
  auto clock = std::chrono::steady_clock::now();
  auto lap = [&](int k) {
    const auto now = std::chrono::steady_clock::now();
    phase_ms[k] += std::chrono::duration<double, std::milli>(now - clock).count();
    clock = now;
  };
  Log log;
  cosims_setup *s = new cosims_setup();
  s->cfg = *cfg;
  s->ff = default_force_field();
  if (atom_path && *atom_path && !read_atom_file(atom_path, s->ff, log)) {
    log.copy_to(log_out, log_cap);
    delete s;
    return fail(COSIMS_ERR_IO, "cannot read atom file %s", atom_path);
  }
  // molecule type from the extension (fileParams::checkMolFileType, fileParams.cpp:680-694)
  std::string path = mol_path;
  if (path.size() < 4 || path[path.size() - 4] != '.') {
    delete s;
    return fail(COSIMS_ERR_IO, "molecule file must end in .pdb or .mfj: %s", mol_path);
  }
  std::string ext = path.substr(path.size() - 3);
  std::transform(ext.begin(), ext.end(), ext.begin(), ::tolower);
  RawMolecule raw;
  s->flags.charged = cfg->charged != 0;
  s->flags.total_charge = cfg->charge;
  bool ok;
  if (ext == "pdb") ok = read_pdb(path, raw, log, structure);
  else if (ext == "mfj") ok = read_mfj(path, s->ff, raw, s->flags, log, structure);
  else {
    delete s;
    return fail(COSIMS_ERR_IO, "molecule file must end in .pdb or .mfj: %s", mol_path);
  }
  if (!ok) {
    log.copy_to(log_out, log_cap);
    delete s;
    // the reader's last error line says what is wrong with the file
    std::string why;
    const size_t at = log.text.rfind("Error");
    if (at != std::string::npos) {
      why = log.text.substr(at);
      why = why.substr(0, why.find('\n'));
    }
    return fail(COSIMS_ERR_IO, "cannot read molecule file %s%s%s", mol_path,
                why.empty() ? "" : ": ", why.c_str());
  }
  lap(0);
  double r_disp = cfg->dispersion_radius, r_mp = cfg->multipole_radius;
  if (!set_properties(raw, s->ff, s->flags, s->mol, r_disp, r_mp, cfg->dispersion_cutoff != 0,
                      cfg->multipole != 0, log)) {
    log.copy_to(log_out, log_cap);
    delete s;
    return fail(COSIMS_ERR_IO, "unknown atom type in %s", mol_path);
  }
  rotate_to_inertia_frame(s->mol, log);
  lap(1);
  Molecule &m = s->mol;
  const bool charged = s->flags.charged;
  // monteTraj::monteTraj (monteTraj.cpp:31-94)
  const double mu = m.totalMass * kHeliumMass / (m.totalMass + kHeliumMass);
  const double beta = mu / (kBoltzmann * cfg->temp);
  const int distrPower = 5;
  const double va = beta / 2.0;
  double norm = vd_norm(distrPower, va);
  const double mean = vd_mean(distrPower, va), sd = vd_std(distrPower, va);
  const double gMin = mean - 2 * sd, gMax = mean + 4 * sd;
  norm = norm / (vd_cdf(distrPower, va, gMax) - vd_cdf(distrPower, va, gMin));
  const double mode = vd_mode(distrPower, va);
  const double maxVelDistr = std::pow(mode, distrPower) * std::exp(-va * mode * mode) * norm;
  const double dipole_scalar = kDipoleScalar / mu;
  const double minKin = 0.5 * mu * std::pow(vd_mean(2, beta / 2.0) - 2 * vd_std(2, beta / 2.0), 2);
  lap(2);
  int threads = cfg->threads > 0 ? cfg->threads : 1;
  if (threads == 1) threads = std::max(1u, std::thread::hardware_concurrency());
  if (!boundary_scan(m, charged, dipole_scalar, minKin, threads, device, s->boundary, log)) {
    log.copy_to(log_out, log_cap);
    delete s;
    return fail(COSIMS_ERR_INVALID, "potential-energy boundary scan failed");
  }
  lap(3);
  fit_ellipsoid(s->boundary, s->ell);
  Ellipsoid fitted = s->ell;
  enlarge_ellipsoid(s->boundary, s->ell);
  lap(4);
  const double bMax = std::max(s->ell.a, std::max(s->ell.b, s->ell.c));   // impactParam.cpp:417
  // forceAccel::setClusters (forceAccel.cpp:63-140)
  const bool clusters = cfg->multipole || cfg->dispersion_cutoff;
  if (clusters && !form_clusters(m, cfg->max_cluster_size, s->cl, log)) {
    log.copy_to(log_out, log_cap);
    delete s;
    return fail(COSIMS_ERR_INVALID, "cluster formation failed");
  }
  lap(5);
  int force_type;
  if (charged)
    force_type = cfg->multipole ? (cfg->dispersion_cutoff ? 1 : 2)
                                : (cfg->dispersion_cutoff ? 3 : 4);
  else
    force_type = cfg->dispersion_cutoff ? 5 : 6;
  double const1 = std::pow(beta, 3) / (64 * kPi);
  const1 = const1 * 8 * kPi * kPi;
  const1 = const1 / norm;
  const double const2 = bMax * bMax;

  cosims_params &p = s->par;
  std::memset(&p, 0, sizeof p);
  p.force_type = force_type;
  p.multipole_order = cfg->multipole_order;
  p.projection = cfg->proj != 0;
  p.charged = charged;
  p.dt = cfg->dt;
  p.mu = mu;
  p.dipole_scalar = dipole_scalar;
  p.r_disp = r_disp;
  p.r_mp = r_mp;
  p.ell_a = s->ell.a; p.ell_b = s->ell.b; p.ell_c = s->ell.c;
  p.b_max = bMax;
  p.start_dist = (double)(float)bMax;      // monteTraj::maxDist is a float (monteTraj.h)
  p.g_min = gMin; p.g_max = gMax;
  p.vdist_a = va;
  p.vdist_norm = norm;
  p.vdist_max = maxVelDistr;
  p.ccs_const = const1 * const2;
  p.max_steps = 0;

  const int n = (int)m.atoms.size();
  s->x.resize(n); s->y.resize(n); s->z.resize(n); s->q.resize(n);
  s->sig6.resize(n); s->eps24m.resize(n); s->eps4.resize(n);
  for (int i = 0; i < n; i++) {
    const Atom &a = m.atoms[i];
    s->x[i] = a.x; s->y[i] = a.y; s->z[i] = a.z; s->q[i] = a.charge;
    s->sig6[i] = a.sig6; s->eps24m[i] = a.eps24m; s->eps4[i] = a.eps4;
  }
  cosims_setup_info &in = s->info;
  std::memset(&in, 0, sizeof in);
  in.n_atoms = n;
  in.n_clusters = clusters ? (int)s->cl.radius.size() : 0;
  in.n_boundary = (int)s->boundary.size();
  in.force_type = force_type;
  in.total_mass = m.totalMass;
  in.mu = mu;
  in.total_charge = s->flags.total_charge;
  for (int k = 0; k < 3; k++) in.center[k] = m.center[k];
  in.radius_gyration = m.radius_gyration;
  for (int k = 0; k < 9; k++) {
    in.inertia[k] = m.inertia[k];
    in.rotation[k] = m.rotation[k];
    in.quadrupole[k] = m.quad[k];
    in.cov[k] = fitted.cov[k];
  }
  for (int k = 0; k < 3; k++) {
    in.dipole[k] = m.dipole[k];
    in.ell_unc[k] = fitted.unc[k];
  }
  in.ell_a = s->ell.a; in.ell_b = s->ell.b; in.ell_c = s->ell.c;
  in.rmsd = fitted.rmsd;
  in.avg_axes = fitted.avg_axes;
  in.avg_axes_unc = fitted.avg_axes_unc;
  in.surf_area = fitted.surf_area;
  in.surf_area_unc = fitted.surf_area_unc;
  in.enlarge = s->ell.enlarge;
  in.b_max = bMax;
  in.g_min = gMin; in.g_max = gMax;
  in.g_mean = mean; in.g_mode = mode;
  in.pct_used = 100 * (vd_cdf(distrPower, va, gMax) - vd_cdf(distrPower, va, gMin));
  in.beta = beta;
  in.ccs_const = p.ccs_const;
  in.r_disp = r_disp;
  in.r_mp = r_mp;
  in.centers_replaced = s->cl.n_replaced;
  in.avg_cluster_size = s->cl.avg_size;
  in.avg_cluster_radius = s->cl.avg_radius;
  for (int k = 0; k < 6; k++) in.setup_ms[k] = phase_ms[k];
  s->info.n_clusters = in.n_clusters;
  // axes of the fit before enlargement are kept in fitted; the path uses the enlarged ones
  (void)fitted;
  log.copy_to(log_out, log_cap);
  *out = s;
  return COSIMS_OK;
}

cosims_status cosims_setup_create(const cosims_config *cfg, const char *mol_path,
                                  const char *atom_path, char *log_out, int64_t log_cap,
                                  cosims_setup **out) {
  return setup_create(cfg, mol_path, atom_path, -1, -1, log_out, log_cap, out);
}

cosims_status cosims_setup_create_device(const cosims_config *cfg, const char *mol_path,
                                         const char *atom_path, int32_t device, char *log_out,
                                         int64_t log_cap, cosims_setup **out) {
  if (device < 0) return fail(COSIMS_ERR_INVALID, "device must be >= 0");
  return setup_create(cfg, mol_path, atom_path, device, -1, log_out, log_cap, out);
}

static bool is_pdb_path(const char *p) {
  std::string path = p;
  if (path.size() < 4) return false;
  std::string ext = path.substr(path.size() - 3);
  std::transform(ext.begin(), ext.end(), ext.begin(), ::tolower);
  return ext == "pdb";
}

cosims_status cosims_molecule_file_structures(const char *mol_path, int32_t *count) {
  if (!mol_path || !count) return fail(COSIMS_ERR_INVALID, "molecule path and count are required");
  const int k = count_structures(mol_path, is_pdb_path(mol_path));
  if (k < 0) return fail(COSIMS_ERR_IO, "cannot read molecule file %s", mol_path);
  *count = k;
  return COSIMS_OK;
}

cosims_status cosims_setup_create_structure(const cosims_config *cfg, const char *mol_path,
                                            const char *atom_path, int32_t structure,
                                            int32_t device, char *log_out, int64_t log_cap,
                                            cosims_setup **out) {
  if (!mol_path) return fail(COSIMS_ERR_INVALID, "molecule path is required");
  const int k = count_structures(mol_path, is_pdb_path(mol_path));
  if (k < 0) return fail(COSIMS_ERR_IO, "cannot read molecule file %s", mol_path);
  if (structure < 0 || structure >= k)
    return fail(COSIMS_ERR_INVALID, "structure %d of a file with %d", structure, k);
  // a single-structure file is read exactly as cosims_setup_create reads it
  return setup_create(cfg, mol_path, atom_path, device, k == 1 ? -1 : structure, log_out,
                      log_cap, out);
}

cosims_status cosims_setup_molecule(const cosims_setup *s, cosims_molecule *m, cosims_params *p) {
  if (!s || !m || !p) return fail(COSIMS_ERR_INVALID, "setup, molecule and params are required");
  std::memset(m, 0, sizeof *m);
  m->n_atoms = (int32_t)s->x.size();
  m->x = s->x.data(); m->y = s->y.data(); m->z = s->z.data();
  m->charge = s->q.data(); m->sig6 = s->sig6.data(); m->eps24m = s->eps24m.data();
  m->eps4 = s->eps4.data();
  m->n_clusters = s->info.n_clusters;
  if (m->n_clusters) {
    m->cluster_offset = s->cl.offset.data();
    m->cluster_atoms = s->cl.atoms.data();
    m->cluster_pos = s->cl.pos.data();
    m->cluster_radius = s->cl.radius.data();
    m->cluster_charge = s->cl.charge.data();
    m->cluster_dipole = s->cl.dipole.data();
    m->cluster_quad = s->cl.quad.data();
    m->cluster_replaced = s->cl.replaced.data();
  }
  *p = s->par;
  return COSIMS_OK;
}

cosims_status cosims_setup_get_info(const cosims_setup *s, cosims_setup_info *info) {
  if (!s || !info) return fail(COSIMS_ERR_INVALID, "setup and info are required");
  *info = s->info;
  return COSIMS_OK;
}

int64_t cosims_setup_boundary(const cosims_setup *s, double *xyz, int64_t cap) {
  if (!s) return 0;
  const int64_t n = (int64_t)s->boundary.size();
  for (int64_t i = 0; i < n && i < cap && xyz; i++) {
    xyz[3 * i] = s->boundary[i].X;
    xyz[3 * i + 1] = s->boundary[i].Y;
    xyz[3 * i + 2] = s->boundary[i].Z;
  }
  return n;
}

const char *cosims_setup_atom_symbol(const cosims_setup *s, int32_t i) {
  if (!s || i < 0 || i >= (int32_t)s->mol.atoms.size()) return "";
  return s->mol.atoms[i].symbol.c_str();
}

void cosims_setup_destroy(cosims_setup *s) { delete s; }

}  // extern "C"
