// cosims_gpu -- command-line CCS run on the GPU engine: the same command line,
// input file and omega_<name>.txt output as the reference program
// (main.cpp:93-150, fileParams::interpretCMD fileParams.cpp:78-202,
// monteTraj::runTraj monteTraj.cpp:281-453), with two extra options.
//
//   cosims_gpu -m <molecule .pdb|.mfj> [-i <input file>] [-a <atoms.dat>]
//              [-s <seed>] [-n <host threads>] [-p plain|mixed] [-g <device>]
//
// -p plain (default) is the reference method in FP64; -p mixed the mixed
// precision form.  Trajectory inputs come from the engine's counter-based
// sampler keyed by the seed (integral k draws trajectories k*traj ...
// (k+1)*traj-1), so a run reproduces itself for a given seed but not the
// reference's mt19937_64 stream.  The per-integral and summary lines keep the
// reference's text and number formats, so tools that read its omega files
// read these.
#include <unistd.h>
#include <algorithm>
#include <chrono>
#include <cstdarg>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <string>
#include <vector>
#include "cosims_cuda.h"
#include "cosims_host.h"

namespace {

struct Out {
  FILE *f = nullptr;
  void printf(const char *fmt, ...) __attribute__((format(printf, 2, 3)));
};

void Out::printf(const char *fmt, ...) {
  char buf[4096];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  fputs(buf, stdout);
  if (f) {
    fputs(buf, f);
    fflush(f);
  }
}

bool is_int(const char *s) {
  if (!*s) return false;
  if (*s == '-' || *s == '+') s++;
  if (!*s) return false;
  for (; *s; s++)
    if (*s < '0' || *s > '9') return false;
  return true;
}

int digits(double v) {   // the reference's (int)log10(x) + 3 field widths
  return v > 0 ? (int)std::log10(v) + 3 : 3;
}

void usage() {
  std::fprintf(stderr,
               "usage: cosims_gpu -m <molecule.pdb|.mfj> [-i <input>] [-a <atoms.dat>] "
               "[-s <seed>] [-n <threads>] [-p plain|mixed] [-g <device>]\n");
}


// monteTraj::printData's line (monteTraj.cpp:555-571)
void write_data_line(FILE *f, const cosims_traj_in &in, const cosims_traj_out &o,
                     const double *p0, const double *v0) {
  std::fprintf(f, "%8.3g  %8.3g  %8.3g  %8.3g  %8.3g  %8.3g  %8i  %8.3g  %8.3g  %8.3g  %8.3g  "
               "%8.3g  %8.3g \n", in.phi, in.theta, in.gamma, in.g, in.b, o.chi, o.steps, p0[0],
               p0[1], p0[2], v0[0], v0[1], v0[2]);
}

// monteTraj::storeTraj's frame (monteTraj.cpp:573-585), one per integration step
void write_frame(FILE *f, const double *fr) {
  std::fprintf(f, "1\nno comments available \nHe     %.15f       %.15f       %.15f     "
               "%.15f       %.15f       %.15f\n", fr[0], fr[1], fr[2], fr[3], fr[4], fr[5]);
}

// Trajectories traced per integral for print_traj, and the frames kept of each.
constexpr int kTracedPerIntegral = 16;
constexpr int kTraceFrames = 100000;

// One coordinate set: setup, context, the integrals and the summary block of
// monteTraj::runTraj (monteTraj.cpp:281-453).  Returns false after an error.
bool run_set(cosims_config &cfg, const std::string &mol_path, const std::string &atom_path,
             int set, int n_sets, int device, int precision, const std::string &path,
             std::vector<char> &log, Out &out, double &ccs, double &ccs_err) {
  cosims_setup *setup = nullptr;
  std::fill(log.begin(), log.end(), 0);
  cosims_status st =
      n_sets > 1 ? cosims_setup_create_structure(&cfg, mol_path.c_str(), atom_path.c_str(), set,
                                                 device, log.data(), (int64_t)log.size(), &setup)
                 : cosims_setup_create_device(&cfg, mol_path.c_str(), atom_path.c_str(), device,
                                              log.data(), (int64_t)log.size(), &setup);
  out.printf("%s", log.data());
  if (st != COSIMS_OK) {
    out.printf("ERROR: Cannot read molecule file (%s).\nProgram will now exit...\n",
               cosims_last_error());
    return false;
  }
  cosims_setup_info info;
  cosims_setup_get_info(setup, &info);
  out.printf("\n Molecule: %d atoms, mass %.4f, reduced mass %.6f, total charge %.3f\n",
             info.n_atoms, info.total_mass, info.mu, info.total_charge);
  out.printf(" Radius of gyration: %.4f\n", info.radius_gyration);
  out.printf(" Ellipsoid axes (enlarged): %.4f %.4f %.4f; b_max %.4f\n", info.ell_a, info.ell_b,
             info.ell_c, info.b_max);
  out.printf(" Relative speeds: %.4f - %.4f; fraction of the distribution %.4f %%\n", info.g_min,
             info.g_max, info.pct_used);
  out.printf(" Force variant %d; clusters %d; parameters: dt %g ps, T %g K, %lld trajectories x "
             "%d integrals, seed %lld\n",
             info.force_type, info.n_clusters, cfg.dt, cfg.temp, (long long)cfg.traj, cfg.iter,
             (long long)cfg.seed);

  cosims_molecule mol;
  cosims_params par;
  cosims_setup_molecule(setup, &mol, &par);
  const std::string tag = n_sets > 1 ? "_set" + std::to_string(set + 1) : std::string();
  if (cfg.print_mol) {
    // monteTraj::printMolecule (monteTraj.cpp:587-600): the rotated molecule
    const std::string mp = path + "outMol_" + cfg.name + tag + ".xyz";
    if (FILE *f = std::fopen(mp.c_str(), "w")) {
      std::fprintf(f, "%d\nRotated Molecule \n", mol.n_atoms);
      for (int i = 0; i < mol.n_atoms; i++)
        std::fprintf(f, "%s %9.4g %9.4g %9.4g\n", cosims_setup_atom_symbol(setup, i), mol.x[i],
                     mol.y[i], mol.z[i]);
      std::fclose(f);
    }
  }
  cosims_ctx *ctx = nullptr;
  st = cosims_ctx_create(&mol, &par, precision, device, &ctx);
  cosims_ctx *tracer = nullptr;
  if (st == COSIMS_OK && cfg.print_traj)
    st = precision == COSIMS_PRECISION_PLAIN_F64
             ? COSIMS_OK
             : cosims_ctx_create(&mol, &par, COSIMS_PRECISION_PLAIN_F64, device, &tracer);
  if (st != COSIMS_OK) {
    out.printf("ERROR: %s\nProgram will now exit...\n", cosims_last_error());
    cosims_ctx_destroy(ctx);
    cosims_setup_destroy(setup);
    return false;
  }
  if (cfg.print_traj && !tracer) tracer = ctx;
  FILE *data_f = nullptr, *xyz_f = nullptr;
  if (cfg.print_data) data_f = std::fopen((path + "data_" + cfg.name + tag + ".txt").c_str(), "a");
  if (cfg.print_traj) xyz_f = std::fopen((path + "xyz_" + cfg.name + tag + ".xyz").c_str(), "w");

  out.printf(" Starting Trajectory Calculations:\n _________________________________\n\n");
  const int iters = cfg.iter > 0 ? cfg.iter : 1;
  const int64_t n_traj = cfg.traj;
  std::vector<double> omega(iters), err(iters);
  double total_time = 0, max_de = 0;
  const int64_t update_every = cfg.print_rate > 0 ? cfg.print_rate : 0;
  const bool dumps = data_f || xyz_f;
  std::vector<cosims_traj_in> ins(dumps ? n_traj : 0);
  std::vector<cosims_traj_out> outs(dumps ? n_traj : 0);
  std::vector<double> p0(dumps ? 3 * n_traj : 0), v0(dumps ? 3 * n_traj : 0);
  std::vector<int32_t> hit(dumps ? n_traj : 0);
  bool ok = true;
  // Without dumps every integral runs in one cosims_run_integrals call (the
  // same sums as one call per integral, in fewer launches); each integral's
  // "Total time" line then shows its share of that call's time.
  std::vector<cosims_ccs_sums> all(dumps ? 0 : iters);
  double all_time = 0;
  if (!dumps) {
    const auto t0 = std::chrono::steady_clock::now();
    st = cosims_run_integrals(ctx, (uint64_t)cfg.seed, 0, n_traj, iters, update_every, all.data(),
                              nullptr, nullptr);
    all_time = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (st != COSIMS_OK) {
      out.printf("ERROR: %s\n", cosims_last_error());
      ok = false;
    }
  }
  for (int k = 0; ok && k < iters; k++) {
    out.printf("\n Computing CCS integral %i / %i on GPU %d (%s form)\n", k + 1, iters, device,
               precision == COSIMS_PRECISION_MIXED ? "mixed" : "plain FP64");
    const auto t0 = std::chrono::steady_clock::now();
    cosims_ccs_sums s;
    if (dumps) {
      st = cosims_run_sampled(ctx, (uint64_t)cfg.seed, (int64_t)k * n_traj, n_traj, update_every,
                              &s, ins.data(), outs.data(), nullptr);
    } else {
      s = all[k];
    }
    if (st != COSIMS_OK) {
      out.printf("ERROR: %s\n", cosims_last_error());
      ok = false;
      break;
    }
    total_time += dumps ? std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count()
                        : all_time / iters;
    if (dumps) {
      // the debugging dumps: successful trajectories, or failed ones with *_fail
      // (the same draws as the integral: its inputs again, with start states and hits)
      st = cosims_sample_inputs(ctx, (uint64_t)cfg.seed, (int64_t)k * n_traj, n_traj, ins.data(),
                                p0.data(), v0.data(), hit.data(), nullptr);
      std::vector<int64_t> traced;
      for (int64_t i = 0; st == COSIMS_OK && i < n_traj; i++) {
        if (!hit[i]) continue;
        const bool success = (outs[i].status & COSIMS_TRAJ_SUCCESS) != 0;
        if (data_f && success != (cfg.print_data_fail != 0))
          write_data_line(data_f, ins[i], outs[i], &p0[3 * i], &v0[3 * i]);
        if (xyz_f && success != (cfg.print_traj_fail != 0) &&
            (int)traced.size() < kTracedPerIntegral)
          traced.push_back(i);
      }
      if (st == COSIMS_OK && xyz_f && !traced.empty()) {
        const int64_t nt = (int64_t)traced.size();
        std::vector<double> tp(3 * nt), tv(3 * nt), frames((size_t)nt * kTraceFrames * 6);
        std::vector<int32_t> nframes(nt);
        std::vector<cosims_traj_out> to(nt);
        for (int64_t j = 0; j < nt; j++)
          for (int c = 0; c < 3; c++) {
            tp[3 * j + c] = p0[3 * traced[j] + c];
            tv[3 * j + c] = v0[3 * traced[j] + c];
          }
        st = cosims_trace_list(tracer, tp.data(), tv.data(), nt, kTraceFrames, frames.data(),
                               nframes.data(), to.data(), nullptr);
        for (int64_t j = 0; st == COSIMS_OK && j < nt; j++) {
          const int nf = std::min(nframes[j], kTraceFrames);
          for (int f = 0; f < nf; f++) write_frame(xyz_f, &frames[((size_t)j * kTraceFrames + f) * 6]);
        }
      }
      if (st != COSIMS_OK) out.printf("ERROR: debugging dumps: %s\n", cosims_last_error());
    }
    // Omega and its error as monteTraj::runTraj forms them (monteTraj.cpp:380-387)
    const double n_eff = (double)s.n_eff;
    omega[k] = s.sum / n_eff;
    err[k] = std::sqrt((s.sum2 / n_eff - omega[k] * omega[k]) / n_eff);
    max_de = std::max(max_de, s.max_de_pct);
    out.printf(" Number of completed trajectories: %lli\n", (long long)n_traj);
    out.printf(" Omega: %11.2f +/- %-*.2f (%*.2f %%)\n", omega[k], digits(err[k]), err[k],
               digits(100 * err[k] / omega[k]), 100 * err[k] / omega[k]);
    out.printf(" Total time: %5.3f; estimated time remaining: %5.3f\n", total_time,
               total_time * (iters - k - 1) / (k + 1));
  }
  if (data_f) std::fclose(data_f);
  if (xyz_f) std::fclose(xyz_f);
  if (tracer && tracer != ctx) cosims_ctx_destroy(tracer);
  cosims_ctx_destroy(ctx);
  cosims_setup_destroy(setup);
  if (!ok) return false;

  double mean = 0, sd = 0, wsum = 0, wmean = 0;
  for (int k = 0; k < iters; k++) mean += omega[k];
  mean /= iters;
  for (int k = 0; k < iters; k++) {
    sd += (omega[k] - mean) * (omega[k] - mean);
    wsum += 1.0 / (err[k] * err[k]);
    wmean += omega[k] / (err[k] * err[k]);
  }
  wmean /= wsum;
  sd = std::sqrt(sd / iters);
  const double werr = 1.0 / std::sqrt(wsum);
  out.printf("\n\n ___________________________________\n");
  out.printf("   Mean Cross-section:   %9.3f\n", mean);
  out.printf("   Standard Dev:         %9.3f\n", sd);
  out.printf("   StdDev Percent:       %9.3f\n\n", sd * 100 / mean);
  out.printf("   Weighted CCS Mean:    %9.3f\n", wmean);
  out.printf("   Weighted Error:       %9.3f\n", werr);
  out.printf("   Weighted Pct. Error:  %9.4f\n", werr * 100 / wmean);
  out.printf("   Max Energy Deviation: %9.4f\n", max_de);
  out.printf(" ___________________________________\n");
  ccs = wmean;
  ccs_err = werr;
  return true;
}

}  // namespace

int main(int argc, char **argv) {
  std::string mol_path, input_path, atom_path;
  bool seed_set = false, threads_set = false;
  long long seed = 0;
  int threads = 0, device = 0;
  int precision = COSIMS_PRECISION_PLAIN_F64;
  // options come in "-x value" pairs, as in fileParams::interpretCMD
  for (int i = 1; i < argc; i += 2) {
    if (i + 1 >= argc || argv[i][0] != '-' || std::strlen(argv[i]) != 2 || argv[i + 1][0] == '-') {
      std::printf("ERROR: Check command line arguments.\nProgram will now exit...\n");
      usage();
      return 0;
    }
    const char o = argv[i][1];
    const char *v = argv[i + 1];
    if (o == 'm') mol_path = v;
    else if (o == 'i') input_path = v;
    else if (o == 'a') atom_path = v;
    else if (o == 's' && is_int(v)) { seed = std::atoll(v); seed_set = true; }
    else if (o == 'n' && is_int(v)) { threads = std::atoi(v); threads_set = true; }
    else if (o == 'g' && is_int(v)) device = std::atoi(v);
    else if (o == 'p' && !std::strcmp(v, "plain")) precision = COSIMS_PRECISION_PLAIN_F64;
    else if (o == 'p' && !std::strcmp(v, "mixed")) precision = COSIMS_PRECISION_MIXED;
    else {
      std::printf("ERROR: Check command line arguments.\nProgram will now exit...\n");
      usage();
      return 0;
    }
  }
  if (mol_path.empty()) {
    std::printf("ERROR: No molecule file was given. Check command-line aguments\n");
    usage();
    return 0;
  }

  cosims_config cfg;
  std::memset(&cfg, 0, sizeof cfg);
  if (seed_set) { cfg.seed = seed; cfg.changed |= COSIMS_KEY_SEED; }
  if (threads_set) { cfg.threads = threads; cfg.changed |= COSIMS_KEY_THREADS; }
  std::vector<char> log(1 << 16, 0);
  cosims_status st = input_path.empty()
                         ? cosims_config_defaults(&cfg, mol_path.c_str())
                         : cosims_config_read(&cfg, input_path.c_str(), mol_path.c_str(),
                                              log.data(), (int64_t)log.size());
  if (st != COSIMS_OK) {
    std::printf("%s", log.data());
    std::printf("ERROR: %s\nProgram will now exit...\n", cosims_last_error());
    return 0;
  }

  // output location: the input file's dir key, relative to the working directory
  char cwd[4096] = ".";
  if (!getcwd(cwd, sizeof cwd)) std::strcpy(cwd, ".");
  std::string dir = cfg.dir;
  std::string path = dir.empty() ? std::string(cwd) + "/"
                                 : (dir[0] == '/' ? dir : std::string(cwd) + "/" + dir);
  const std::string omega_path = path + "omega_" + cfg.name + ".txt";
  Out out;
  out.f = std::fopen(omega_path.c_str(), "w");

  const time_t now = std::time(nullptr);
  out.printf("\n Starting Program \n Current Date/Time: %s\n", std::ctime(&now));
  out.printf(" Importing and assigning molecule information...\n");
  out.printf("%s", log.data());
  out.printf(" Importing files complete.\n");
  const auto t_start = std::chrono::steady_clock::now();

  int32_t n_sets = 1;
  if (cosims_molecule_file_structures(mol_path.c_str(), &n_sets) != COSIMS_OK) n_sets = 1;
  std::vector<double> set_ccs, set_err;
  for (int set = 0; set < n_sets; set++) {
    if (n_sets > 1) out.printf("\n Coordinate set %d / %d\n", set + 1, n_sets);
    double ccs = 0, ccs_err = 0;
    if (!run_set(cfg, mol_path, atom_path, set, n_sets, device, precision, path, log, out, ccs,
                 ccs_err))
      break;
    set_ccs.push_back(ccs);
    set_err.push_back(ccs_err);
  }
  if (n_sets > 1 && (int)set_ccs.size() == n_sets) {
    // the average over coordinate sets (conformers), each set's weighted mean
    double mean = 0, e2 = 0, sd = 0;
    for (int k = 0; k < n_sets; k++) { mean += set_ccs[k]; e2 += set_err[k] * set_err[k]; }
    mean /= n_sets;
    for (int k = 0; k < n_sets; k++) sd += (set_ccs[k] - mean) * (set_ccs[k] - mean);
    sd = std::sqrt(sd / n_sets);
    out.printf("\n\n ___________________________________\n");
    out.printf("   Coordinate sets:      %9d\n", n_sets);
    out.printf("   Average CCS:          %9.3f\n", mean);
    out.printf("   Propagated Error:     %9.3f\n", std::sqrt(e2) / n_sets);
    out.printf("   StdDev over sets:     %9.3f\n", sd);
    out.printf(" ___________________________________\n");
  }
  const double wall =
      std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
  const time_t end = std::time(nullptr);
  out.printf("\n Program finished: %s Total run time: %.3f s\n", std::ctime(&end), wall);
  if (out.f) std::fclose(out.f);
  return 0;
}
