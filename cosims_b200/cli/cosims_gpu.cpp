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

  cosims_setup *setup = nullptr;
  std::fill(log.begin(), log.end(), 0);
  st = cosims_setup_create_device(&cfg, mol_path.c_str(), atom_path.c_str(), device, log.data(),
                                  (int64_t)log.size(), &setup);
  out.printf("%s", log.data());
  if (st != COSIMS_OK) {
    out.printf("ERROR: Cannot read molecule file (%s).\nProgram will now exit...\n",
               cosims_last_error());
    if (out.f) std::fclose(out.f);
    return 0;
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
  cosims_ctx *ctx = nullptr;
  st = cosims_ctx_create(&mol, &par, precision, device, &ctx);
  if (st != COSIMS_OK) {
    out.printf("ERROR: %s\nProgram will now exit...\n", cosims_last_error());
    cosims_setup_destroy(setup);
    if (out.f) std::fclose(out.f);
    return 1;
  }

  out.printf(" Starting Trajectory Calculations:\n _________________________________\n\n");
  const int iters = cfg.iter > 0 ? cfg.iter : 1;
  const int64_t n_traj = cfg.traj;
  std::vector<double> omega(iters), err(iters);
  double total_time = 0, max_de = 0;
  const int64_t update_every = cfg.print_rate > 0 ? cfg.print_rate : 0;
  for (int k = 0; k < iters; k++) {
    out.printf("\n Computing CCS integral %i / %i on GPU %d (%s form)\n", k + 1, iters, device,
               precision == COSIMS_PRECISION_MIXED ? "mixed" : "plain FP64");
    const auto t0 = std::chrono::steady_clock::now();
    cosims_ccs_sums s;
    st = cosims_run_sampled(ctx, (uint64_t)cfg.seed, (int64_t)k * n_traj, n_traj, update_every,
                            &s, nullptr, nullptr, nullptr);
    if (st != COSIMS_OK) {
      out.printf("ERROR: %s\n", cosims_last_error());
      break;
    }
    total_time += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
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
  const double wall =
      std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
  const time_t end = std::time(nullptr);
  out.printf("\n Program finished: %s Total run time: %.3f s\n", std::ctime(&end), wall);
  cosims_ctx_destroy(ctx);
  cosims_setup_destroy(setup);
  if (out.f) std::fclose(out.f);
  return 0;
}
