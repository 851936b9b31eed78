// reduce.cu -- CCS sums of one integral from per-trajectory records.
//
// Replaces the per-thread accumulation of monteTraj::runThreads
// (monteTraj.cpp:456-502) and the omp-critical merge (monteTraj.cpp:372-378).
// The sums are formed in a fixed tree order (no floating-point atomics), so a
// result depends only on the records, not on the launch or on timing.
//
// n_eff reproduces the reference's success count with one thread: an
// ellipsoid miss keeps the previous trajectory's success flag
// (monteTraj.cpp:326-367), and only the failures since the last progress
// update -- the final partial window of update_every trajectories -- are
// subtracted (monteTraj.cpp:380, :504-521).
#include <cuda_runtime.h>
#include "engine.h"

namespace cosims {

constexpr int kRedThreads = 256;
constexpr int kRedMaxBlocks = 512;
constexpr int kFinalThreads = 512;

struct Part { double sum, sum2, max_de; long long hit, succ; };

__device__ __forceinline__ double contribution(const cosims_traj_out &r, double c, int half) {
  if (!(r.status & COSIMS_TRAJ_HIT)) return 0.0;
  const double chi = fabs(r.chi);
  if (half) {
    const double s = sin(0.5 * chi);
    return c * (2.0 * s * s);
  }
  return c * (1.0 - cos(chi));
}

__global__ void reduce_parts(const cosims_traj_out *__restrict__ recs, long long n, double c,
                             int half, long long chunk, Part *parts) {
  __shared__ double s_sum[kRedThreads], s_sum2[kRedThreads], s_max[kRedThreads];
  __shared__ long long s_hit[kRedThreads], s_succ[kRedThreads];
  const long long b0 = (long long)blockIdx.x * chunk;
  const long long b1 = min(n, b0 + chunk);
  double sum = 0, sum2 = 0, mx = 0;
  long long hit = 0, succ = 0;
  for (long long i = b0 + threadIdx.x; i < b1; i += kRedThreads) {
    const cosims_traj_out r = recs[i];
    const double v = contribution(r, c, half);
    sum += v;
    sum2 += v * v;
    if (r.status & COSIMS_TRAJ_HIT) {
      hit++;
      if (r.status & COSIMS_TRAJ_SUCCESS) {
        succ++;
        mx = fmax(mx, r.de_pct);
      }
    }
  }
  s_sum[threadIdx.x] = sum; s_sum2[threadIdx.x] = sum2; s_max[threadIdx.x] = mx;
  s_hit[threadIdx.x] = hit; s_succ[threadIdx.x] = succ;
  __syncthreads();
  for (int o = kRedThreads / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      s_sum[threadIdx.x] += s_sum[threadIdx.x + o];
      s_sum2[threadIdx.x] += s_sum2[threadIdx.x + o];
      s_max[threadIdx.x] = fmax(s_max[threadIdx.x], s_max[threadIdx.x + o]);
      s_hit[threadIdx.x] += s_hit[threadIdx.x + o];
      s_succ[threadIdx.x] += s_succ[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    Part p = {s_sum[0], s_sum2[0], s_max[0], s_hit[0], s_succ[0]};
    parts[blockIdx.x] = p;
  }
}

// Effective success flag of a record given the flag carried in.
__device__ __forceinline__ int eff_of(const cosims_traj_out &r, int carried) {
  if (r.status & COSIMS_TRAJ_HIT) return (r.status & COSIMS_TRAJ_SUCCESS) ? 1 : 0;
  return carried;
}

__global__ void reduce_final(const cosims_traj_out *__restrict__ recs, long long n,
                             long long update_every, const Part *parts, int nparts,
                             const unsigned long long *counters, cosims_ccs_sums *out) {
  __shared__ double s_sum[kFinalThreads], s_sum2[kFinalThreads], s_max[kFinalThreads];
  __shared__ long long s_hit[kFinalThreads], s_succ[kFinalThreads];
  __shared__ long long s_f0[kFinalThreads], s_f1[kFinalThreads];
  __shared__ int s_e0[kFinalThreads], s_e1[kFinalThreads];
  const int t = threadIdx.x;
  // 1) partials, fixed pairing
  Part p = {0, 0, 0, 0, 0};
  if (t < nparts) p = parts[t];
  s_sum[t] = p.sum; s_sum2[t] = p.sum2; s_max[t] = p.max_de; s_hit[t] = p.hit; s_succ[t] = p.succ;
  // 2) failures in the final window [w0, n), as a two-state automaton per segment
  long long w0 = 0;
  if (update_every > 0) w0 = n - n % update_every;
  if (w0 == n) w0 = n;   // empty window when n is a multiple of update_every
  const long long wl = n - w0;
  const long long seg = (wl + kFinalThreads - 1) / kFinalThreads;
  const long long s0 = w0 + (long long)t * seg, s1 = min(n, s0 + seg);
  int e0 = 0, e1 = 1;
  long long f0 = 0, f1 = 0;
  for (long long i = s0; i < s1; i++) {
    const cosims_traj_out r = recs[i];
    e0 = eff_of(r, e0);
    e1 = eff_of(r, e1);
    f0 += !e0;
    f1 += !e1;
  }
  s_f0[t] = f0; s_f1[t] = f1; s_e0[t] = e0; s_e1[t] = e1;
  __syncthreads();
  for (int o = kFinalThreads / 2; o > 0; o >>= 1) {
    if (t < o) {
      s_sum[t] += s_sum[t + o];
      s_sum2[t] += s_sum2[t + o];
      s_max[t] = fmax(s_max[t], s_max[t + o]);
      s_hit[t] += s_hit[t + o];
      s_succ[t] += s_succ[t + o];
    }
    __syncthreads();
  }
  if (t == 0) {
    // success flag carried into the window: that of the last hit before w0
    int carried = 0;
    for (long long i = w0 - 1; i >= 0; i--) {
      const cosims_traj_out r = recs[i];
      if (r.status & COSIMS_TRAJ_HIT) { carried = (r.status & COSIMS_TRAJ_SUCCESS) ? 1 : 0; break; }
    }
    long long fails = 0;
    for (int k = 0; k < kFinalThreads; k++) {
      const long long k0 = w0 + (long long)k * seg;
      if (k0 >= n) break;
      fails += carried ? s_f1[k] : s_f0[k];
      carried = carried ? s_e1[k] : s_e0[k];
    }
    cosims_ccs_sums s;
    s.sum = s_sum[0];
    s.sum2 = s_sum2[0];
    s.max_de_pct = s_max[0];
    s.n = n;
    s.n_hit = s_hit[0];
    s.n_success = s_succ[0];
    s.n_eff = n - fails;
    // work counters of the launch (NULL: a slice of a multi-integral launch,
    // whose work is reported for the whole call)
    s.steps = counters ? (int64_t)counters[C_STEPS] : 0;
    s.force_evals = counters ? (int64_t)counters[C_FORCE_EVALS] : 0;
    s.pot_evals = counters ? (int64_t)counters[C_POT_EVALS] : 0;
    s.pair_lj = counters ? (int64_t)counters[C_PAIR_LJ] : 0;
    s.pair_es = counters ? (int64_t)counters[C_PAIR_ES] : 0;
    s.pair_pot = counters ? (int64_t)counters[C_PAIR_POT] : 0;
    s.far_terms = counters ? (int64_t)counters[C_FAR] : 0;
    s.pair_es_nolj = counters ? (int64_t)counters[C_PAIR_ESNL] : 0;
    *out = s;
  }
}

// Adds one launch's work counters to a record's work fields (steps .. far
// terms); zero_first clears the whole record first.
__global__ void add_work_kernel(const unsigned long long *counters, cosims_ccs_sums *w,
                                int zero_first) {
  if (threadIdx.x != 0) return;
  if (zero_first) memset(w, 0, sizeof *w);
  w->steps += (int64_t)counters[C_STEPS];
  w->force_evals += (int64_t)counters[C_FORCE_EVALS];
  w->pot_evals += (int64_t)counters[C_POT_EVALS];
  w->pair_lj += (int64_t)counters[C_PAIR_LJ];
  w->pair_es += (int64_t)counters[C_PAIR_ES];
  w->pair_pot += (int64_t)counters[C_PAIR_POT];
  w->far_terms += (int64_t)counters[C_FAR];
  w->pair_es_nolj += (int64_t)counters[C_PAIR_ESNL];
}

int add_work_launch(const unsigned long long *counters, cosims_ccs_sums *d_work, int zero_first,
                    void *stream) {
  add_work_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(counters, d_work, zero_first);
  return (int)cudaGetLastError();
}

int64_t reduce_scratch_len(int64_t n) {
  (void)n;
  return (int64_t)(kRedMaxBlocks * sizeof(Part) / sizeof(double)) + 8;
}

int reduce_launch(const cosims_traj_out *recs, int64_t n, double ccs_const, int half_angle,
                  int64_t update_every, const unsigned long long *counters,
                  cosims_ccs_sums *d_sums, double *scratch, int64_t scratch_len,
                  void *stream) {
  if (scratch_len < reduce_scratch_len(n)) return (int)cudaErrorInvalidValue;
  cudaStream_t s = (cudaStream_t)stream;
  long long nb = (n + 4095) / 4096;
  if (nb < 1) nb = 1;
  if (nb > kRedMaxBlocks) nb = kRedMaxBlocks;
  const long long chunk = (n + nb - 1) / nb > 0 ? (n + nb - 1) / nb : 1;
  Part *parts = reinterpret_cast<Part *>(scratch);
  reduce_parts<<<(int)nb, kRedThreads, 0, s>>>(recs, n, ccs_const, half_angle, chunk, parts);
  reduce_final<<<1, kFinalThreads, 0, s>>>(recs, n, update_every, parts, (int)nb, counters,
                                           d_sums);
  return (int)cudaGetLastError();
}

}  // namespace cosims

namespace cosims {

// ---- batched reduction: one CTA per molecule ------------------------------------------
// The same fixed-order sums and one-thread n_eff bookkeeping as reduce_final,
// over each molecule's records [base, base + n_traj).  Contributions use
// 2 sin^2(chi/2) (the batched form is the mixed form).  Work counters are
// reported for the whole batch by cosims_batch_counters, so they are 0 here.
__global__ void batch_reduce_kernel(const BatchMol *mols, const cosims_traj_out *__restrict__ recs,
                                    long long update_every, cosims_ccs_sums *sums) {
  __shared__ double s_sum[kFinalThreads], s_sum2[kFinalThreads], s_max[kFinalThreads];
  __shared__ long long s_hit[kFinalThreads], s_succ[kFinalThreads];
  __shared__ long long s_f0[kFinalThreads], s_f1[kFinalThreads];
  __shared__ int s_e0[kFinalThreads], s_e1[kFinalThreads];
  const BatchMol &bm = mols[blockIdx.x];
  const cosims_traj_out *r = recs + bm.base;
  const long long n = bm.n_traj;
  const double c = bm.par.ccs_const;
  const int t = threadIdx.x;
  const long long chunk = (n + kFinalThreads - 1) / kFinalThreads;
  double sum = 0, sum2 = 0, mx = 0;
  long long hit = 0, succ = 0;
  for (long long i = (long long)t * chunk; i < n && i < (long long)(t + 1) * chunk; i++) {
    const cosims_traj_out x = r[i];
    const double v = contribution(x, c, 1);
    sum += v;
    sum2 += v * v;
    if (x.status & COSIMS_TRAJ_HIT) {
      hit++;
      if (x.status & COSIMS_TRAJ_SUCCESS) { succ++; mx = fmax(mx, x.de_pct); }
    }
  }
  s_sum[t] = sum; s_sum2[t] = sum2; s_max[t] = mx; s_hit[t] = hit; s_succ[t] = succ;
  long long w0 = 0;
  if (update_every > 0) w0 = n - n % update_every;
  const long long wl = n - w0;
  const long long seg = (wl + kFinalThreads - 1) / kFinalThreads;
  const long long s0 = w0 + (long long)t * seg, s1 = min(n, s0 + seg);
  int e0 = 0, e1 = 1;
  long long f0 = 0, f1 = 0;
  for (long long i = s0; i < s1; i++) {
    const cosims_traj_out x = r[i];
    e0 = eff_of(x, e0);
    e1 = eff_of(x, e1);
    f0 += !e0;
    f1 += !e1;
  }
  s_f0[t] = f0; s_f1[t] = f1; s_e0[t] = e0; s_e1[t] = e1;
  __syncthreads();
  for (int o = kFinalThreads / 2; o > 0; o >>= 1) {
    if (t < o) {
      s_sum[t] += s_sum[t + o];
      s_sum2[t] += s_sum2[t + o];
      s_max[t] = fmax(s_max[t], s_max[t + o]);
      s_hit[t] += s_hit[t + o];
      s_succ[t] += s_succ[t + o];
    }
    __syncthreads();
  }
  if (t == 0) {
    int carried = 0;
    for (long long i = w0 - 1; i >= 0; i--) {
      const cosims_traj_out x = r[i];
      if (x.status & COSIMS_TRAJ_HIT) { carried = (x.status & COSIMS_TRAJ_SUCCESS) ? 1 : 0; break; }
    }
    long long fails = 0;
    for (int k = 0; k < kFinalThreads; k++) {
      if (w0 + (long long)k * seg >= n) break;
      fails += carried ? s_f1[k] : s_f0[k];
      carried = carried ? s_e1[k] : s_e0[k];
    }
    cosims_ccs_sums s;
    memset(&s, 0, sizeof s);
    s.sum = s_sum[0]; s.sum2 = s_sum2[0]; s.max_de_pct = s_max[0];
    s.n = n; s.n_hit = s_hit[0]; s.n_success = s_succ[0]; s.n_eff = n - fails;
    sums[blockIdx.x] = s;
  }
}

int batch_reduce_launch(const BatchMol *mols, int n_mols, const cosims_traj_out *recs,
                        int64_t update_every, cosims_ccs_sums *sums, void *stream) {
  if (n_mols <= 0) return 0;
  batch_reduce_kernel<<<n_mols, kFinalThreads, 0, (cudaStream_t)stream>>>(mols, recs, update_every,
                                                                          sums);
  return (int)cudaGetLastError();
}

}  // namespace cosims
