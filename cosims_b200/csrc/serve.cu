// serve.cu -- continuous-batching CCS service (include/cosims_cuda.h).
//
// Jobs (a molecule, a seed and a target relative standard error) are admitted
// while their device footprint fits the server's HBM budget and a job slot is
// free.  Each admitted molecule's images and its running sums stay on the
// device until the job is released.  A round integrates the next chunk of
// round_traj trajectories of every active job in one launch of the persistent
// multi-molecule kernel, adds each job's chunk sums to its running sums (on
// the device, in round order) and retires the jobs whose relative standard
// error reached the target.  A job's first chunk is round_traj trajectories;
// each later chunk is the job's own estimate of what it still needs, from its
// running error (at most 16 round_traj), so a job typically retires in two or
// three rounds.  The chunks are always the next trajectories of the job's own
// Philox stream and their sizes follow from the job alone, so its result is
// the same whether it ran alone or among other jobs; a round takes jobs in
// submission order while their chunks fit the server's trajectory slots, and
// a job that does not fit waits for the next round.
#include <cuda_runtime.h>
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <vector>
#include "capi_internal.h"

namespace cosims {
int tuned_group_lanes(int type, int n_atoms);   // batch.cu

namespace {

constexpr int kServeBlock = kBatchMaxBlock;
constexpr uint32_t kServeImageCap = 96 * 1024;
constexpr int64_t kMaxChunkRounds = 16;   // a chunk is at most 16 round_traj

struct Job {
  int64_t id = 0;
  int32_t state = COSIMS_JOB_RUNNING;
  int32_t slot = 0;
  int32_t rounds = 0;
  int32_t n_atoms = 0;
  double target = 0;
  int64_t min_traj = 0, max_traj = 0, done = 0;
  int64_t next_chunk = 0;          // trajectories of the job's next round
  int64_t footprint = 0;
  unsigned char *d_img = nullptr;
  BatchMol bm{};
  cosims_ccs_sums sums{};
  double submitted_ms = 0, finished_ms = 0;
};

// slots[j] >= 0: add round j to that slot's running sums; slots[j] = -(s+1):
// the job's first round, which replaces slot s's previous contents.
__global__ void accumulate_sums(const cosims_ccs_sums *round, const int32_t *slots, int n,
                                cosims_ccs_sums *running) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int32_t sl = slots[j];
  cosims_ccs_sums &r = running[sl >= 0 ? sl : -sl - 1];
  const cosims_ccs_sums &c = round[j];
  if (sl < 0) {
    r = c;
    return;
  }
  r.sum += c.sum;
  r.sum2 += c.sum2;
  r.max_de_pct = fmax(r.max_de_pct, c.max_de_pct);
  r.n += c.n;
  r.n_hit += c.n_hit;
  r.n_success += c.n_success;
  r.n_eff += c.n_eff;
}

}  // namespace
}  // namespace cosims

using namespace cosims;

struct cosims_server {
  int device = 0, sm_count = 0, max_smem = 0;
  int64_t budget = 0, in_use = 0, round_traj = 0, next_id = 1;
  int32_t max_jobs = 0;
  std::map<int64_t, Job> jobs;
  std::vector<int32_t> free_slots;
  // round buffers
  BatchMol *d_mols = nullptr;
  BatchItem *d_items = nullptr;
  int64_t items_cap = 0;
  double *d_pos0 = nullptr, *d_vel0 = nullptr;
  int32_t *d_hit = nullptr, *d_slots = nullptr;
  cosims_traj_out *d_out = nullptr;
  unsigned long long *d_ctrl = nullptr;
  cosims_ccs_sums *d_round = nullptr, *d_running = nullptr;
  std::vector<cosims_ccs_sums> running_host;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  double clock_ms() const {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
};

extern "C" {

cosims_status cosims_serve_create(int32_t device, int64_t hbm_budget_bytes, int32_t max_jobs,
                                  int64_t round_traj, cosims_server **out) {
  if (!out) return fail(COSIMS_ERR_INVALID, "out is NULL");
  *out = nullptr;
  if (max_jobs <= 0 || max_jobs > 4096 || round_traj <= 0 || round_traj > (1 << 24) ||
      hbm_budget_bytes <= 0)
    return fail(COSIMS_ERR_INVALID, "max_jobs, round_traj and the HBM budget must be positive");
  int sm = 0, smem = 0;
  cosims_status st = check_device(device, &sm, &smem);
  if (st != COSIMS_OK) return st;
  DeviceGuard g(device);
  cosims_server *s = new cosims_server();
  s->device = device;
  s->sm_count = sm;
  s->max_smem = smem;
  s->budget = hbm_budget_bytes;
  s->max_jobs = max_jobs;
  s->round_traj = round_traj;
  const int64_t slots = (int64_t)max_jobs * round_traj;
  cudaError_t e = cudaMalloc((void **)&s->d_mols, sizeof(BatchMol) * max_jobs);
  if (e == cudaSuccess) e = cudaMalloc((void **)&s->d_pos0, sizeof(double) * 3 * slots);
  if (e == cudaSuccess) e = cudaMalloc((void **)&s->d_vel0, sizeof(double) * 3 * slots);
  if (e == cudaSuccess) e = cudaMalloc((void **)&s->d_hit, sizeof(int32_t) * slots);
  if (e == cudaSuccess) e = cudaMalloc((void **)&s->d_out, sizeof(cosims_traj_out) * slots);
  if (e == cudaSuccess) e = cudaMalloc((void **)&s->d_slots, sizeof(int32_t) * max_jobs);
  if (e == cudaSuccess) e = cudaMalloc((void **)&s->d_ctrl, sizeof(unsigned long long) * (1 + C_COUNT));
  if (e == cudaSuccess) e = cudaMalloc((void **)&s->d_round, sizeof(cosims_ccs_sums) * max_jobs);
  if (e == cudaSuccess) e = cudaMalloc((void **)&s->d_running, sizeof(cosims_ccs_sums) * max_jobs);
  if (e == cudaSuccess) e = cudaMemset(s->d_running, 0, sizeof(cosims_ccs_sums) * max_jobs);
  if (e != cudaSuccess) {
    cosims_serve_destroy(s);
    return fail(COSIMS_ERR_NOMEM, "server allocation: %s", cudaGetErrorString(e));
  }
  s->in_use = slots * (48 + 4 + 24);
  s->running_host.resize(max_jobs);
  for (int k = max_jobs - 1; k >= 0; k--) s->free_slots.push_back(k);
  *out = s;
  return COSIMS_OK;
}

void cosims_serve_destroy(cosims_server *s) {
  if (!s) return;
  DeviceGuard g(s->device);
  for (auto &kv : s->jobs) cudaFree(kv.second.d_img);
  cudaFree(s->d_mols); cudaFree(s->d_items); cudaFree(s->d_pos0); cudaFree(s->d_vel0);
  cudaFree(s->d_hit); cudaFree(s->d_out); cudaFree(s->d_slots); cudaFree(s->d_ctrl);
  cudaFree(s->d_round); cudaFree(s->d_running);
  delete s;
}

cosims_status cosims_serve_submit(cosims_server *s, const cosims_molecule *mol,
                                  const cosims_params *par, uint64_t seed, double target_rel_se,
                                  int64_t min_traj, int64_t max_traj, int64_t *job_id) {
  if (!s || !job_id) return fail(COSIMS_ERR_INVALID, "server and job_id are required");
  if (!(target_rel_se > 0) || min_traj < 0 || max_traj <= 0 || max_traj < min_traj)
    return fail(COSIMS_ERR_INVALID, "target > 0 and 0 <= min_traj <= max_traj are required");
  cosims_status st = validate(mol, par);
  if (st != COSIMS_OK) return st;
  DeviceGuard g(s->device);
  HostImage h64, h32;
  build_images(mol, par, h64, h32);
  const int64_t fp = (int64_t)((h64.img.bytes + 255) & ~255u) + ((h32.img.bytes + 255) & ~255u);
  if (s->free_slots.empty() || s->in_use + fp > s->budget)
    return fail(COSIMS_ERR_BUSY, "no room: %zu active jobs, %lld of %lld bytes in use",
                s->jobs.size(), (long long)s->in_use, (long long)s->budget);
  Job j;
  j.id = s->next_id++;
  j.slot = s->free_slots.back();
  j.target = target_rel_se;
  j.min_traj = min_traj;
  j.max_traj = max_traj;
  j.n_atoms = mol->n_atoms;
  j.footprint = fp;
  j.next_chunk = std::max<int64_t>(s->round_traj, std::min<int64_t>(min_traj, kMaxChunkRounds * s->round_traj));
  const size_t o32 = (h64.img.bytes + 255) & ~size_t(255);
  cudaError_t e = cudaMalloc((void **)&j.d_img, o32 + h32.img.bytes);
  if (e == cudaSuccess) e = cudaMemcpy(j.d_img, h64.bytes.data(), h64.img.bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(j.d_img + o32, h32.bytes.data(), h32.img.bytes, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(j.d_img);
    return fail(COSIMS_ERR_NOMEM, "job images: %s", cudaGetErrorString(e));
  }
  BatchMol &bm = j.bm;
  std::memset(&bm, 0, sizeof bm);
  bm.img64 = h64.img;
  bm.img64.gbase = j.d_img;
  bm.img32 = h32.img;
  bm.img32.gbase = j.d_img + o32;
  bm.par = make_dev_params(par);
  bm.type = par->force_type;
  bm.group_lanes = tuned_group_lanes(bm.type, mol->n_atoms);
  bm.seed = seed;
  j.submitted_ms = s->clock_ms();
  s->free_slots.pop_back();
  s->in_use += fp;
  *job_id = j.id;
  s->jobs.emplace(j.id, j);
  return COSIMS_OK;
}

cosims_status cosims_serve_step(cosims_server *s, void *stream, int32_t *n_finished) {
  if (!s) return fail(COSIMS_ERR_INVALID, "server is NULL");
  if (n_finished) *n_finished = 0;
  DeviceGuard g(s->device);
  cudaStream_t st = (cudaStream_t)stream;
  // jobs in submission order while their chunks fit the trajectory slots
  const int64_t pool = (int64_t)s->max_jobs * s->round_traj;
  std::vector<Job *> act;
  std::vector<int64_t> chunk;
  int64_t packed = 0;
  for (auto &kv : s->jobs) {
    Job &j = kv.second;
    if (j.state != COSIMS_JOB_RUNNING) continue;
    const int64_t c = std::min<int64_t>(j.next_chunk, j.max_traj - j.done);
    if (packed + c > pool) continue;
    act.push_back(&j);
    chunk.push_back(c);
    packed += c;
  }
  if (act.empty()) return COSIMS_OK;
  std::vector<BatchMol> mols;
  std::vector<int32_t> slots;
  std::vector<BatchItem> items;
  int64_t base = 0;
  size_t smem = 0;
  const int budget = s->max_smem - 1024 - (int)sizeof(BatchMol) - 64;
  for (size_t k = 0; k < act.size(); k++) {
    Job &j = *act[k];
    BatchMol bm = j.bm;
    bm.base = base;
    bm.n_traj = chunk[k];
    bm.first_index = j.done;
    const size_t need = batch_mol_smem(bm, kServeBlock, budget, kServeImageCap);
    if ((int)need > budget)
      return fail(COSIMS_ERR_UNSUPPORTED, "job %lld needs %zu bytes of shared memory",
                  (long long)j.id, need);
    smem = std::max(smem, need);
    base += bm.n_traj;
    mols.push_back(bm);
    slots.push_back(j.rounds == 0 ? -j.slot - 1 : j.slot);
  }
  int per_sm = 1;
  int orc = batch_occupancy(kServeBlock, smem, &per_sm);
  if (orc != 0) return cuda_fail((cudaError_t)orc, "round occupancy");
  per_sm = std::max(1, per_sm);
  {
    std::vector<int64_t> nt;
    std::vector<int> na, lanes;
    for (size_t k = 0; k < act.size(); k++) {
      nt.push_back(mols[k].n_traj);
      na.push_back(act[k]->n_atoms);
      lanes.push_back(mols[k].group_lanes);
    }
    balanced_items(nt, na, lanes, kServeBlock, per_sm * s->sm_count, items);
  }
  if ((int64_t)items.size() > s->items_cap) {
    cudaFree(s->d_items);
    s->d_items = nullptr;
    cudaError_t e = cudaMalloc((void **)&s->d_items, sizeof(BatchItem) * items.size());
    if (e != cudaSuccess) return fail(COSIMS_ERR_NOMEM, "round items: %s", cudaGetErrorString(e));
    s->items_cap = (int64_t)items.size();
  }
  const int n = (int)act.size();
  cudaError_t e = cudaMemcpyAsync(s->d_mols, mols.data(), sizeof(BatchMol) * n,
                                  cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(s->d_items, items.data(), sizeof(BatchItem) * items.size(),
                        cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(s->d_slots, slots.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(s->d_ctrl, 0, sizeof(unsigned long long) * (1 + C_COUNT), st);
  if (e != cudaSuccess) return cuda_fail(e, "round descriptors");
  int rc = batch_sample_launch(s->d_mols, n, base, s->d_pos0, s->d_vel0, s->d_hit, st);

  BatchArgs a;
  std::memset(&a, 0, sizeof a);
  a.mols = s->d_mols;
  a.items = s->d_items;
  a.n_items = (int32_t)items.size();
  a.n_mols = n;
  a.smem_bytes = (uint32_t)smem;
  a.pos0 = s->d_pos0;
  a.vel0 = s->d_vel0;
  a.hit = s->d_hit;
  a.out = s->d_out;
  a.item_queue = s->d_ctrl;
  a.counters = s->d_ctrl + 1;
  if (rc == 0) rc = batch_launch(a, kServeBlock, per_sm * s->sm_count, smem, st);
  if (rc == 0) rc = batch_reduce_launch(s->d_mols, n, s->d_out, 0, s->d_round, st);
  if (rc != 0) return cuda_fail((cudaError_t)rc, "round launch");
  accumulate_sums<<<(n + 127) / 128, 128, 0, st>>>(s->d_round, s->d_slots, n, s->d_running);
  e = cudaMemcpyAsync(s->running_host.data(), s->d_running,
                      sizeof(cosims_ccs_sums) * s->max_jobs, cudaMemcpyDeviceToHost, st);
  unsigned long long flag = 0;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&flag, s->d_ctrl + 1 + C_ERROR, sizeof flag, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, "round");
  if (flag) return fail(COSIMS_ERR_TIMEOUT, "shared-memory staging wait gave up");
  const double now = s->clock_ms();
  int finished = 0;
  for (int k = 0; k < n; k++) {
    Job &j = *act[k];
    j.done += mols[k].n_traj;
    j.rounds++;
    j.sums = s->running_host[j.slot];
    const double ne = (double)j.sums.n_eff;
    bool done = j.done >= j.max_traj;
    double rel = 0;
    if (!done && ne > 1 && j.sums.sum > 0) {
      const double m = j.sums.sum / ne;
      const double se = std::sqrt(std::max(j.sums.sum2 / ne - m * m, 0.0) / ne);
      rel = se / m;
      done = j.done >= j.min_traj && rel <= j.target;
    }
    if (!done) {
      // the error falls as 1/sqrt(n): trajectories still needed, plus 5 %
      int64_t want = s->round_traj;
      if (rel > 0) {
        const double need = (double)j.done * ((rel / j.target) * (rel / j.target) - 1.0) * 1.05;
        want = (int64_t)std::ceil(std::max(need, 0.0) / (double)s->round_traj) * s->round_traj;
      }
      want = std::max<int64_t>(want, j.min_traj - j.done);
      const int64_t cap = std::min<int64_t>(kMaxChunkRounds * s->round_traj, pool);
      j.next_chunk = std::min<int64_t>(std::max<int64_t>(want, s->round_traj), cap);
    }
    if (done) {
      j.state = COSIMS_JOB_DONE;
      j.finished_ms = now;
      finished++;
    }
  }
  if (n_finished) *n_finished = finished;
  return COSIMS_OK;
}

cosims_status cosims_serve_poll(cosims_server *s, int64_t job_id, cosims_job_status *out) {
  if (!s || !out) return fail(COSIMS_ERR_INVALID, "server and out are required");
  auto it = s->jobs.find(job_id);
  if (it == s->jobs.end()) return fail(COSIMS_ERR_INVALID, "unknown job %lld", (long long)job_id);
  const Job &j = it->second;
  std::memset(out, 0, sizeof *out);
  out->job_id = j.id;
  out->state = j.state;
  out->rounds = j.rounds;
  out->sums = j.sums;
  const double ne = (double)j.sums.n_eff;
  if (ne > 0) {
    out->omega = j.sums.sum / ne;
    out->se = std::sqrt(std::max(j.sums.sum2 / ne - out->omega * out->omega, 0.0) / ne);
    out->rel_se = out->omega > 0 ? out->se / out->omega : 0;
  }
  out->device_ms = j.state == COSIMS_JOB_DONE ? j.finished_ms - j.submitted_ms : 0;
  return COSIMS_OK;
}

cosims_status cosims_serve_release(cosims_server *s, int64_t job_id) {
  if (!s) return fail(COSIMS_ERR_INVALID, "server is NULL");
  auto it = s->jobs.find(job_id);
  if (it == s->jobs.end()) return fail(COSIMS_ERR_INVALID, "unknown job %lld", (long long)job_id);
  DeviceGuard g(s->device);
  Job &j = it->second;
  cudaFree(j.d_img);
  s->in_use -= j.footprint;
  s->free_slots.push_back(j.slot);
  s->jobs.erase(it);
  return COSIMS_OK;
}

cosims_status cosims_serve_info(const cosims_server *s, int32_t *active, int64_t *bytes_in_use) {
  if (!s) return fail(COSIMS_ERR_INVALID, "server is NULL");
  int32_t a = 0;
  for (auto &kv : s->jobs) a += kv.second.state == COSIMS_JOB_RUNNING;
  if (active) *active = a;
  if (bytes_in_use) *bytes_in_use = s->in_use;
  return COSIMS_OK;
}

}  // extern "C"
