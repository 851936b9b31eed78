// serve.cu -- continuous-batching CCS service (include/cosims_cuda.h).
//
// Jobs (a molecule, a seed and a target relative standard error) are admitted
// while their device footprint fits the server's HBM budget and a job slot is
// free.  Each admitted molecule's images live in a device arena allocated once
// at creation (a first-fit free list on the host: admission allocates no
// device memory and never synchronises the device) and stay there, with the
// job's running sums, until the job is released.
//
// A round integrates the next chunk of every runnable job in one launch of
// the persistent multi-molecule kernel, adds each job's chunk sums to its
// running sums on the device and copies the updated sums to pinned host
// memory.  Up to kRounds rounds are in flight at once, each on its own stream
// with its own buffers: a job belongs to at most one round in flight, and a
// round launched while others run takes the jobs that arrived or finished a
// chunk meanwhile, so new work starts as SMs free up instead of after the
// slowest chunk of the previous round.  cosims_serve_step harvests the rounds
// that have completed (it never waits while it can launch), retires the jobs
// whose relative standard error reached the target, and launches the next
// round.
//
// A job's first chunk is round_traj trajectories (or min_traj); each later
// chunk is the job's own estimate of what it still needs from its running
// error (+5 %, at most 64 round_traj by default).  The chunks are always the next
// trajectories of the job's own Philox stream and their sizes follow from the
// job alone, so its result is the same whether it ran alone or among other
// jobs, whatever the timing of the rounds.
#include <cuda_runtime.h>
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <thread>
#include <vector>
#include "capi_internal.h"

namespace cosims {
int tuned_group_lanes(int type, int n_atoms);   // batch.cu

namespace {

constexpr int kServeBlock = kBatchMaxBlock;
constexpr uint32_t kServeImageCap = 96 * 1024;
// default chunk cap: 64 round_traj.  Against 16 on the configuration-4 mix (3.8
// requests/s offered, 90 s): p99 latency 20 s instead of 33 s, the 0.2 % requests'
// median 17 s instead of 27 s, throughput 1.84 M instead of 1.77 M trajectories/s
constexpr int64_t kMaxChunkRounds = 64;
constexpr int kRounds = 3;                // rounds in flight at most
constexpr size_t kArenaAlign = 256;
constexpr size_t kStageBytes = size_t(8) << 20;   // pinned staging of job images
constexpr double kStepWaitMs = 5.0;       // cosims_serve_step waits at most this long

struct Job {
  int64_t id = 0;
  int32_t state = COSIMS_JOB_RUNNING;
  int32_t slot = 0;
  int32_t rounds = 0;
  int32_t n_atoms = 0;
  int32_t in_round = -1;           // round buffer it is in flight in, or -1
  double target = 0;
  int64_t min_traj = 0, max_traj = 0, done = 0;
  int64_t next_chunk = 0;          // trajectories of the job's next round
  int64_t footprint = 0;
  size_t arena_off = 0;
  BatchMol bm{};
  cosims_ccs_sums sums{};
  double submitted_ms = 0, finished_ms = 0;
};

// slots[j] >= 0: add round j to that slot's running sums; slots[j] = -(s+1):
// the job's first round, which replaces slot s's previous contents.  The
// updated record of job j also goes to out[j] (the round's copy to the host).
__global__ void accumulate_sums(const cosims_ccs_sums *round, const int32_t *slots, int n,
                                cosims_ccs_sums *running, cosims_ccs_sums *out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int32_t sl = slots[j];
  cosims_ccs_sums &r = running[sl >= 0 ? sl : -sl - 1];
  const cosims_ccs_sums &c = round[j];
  if (sl < 0) {
    r = c;
  } else {
    r.sum += c.sum;
    r.sum2 += c.sum2;
    r.max_de_pct = fmax(r.max_de_pct, c.max_de_pct);
    r.n += c.n;
    r.n_hit += c.n_hit;
    r.n_success += c.n_success;
    r.n_eff += c.n_eff;
  }
  out[j] = r;
}

// One round buffer: its stream, device arrays for max_jobs * round_traj
// trajectory slots, and pinned host descriptors and results.
struct Round {
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  bool busy = false;
  BatchMol *d_mols = nullptr;
  BatchItem *d_items = nullptr;
  double *d_pos0 = nullptr, *d_vel0 = nullptr;
  int32_t *d_hit = nullptr, *d_slots = nullptr;
  cosims_traj_out *d_out = nullptr;
  unsigned long long *d_ctrl = nullptr;      // [0] item queue, [1..] counters
  cosims_ccs_sums *d_round = nullptr, *d_result = nullptr;
  BatchMol *h_mols = nullptr;
  BatchItem *h_items = nullptr;
  int32_t *h_slots = nullptr;
  cosims_ccs_sums *h_result = nullptr;
  unsigned long long *h_flag = nullptr;
  std::vector<int64_t> jobs;                 // job ids, in the round's molecule order
  std::vector<int64_t> chunk;
};

}  // namespace
}  // namespace cosims

using namespace cosims;

struct cosims_server {
  int device = 0, sm_count = 0, max_smem = 0;
  int64_t budget = 0, in_use = 0, round_traj = 0, next_id = 1;
  int64_t max_chunk = 0;                     // trajectories of one job in one round, at most
  int32_t max_jobs = 0;
  int items_cap = 0;
  std::map<int64_t, Job> jobs;
  std::vector<int32_t> free_slots;
  cosims_ccs_sums *d_running = nullptr;
  Round rounds[kRounds];
  int64_t launched = 0;                      // rounds launched (age order of the buffers)
  int64_t round_seq[kRounds] = {};
  // image arena: device bytes and a first-fit list of free ranges (offset -> size)
  unsigned char *d_arena = nullptr;
  size_t arena_bytes = 0;
  std::map<size_t, size_t> arena_free;
  // pinned staging of job images, uploaded on their own stream
  unsigned char *h_stage = nullptr;
  size_t stage_head = 0;
  cudaStream_t upload = nullptr;
  cudaEvent_t uploaded = nullptr;
  bool pending_upload = false;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  double clock_ms() const {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
};

namespace cosims {
namespace {

bool arena_take(cosims_server *s, size_t bytes, size_t *off) {
  for (auto it = s->arena_free.begin(); it != s->arena_free.end(); ++it) {
    if (it->second < bytes) continue;
    *off = it->first;
    const size_t rest = it->second - bytes;
    s->arena_free.erase(it);
    if (rest) s->arena_free.emplace(*off + bytes, rest);
    return true;
  }
  return false;
}

void arena_give(cosims_server *s, size_t off, size_t bytes) {
  auto it = s->arena_free.emplace(off, bytes).first;
  auto nx = std::next(it);
  if (nx != s->arena_free.end() && it->first + it->second == nx->first) {
    it->second += nx->second;
    s->arena_free.erase(nx);
  }
  if (it != s->arena_free.begin()) {
    auto pv = std::prev(it);
    if (pv->first + pv->second == it->first) {
      pv->second += it->second;
      s->arena_free.erase(it);
    }
  }
}

// Copies `bytes` of host data to device `dst` through the pinned staging
// buffer on the upload stream (never the legacy stream, so no in-flight
// round is waited for; the staging buffer is reused once its uploads ended).
cudaError_t stage_upload(cosims_server *s, unsigned char *dst, const void *src, size_t bytes) {
  size_t done = 0;
  while (done < bytes) {
    if (s->stage_head == kStageBytes) {
      cudaError_t e = cudaStreamSynchronize(s->upload);   // uploads only
      if (e != cudaSuccess) return e;
      s->stage_head = 0;
    }
    const size_t n = std::min(bytes - done, kStageBytes - s->stage_head);
    std::memcpy(s->h_stage + s->stage_head, (const unsigned char *)src + done, n);
    cudaError_t e = cudaMemcpyAsync(dst + done, s->h_stage + s->stage_head, n,
                                    cudaMemcpyHostToDevice, s->upload);
    if (e != cudaSuccess) return e;
    s->stage_head += (n + 255) & ~size_t(255);
    if (s->stage_head > kStageBytes) s->stage_head = kStageBytes;
    done += n;
  }
  s->pending_upload = true;
  return cudaSuccess;
}

// Takes the results of a completed round: running sums to the jobs, the
// retirement test, the next chunk sizes.  Returns the jobs retired.
cosims_status harvest(cosims_server *s, int r, int *finished) {
  Round &R = s->rounds[r];
  cudaError_t e = cudaEventSynchronize(R.done);
  if (e != cudaSuccess) return cuda_fail(e, "round");
  R.busy = false;
  const bool timed_out = *R.h_flag != 0;
  const double now = s->clock_ms();
  const int64_t pool = (int64_t)s->max_jobs * s->round_traj;
  for (size_t k = 0; k < R.jobs.size(); k++) {
    auto it = s->jobs.find(R.jobs[k]);
    if (it == s->jobs.end()) continue;
    Job &j = it->second;
    j.in_round = -1;
    j.done += R.chunk[k];
    j.rounds++;
    j.sums = R.h_result[k];
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
      const int64_t cap = std::min<int64_t>(s->max_chunk, pool);
      j.next_chunk = std::min<int64_t>(std::max<int64_t>(want, s->round_traj), cap);
    } else {
      j.state = COSIMS_JOB_DONE;
      j.finished_ms = now;
      (*finished)++;
    }
  }
  R.jobs.clear();
  R.chunk.clear();
  if (timed_out) return fail(COSIMS_ERR_TIMEOUT, "shared-memory staging wait gave up");
  return COSIMS_OK;
}

// Launches a round on buffer r with the runnable jobs (submission order,
// while their chunks fit the trajectory slots).  *launched: a round started.
cosims_status launch_round(cosims_server *s, int r, cudaStream_t after, bool *launched) {
  *launched = false;
  Round &R = s->rounds[r];
  const int64_t pool = (int64_t)s->max_jobs * s->round_traj;
  std::vector<Job *> act;
  std::vector<int64_t> chunk;
  int64_t packed = 0;
  for (auto &kv : s->jobs) {
    Job &j = kv.second;
    if (j.state != COSIMS_JOB_RUNNING || j.in_round >= 0) continue;
    const int64_t c = std::min<int64_t>(j.next_chunk, j.max_traj - j.done);
    if (packed + c > pool) continue;
    act.push_back(&j);
    chunk.push_back(c);
    packed += c;
  }
  if (act.empty()) return COSIMS_OK;
  const int n = (int)act.size();
  size_t smem = 0;
  int64_t base = 0;
  const int budget = s->max_smem - 1024 - (int)sizeof(BatchMol) - 64;
  for (int k = 0; k < n; k++) {
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
    R.h_mols[k] = bm;
    R.h_slots[k] = j.rounds == 0 ? -j.slot - 1 : j.slot;
  }
  int per_sm = 1;
  int orc = batch_occupancy(kServeBlock, smem, &per_sm);
  if (orc != 0) return cuda_fail((cudaError_t)orc, "round occupancy");
  per_sm = std::max(1, per_sm);
  std::vector<BatchItem> items;
  {
    std::vector<int64_t> nt;
    std::vector<int> na, lanes;
    for (int k = 0; k < n; k++) {
      nt.push_back(R.h_mols[k].n_traj);
      na.push_back(act[k]->n_atoms);
      lanes.push_back(R.h_mols[k].group_lanes);
    }
    balanced_items(nt, na, lanes, kServeBlock, per_sm * s->sm_count, items);
  }
  if ((int)items.size() > s->items_cap)
    return fail(COSIMS_ERR_UNSUPPORTED, "round of %zu work items (at most %d)", items.size(),
                s->items_cap);
  std::memcpy(R.h_items, items.data(), sizeof(BatchItem) * items.size());
  cudaStream_t st = R.stream;
  cudaError_t e = cudaSuccess;
  // after the caller's stream and the image uploads
  if (after) {
    e = cudaEventRecord(R.done, after);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, R.done, 0);
  }
  if (e == cudaSuccess && s->pending_upload) {
    e = cudaEventRecord(s->uploaded, s->upload);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, s->uploaded, 0);
    s->pending_upload = false;
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(R.d_mols, R.h_mols, sizeof(BatchMol) * n, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(R.d_items, R.h_items, sizeof(BatchItem) * items.size(),
                        cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(R.d_slots, R.h_slots, sizeof(int32_t) * n, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(R.d_ctrl, 0, sizeof(unsigned long long) * (1 + C_COUNT), st);
  if (e != cudaSuccess) return cuda_fail(e, "round descriptors");
  int rc = batch_sample_launch(R.d_mols, n, base, R.d_pos0, R.d_vel0, R.d_hit, st);
  BatchArgs a;
  std::memset(&a, 0, sizeof a);
  a.mols = R.d_mols;
  a.items = R.d_items;
  a.n_items = (int32_t)items.size();
  a.n_mols = n;
  a.smem_bytes = (uint32_t)smem;
  a.pos0 = R.d_pos0;
  a.vel0 = R.d_vel0;
  a.hit = R.d_hit;
  a.out = R.d_out;
  a.item_queue = R.d_ctrl;
  a.counters = R.d_ctrl + 1;
  if (rc == 0) rc = batch_launch(a, kServeBlock, per_sm * s->sm_count, smem, st);
  if (rc == 0) rc = batch_reduce_launch(R.d_mols, n, R.d_out, 0, R.d_round, st);
  if (rc != 0) return cuda_fail((cudaError_t)rc, "round launch");
  accumulate_sums<<<(n + 127) / 128, 128, 0, st>>>(R.d_round, R.d_slots, n, s->d_running,
                                                   R.d_result);
  e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(R.h_result, R.d_result, sizeof(cosims_ccs_sums) * n,
                        cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(R.h_flag, R.d_ctrl + 1 + C_ERROR, sizeof(unsigned long long),
                        cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaEventRecord(R.done, st);
  if (e != cudaSuccess) return cuda_fail(e, "round");
  R.busy = true;
  R.jobs.clear();
  R.chunk.clear();
  for (int k = 0; k < n; k++) {
    act[k]->in_round = r;
    R.jobs.push_back(act[k]->id);
    R.chunk.push_back(chunk[k]);
  }
  s->round_seq[r] = ++s->launched;
  *launched = true;
  return COSIMS_OK;
}

void free_round(Round &R) {
  if (R.stream) cudaStreamSynchronize(R.stream);
  cudaFree(R.d_mols); cudaFree(R.d_items); cudaFree(R.d_pos0); cudaFree(R.d_vel0);
  cudaFree(R.d_hit); cudaFree(R.d_slots); cudaFree(R.d_out); cudaFree(R.d_ctrl);
  cudaFree(R.d_round); cudaFree(R.d_result);
  cudaFreeHost(R.h_mols); cudaFreeHost(R.h_items); cudaFreeHost(R.h_slots);
  cudaFreeHost(R.h_result); cudaFreeHost(R.h_flag);
  if (R.done) cudaEventDestroy(R.done);
  if (R.stream) cudaStreamDestroy(R.stream);
  R = Round();
}

}  // namespace
}  // namespace cosims

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
  s->max_chunk = kMaxChunkRounds * round_traj;
  // at most three items per CTA of two resident CTAs per SM, plus one per job
  s->items_cap = 3 * 2 * sm + max_jobs + 64;
  const int64_t slots = (int64_t)max_jobs * round_traj;
  cudaError_t e = cudaMalloc((void **)&s->d_running, sizeof(cosims_ccs_sums) * max_jobs);
  if (e == cudaSuccess) e = cudaMemset(s->d_running, 0, sizeof(cosims_ccs_sums) * max_jobs);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->upload, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->uploaded, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaHostAlloc((void **)&s->h_stage, kStageBytes, cudaHostAllocDefault);
  for (int r = 0; r < kRounds && e == cudaSuccess; r++) {
    Round &R = s->rounds[r];
    e = cudaStreamCreateWithFlags(&R.stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&R.done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMalloc((void **)&R.d_mols, sizeof(BatchMol) * max_jobs);
    if (e == cudaSuccess) e = cudaMalloc((void **)&R.d_items, sizeof(BatchItem) * s->items_cap);
    if (e == cudaSuccess) e = cudaMalloc((void **)&R.d_pos0, sizeof(double) * 3 * slots);
    if (e == cudaSuccess) e = cudaMalloc((void **)&R.d_vel0, sizeof(double) * 3 * slots);
    if (e == cudaSuccess) e = cudaMalloc((void **)&R.d_hit, sizeof(int32_t) * slots);
    if (e == cudaSuccess) e = cudaMalloc((void **)&R.d_out, sizeof(cosims_traj_out) * slots);
    if (e == cudaSuccess) e = cudaMalloc((void **)&R.d_slots, sizeof(int32_t) * max_jobs);
    if (e == cudaSuccess)
      e = cudaMalloc((void **)&R.d_ctrl, sizeof(unsigned long long) * (1 + C_COUNT));
    if (e == cudaSuccess) e = cudaMalloc((void **)&R.d_round, sizeof(cosims_ccs_sums) * max_jobs);
    if (e == cudaSuccess) e = cudaMalloc((void **)&R.d_result, sizeof(cosims_ccs_sums) * max_jobs);
    if (e == cudaSuccess) e = cudaHostAlloc((void **)&R.h_mols, sizeof(BatchMol) * max_jobs, 0);
    if (e == cudaSuccess)
      e = cudaHostAlloc((void **)&R.h_items, sizeof(BatchItem) * s->items_cap, 0);
    if (e == cudaSuccess) e = cudaHostAlloc((void **)&R.h_slots, sizeof(int32_t) * max_jobs, 0);
    if (e == cudaSuccess)
      e = cudaHostAlloc((void **)&R.h_result, sizeof(cosims_ccs_sums) * max_jobs, 0);
    if (e == cudaSuccess) e = cudaHostAlloc((void **)&R.h_flag, sizeof(unsigned long long), 0);
  }
  if (e != cudaSuccess) {
    cosims_serve_destroy(s);
    return fail(COSIMS_ERR_NOMEM, "server allocation: %s", cudaGetErrorString(e));
  }
  // the round buffers count against the budget; the rest, up to 4 GiB, is the
  // image arena that admission sub-allocates
  s->in_use = kRounds * slots * (48 + 4 + 24) + (int64_t)sizeof(cosims_ccs_sums) * max_jobs;
  const int64_t rest = s->budget - s->in_use;
  if (rest > 0) {
    s->arena_bytes = (size_t)std::min<int64_t>(rest, int64_t(4) << 30) & ~(kArenaAlign - 1);
    if (s->arena_bytes) {
      e = cudaMalloc((void **)&s->d_arena, s->arena_bytes);
      if (e != cudaSuccess) {
        cosims_serve_destroy(s);
        return fail(COSIMS_ERR_NOMEM, "server image arena: %s", cudaGetErrorString(e));
      }
      s->arena_free.emplace(0, s->arena_bytes);
    }
  }
  for (int k = max_jobs - 1; k >= 0; k--) s->free_slots.push_back(k);
  *out = s;
  return COSIMS_OK;
}

void cosims_serve_destroy(cosims_server *s) {
  if (!s) return;
  DeviceGuard g(s->device);
  for (int r = 0; r < kRounds; r++) free_round(s->rounds[r]);
  if (s->upload) cudaStreamSynchronize(s->upload);
  cudaFree(s->d_arena);
  cudaFree(s->d_running);
  cudaFreeHost(s->h_stage);
  if (s->uploaded) cudaEventDestroy(s->uploaded);
  if (s->upload) cudaStreamDestroy(s->upload);
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
  const size_t o32 = (h64.img.bytes + kArenaAlign - 1) & ~(kArenaAlign - 1);
  const size_t bytes = (o32 + h32.img.bytes + kArenaAlign - 1) & ~(kArenaAlign - 1);
  const int64_t fp = (int64_t)bytes;
  size_t off = 0;
  if (s->free_slots.empty() || s->in_use + fp > s->budget || !arena_take(s, bytes, &off))
    return fail(COSIMS_ERR_BUSY, "no room: %zu active jobs, %lld of %lld bytes in use",
                s->jobs.size(), (long long)s->in_use, (long long)s->budget);
  unsigned char *d_img = s->d_arena + off;
  cudaError_t e = stage_upload(s, d_img, h64.bytes.data(), h64.img.bytes);
  if (e == cudaSuccess) e = stage_upload(s, d_img + o32, h32.bytes.data(), h32.img.bytes);
  if (e != cudaSuccess) {
    arena_give(s, off, bytes);
    return cuda_fail(e, "job image upload");
  }
  Job j;
  j.id = s->next_id++;
  j.slot = s->free_slots.back();
  j.target = target_rel_se;
  j.min_traj = min_traj;
  j.max_traj = max_traj;
  j.n_atoms = mol->n_atoms;
  j.footprint = fp;
  j.arena_off = off;
  j.next_chunk = std::max<int64_t>(s->round_traj, std::min<int64_t>(min_traj, s->max_chunk));
  j.next_chunk = std::min<int64_t>(j.next_chunk, (int64_t)s->max_jobs * s->round_traj);
  BatchMol &bm = j.bm;
  std::memset(&bm, 0, sizeof bm);
  bm.img64 = h64.img;
  bm.img64.gbase = d_img;
  bm.img32 = h32.img;
  bm.img32.gbase = d_img + o32;
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
  int finished = 0;
  cosims_status st = COSIMS_OK;
  // 1. harvest every round that has completed
  for (int r = 0; r < kRounds && st == COSIMS_OK; r++) {
    Round &R = s->rounds[r];
    if (!R.busy) continue;
    const cudaError_t q = cudaEventQuery(R.done);
    if (q == cudaErrorNotReady) continue;
    if (q != cudaSuccess) return cuda_fail(q, "round");
    st = harvest(s, r, &finished);
  }
  if (st != COSIMS_OK) return st;
  // 2. launch a round of the runnable jobs on a free buffer
  bool launched = false;
  for (int r = 0; r < kRounds && !launched; r++) {
    if (s->rounds[r].busy) continue;
    st = launch_round(s, r, (cudaStream_t)stream, &launched);
    if (st != COSIMS_OK) return st;
    break;                                   // no runnable job: nothing to launch
  }
  // 3. nothing launched and nothing retired: wait for a round to complete, at
  // most kStepWaitMs, so that the caller can admit new arrivals meanwhile
  if (!launched && finished == 0) {
    const double t_end = s->clock_ms() + kStepWaitMs;
    for (bool any = true; any && finished == 0 && st == COSIMS_OK;) {
      any = false;
      for (int r = 0; r < kRounds && st == COSIMS_OK; r++) {
        Round &R = s->rounds[r];
        if (!R.busy) continue;
        any = true;
        const cudaError_t q = cudaEventQuery(R.done);
        if (q == cudaErrorNotReady) continue;
        if (q != cudaSuccess) return cuda_fail(q, "round");
        st = harvest(s, r, &finished);
      }
      if (!any || finished || s->clock_ms() > t_end) break;
      std::this_thread::sleep_for(std::chrono::microseconds(100));
    }
  }
  if (n_finished) *n_finished = finished;
  return st;
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
  if (j.in_round >= 0) {
    // a running job leaves only after its round in flight has ended
    int finished = 0;
    cosims_status st = harvest(s, j.in_round, &finished);
    if (st != COSIMS_OK) return st;
  }
  arena_give(s, j.arena_off, (size_t)j.footprint);
  s->in_use -= j.footprint;
  s->free_slots.push_back(j.slot);
  s->jobs.erase(it);
  return COSIMS_OK;
}

cosims_status cosims_serve_set_max_chunk(cosims_server *s, int64_t max_chunk_traj) {
  if (!s) return fail(COSIMS_ERR_INVALID, "server is NULL");
  if (max_chunk_traj < 0) return fail(COSIMS_ERR_INVALID, "max_chunk_traj must be >= 0");
  s->max_chunk = max_chunk_traj == 0 ? kMaxChunkRounds * s->round_traj
                                     : std::max<int64_t>(max_chunk_traj, s->round_traj);
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
