// batch.cu -- many molecules in one persistent launch (include/cosims_cuda.h).
//
// All molecules' F64 and F32 images live in one device arena.  A run samples
// every molecule's start states in one kernel, then one persistent kernel
// (batch_mixed_kernel) takes work items -- a molecule and a range of its
// trajectories, the most expensive items first -- from a device queue, and
// one CTA per molecule reduces its records.  The sequence is captured once in
// a CUDA graph and replayed while the number of items and slots stays the
// same.  cosims_batch_autotune picks lanes per trajectory per molecule size
// class by timing short single-molecule runs of the same kernel.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <vector>
#include "capi_internal.h"

namespace cosims {
namespace {

constexpr uint32_t kBatchImageCap = 96 * 1024;   // larger F32 images are read through L1/L2
constexpr int kBatchBlock = kBatchMaxBlock;
constexpr int kItemsPerCta = 3;          // items of about equal cost per CTA of a run
constexpr int kMinTrajPerGroup = 4;      // an item gives every group some trajectories

// process-wide tuning cache: (force type, atom-count class) -> lanes per trajectory
std::mutex g_tune_mu;
std::map<std::pair<int, int>, int> g_tune;

int size_class(int n_atoms) {
  int c = 0;
  while ((64 << c) < n_atoms && c < 12) c++;
  return c;
}

}  // namespace

// Dynamic shared memory one batched-kernel CTA of `block` threads needs for
// molecule bm: its F32 image when staged (at most img_cap bytes, and only if
// it fits the budget) plus each group's trajectory state and mode scratch.
// Sets bm.use_smem and bm.mode_stride.
size_t batch_mol_smem(BatchMol &bm, int block, int budget, uint32_t img_cap) {
  bm.use_smem = bm.img32.bytes <= img_cap ? 1 : 0;
  bm.mode_stride = mode_stride_for(bm.img32, bm.type);
  const size_t groups = (size_t)(block / bm.group_lanes);
  const size_t scratch = groups * ((size_t)kGroupStateBytes + (size_t)bm.mode_stride);
  size_t need = (bm.use_smem ? ((bm.img32.bytes + 15u) & ~15u) : 0) + scratch;
  if ((int)need > budget && bm.use_smem) {
    bm.use_smem = 0;
    need = scratch;
  }
  return need;
}

// Work items for one persistent launch: molecule i's n_traj[i] trajectories
// cut into items of about equal cost (atoms x trajectories), about
// kItemsPerCta per CTA, so a CTA works on few molecules and rarely waits for
// its groups to restage; every group of a CTA gets at least kMinTrajPerGroup
// trajectories of an item.  Largest first, a molecule's items adjacent.
void balanced_items(const std::vector<int64_t> &n_traj, const std::vector<int> &n_atoms,
                    const std::vector<int> &group_lanes, int block, int grid,
                    std::vector<BatchItem> &items) {
  items.clear();
  double total = 0;
  for (size_t m = 0; m < n_traj.size(); m++) total += (double)n_atoms[m] * (double)n_traj[m];
  const double target = total / (double)std::max(1, kItemsPerCta * std::max(grid, 1));
  for (size_t m = 0; m < n_traj.size(); m++) {
    if (n_traj[m] <= 0) continue;
    const double cost = (double)n_atoms[m] * (double)n_traj[m];
    int64_t k = std::max<int64_t>(1, (int64_t)std::ceil(cost / std::max(target, 1.0)));
    const int64_t min_size = (int64_t)(block / std::max(group_lanes[m], 1)) * kMinTrajPerGroup;
    k = std::min<int64_t>(k, std::max<int64_t>(1, n_traj[m] / std::max<int64_t>(min_size, 1)));
    const int64_t per = (n_traj[m] + k - 1) / k;
    for (int64_t t0 = 0; t0 < n_traj[m]; t0 += per) {
      BatchItem it;
      it.mol = (int32_t)m;
      it.pad = 0;
      it.t0 = t0;
      it.t1 = std::min<int64_t>(n_traj[m], t0 + per);
      items.push_back(it);
    }
  }
  std::stable_sort(items.begin(), items.end(), [&](const BatchItem &x, const BatchItem &y) {
    const double cx = (double)n_atoms[x.mol] * (double)(x.t1 - x.t0);
    const double cy = (double)n_atoms[y.mol] * (double)(y.t1 - y.t0);
    return cx > cy;
  });
}

// Lanes per trajectory of the batched (and serving) kernel for a size class
// the autotuner has not measured in this process: its picks on a library of
// 256 molecules of 50-5000 atoms (B200, 640-thread CTAs), 4 lanes up to 128
// atoms and 32 above.  They differ from the single-molecule kernel's defaults;
// a server that ran on those measured 2.98 requests/s of capacity against
// 4.81 on these.
int batch_default_lanes(int n_atoms) { return n_atoms <= 128 ? 4 : 32; }

// Lanes per trajectory for a molecule: the tuned value of its size class if
// cosims_batch_autotune has measured one in this process, else the default.
int tuned_group_lanes(int type, int n_atoms) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tune.find({type, size_class(n_atoms)});
  return it != g_tune.end() ? it->second : batch_default_lanes(n_atoms);
}

}  // namespace cosims

using namespace cosims;

struct cosims_batch {
  int device = 0, sm_count = 0, max_smem = 0, n_mol = 0;
  std::vector<HostImage> h64, h32;
  std::vector<BatchMol> mols;
  std::vector<int> n_atoms;
  unsigned char *d_arena = nullptr;
  BatchMol *d_mols = nullptr;
  BatchItem *d_items = nullptr;
  int64_t items_cap = 0;
  double *d_pos0 = nullptr, *d_vel0 = nullptr;
  int32_t *d_hit = nullptr;
  cosims_traj_out *d_out = nullptr;
  int64_t slots_cap = 0;
  unsigned long long *d_ctrl = nullptr;      // [0] item queue, [1..] counters
  cosims_ccs_sums *d_sums = nullptr;
  int block = kBatchBlock, grid = 0;
  size_t smem = 0;
  cudaStream_t cap_stream = nullptr;
  cudaGraphExec_t exec = nullptr;
  int graph_items = -1;
  int64_t graph_total = -1;
  int64_t update_every = 0;
  int64_t graph_update_every = -1;
  std::vector<BatchItem> items;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace cosims {
namespace {

cosims_status shape_launch(cosims_batch *b) {
  const int budget = b->max_smem - 1024 - (int)sizeof(BatchMol) - 64;
  size_t smem = 0;
  for (int m = 0; m < b->n_mol; m++) {
    BatchMol &bm = b->mols[m];
    const size_t need = batch_mol_smem(bm, kBatchBlock, budget, kBatchImageCap);
    if ((int)need > budget)
      return fail(COSIMS_ERR_UNSUPPORTED, "molecule %d needs %zu bytes of shared memory", m, need);
    smem = std::max(smem, need);
  }
  b->smem = smem;
  int per_sm = 1;
  int rc = batch_occupancy(b->block, smem, &per_sm);
  if (rc != 0) return cuda_fail((cudaError_t)rc, "batch occupancy");
  b->grid = std::max(1, per_sm) * b->sm_count;
  return COSIMS_OK;
}

template <typename T>
cosims_status grow_buf(T **p, int64_t *cap, int64_t need) {
  if (*cap >= need) return COSIMS_OK;
  cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  cudaError_t e = cudaMalloc((void **)p, sizeof(T) * (size_t)std::max<int64_t>(need, 1));
  if (e != cudaSuccess) return fail(COSIMS_ERR_NOMEM, "batch buffer: %s", cudaGetErrorString(e));
  *cap = need;
  return COSIMS_OK;
}

void drop_graph(cosims_batch *b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  b->exec = nullptr;
  b->graph_items = -1;
  b->graph_total = -1;
}

// Per-run descriptors and work items; items of expensive molecules first.
cosims_status prepare(cosims_batch *b, const uint64_t *seed, const int64_t *first,
                      const int64_t *n_traj, int64_t *total_out) {
  int64_t total = 0;
  for (int m = 0; m < b->n_mol; m++) {
    if (n_traj[m] < 0 || first[m] < 0)
      return fail(COSIMS_ERR_INVALID, "molecule %d: n_traj and first_index must be >= 0", m);
    BatchMol &bm = b->mols[m];
    bm.base = total;
    bm.n_traj = n_traj[m];
    bm.seed = seed[m];
    bm.first_index = first[m];
    total += n_traj[m];
  }
  if (total > INT32_MAX) return fail(COSIMS_ERR_UNSUPPORTED, "at most 2^31-1 trajectories per run");
  std::vector<int64_t> nt(b->n_mol);
  std::vector<int> lanes(b->n_mol);
  for (int m = 0; m < b->n_mol; m++) {
    nt[m] = b->mols[m].n_traj;
    lanes[m] = b->mols[m].group_lanes;
  }
  balanced_items(nt, b->n_atoms, lanes, b->block, b->grid, b->items);
  *total_out = total;
  return COSIMS_OK;
}

cosims_status enqueue(cosims_batch *b, int64_t total, cudaStream_t s) {
  const int64_t items_before = b->items_cap;
  cosims_status st = grow_buf(&b->d_items, &b->items_cap, (int64_t)b->items.size());
  if (st == COSIMS_OK && b->items_cap != items_before) drop_graph(b);   // new pointer
  if (st == COSIMS_OK) {
    const int64_t before = b->slots_cap;
    st = grow_buf(&b->d_out, &b->slots_cap, total);
    if (st == COSIMS_OK && b->slots_cap != before) {
      cudaFree(b->d_pos0); cudaFree(b->d_vel0); cudaFree(b->d_hit);
      cudaError_t e = cudaMalloc((void **)&b->d_pos0, sizeof(double) * 3 * b->slots_cap);
      if (e == cudaSuccess) e = cudaMalloc((void **)&b->d_vel0, sizeof(double) * 3 * b->slots_cap);
      if (e == cudaSuccess) e = cudaMalloc((void **)&b->d_hit, sizeof(int32_t) * b->slots_cap);
      if (e != cudaSuccess) return fail(COSIMS_ERR_NOMEM, "batch slots: %s", cudaGetErrorString(e));
      drop_graph(b);
    }
  }
  if (st != COSIMS_OK) return st;
  cudaError_t e = cudaMemcpyAsync(b->d_mols, b->mols.data(), sizeof(BatchMol) * b->n_mol,
                                  cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && !b->items.empty())
    e = cudaMemcpyAsync(b->d_items, b->items.data(), sizeof(BatchItem) * b->items.size(),
                        cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return cuda_fail(e, "batch descriptors");
  const int n_items = (int)b->items.size();
  if (!b->exec || b->graph_items != n_items || b->graph_total != total ||
      b->graph_update_every != b->update_every) {
    drop_graph(b);
    cudaGraph_t g = nullptr;
    e = cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_fail(e, "graph capture");
    cudaMemsetAsync(b->d_ctrl, 0, sizeof(unsigned long long) * (1 + C_COUNT), b->cap_stream);
    int rc = batch_sample_launch(b->d_mols, b->n_mol, total, b->d_pos0, b->d_vel0, b->d_hit,
                                 b->cap_stream);
    BatchArgs a;
    std::memset(&a, 0, sizeof a);
    a.mols = b->d_mols;
    a.items = b->d_items;
    a.n_items = n_items;
    a.n_mols = b->n_mol;
    a.smem_bytes = (uint32_t)b->smem;
    a.pos0 = b->d_pos0;
    a.vel0 = b->d_vel0;
    a.hit = b->d_hit;
    a.out = b->d_out;
    a.item_queue = b->d_ctrl;
    a.counters = b->d_ctrl + 1;
    if (rc == 0) rc = batch_launch(a, b->block, b->grid, b->smem, b->cap_stream);
    if (rc == 0)
      rc = batch_reduce_launch(b->d_mols, b->n_mol, b->d_out, b->update_every, b->d_sums,
                               b->cap_stream);
    e = cudaStreamEndCapture(b->cap_stream, &g);
    if (rc != 0) {
      if (g) cudaGraphDestroy(g);
      return cuda_fail((cudaError_t)rc, "batch capture");
    }
    if (e != cudaSuccess) return cuda_fail(e, "graph capture end");
    e = cudaGraphInstantiate(&b->exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(e, "graph instantiate");
    b->graph_items = n_items;
    b->graph_total = total;
    b->graph_update_every = b->update_every;
  }
  cudaEventRecord(b->ev0, s);
  e = cudaGraphLaunch(b->exec, s);
  cudaEventRecord(b->ev1, s);
  if (e != cudaSuccess) return cuda_fail(e, "graph launch");
  return COSIMS_OK;
}

cosims_status finish_run(cosims_batch *b, cosims_ccs_sums *sums, cudaStream_t s) {
  unsigned long long flag = 0;
  cudaError_t e = cudaMemcpyAsync(sums, b->d_sums, sizeof(cosims_ccs_sums) * b->n_mol,
                                  cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&flag, b->d_ctrl + 1 + C_ERROR, sizeof flag, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "batch run");
  if (flag) return fail(COSIMS_ERR_TIMEOUT, "shared-memory staging wait gave up");
  return COSIMS_OK;
}

}  // namespace
}  // namespace cosims

extern "C" {

cosims_status cosims_batch_create(const cosims_molecule *mols, const cosims_params *pars,
                                  int32_t n_mol, int32_t precision, int32_t device,
                                  cosims_batch **out) {
  if (!out) return fail(COSIMS_ERR_INVALID, "out is NULL");
  *out = nullptr;
  if (precision != COSIMS_PRECISION_MIXED)
    return fail(COSIMS_ERR_UNSUPPORTED, "the batched form runs the mixed precision only");
  if (!mols || !pars || n_mol <= 0) return fail(COSIMS_ERR_INVALID, "molecules are required");
  for (int m = 0; m < n_mol; m++) {
    cosims_status st = validate(&mols[m], &pars[m]);
    if (st != COSIMS_OK) return st;
  }
  int sm = 0, smem = 0;
  cosims_status st = check_device(device, &sm, &smem);
  if (st != COSIMS_OK) return st;
  DeviceGuard g(device);
  cosims_batch *b = new cosims_batch();
  b->device = device;
  b->sm_count = sm;
  b->max_smem = smem;
  b->n_mol = n_mol;
  b->h64.resize(n_mol);
  b->h32.resize(n_mol);
  b->mols.resize(n_mol);
  b->n_atoms.resize(n_mol);
  size_t arena = 0;
  std::vector<size_t> off64(n_mol), off32(n_mol);
  for (int m = 0; m < n_mol; m++) {
    build_images(&mols[m], &pars[m], b->h64[m], b->h32[m]);
    off64[m] = arena;
    arena += (b->h64[m].img.bytes + 255) & ~size_t(255);
    off32[m] = arena;
    arena += (b->h32[m].img.bytes + 255) & ~size_t(255);
    b->n_atoms[m] = mols[m].n_atoms;
  }
  cudaError_t e = cudaMalloc((void **)&b->d_arena, arena);
  if (e == cudaSuccess) e = cudaMalloc((void **)&b->d_mols, sizeof(BatchMol) * n_mol);
  if (e == cudaSuccess) e = cudaMalloc((void **)&b->d_ctrl, sizeof(unsigned long long) * (1 + C_COUNT));
  if (e == cudaSuccess) e = cudaMalloc((void **)&b->d_sums, sizeof(cosims_ccs_sums) * n_mol);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&b->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&b->ev1);
  for (int m = 0; m < n_mol && e == cudaSuccess; m++) {
    e = cudaMemcpy(b->d_arena + off64[m], b->h64[m].bytes.data(), b->h64[m].img.bytes,
                   cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMemcpy(b->d_arena + off32[m], b->h32[m].bytes.data(), b->h32[m].img.bytes,
                     cudaMemcpyHostToDevice);
    BatchMol &bm = b->mols[m];
    std::memset(&bm, 0, sizeof bm);
    bm.img64 = b->h64[m].img;
    bm.img64.gbase = b->d_arena + off64[m];
    bm.img32 = b->h32[m].img;
    bm.img32.gbase = b->d_arena + off32[m];
    bm.par = make_dev_params(&pars[m]);
    bm.type = pars[m].force_type;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find({bm.type, size_class(mols[m].n_atoms)});
    bm.group_lanes = it != g_tune.end() ? it->second : batch_default_lanes(mols[m].n_atoms);
  }
  if (e != cudaSuccess) {
    cosims_batch_destroy(b);
    return fail(COSIMS_ERR_NOMEM, "batch allocation: %s", cudaGetErrorString(e));
  }
  st = shape_launch(b);
  if (st != COSIMS_OK) { cosims_batch_destroy(b); return st; }
  *out = b;
  return COSIMS_OK;
}

void cosims_batch_destroy(cosims_batch *b) {
  if (!b) return;
  DeviceGuard g(b->device);
  drop_graph(b);
  cudaFree(b->d_arena); cudaFree(b->d_mols); cudaFree(b->d_items); cudaFree(b->d_pos0);
  cudaFree(b->d_vel0); cudaFree(b->d_hit); cudaFree(b->d_out); cudaFree(b->d_ctrl);
  cudaFree(b->d_sums);
  if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  delete b;
}

cosims_status cosims_batch_run_async(cosims_batch *b, const uint64_t *seed,
                                     const int64_t *first_index, const int64_t *n_traj,
                                     cosims_ccs_sums *d_sums, void *stream) {
  if (!b || !seed || !first_index || !n_traj)
    return fail(COSIMS_ERR_INVALID, "batch, seeds, first indices and counts are required");
  DeviceGuard g(b->device);
  int64_t total = 0;
  cosims_status st = prepare(b, seed, first_index, n_traj, &total);
  if (st == COSIMS_OK) st = enqueue(b, total, (cudaStream_t)stream);
  if (st != COSIMS_OK) return st;
  if (d_sums) {
    cudaError_t e = cudaMemcpyAsync(d_sums, b->d_sums, sizeof(cosims_ccs_sums) * b->n_mol,
                                    cudaMemcpyDeviceToDevice, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "batch sums");
  }
  return COSIMS_OK;
}

cosims_status cosims_batch_run(cosims_batch *b, const uint64_t *seed, const int64_t *first_index,
                               const int64_t *n_traj, cosims_ccs_sums *sums, void *stream) {
  if (!sums) return fail(COSIMS_ERR_INVALID, "sums is NULL");
  cosims_status st = cosims_batch_run_async(b, seed, first_index, n_traj, nullptr, stream);
  if (st != COSIMS_OK) return st;
  DeviceGuard g(b->device);
  return finish_run(b, sums, (cudaStream_t)stream);
}

cosims_status cosims_batch_autotune(cosims_batch *b, void *stream) {
  if (!b) return fail(COSIMS_ERR_INVALID, "batch is NULL");
  DeviceGuard g(b->device);
  std::map<std::pair<int, int>, int> rep;    // size class -> representative molecule
  for (int m = 0; m < b->n_mol; m++) {
    auto key = std::make_pair(b->mols[m].type, size_class(b->n_atoms[m]));
    if (!rep.count(key)) rep[key] = m;
  }
  const std::vector<int> saved = [&] {
    std::vector<int> v;
    for (auto &bm : b->mols) v.push_back(bm.group_lanes);
    return v;
  }();
  std::vector<uint64_t> seeds(b->n_mol, 12345);
  std::vector<int64_t> first(b->n_mol, 0), n(b->n_mol, 0);
  std::vector<cosims_ccs_sums> sums(b->n_mol);
  std::map<std::pair<int, int>, int> best_g;
  for (auto &kv : rep) {
    const int m = kv.second;
    const int slots = b->mols[m].img32.n_slots;
    float best = 1e30f;
    int best_lanes = b->mols[m].group_lanes;
    // about fifty million atom-trajectories per trial (some 50 ms), so that
    // throughput, not the single longest trajectory, decides; lanes that
    // leave each lane between 8 and 256 atom slots
    const int64_t trials =
        std::min<int64_t>(200000, std::max<int64_t>(4096, (int64_t)50000000 / slots));
    bool warmed = false;
    for (int lanes : {2, 4, 8, 16, 32}) {
      if (slots / lanes > 256 && lanes != 32) continue;
      if (slots / lanes < 8 && lanes != 2) continue;
      b->mols[m].group_lanes = lanes;
      if (shape_launch(b) != COSIMS_OK) continue;
      drop_graph(b);
      std::fill(n.begin(), n.end(), 0);
      n[m] = trials;
      float ms = 0;
      bool ok = true;
      for (int rep_i = 0; rep_i < (warmed ? 1 : 2) && ok; rep_i++) {
        if (cosims_batch_run(b, seeds.data(), first.data(), n.data(), sums.data(), stream) !=
            COSIMS_OK) ok = false;
      }
      warmed = true;
      if (!ok) continue;
      cudaEventElapsedTime(&ms, b->ev0, b->ev1);
      if (ms < best) { best = ms; best_lanes = lanes; }
    }
    best_g[kv.first] = best_lanes;
  }
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (auto &kv : best_g) g_tune[kv.first] = kv.second;
  }
  for (int m = 0; m < b->n_mol; m++) {
    auto key = std::make_pair(b->mols[m].type, size_class(b->n_atoms[m]));
    b->mols[m].group_lanes = best_g.count(key) ? best_g[key] : saved[m];
  }
  drop_graph(b);
  return shape_launch(b);
}

cosims_status cosims_batch_get_launch(const cosims_batch *b, int32_t mol, int32_t *group_lanes,
                                      int32_t *item_traj) {
  if (!b || mol < 0 || mol >= b->n_mol) return fail(COSIMS_ERR_INVALID, "bad batch or molecule");
  const int lanes = b->mols[mol].group_lanes;
  if (group_lanes) *group_lanes = lanes;
  if (item_traj) {   // trajectories in the molecule's first item of the last run
    *item_traj = 0;
    for (const BatchItem &it : b->items)
      if (it.mol == mol) { *item_traj = (int32_t)(it.t1 - it.t0); break; }
  }
  return COSIMS_OK;
}

cosims_status cosims_batch_set_update_every(cosims_batch *b, int64_t update_every) {
  if (!b || update_every < 0) return fail(COSIMS_ERR_INVALID, "bad batch or interval");
  b->update_every = update_every;
  return COSIMS_OK;
}

cosims_status cosims_batch_counters(cosims_batch *b, cosims_ccs_sums *work, float *ms) {
  if (!b || !work) return fail(COSIMS_ERR_INVALID, "batch and work are required");
  DeviceGuard g(b->device);
  unsigned long long c[C_COUNT];
  cudaError_t e = cudaMemcpy(c, b->d_ctrl + 1, sizeof c, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "batch counters");
  std::memset(work, 0, sizeof *work);
  work->steps = (int64_t)c[C_STEPS];
  work->force_evals = (int64_t)c[C_FORCE_EVALS];
  work->pot_evals = (int64_t)c[C_POT_EVALS];
  work->pair_lj = (int64_t)c[C_PAIR_LJ];
  work->pair_es = (int64_t)c[C_PAIR_ES];
  work->pair_pot = (int64_t)c[C_PAIR_POT];
  work->far_terms = (int64_t)c[C_FAR];
  work->pair_es_nolj = (int64_t)c[C_PAIR_ESNL];
  if (ms) {
    e = cudaEventElapsedTime(ms, b->ev0, b->ev1);
    if (e != cudaSuccess) return cuda_fail(e, "batch timing");
  }
  return COSIMS_OK;
}

}  // extern "C"
