// noalloc.cu -- a list-form trajectory run that allocates no device memory.
//
// Some callers cannot allocate device memory from inside this library: a
// host program that owns the GPU's memory through its own pool or arena, or
// one that forbids allocation on its hot path (cudaMalloc synchronises the
// device and can fail mid-run).  cosims_run_list_noalloc serves them: the
// caller passes device buffers for the start states and the results; the
// molecule image, the work queue, the work order and the counters live in a
// fixed static device array (kNoallocScratchBytes), which every GPU that
// loads this library holds until the process exits.
//
// Set-up: the first call on a device looks up that device's copy of the
// array with cudaGetSymbolAddress (the device must be current; the address is
// cached per device, so the device's primary context -- the one the CUDA
// runtime uses -- is the one supported).  That first call should come before
// any stream capture.  Every call shares the array and leaves its contents
// behind; the call clears what must start at zero (queue, counters,
// histogram).  Calls that overlap on the GPU -- two streams, or two host
// threads -- race on the array: run them one after another.
//
// The run has no long-trajectory hand-off (its records would need 200 bytes
// per trajectory of scratch): every trajectory is integrated to its end by
// the group that started it.  The mixed form's results are those of a context
// with the hand-off off (cosims_ctx_set_handoff(ctx, -1, 0)); with the hand-off
// on, a trajectory past its 2048-step budget is finished by a wide group whose
// FP32 sums run in another order.  The plain form's results are bit for bit
// the context's either way, but its longest trajectories then run on one
// thread each, so a 1e5-trajectory call takes about 5x as long as with the
// hand-off (1.3-1.6 s against 0.27 s for the 512-atom ion).
//
// The molecule images are copied from pageable host memory (the call may wait
// for that copy before it returns).
#include <cuda_runtime.h>
#include <cstring>
#include <mutex>
#include <vector>
#include "capi_internal.h"

namespace cosims {

namespace {

constexpr size_t kNoallocScratchBytes = 12u << 20;       // 12 MiB per device
constexpr size_t kCtrlBytes = 4096;                       // queue, counters, order scratch
// molecule images (F64 + F32): about 100 bytes per atom and at most 850 per
// cluster (its records, far-field table entry and the padding of its last slot
// block), so every molecule of the 16384-atom limit fits with up to 3000 clusters
constexpr size_t kImageBytes = 4u << 20;
constexpr size_t kOrderBytes = kNoallocScratchBytes - kCtrlBytes - kImageBytes;
constexpr int64_t kNoallocMaxTraj = (int64_t)(kOrderBytes / sizeof(int32_t));
constexpr int kMaxDevices = 64;

static_assert(sizeof(unsigned long long) * (1 + C_COUNT) + sizeof(int32_t) * 2 *
                  (kOrderBuckets + 1) <= kCtrlBytes, "control region too small");

std::mutex g_mu;
void *g_scratch[kMaxDevices] = {nullptr};

}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

// Device address of this device's scratch array (set-up on first use).
static cosims_status scratch_of(int dev, unsigned char **out) {
  if (dev < 0 || dev >= kMaxDevices) return fail(COSIMS_ERR_UNSUPPORTED, "device %d", dev);
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress of the no-alloc scratch");
    g_scratch[dev] = p;
  }
  *out = static_cast<unsigned char *>(g_scratch[dev]);
  return COSIMS_OK;
}

}  // namespace cosims

using namespace cosims;

extern "C" cosims_status cosims_run_list_noalloc(const cosims_molecule *mol,
                                                 const cosims_params *par, int32_t precision,
                                                 int32_t group_lanes, const double *d_pos0,
                                                 const double *d_vel0, int64_t n,
                                                 cosims_traj_out *d_out, void *stream) {
  if (precision != COSIMS_PRECISION_PLAIN_F64 && precision != COSIMS_PRECISION_MIXED)
    return fail(COSIMS_ERR_INVALID, "unknown precision %d", precision);
  const int G = precision == COSIMS_PRECISION_PLAIN_F64 ? 1 : group_lanes;
  if (G < 1 || G > 32 || (G & (G - 1)))
    return fail(COSIMS_ERR_INVALID, "group_lanes must be a power of two in 1..32");
  if (n < 0) return fail(COSIMS_ERR_INVALID, "n must be >= 0");
  if (n > kNoallocMaxTraj)
    return fail(COSIMS_ERR_UNSUPPORTED,
                "n = %lld exceeds the no-alloc limit of %lld trajectories per call",
                (long long)n, (long long)kNoallocMaxTraj);
  if (n > 0 && (!d_pos0 || !d_vel0 || !d_out))
    return fail(COSIMS_ERR_INVALID, "pos0, vel0 and out are required");
  cosims_status st = validate(mol, par);
  if (st != COSIMS_OK) return st;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  int sm = 0, max_smem = 0;
  st = check_device(dev, &sm, &max_smem);
  if (st != COSIMS_OK) return st;

  HostImage h64, h32;
  build_images(mol, par, h64, h32);
  if ((size_t)h64.img.bytes + h32.img.bytes > kImageBytes)
    return fail(COSIMS_ERR_UNSUPPORTED,
                "molecule image of %u bytes exceeds the no-alloc limit of %zu bytes",
                h64.img.bytes + h32.img.bytes, kImageBytes);
  unsigned char *base = nullptr;
  st = scratch_of(dev, &base);
  if (st != COSIMS_OK) return st;
  unsigned long long *queue = reinterpret_cast<unsigned long long *>(base);
  unsigned long long *counters = queue + 1;
  int32_t *order_scratch =
      reinterpret_cast<int32_t *>(base + sizeof(unsigned long long) * (1 + C_COUNT));
  unsigned char *img64 = base + kCtrlBytes;
  unsigned char *img32 = img64 + h64.img.bytes;
  int32_t *order = reinterpret_cast<int32_t *>(base + kCtrlBytes + kImageBytes);

  cudaStream_t s = (cudaStream_t)stream;
  // pageable host -> device: returns once the host images have been staged
  e = cudaMemcpyAsync(img64, h64.bytes.data(), h64.img.bytes, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(img32, h32.bytes.data(), h32.img.bytes, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(queue, 0, sizeof(unsigned long long) * (1 + C_COUNT), s);
  if (e != cudaSuccess) return cuda_fail(e, "no-alloc staging");
  if (n == 0) return COSIMS_OK;

  const DevParams dp = make_dev_params(par);
  int rc = order_launch(dp, d_vel0, nullptr, n, order, order_scratch, stream);
  if (rc != 0) return cuda_fail((cudaError_t)rc, "work-order launch");

  // launch shape: the image staged in shared memory when it fits
  const bool plain = precision == COSIMS_PRECISION_PLAIN_F64;
  MolImage img = plain ? h64.img : h32.img;
  img.gbase = plain ? img64 : img32;
  MolImage i64 = h64.img;
  i64.gbase = img64;
  LaunchShape ls;
  cosims_status shs = shape_for(plain, img, G, plain ? 128 : 0, 0, par->force_type, sm, max_smem, n, ls);
  if (shs != COSIMS_OK) return shs;

  TrajArgs a;
  std::memset(&a, 0, sizeof a);
  a.img = img;
  a.img64 = i64;
  a.par = dp;
  a.group_lanes = G;
  a.use_smem = ls.use_smem;
  a.mode_stride = ls.mode_stride;
  a.stage_limit = kStageSpinLimit;
  a.pos0 = d_pos0;
  a.vel0 = d_vel0;
  a.hit = nullptr;
  a.order = order;
  a.n = n;
  a.out = d_out;
  a.queue = queue;
  a.counters = counters;
  rc = plain ? plain_launch(a, ls.block, ls.grid, ls.smem, stream)
             : mixed_launch(a, ls.block, ls.grid, ls.smem, stream);
  if (rc != 0) return cuda_fail((cudaError_t)rc, "trajectory kernel launch");
  return COSIMS_OK;
}
