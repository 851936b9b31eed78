// batch.cu -- many molecules in one persistent launch (filled in below).
#include <cuda_runtime.h>
#include "capi_internal.h"

using namespace cosims;

struct cosims_batch { int dummy; };

extern "C" {
cosims_status cosims_batch_create(const cosims_molecule *, const cosims_params *, int32_t,
                                  int32_t, int32_t, cosims_batch **out) {
  if (out) *out = nullptr;
  return fail(COSIMS_ERR_UNSUPPORTED, "batched form not built");
}
void cosims_batch_destroy(cosims_batch *b) { delete b; }
cosims_status cosims_batch_autotune(cosims_batch *, void *) {
  return fail(COSIMS_ERR_UNSUPPORTED, "batched form not built");
}
cosims_status cosims_batch_run(cosims_batch *, const uint64_t *, const int64_t *,
                               const int64_t *, cosims_ccs_sums *, void *) {
  return fail(COSIMS_ERR_UNSUPPORTED, "batched form not built");
}
cosims_status cosims_batch_run_async(cosims_batch *, const uint64_t *, const int64_t *,
                                     const int64_t *, cosims_ccs_sums *, void *) {
  return fail(COSIMS_ERR_UNSUPPORTED, "batched form not built");
}
cosims_status cosims_batch_get_launch(const cosims_batch *, int32_t, int32_t *, int32_t *) {
  return fail(COSIMS_ERR_UNSUPPORTED, "batched form not built");
}
}
