// egpu_batch.cu -- batched persistent solver (entry points; implementation follows)
#include "egpu_internal.cuh"

struct egpu_batch {
  egpu_ctx *ctx;
};

extern "C" int egpu_batch_create(egpu_ctx *ctx, egpu_batch **out) {
  (void)ctx;
  if (out) *out = nullptr;
  return EGPU_ERR_STATE;
}
extern "C" int egpu_batch_add(egpu_batch *, int, const int *, const int *, const int *, const double *,
                              const double *) {
  return EGPU_ERR_STATE;
}
extern "C" int egpu_batch_solve(egpu_batch *, const egpu_params *, egpu_result *) { return EGPU_ERR_STATE; }
extern "C" int egpu_batch_solution(egpu_batch *, int, double *) { return EGPU_ERR_STATE; }
extern "C" int egpu_batch_tune(egpu_batch *, const egpu_params *, int *) { return EGPU_ERR_STATE; }
extern "C" void egpu_batch_free(egpu_batch *) {}
