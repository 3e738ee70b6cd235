// Entry points whose kernels are not built yet report NSPB_ERR_UNSUPPORTED.
#include "spgemm_host.h"

namespace nspb {
int run_numeric_mode(Call &call, nspb_csr_out *C) {
  if (call.opts.precision == NSPB_PREC_FP64) return call.numeric(C->rowptr, C->col, C->val);
  return NSPB_ERR_UNSUPPORTED;
}
}  // namespace nspb

extern "C" {
int nspb_spgemm_batched(int, const nspb_csr_in *, const nspb_csr_in *, nspb_csr_out *,
                        const nspb_opts *, nspb_stats *) { return NSPB_ERR_UNSUPPORTED; }
int nspb_spgemm_rowblocked(const nspb_csr_in *, const nspb_csr_in *, int64_t, int32_t *, int32_t *,
                           double *, int64_t, int64_t *, int32_t *, const nspb_opts *) { return NSPB_ERR_UNSUPPORTED; }
}
