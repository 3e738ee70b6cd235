// Numeric step in the call's precision mode.
#include "spgemm_host.h"

namespace nspb {
int run_numeric_mode(Call &call, nspb_csr_out *C) {
  return call.numeric(C->rowptr, C->col, C->val);
}
}  // namespace nspb

