// Autotuner: threads per row and numeric table size chosen by timing the
// caller's own product (the reference fixes both per bin at compile time,
// nsp/inc/nsp.h:25-98).
#include <cuda_runtime.h>

#include <cstring>

#include "internal.h"
#include "spgemm_host.h"

using namespace nspb;

extern "C" int nspb_autotune(const nspb_csr_in *A, const nspb_csr_in *B, const nspb_opts *base,
                             int reps, nspb_opts *best, nspb_tune_entry *report,
                             int32_t *n_report) {
  if (!A || !B || !best || reps < 1) return NSPB_ERR_INVALID;
  nspb_opts o;
  nspb_default_opts(&o);
  if (base) o = *base;
  cudaStream_t s = static_cast<cudaStream_t>(o.stream);
  // C sized and allocated by one checked call, then reused by every candidate
  nspb_csr_out C;
  std::memset(&C, 0, sizeof(C));
  int st = nspb_spgemm(A, B, &C, &o, nullptr);
  if (st) return st;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t ce = cudaEventCreate(&e0);
  if (ce == cudaSuccess) ce = cudaEventCreate(&e1);
  const int lanes[3] = {8, 16, 32};
  float best_ms = -1.f;
  int n = 0;
  for (int li = 0; li < 3 && !st && ce == cudaSuccess; ++li) {
    for (int ts = 0; ts < 2 && !st && ce == cudaSuccess; ++ts) {
      nspb_opts c = o;
      c.group_lanes = lanes[li];
      c.num_table_shift = ts;
      c.check_errors = 0;
      c.timing = 0;
      st = nspb_spgemm(A, B, &C, &c, nullptr);  // warm-up
      if (st) break;
      ce = cudaEventRecord(e0, s);
      for (int r = 0; r < reps && !st && ce == cudaSuccess; ++r) st = nspb_spgemm(A, B, &C, &c, nullptr);
      if (ce == cudaSuccess) ce = cudaEventRecord(e1, s);
      if (ce == cudaSuccess) ce = cudaEventSynchronize(e1);
      float ms = 0.f;
      if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, e0, e1);
      if (st || ce != cudaSuccess) break;
      ms /= (float)reps;
      if (report) report[n] = nspb_tune_entry{c.group_lanes, c.num_table_shift, ms, 0};
      ++n;
      if (best_ms < 0.f || ms < best_ms) {
        best_ms = ms;
        *best = o;
        best->group_lanes = c.group_lanes;
        best->num_table_shift = c.num_table_shift;
      }
    }
  }
  if (!st && ce != cudaSuccess) {
    g_last_cuda = (int)ce;
    cudaGetLastError();
    st = NSPB_ERR_CUDA;
  }
  // one checked call with the winner (device error words of the timed runs)
  if (!st) st = nspb_spgemm(A, B, &C, best, nullptr);
  if (n_report) *n_report = n;
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaStreamSynchronize(s);
  nspb_free(C.rowptr);
  nspb_free(C.col);
  nspb_free(C.val);
  return st;
}
