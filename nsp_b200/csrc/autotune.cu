// Autotuner: the row-group kernels' threads per row, kernel family and table
// size, and the symbolic and numeric bin thresholds, chosen by timing the
// caller's own product (the reference fixes all of them per bin at compile
// time: nsp/inc/nsp.h:25-98, bin limits nsp/src/nsp.cu:336-345, 1150-1162).
//
// A coordinate search from the library's defaults: each knob in turn is tried
// at every candidate value with the best values found so far for the others,
// and kept at its fastest. Candidates, in search order:
//   group_lanes     8, 16, 32
//   row_kernel      1 (hash tables, in-table sort), 2 (staged walk), 7 (entry maps)
//   table size      hash-sort: num_table_shift 0, 1; staged: row_kernel 2, 3
//   sym_fill_pct    50, 75, 90
//   num_fill_pct    25, 37, 50
// 13 timed candidates at most (the default of each knob is timed once).
#include <cuda_runtime.h>

#include <cstring>
#include <vector>

#include "internal.h"
#include "spgemm_host.h"

using namespace nspb;

namespace {

struct Knobs {
  int lanes, tshift, rk, sym_fill, num_fill;
  bool operator==(const Knobs &o) const {
    return lanes == o.lanes && tshift == o.tshift && rk == o.rk && sym_fill == o.sym_fill &&
           num_fill == o.num_fill;
  }
};

struct Tuner {
  const nspb_csr_in *A, *B;
  nspb_opts base;
  nspb_csr_out *C;
  int reps;
  cudaStream_t s;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  std::vector<std::pair<Knobs, float>> seen;

  nspb_opts opts_of(const Knobs &k) const {
    nspb_opts c = base;
    c.group_lanes = k.lanes;
    c.num_table_shift = k.tshift;
    c.row_kernel = k.rk;
    c.sym_fill_pct = k.sym_fill;
    c.num_fill_pct = k.num_fill;
    c.check_errors = 0;
    c.timing = 0;
    return c;
  }

  // mean ms of `reps` products with knobs k (after one warm-up); cached
  int time(const Knobs &k, float *ms) {
    for (auto &p : seen)
      if (p.first == k) {
        *ms = p.second;
        return NSPB_OK;
      }
    const nspb_opts c = opts_of(k);
    int st = nspb_spgemm(A, B, C, &c, nullptr);  // warm-up
    if (st) return st;
    cudaError_t ce = cudaEventRecord(e0, s);
    for (int r = 0; r < reps && !st && ce == cudaSuccess; ++r) st = nspb_spgemm(A, B, C, &c, nullptr);
    if (st) return st;
    if (ce == cudaSuccess) ce = cudaEventRecord(e1, s);
    if (ce == cudaSuccess) ce = cudaEventSynchronize(e1);
    float t = 0.f;
    if (ce == cudaSuccess) ce = cudaEventElapsedTime(&t, e0, e1);
    if (ce != cudaSuccess) {
      g_last_cuda = (int)ce;
      cudaGetLastError();
      return NSPB_ERR_CUDA;
    }
    *ms = t / (float)reps;
    seen.push_back({k, *ms});
    return NSPB_OK;
  }

  // try every value of one knob (set by `put`) around `best`
  template <typename Put>
  int sweep(Knobs &best, float &best_ms, const int *vals, int nv, Put put) {
    for (int i = 0; i < nv; ++i) {
      Knobs k = best;
      put(k, vals[i]);
      float ms = 0.f;
      const int st = time(k, &ms);
      if (st) return st;
      if (ms < best_ms) {
        best_ms = ms;
        best = k;
      }
    }
    return NSPB_OK;
  }
};

}  // namespace

extern "C" int nspb_autotune(const nspb_csr_in *A, const nspb_csr_in *B, const nspb_opts *base,
                             int reps, nspb_opts *best, nspb_tune_entry *report,
                             int32_t *n_report) {
  if (!A || !B || !best || reps < 1) return NSPB_ERR_INVALID;
  nspb_opts o;
  nspb_default_opts(&o);
  if (base) o = *base;
  // C sized and allocated by one checked call, then reused by every candidate
  nspb_csr_out C;
  std::memset(&C, 0, sizeof(C));
  int st = nspb_spgemm(A, B, &C, &o, nullptr);
  if (st) return st;
  Tuner t{A, B, o, &C, reps, static_cast<cudaStream_t>(o.stream)};
  cudaError_t ce = cudaEventCreate(&t.e0);
  if (ce == cudaSuccess) ce = cudaEventCreate(&t.e1);
  if (ce != cudaSuccess) {
    g_last_cuda = (int)ce;
    cudaGetLastError();
    st = NSPB_ERR_CUDA;
  }
  Knobs k{32, 0, 1, 75, 50};
  float k_ms = 1e30f;
  if (!st) st = t.time(k, &k_ms);
  static const int lanes[] = {8, 16, 32}, kinds[] = {1, 2, 7}, fills_s[] = {50, 75, 90},
                   fills_n[] = {25, 37, 50};
  if (!st) st = t.sweep(k, k_ms, lanes, 3, [](Knobs &x, int v) { x.lanes = v; });
  if (!st) st = t.sweep(k, k_ms, kinds, 3, [](Knobs &x, int v) { x.rk = v; });
  if (!st) {
    if (k.rk == 7) {
      // entry maps have no table size
    } else if (k.rk == 1) {
      static const int shifts[] = {0, 1};
      st = t.sweep(k, k_ms, shifts, 2, [](Knobs &x, int v) { x.tshift = v; });
    } else {
      static const int staged[] = {2, 3};
      st = t.sweep(k, k_ms, staged, 2, [](Knobs &x, int v) { x.rk = v; });
    }
  }
  if (!st) st = t.sweep(k, k_ms, fills_s, 3, [](Knobs &x, int v) { x.sym_fill = v; });
  if (!st) st = t.sweep(k, k_ms, fills_n, 3, [](Knobs &x, int v) { x.num_fill = v; });
  if (!st) {
    *best = t.opts_of(k);
    best->check_errors = o.check_errors;
    best->timing = o.timing;
    // one checked call with the winner (device error words of the timed runs)
    nspb_opts chk = *best;
    chk.check_errors = 1;
    st = nspb_spgemm(A, B, &C, &chk, nullptr);
  }
  int n = 0;
  for (auto &p : t.seen) {
    if (report && n < NSPB_TUNE_MAX_REPORT)
      report[n] = nspb_tune_entry{p.first.lanes, p.first.tshift, p.second, p.first.rk,
                                  p.first.sym_fill, p.first.num_fill};
    ++n;
  }
  if (n_report) *n_report = n < NSPB_TUNE_MAX_REPORT ? n : NSPB_TUNE_MAX_REPORT;
  if (t.e0) cudaEventDestroy(t.e0);
  if (t.e1) cudaEventDestroy(t.e1);
  cudaStreamSynchronize(t.s);
  nspb_free(C.rowptr);
  nspb_free(C.col);
  nspb_free(C.val);
  return st;
}
