// Host-side state of one product call (shared by the one-call, two-call,
// FP32-compensated, batched and row-blocked entry points).
#pragma once

#include <cuda_runtime.h>

#include "internal.h"

namespace nspb {

extern thread_local int g_last_cuda;

// Device counters of a call, zeroed at the start; read back in one copy.
struct DevCounters {
  int sym_counts[16];
  int num_counts[16];
  int cursor_sym[16];
  int cursor_num[16];
  int flags;
  int err;
  int tile_ctr;
  int redo_count;
  unsigned long long total_ip;
  long long total_nnz;
  float max_row_err;
  int max_comp_deg;  // compensated mode: largest A-row degree of a pair row
  int long_rows;     // rows listed for the block-per-row intermediate-product count
  int pad;
  int ticket[32];    // row tickets of the block-per-row launches (symbolic
                     // bin b at b, numeric bin b at 16 + b)
};

struct HostStage {
  DevCounters c;
};

HostStage *host_stage();
int scratch_alloc(void **p, size_t bytes, cudaStream_t s);
void scratch_free(void *p, cudaStream_t s);
int alloc_out(void **p, size_t bytes);

struct Call {
  nspb_opts opts{};
  cudaStream_t s = nullptr;
  CsrDev A, B;  // one product's operands (a table of one); see set_table for batches
  // what the kernels read: one product by value, or a device table of products
  ProdTable<double> t64;
  ProdTable<float> t32;
  ProdInfo info;
  BinLimits lim{};                  // bin thresholds (opts.sym_fill_pct, num_fill_pct)
  int64_t a_nnz = 0;                // entries of A over all products
  bool table = false;               // several products through a device table
  const Operands<void> *ops = nullptr;
  int n = 0;
  int lanes = 32;
  // scratch (one stream-ordered block)
  char *ws = nullptr;
  size_t ws_bytes = 0;
  size_t off_row_nz = 0, off_perm = 0, off_counters = 0, off_tiles = 0;
  int *row_nz = nullptr;
  int *perm = nullptr;
  DevCounters *ctr = nullptr;
  unsigned long long *tile_state = nullptr;
  // host copies
  DevCounters h{};
  bool b_sorted = true;
  bool num_counts_ready = false;
  int64_t intprod = 0;
  int launches = 0;
  // Caller-supplied scratch and host staging (set by nspb_spgemm_noalloc);
  // when null the pool and the pinned per-thread stage are used.
  char *ext_ws = nullptr;
  size_t ext_bytes = 0;
  bool ws_external = false;
  HostStage *stage = nullptr;
  // Entry maps (k_sym_map / k_num_map): the symbolic phase records, for each
  // intermediate product, its column's index among the row's distinct
  // columns; the numeric row-group bins of at most 256 entries then add every
  // product at its index with no hash table. allow_map false: entry points
  // whose numeric phase runs in another call, or that may not allocate.
  bool allow_map = true;
  bool use_map = false;
  void *map_block = nullptr;   // pool block: map_off (n entries), B row shift bits, the map
  unsigned char *map = nullptr;
  unsigned *map_off = nullptr;
  unsigned *bshift = nullptr;  // B row shift bits for the row templates (one product)
  bool map_wanted() const;
  // opts.timing: events around rowinfo, symbolic, scan, numeric
  cudaEvent_t ev[8] = {};
  bool timing = false;
  // Numeric row-group bins through the staged-walk kernels (rowgroup.cu)?
  // opts.row_kernel 2 or 3 always, 1 never, 0 when the rows compress: at
  // least 1.5 intermediate products per entry of C (measured on B200: the
  // staged walk wins on stencils, 1.04x, and 7-point Laplacians, 1.27x, and
  // loses on random and power-law rows, where almost every product is a new
  // entry). Needs B rows strictly increasing.
  bool use_staged() const {
    const int k = opts.row_kernel & 0xff;
    if (k == 2 || k == 3) return true;
    if (k != 0) return false;
    return h.total_nnz > 0 && (double)intprod >= 1.5 * (double)h.total_nnz;
  }
  // B rows whose loads the staged walk issues ahead: bits 8.. of row_kernel (0 = 4)
  // Rows a group takes in a run on the entry-map path (row templates): bits
  // 20..27 of row_kernel, taken as given (returned negative, see
  // template_chunk), or kTemplateRun, shortened for small bins; 1 with
  // templates turned off.
  int template_run() const {
    if (opts.row_kernel & kNoRowTemplates) return 1;
    const int r = (opts.row_kernel >> 20) & 0xff;
    return r ? -r : kTemplateRun;
  }
  int rg_depth() const {
    const int d = (opts.row_kernel >> 8) & 0xff;
    return d ? d : 4;
  }
  void mark(int i) {
    if (timing && ev[i]) cudaEventRecord(ev[i], s);
  }

  int init(const nspb_csr_in *a, const nspb_csr_in *b, const nspb_opts *o);
  // Batched call: the products of a device table instead of init's A and B
  // (init must have run with any valid operands first; opts are kept).
  void set_table(const ProdTable<double> &d, const ProdTable<float> &f, const ProdInfo &pi,
                 int64_t total_a_nnz);
  size_t scratch_bytes();  // sets the scratch offsets; bytes alloc_scratch needs
  int alloc_scratch();
  int cuda_fail(cudaError_t e);
  int fetch_counters();
  // heaviest rows first in the block-per-row bins [first, end) of perm
  cudaError_t order_block_bins(const int *key, int kind, const int *counts, int first, int end,
                               const BinOffsets &off);
  int symbolic(int *crpt, int64_t *nnz_out);
  int prepare_numeric(const int *crpt);
  int numeric(const int *crpt, int *ccol, double *cval);
  int finish(nspb_stats *stats);
  ~Call();
};

// Compensated mode: longest A row accumulated in fp32 pairs for a tolerance,
// and the relative error bound of a pair row with n A entries.
int comp_nmax(double tol);
double comp_bound(int n);

}  // namespace nspb
