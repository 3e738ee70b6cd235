// Host-side interfaces between the orchestration (spgemm.cu) and the kernel
// translation units. Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/nspb.h"

namespace nspb {

struct DevInfo {
  int device = -1;
  int sms = 0;
  int smem_optin = 0;  // max dynamic shared memory per block (opt-in)
  size_t total_mem = 0;  // device memory in bytes
};
// Properties of the current device (cached per device).
const DevInfo &dev_info();

// Internal device view of a CSR operand (fp64 values unless noted).
struct CsrDev {
  int nrows = 0, ncols = 0;
  int64_t nnz = 0;
  const int *rpt = nullptr;
  const int *col = nullptr;
  const double *val = nullptr;
  const float *val32 = nullptr;  // fp32 operands (FP32_COMP mode)
};

// One product's operands as the row kernels read them (device pointers).
// Layout-identical for every VT, so a table can be viewed as Operands<void>
// by the kernels that read no values.
template <typename VT>
struct Operands {
  const int *arpt = nullptr;
  const int *acol = nullptr;
  const VT *aval = nullptr;
  const int *brpt = nullptr;
  const int *bcol = nullptr;
  const VT *bval = nullptr;
  int ncols = 0;  // columns of B
  int brows = 0;  // rows of B
};

// The products a call computes, as the row kernels see them. A call's rows
// are numbered globally; one product (prod_of_row null) is `one`, held by
// value in the kernel parameters. A batch of products keeps a device array of
// Operands, the product of every global A row and each product's first global
// row: kernels read A and B where they lie, and nothing is concatenated.
template <typename VT>
struct ProdTable {
  Operands<VT> one;
  const Operands<VT> *ops = nullptr;
  const int *prod_of_row = nullptr;
  const int *row_off = nullptr;
};

template <typename VT>
inline ProdTable<void> structure_of(const ProdTable<VT> &t) {
  ProdTable<void> s;
  s.one.arpt = t.one.arpt;
  s.one.acol = t.one.acol;
  s.one.aval = t.one.aval;
  s.one.brpt = t.one.brpt;
  s.one.bcol = t.one.bcol;
  s.one.bval = t.one.bval;
  s.one.ncols = t.one.ncols;
  s.one.brows = t.one.brows;
  s.ops = reinterpret_cast<const Operands<void> *>(t.ops);
  s.prod_of_row = t.prod_of_row;
  s.row_off = t.row_off;
  return s;
}

// What the host launchers need besides the table: the call's rows, the
// largest B column count (bitmap windows of the long-row kernels) and the
// number of products.
struct ProdInfo {
  int n = 0;
  int max_ncols = 0;
  int nprod = 1;
  int max_brows = 0;
};

// Inclusive row limits of the symbolic and numeric bins (the last bin of each
// is unbounded). The kernel of bin b has a table of 32 << b slots; a limit
// only moves rows between bins, never past what a bin's kernel holds.
struct BinLimits {
  int sym[16];
  int num[16];
};
// From the fill percentages of nspb_opts (0: the defaults, 75% and 50%).
BinLimits bin_limits(int sym_fill_pct, int num_fill_pct);
int sym_bin_of(int ub, const BinLimits &l);
int num_bin_of(int nz, const BinLimits &l);

// Flag bits: B_UNSORTED written by launch_check_sorted (and k_rowinfo);
// MAP_OVERFLOW by the map-recording symbolic kernels when a row has more
// intermediate products than its map stride (the call then drops the map).
enum : int { B_UNSORTED = 1, MAP_OVERFLOW = 2 };

// ---- entry maps ------------------------------------------------------------------
// The symbolic row-group kernels can record, for every intermediate product
// of a row, the index of its column among the row's distinct columns in
// order of first appearance (one byte; rows of more than 256 entries are not
// served). map_off[row] gives the row's map in 16-byte units from the map
// base, or kNoMap.
constexpr unsigned kNoMap = 0xffffffffu;
constexpr unsigned kMapEmpty = 0xffffffffu;   // empty slot of the map tables
constexpr int kMapMaxCols = (1 << 24) - 2;    // column offsets take 24 bits
constexpr int kMapNumBins = 5;                // numeric bins served: <= 256 entries
struct MapArgs {
  unsigned char *map = nullptr;  // the call's map
  long long bin_off = 0;         // bytes from map to this bin's first row
  int stride = 0;                // bytes per row (a multiple of 16)
  unsigned *map_off = nullptr;   // per global row
  int *flags = nullptr;          // MAP_OVERFLOW
  int chunk = 1;                 // rows a group takes in a run; > 1: row templates
                                 // (negative: exactly -chunk, see template_chunk)
  const unsigned *bshift = nullptr;  // B row shift bits (launch_brow_shift), or none
};
// Row templates of the map symbolic pass: consecutive rows a group takes in a
// run, and the opts.row_kernel bit that turns templates off.
constexpr int kTemplateRun = 16;
constexpr int kNoRowTemplates = 0x10000;

// fp32 input modes (compensated pairs, or fp64 accumulation of exact products).
inline bool fp32_inputs(int precision) {
  return precision == NSPB_PREC_FP32_COMP || precision == NSPB_PREC_FP32_WIDE;
}

// Compensated-mode parameters of a numeric launch (fp32 inputs).
struct CompArgs {
  int nmax;        // rows with at most nmax A entries accumulate error-free in
                   // fp32 pairs; longer rows accumulate in fp64
  int *redo;       // counter of rows accumulated in fp64
  int *max_deg;    // largest A-row degree among the pair-accumulated rows
};

// ---- rowinfo.cu -----------------------------------------------------------------
cudaError_t launch_check_sorted(const CsrDev &B, int *flags, cudaStream_t s);
// The B rows of every product of a table (ops: device array of nprod entries).
cudaError_t launch_check_sorted_table(const Operands<void> *ops, int nprod, int max_brows,
                                      int *flags, cudaStream_t s);
// row_nz[i] = min(intprod_i, ncols(B)); sym_counts[b] += rows of symbolic bin b
// (rows with zero products are not binned); *total_ip += sum of intprod_i.
// row_ip (optional) receives intprod_i as int64.
// flags (may be NULL): when B is A, B_UNSORTED is set there as launch_check_sorted
// would, from the rows read here. long_list / long_count (may be NULL; n ints and
// a zeroed counter): rows of more than 1024 A entries are listed there and
// counted by a second kernel, a block per row.
cudaError_t launch_rowinfo(const ProdTable<void> &t, int n, int64_t a_nnz, const BinLimits &lim,
                           int *row_nz,
                           int64_t *row_ip, int *sym_counts,
                           unsigned long long *total_ip, int *flags, int *long_list,
                           int *long_count, cudaStream_t s);
// Scatter rows into bin-contiguous order. kind 0: key = ub (symbolic bins),
// kind 1: key = crpt[i+1]-crpt[i] (numeric bins). offsets: 16 bin starts.
struct BinOffsets {
  int v[16];
};
cudaError_t launch_perm(const int *key, int n, int kind, BinOffsets offsets,
                        const BinLimits &lim, int *cursor, int *perm, cudaStream_t s);
// Reorder row lists of perm (list i: perm[off[i] .. off[i]+count[i])) so that
// rows of the heaviest weight class come first; weight as in launch_perm.
// Lists of more than kOrderCap rows are left as they are.
constexpr int kOrderCap = 32768;
struct RowLists {
  int off[16];
  int count[16];
  int n;
};
cudaError_t launch_order_rows(const int *key, int kind, const RowLists &lists, int *perm,
                              cudaStream_t s);
// Single-pass exclusive scan of row_nz into crpt[0..n] (crpt[n] = total) with
// the numeric-bin histogram of the counts. Workspace: tile_state (zeroed,
// scan_tiles(n) entries) and tile_ctr (zeroed).
int scan_tiles(int n);
cudaError_t launch_scan(const int *row_nz, int n, int *crpt, long long *total,
                        unsigned long long *tile_state, int *tile_ctr, const BinLimits &lim,
                        int *num_counts, int *err, cudaStream_t s);
// Numeric-bin histogram from an existing row pointer.
cudaError_t launch_num_hist(const int *crpt, int n, const BinLimits &lim, int *num_counts,
                            cudaStream_t s);

// ---- symbolic.cu ----------------------------------------------------------------
// ticket: a zeroed counter for this launch (block-per-row kernels hand out
// rows with it). b_sorted: B rows strictly increasing (a row's column span
// then comes from the ends of the B rows it touches).
cudaError_t launch_symbolic_bin(int bin, int lanes, bool b_sorted, const ProdTable<void> &t,
                                const ProdInfo &info, const int *rows, int count,
                                int *row_nz, int *err, int *ticket, cudaStream_t s);

// Row-group symbolic bin (bin < kSymGroupBins) that also writes the entry
// map of each row (B rows strictly increasing; every product's B has at
// most kMapMaxCols columns).
// Bit k of bits (nb / 32 + 1 words): B row k is B row k-1 moved by one
// column shift (same length, same column differences).
cudaError_t launch_brow_shift(const int *brpt, const int *bcol, int nb, unsigned *bits,
                              cudaStream_t s);
cudaError_t launch_symbolic_map(int bin, int lanes, const ProdTable<void> &t, const int *rows,
                                int count, int *row_nz, int *err, const MapArgs &m,
                                cudaStream_t s);

// ---- numeric.cu -----------------------------------------------------------------
// owned: B rows hold no duplicate columns (deterministic plain accumulation).
// tshift: the row-group bins use tables 2^tshift times their default size.
// b_sorted: B rows strictly increasing (long rows take their column span
// from the ends of the B rows they touch).
cudaError_t launch_numeric_bin(int bin, int lanes, bool owned, bool b_sorted,
                               const ProdTable<double> &t, const ProdInfo &info,
                               const int *crpt, int *ccol, double *cval,
                               const int *rows, int count, int *err, int *ticket,
                               int tshift, cudaStream_t s);

// Compensated numeric step (fp32 inputs): rows with at most nmax A entries
// accumulate error-free fp32 pairs (TwoProduct + TwoSum) collapsed to fp64;
// the other rows accumulate fp64 products of the widened inputs. *redo
// counts the fp64 rows, *max_deg receives the largest A-row degree among the
// pair rows.
cudaError_t launch_numeric_comp_bin(int bin, int lanes, bool owned, bool b_sorted,
                                    const ProdTable<float> &t, const ProdInfo &info,
                                    const int *crpt, int *ccol, double *cval, const int *rows,
                                    int count, int nmax, int *redo, int *max_deg, int *err,
                                    int *ticket, int tshift, cudaStream_t s);

// ---- rowgroup.cu ----------------------------------------------------------------
// Staged-walk numeric kernels of the row-group bins (numeric bins <
// kNumGroupBins) with lane groups of `lanes` lanes; B rows strictly
// increasing. tshift 0 gives tables of four times the bin's row limit, -1
// twice. depth: B rows whose loads are issued together before their inserts
// (1, 2 or 4).
cudaError_t launch_numeric_rg(int bin, int lanes, int tshift, int depth,
                              const ProdTable<double> &t, const int *crpt, int *ccol,
                              double *cval, const int *rows, int count, int *err,
                              cudaStream_t s);
cudaError_t launch_numeric_comp_rg(int bin, int lanes, int tshift, int depth,
                                   const ProdTable<float> &t, const int *crpt, int *ccol,
                                   double *cval, const int *rows, int count, int nmax,
                                   int *redo, int *max_deg, int *err, cudaStream_t s);

// ---- rowmap.cu ------------------------------------------------------------------
// Numeric row-group bin (bin < kMapNumBins) from the entry maps of a
// map-recording symbolic phase: no hash table; B rows strictly increasing.
// prefetch_a (single products only): cp.async copies each group's next row's
// first A entries into shared memory while the current row is computed.
// run > 1: groups take runs of `run` consecutive rows and reuse the sort of a
// row for the rows that share its map (row templates of the symbolic pass) or
// whose B rows are its B rows moved by one shift (bshift, one product).
cudaError_t launch_numeric_map(int bin, int lanes, const ProdTable<double> &t,
                               const unsigned char *map, const unsigned *map_off,
                               const int *crpt, int *ccol, double *cval, const int *rows,
                               int count, bool prefetch_a, int run, const unsigned *bshift,
                               int *err, cudaStream_t s);
// The same for fp32 inputs: rows of at most nmax A entries in fp32 pairs, the
// others in fp64 from exact products (see launch_numeric_comp_bin).
cudaError_t launch_numeric_comp_map(int bin, int lanes, const ProdTable<float> &t,
                                    const unsigned char *map, const unsigned *map_off,
                                    const int *crpt, int *ccol, double *cval, const int *rows,
                                    int count, bool prefetch_a, int run, const unsigned *bshift, int nmax, int *redo,
                                    int *max_deg, int *err, cudaStream_t s);
}  // namespace nspb
