/*
 * nspb.h — C ABI of the B200-native CSR sparse matrix product C = A·B.
 *
 * Every entry point is `extern "C"`, takes plain pointers and sizes and
 * returns an int status (0 = success, negative = nspb_status). Device
 * pointers are CUDA device addresses on the current device; streams are
 * passed as `void*` (a cudaStream_t, NULL = the legacy default stream).
 *
 * Reference interfaces replaced (file:line in amavliut/nsp):
 *   nspb_spgemm            <- nsp_spgemm_kernel_hash   nsp/inc/nsp.h:105,
 *                             nsp/src/nsp.cu:2448-2488 (one call, C allocated
 *                             inside, row_ptr/col/val device arrays)
 *   nspb_spgemm_symbolic   <- nsp_set_max_bin + nsp_set_row_nnz
 *                             nsp/src/nsp.cu:417-471, 921-1130 (row counts and
 *                             the exclusive scan to row_ptr)
 *   nspb_spgemm_numeric    <- nsp_set_min_bin + nsp_calculate_value_col_bin
 *                             nsp/src/nsp.cu:1241-1300, 2178-2440
 *   nspb_intprod           <- nsp_set_intprod_num      nsp/src/nsp.cu:306-320
 *   nspb_getmct            <- getmct                   src/getmct.cu:41-92
 *   nspb_compactcol        <- compactcol / cuCompactor src/compactcol.cu:160-163
 *   nspb_shrink_col        <- get_shrinked_col / apply_mask_permut_GPU_noSideEffects
 *                             src/spspmpi.cu:58-104, 106-182
 *   nspb_spgemm_batched    <- no single reference entry point: replaces a host
 *                             loop of nsp_spgemm_kernel_hash calls (one per
 *                             Galerkin product), src/spspmpi.cu:266-313
 *   nspb_spgemm_rowblocked <- nsparseMGPU_version1's shrink + local product,
 *                             src/spspmpi.cu:906-935, run per row block on one GPU
 *
 * C++ drop-in shims with the reference's own signatures (sfCSR, CSR,
 * nsparseMGPU_version0/1) are declared in nspb_compat.h.
 */
#ifndef NSPB_H
#define NSPB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
typedef enum {
  NSPB_OK = 0,
  NSPB_ERR_INVALID = -1,   /* null pointer, negative size, dimension mismatch   */
  NSPB_ERR_OVERFLOW = -2,  /* nnz(C) or a row count does not fit int32          */
  NSPB_ERR_ALLOC = -3,     /* device or pinned-host allocation failed           */
  NSPB_ERR_CUDA = -4,      /* a CUDA runtime call failed (see nspb_last_cuda_error) */
  NSPB_ERR_DEVICE = -5,    /* a kernel raised its error word (bounded probe or
                              bounded wait exhausted); results are invalid      */
  NSPB_ERR_NO_DEVICE = -6, /* no CUDA device visible                            */
  NSPB_ERR_UNSUPPORTED = -7,
  NSPB_ERR_CAPACITY = -8,  /* a size exceeds a fixed capacity of the call       */
  NSPB_ERR_IO = -9         /* a file could not be opened, read or written       */
} nspb_status;

/* value types */
enum { NSPB_F64 = 0, NSPB_F32 = 1 };

/* precision modes of the product */
enum {
  NSPB_PREC_FP64 = 0,      /* fp64 inputs, fp64 accumulation (the drop-in)       */
  NSPB_PREC_FP32_COMP = 1, /* fp32 inputs, error-free fp32 products and two-sum
                              compensated accumulation, fp64 output; rows whose
                              running error bound exceeds opts.comp_tol are
                              re-accumulated in fp64                            */
  NSPB_PREC_FP32_WIDE = 2  /* fp32 inputs (half the value bytes), products
                              exact in fp64 (24 + 24 significant bits), fp64
                              accumulation in A-row order; |c - c*| <=
                              n 2^-53 sum|a*b| for a row of n A entries         */
};

/* A CSR matrix on the device. rowptr has nrows+1 entries, 0-based, int32.   */
typedef struct {
  int32_t nrows;
  int32_t ncols;
  int64_t nnz;
  const int32_t *rowptr;
  const int32_t *col;
  const void *val;       /* nnz values of val_type                          */
  int32_t val_type;      /* NSPB_F64 or NSPB_F32                            */
  int32_t _pad;
} nspb_csr_in;

/* Output CSR. If `col`/`val` are NULL on entry, the call allocates them with
 * cudaMalloc (release with cudaFree or nspb_free). If they are non-NULL,
 * `capacity` must hold their length in entries; the call fails with
 * NSPB_ERR_CAPACITY when nnz(C) exceeds it. `rowptr` follows the same rule
 * (nrows+1 entries). val is always fp64.                                    */
typedef struct {
  int32_t nrows;
  int32_t ncols;
  int64_t nnz;
  int32_t *rowptr;
  int32_t *col;
  double *val;
  int64_t capacity;
} nspb_csr_out;

typedef struct {
  int32_t precision;     /* NSPB_PREC_*                                      */
  int32_t assume_sorted; /* 1: caller guarantees B rows strictly increasing
                            (skips the B check pass)                         */
  int32_t check_errors;  /* 1: synchronise at the end and report device
                            error words                                      */
  int32_t group_lanes;   /* 0 = auto; else 8, 16 or 32 lanes per row group    */
  int32_t timing;        /* 1: record CUDA events around each phase (stats)  */
  int32_t batch_max_products; /* batched calls and plans: at most this many
                            products per block-diagonal group (0 = no limit
                            beyond the int32 and size-based grouping)        */
  double comp_tol;       /* FP32_COMP: bound on |c - c*| / sum|a*b| per entry;
                            rows whose a-priori Dot2 bound exceeds it are
                            accumulated in fp64 (default 1e-10)              */
  void *stream;          /* cudaStream_t                                     */
  int32_t num_table_shift; /* 0: numeric row-group tables of twice the bin's
                            entry limit (load <= 1/2); 1: four times (load
                            <= 1/4); chosen by nspb_autotune              */
  int32_t row_kernel;    /* numeric row-group kernels (rows of <= 512 entries):
                            0 = automatic: the staged walk when the rows
                            compress (>= 1.5 intermediate products per entry
                            of C), else hash tables with an in-table sort;
                            1 = always the hash-sort kernels; 2 = always the
                            staged walk (tables of 4x the bin's row limit);
                            3 = staged walk with tables of 2x; 7 = entry
                            maps: the symbolic pass records each product's
                            entry index in its row and the numeric rows of
                            <= 256 entries add at that index with no hash
                            table (0 takes maps when the B rows read fill
                            3/4 of the row groups' lanes on average; maps
                            need one-call products, sorted B rows, no row of
                            more than 3072 products, < 2^24 columns).
                            With maps, rows that repeat a neighbour's
                            pattern (the same A and B row lengths, every
                            product column moved by one shift) reuse its
                            count, map and sort (row templates): bit 16
                            (0x10000) turns them off; bits 8..15: B rows
                            the staged walk loads ahead (0 = 4); bits
                            20..27: rows a row group takes in a run (0 =
                            16, shorter for small bins)                    */
  int32_t sym_fill_pct;  /* symbolic bin thresholds: a row goes to the bin
                            whose table (32 << b slots) it fills to at most
                            this percentage at its upper bound of distinct
                            columns; 0 = 75, else 10..90                     */
  int32_t num_fill_pct;  /* numeric bin thresholds: a row of nnz entries goes
                            to the bin whose 32 << b slots it fills to at
                            most this percentage; 0 = 50, else 10..50        */
} nspb_opts;

/* Per-call figures (all optional; pass NULL).                               */
typedef struct {
  int64_t intprod;       /* sum_i sum_{k in A(i,:)} nnz(B(k,:))              */
  int64_t nnz;           /* nnz(C)                                           */
  int32_t sym_bins[16];  /* rows per symbolic bin                            */
  int32_t num_bins[16];  /* rows per numeric bin                             */
  int32_t rows_redone;   /* FP32_COMP: rows accumulated in fp64 instead       */
  int32_t b_sorted;      /* 1 if B rows were found strictly increasing       */
  double max_row_err;    /* FP32_COMP: largest per-row error bound of the
                            fp32-pair rows, relative to sum|a*b|            */
  int32_t launches;      /* kernels this call launched                       */
  float ms_rowinfo;      /* opts.timing: B check + row counts + bins         */
  float ms_symbolic;     /* opts.timing: permutation + symbolic kernels      */
  float ms_scan;         /* opts.timing: row_ptr scan                        */
  float ms_numeric;      /* opts.timing: permutation + numeric kernels       */
  int32_t entry_map;     /* 1 if the symbolic phase recorded entry maps and
                            the numeric row-group bins of <= 256 entries ran
                            from them (opts.row_kernel 0 or 7); batched
                            calls and plans: the number of such groups     */
} nspb_stats;

/* ---- library ------------------------------------------------------------ */
const char *nspb_version(void);
const char *nspb_strerror(int status);
int nspb_last_cuda_error(void);          /* cudaError_t of the last failure  */
void nspb_default_opts(nspb_opts *opts);
int nspb_free(void *device_ptr);         /* cudaFree                         */
int nspb_device_sm_count(int *sms);

/* ---- the product ---------------------------------------------------------- */
/* C = A·B. One call: counts, allocates C (unless provided), fills it. On
 * return C->rowptr/col/val are complete in stream order on opts->stream; the
 * call itself synchronises twice on the host (bin sizes; nnz(C)).           */
int nspb_spgemm(const nspb_csr_in *A, const nspb_csr_in *B, nspb_csr_out *C,
                const nspb_opts *opts, nspb_stats *stats);

/* Two-call form. symbolic writes C->rowptr (allocating it when NULL) and sets
 * C->nnz; numeric fills C->col/C->val (allocating when NULL). The structure
 * of A and B must not change between the two calls.                         */
int nspb_spgemm_symbolic(const nspb_csr_in *A, const nspb_csr_in *B,
                         nspb_csr_out *C, const nspb_opts *opts,
                         nspb_stats *stats);
int nspb_spgemm_numeric(const nspb_csr_in *A, const nspb_csr_in *B,
                        nspb_csr_out *C, const nspb_opts *opts,
                        nspb_stats *stats);

/* No counterpart in the reference. The one-call fp64 product for callers that
 * may not allocate memory during the call (a framework that owns all device
 * memory and forbids allocations inside the calls it dispatches, a loop with
 * memory reserved up front, a process near the HBM limit). C->rowptr, C->col
 * and C->val must be supplied, with C->capacity entries in col/val
 * (NSPB_ERR_CAPACITY with C->nnz = the size needed when too small). Scratch
 * comes from a fixed 32 MiB device array inside the library, so A may have at
 * most about 4.19 million rows (4,000,000 always fit); larger inputs get
 * NSPB_ERR_CAPACITY with C->nnz = -1 before any GPU work. Calls share that
 * array: calls whose GPU work overlaps race, so serialise them. The first
 * call on each device looks up the array's device address, and CUDA's lazy
 * module loading reserves the array's 32 MiB then (and loads the kernels at
 * their first launch): make one small warm-up call at set-up, before any
 * stream capture begins, so that later calls take no memory at all. The
 * looked-up address assumes the device's primary context lives as long as
 * the process (no cudaDeviceReset in between).                              */
int nspb_spgemm_noalloc(const nspb_csr_in *A, const nspb_csr_in *B,
                        nspb_csr_out *C, const nspb_opts *opts,
                        nspb_stats *stats);

/* Per-row intermediate-product counts (device out, int64[nrows]) and their
 * total (host out).                                                          */
int nspb_intprod(const nspb_csr_in *A, const nspb_csr_in *B, int64_t *d_row_ip,
                 int64_t *total, void *stream);

/* ---- batched products ------------------------------------------------------ */
/* `count` independent products C[i] = A[i]·B[i] through one pipeline: the
 * rows of all products form one work list, read through per-product operand
 * descriptors and a row-to-product map (no copies of A or B), with one launch
 * per phase and bin. Products are grouped so that each group's nnz(C) stays
 * below int32; a group reads back to the host the bin counts, nnz(C), the
 * error word (when checked) and C's per-product offsets. C[i] are views into one allocation
 * per group (values, columns, row pointers); their base pointers are written
 * to owners (room for 3*count) and *n_owners; release them with nspb_free.  */
int nspb_spgemm_batched(int count, const nspb_csr_in *A, const nspb_csr_in *B,
                        nspb_csr_out *C, const nspb_opts *opts,
                        nspb_stats *stats, void **owners, int32_t *n_owners);

/* ---- host-memory operands --------------------------------------------------
 * C = A·B with A, B (nspb_csr_in whose pointers are HOST memory, row pointers
 * starting at 0) and C in host memory. Structure is copied first, values in
 * row chunks on a second stream while the symbolic phase runs; the numeric
 * phase runs in `nblocks` row blocks (0 = 16), each once the value chunks it
 * reads are in, whose columns and values are copied back on a third stream
 * while the next block is computed. Pinned host arrays give full-bandwidth,
 * overlapped copies. h_rowptr receives n+1 entries; h_col/h_val must hold
 * h_capacity entries: with fewer than nnz(C) (or NULL) only the row pointer
 * is written, *nnz_out tells the size and NSPB_ERR_CAPACITY is returned.
 * When B's three host arrays are A's, they are copied once.             */
int nspb_spgemm_host(const nspb_csr_in *hA, const nspb_csr_in *hB, int32_t *h_rowptr,
                     int32_t *h_col, double *h_val, int64_t h_capacity, int64_t *nnz_out,
                     int32_t nblocks, const nspb_opts *opts);

/* ---- autotuner ---------------------------------------------------------------
 * Times this product (C sized once, then written into the same arrays) under
 * candidates of the row-group threads per row (group_lanes 8, 16, 32), kernel
 * family (row_kernel 1 hash-sort, 2 staged walk), table size (num_table_shift
 * 0/1, or row_kernel 2/3) and bin thresholds (sym_fill_pct 50/75/90,
 * num_fill_pct 25/37/50), each knob swept in turn with the best values found
 * so far for the others: one warm-up and `reps` timed calls per candidate,
 * CUDA events on opts->stream. *best receives `base` with the fastest
 * candidate's knobs; report (may be NULL; room for NSPB_TUNE_MAX_REPORT) the
 * candidates and their mean ms, *n_report their number.                    */
#define NSPB_TUNE_MAX_REPORT 16
typedef struct {
  int32_t group_lanes;
  int32_t num_table_shift;
  float ms;
  int32_t row_kernel;
  int32_t sym_fill_pct;
  int32_t num_fill_pct;
} nspb_tune_entry;
int nspb_autotune(const nspb_csr_in *A, const nspb_csr_in *B, const nspb_opts *base,
                  int reps, nspb_opts *best, nspb_tune_entry *report, int32_t *n_report);

/* ---- plans: repeated products of a fixed structure --------------------------
 * An AMG setup or a time loop often forms the same products again with new
 * values. nspb_plan_create runs the symbolic phase of `count` products once
 * (as one block-diagonal product when count > 1), allocates every C, runs
 * one numeric pass and captures the numeric phase (counter reset, value
 * concatenation, per-bin kernels, split) in a CUDA graph.
 * nspb_plan_execute replays that graph on `stream`: it reads the CURRENT
 * values behind A[p].val and B[p].val (same pointers, same structure as at
 * creation) and rewrites C's values. C[p] point into plan-owned arrays that
 * stay valid until nspb_plan_destroy. One plan must not be executed on two
 * streams at once. opts.check_errors makes execute synchronise and report the
 * device error word. fp64 or the fp32 compensated mode.                   */
typedef struct nspb_plan_s *nspb_plan;
int nspb_plan_create(int count, const nspb_csr_in *A, const nspb_csr_in *B,
                     nspb_csr_out *C, const nspb_opts *opts, nspb_stats *stats,
                     nspb_plan *plan);
int nspb_plan_execute(nspb_plan plan, void *stream);
int nspb_plan_destroy(nspb_plan plan);

/* ---- column remap (compactcol / getmct) ------------------------------------ */
/* Sorted unique column indices of col[0..nnz) that fall outside [first,last]
 * (when first > last: all columns). d_out must hold nnz entries; *nout is
 * the number written.                                                        */
int nspb_getmct(const int32_t *d_col, int64_t nnz, int32_t first, int32_t last,
                int32_t *d_out, int64_t *nout, void *stream);
/* Stream compaction: d_out[j] = d_in[i] for the i with pred(d_in[i]) in
 * order, pred(x) = (x < lo || x > hi). *nout = count.                        */
int nspb_compactcol(const int32_t *d_in, int64_t n, int32_t lo, int32_t hi,
                    int32_t *d_out, int64_t *nout, void *stream);
/* Remap each column of d_col to its position in the sorted list d_cols
 * (binary search); columns absent from the list map to -1.                  */
int nspb_shrink_col(const int32_t *d_col, int64_t nnz, const int32_t *d_cols,
                    int64_t ncols, int32_t *d_out, void *stream);

/* Row-blocked product for C larger than a device budget: A is split into
 * contiguous row blocks whose C fits `budget_bytes`; per block the B rows it
 * references are gathered (getmct + shrink), the block product runs, and the
 * block of C is copied to the HOST arrays h_rowptr/h_col/h_val (caller sizes
 * them from nspb_spgemm_symbolic or an upper bound `h_capacity`).            */
int nspb_spgemm_rowblocked(const nspb_csr_in *A, const nspb_csr_in *B,
                           int64_t budget_bytes, int32_t *h_rowptr,
                           int32_t *h_col, double *h_val, int64_t h_capacity,
                           int64_t *nnz_out, int32_t *nblocks_out,
                           const nspb_opts *opts);

/* ---- AMG Galerkin driver ----------------------------------------------------
 * T = A^T (CSRm::T, src/CSR.cu:738-785, cuSPARSE csr2csc there): every row of
 * T lists its columns (A's rows) ascending, duplicates in their stored order.
 * fp64 or fp32 values (T keeps A's value type; T->val then holds floats).
 * Output allocation follows nspb_spgemm (NULL arrays are cudaMalloc'ed;
 * caller arrays must hold nnz(A) entries, else NSPB_ERR_CAPACITY).          */
int nspb_transpose(const nspb_csr_in *A, nspb_csr_out *T, const nspb_opts *opts);
/* Smoothed-aggregation prolongator P = P_tent - omega D^-1 (A P_tent), D the
 * diagonal of A (CSRm::diag, src/CSR.cu:1389-1418: the last stored diagonal
 * entry of a row). fp64; A square with every diagonal entry stored. Each
 * value is (-omega * (A P_tent)_ij) / d_i, plus P_tent_ij where P_tent has an
 * entry, rounded in that order. NSPB_ERR_INVALID when a diagonal entry is
 * missing.                                                                   */
int nspb_sa_prolongator(const nspb_csr_in *A, const nspb_csr_in *Ptent, double omega,
                        nspb_csr_out *P, const nspb_opts *opts);
/* Galerkin coarse operator A_c = R (A P) with R = P^T (returned in R when
 * non-NULL). fp64.                                                           */
int nspb_galerkin(const nspb_csr_in *A, const nspb_csr_in *P, nspb_csr_out *R,
                  nspb_csr_out *Ac, const nspb_opts *opts);

/* ---- seeded input generators (host memory) --------------------------------- */
/* Each fills rowptr[nrows+1] and returns nnz (>=0) or a negative status; col
 * and val are filled when non-NULL. Values depend only on (seed, row, slot),
 * never on the thread count.                                                 */
/* 3-D stencil on nx*ny*nz, npts = 7 (diag 6, off -1) or 27 (off uniform[-1,1],
 * diag = sum|off| + 1). fp32_values rounds every value to float first.       */
int64_t nspb_gen_stencil(int32_t nx, int32_t ny, int32_t nz, int32_t npts,
                         uint64_t seed, int32_t fp32_values, int32_t *rowptr,
                         int32_t *col, double *val);
/* Rows of the z-planes [z0, z1) of the same stencil (global column ids):
 * the row block one GPU owns when the grid is split into z-slabs.           */
int64_t nspb_gen_stencil_slab(int32_t nx, int32_t ny, int32_t nz, int32_t z0,
                              int32_t z1, int32_t npts, uint64_t seed,
                              int32_t fp32_values, int32_t *rowptr,
                              int32_t *col, double *val);
/* Power-law rows: degree ~ truncated Pareto(alpha) with its lower bound
 * solved so the mean degree is `mean_deg`, capped at max_deg; columns uniform
 * without duplicates, sorted; values uniform[-1,1].                         */
int64_t nspb_gen_powerlaw(int32_t nrows, int32_t ncols, double alpha,
                          double mean_deg, int32_t max_deg, uint64_t seed,
                          int32_t fp32_values, int32_t *rowptr, int32_t *col,
                          double *val);
/* Uniform random rows: degree uniform in [dmin,dmax] (clamped to ncols),
 * columns uniform without duplicates, sorted; values uniform[-1,1].          */
int64_t nspb_gen_random(int32_t nrows, int32_t ncols, int32_t dmin,
                        int32_t dmax, uint64_t seed, int32_t fp32_values,
                        int32_t *rowptr, int32_t *col, double *val);
/* Lower bound x_min of the truncated Pareto used by nspb_gen_powerlaw.       */
double nspb_powerlaw_xmin(double alpha, double mean_deg, int32_t max_deg);

/* ---- matrix files (host memory) ---------------------------------------------
 * The reference's own formats, so its data files drive this library:
 *  - binary COO (src/READ_MATRIX_MPI.cpp:146-356, read through
 *    load_MatrixMPI, src/distribute.cu:1071-1125): a header of int64
 *    {nr, nc, nt} (header_type 1) or {nr, nt} (header_type 0, nc = nr), then
 *    nt records {ii, jj, aa}: 1-based row and column as int64
 *    (index_bytes 8, what main.cu loads) or int32 (index_bytes 4), and an fp64
 *    value; records sorted by row;
 *  - the same as text (READ_ASCII_MATRIX_MPI, src/READ_MATRIX_MPI.cpp:365):
 *    '%' comment lines, a line "nr nc nt" or "nr nt", then "ii jj aa" lines.
 * As the reference does for one rank, local row 0 is the first row that holds
 * an entry and nrows = last row - first row + 1 (first_row gives the offset;
 * full_nrows is the header's nr), and a row whose columns are out of order is
 * stably sorted by column (src/distribute.cu:1051-1069). Duplicates are kept. */
typedef struct {
  int64_t nrows, ncols, nnz;
  int64_t full_nrows;  /* nr of the header                                  */
  int64_t first_row;   /* 0-based file row of local row 0                   */
  int32_t *rowptr;     /* [nrows+1]; library-allocated, see nspb_host_csr_free */
  int32_t *col;        /* [nnz], 0-based                                     */
  double *val;         /* [nnz]                                              */
} nspb_host_csr;

int nspb_read_coo_bin(const char *path, int header_type, int index_bytes,
                      nspb_host_csr *out);
int nspb_read_coo_ascii(const char *path, nspb_host_csr *out);
void nspb_host_csr_free(nspb_host_csr *m);
/* Binary COO writer of main.cu:468-512 (write_binary_matrix<mtype, otype>):
 * header {nr, nc} as int32 (index_bytes 4) or int64 (8), then nt as int64;
 * records {ii, jj} 1-based in the same width, then the fp64 value. With
 * index_bytes 4 the header is 16 bytes, which the binary reader above (like
 * the reference's) does not accept; index_bytes 8 round-trips.             */
int nspb_write_coo_bin(const char *path, const int32_t *rowptr, const int32_t *col,
                       const double *val, int64_t nrows, int64_t ncols, int index_bytes);
/* MatrixMarket coordinate writer of src/matrixIO.cu:299-339 (1-based).    */
int nspb_write_mtx(const char *path, const int32_t *rowptr, const int32_t *col,
                   const double *val, int64_t nrows, int64_t ncols);

#ifdef __cplusplus
}
#endif
#endif /* NSPB_H */
