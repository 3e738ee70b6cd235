/*
 * nspb_compat.h — drop-in C++ shims with the reference's own signatures.
 *
 * The types below keep the field order and sizes of the reference's structs
 * so that host code written against them links against libnspb.so unchanged:
 *   sfCSR                 <- nsp/inc/nsp.h:57-70
 *   CSRtype<> / CSR       <- src/CSR.h:67-106 (halo_info src/CSR.h:22-42);
 *                            pointers to reference-only types (vector<T>,
 *                            cusparseMatDescr_t, rows_to_get_info) are kept as
 *                            pointers of the same size
 *   stype/gstype/itype/vtype <- src/setting.h:21-28
 *   csrlocinfo            <- src/csrseg.h:3-9
 *
 * Entry points:
 *   void nsp_spgemm_kernel_hash(sfCSR*, sfCSR*, sfCSR*)  <- nsp/inc/nsp.h:105
 *       Same contract: reads a->M, b->N, a->nnz, b->nnz and the d_rpt/d_col/
 *       d_val device arrays; sets c->M, c->N, c->nnz and allocates c->d_rpt,
 *       c->d_col, c->d_val with cudaMalloc (caller frees with cudaFree);
 *       returns with the product complete (device synchronised). On a
 *       failure it prints the reason and exits, as checkCudaErrors does in
 *       the reference.
 *   CSR* nsparseMGPU_version0(CSR*, CSR*, csrlocinfo*, double&) <- src/spspmpi.cu:266
 *   CSR* nsparseMGPU_version1(handles*, CSR*, CSR*, double&)     <- src/spspmpi.h:31
 *       One GPU, no MPI: version1 is version0 (the reference's nprocs == 1
 *       path, src/spspmpi.cu:385). loc_time = wall seconds of the product
 *       bracketed by device synchronisation (src/spspmpi.cu:288-305). The
 *       returned CSR is malloc'ed with n = A->n, m = B->m, nnz,
 *       on_the_device = true, full_n = A->full_n, row_shift = A->row_shift
 *       and device arrays from cudaMalloc; its descr points to a NULL
 *       descriptor (this library does not link cuSPARSE).
 * The status-returning C variant of the kernel-level shim is
 * nspb_nsp_spgemm_kernel_hash (extern "C").
 */
#ifndef NSPB_COMPAT_H
#define NSPB_COMPAT_H

#include "nspb.h"

typedef double real;

typedef struct {
  int *rpt;
  int *col;
  real *val;
  int *d_rpt;
  int *d_col;
  real *d_val;
  unsigned int M;
  unsigned int N;
  int nnz;
  int nnz_max;
  char *matrix_name;
} sfCSR;

typedef struct {
  int fr;
  int lr;
  int *row;
  int *col;
  double *val;
} csrlocinfo;

#ifdef __cplusplus
extern "C" {
#endif
/* C form of nsp_spgemm_kernel_hash: same effect, returns an nspb_status. */
int nspb_nsp_spgemm_kernel_hash(sfCSR *a, sfCSR *b, sfCSR *c);
#ifdef __cplusplus
}

typedef unsigned long stype;
typedef unsigned long gstype;
typedef long gsstype;
typedef int itype;
typedef double vtype;

struct halo_info {
  void *to_receive;
  void *to_receive_d;
  int to_receive_n;
  int *to_receive_counts;
  int *to_receive_spls;
  vtype *what_to_receive;
  vtype *what_to_receive_d;
  void *to_send;
  void *to_send_d;
  int to_send_n;
  int *to_send_counts;
  int *to_send_spls;
  vtype *what_to_send;
  vtype *what_to_send_d;
  bool init;
};

struct rows_info;
struct handles;

template <typename Tst = stype, typename Tgs = gstype, typename Ti = itype>
struct CSRtype {
  Tst nnz;
  Tst n;
  Tgs m;
  Tst shrinked_m;
  gstype full_n;
  gstype full_m;
  bool on_the_device;
  bool is_symmetric;
  bool shrinked_flag;
  bool custom_alloced;
  gsstype col_shifted;
  gstype shrinked_firstrow;
  gstype shrinked_lastrow;
  vtype *val;
  Ti *col;
  Ti *row;
  Ti *shrinked_col;
  gstype row_shift;
  int *bitcol;
  int bitcolsize;
  int post_local;
  void **descr; /* cusparseMatDescr_t* in the reference */
  halo_info halo;
  rows_info *rows_to_get;
};

using CSR = CSRtype<>;

void nsp_spgemm_kernel_hash(sfCSR *a, sfCSR *b, sfCSR *c);
CSR *nsparseMGPU_version0(CSR *Alocal, CSR *Pfull, csrlocinfo *Plocal, double &loc_time);
CSR *nsparseMGPU_version1(handles *h, CSR *Alocal, CSR *Plocal, double &loc_time);
#endif /* __cplusplus */

#endif /* NSPB_COMPAT_H */
