/*
 * TEST INFRASTRUCTURE — the CPU oracle for the CSR product C = A·B.
 * Only tests, the smoke check and the benchmark's CPU-baseline / reference
 * arm may load this library. The product path never calls it.
 *
 * It restates the semantics of amavliut/nsp's hash SpGEMM
 * (nsp/src/nsp.cu:2448-2488, nsp_spgemm_kernel_hash) as a two-pass OpenMP
 * Gustavson product:
 *   - intermediate products per row: nsp_set_intprod_num, nsp/src/nsp.cu:306-320
 *   - structure: the union of B-row patterns over the A-row entries; keys are
 *     inserted whatever their value (hashmap_symbolic_bit, nsp/src/nsp.cu:23-39),
 *     so structural and cancellation zeros are kept
 *   - row_ptr: exclusive scan of the row counts (nsp/src/nsp.cu:1124)
 *   - values: sum over k of a_ik*b_kj in fp64, each product rounded before it
 *     is added (atomicAdd_block(value+hash, coef_B*cval_A),
 *     nsp/src/nsp.cu:1361-1366 with hashmap_bit :64-89); this oracle adds them
 *     in A-row order, then B-row order, starting from 0.0
 *   - columns ascending within each row (rank sort, nsp/src/nsp.cu:1618-1626)
 *   - duplicate entries in A or B are summed (hash merge)
 * Built with -ffp-contract=off so no product is fused into an add.
 *
 * Parity pins: the reference ships no tests or golden vectors. This oracle
 * is pinned by (1) exact structure counts of the stencil products computed
 * independently from 1-D Kronecker factors, (2) scipy's sparse product on
 * small cases, and (3) fixtures produced by the reference's own
 * nsp_spgemm_kernel_hash built for sm_100a (tests/golden).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORACLE_OK 0
#define ORACLE_ERR_INVALID (-1)
#define ORACLE_ERR_OVERFLOW (-2)
#define ORACLE_ERR_ALLOC (-3)

static void set_threads(int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
}

int oracle_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* Per-row intermediate products (nsp_set_intprod_num, nsp/src/nsp.cu:306-320),
 * returned as int64 per row; the total is the return value. */
int64_t oracle_intprod(int32_t n, const int32_t *arpt, const int32_t *acol,
                       const int32_t *brpt, int64_t *row_ip, int nthreads) {
  set_threads(nthreads);
  int64_t total = 0;
#pragma omp parallel for schedule(static) reduction(+ : total)
  for (int32_t i = 0; i < n; ++i) {
    int64_t s = 0;
    for (int32_t j = arpt[i]; j < arpt[i + 1]; ++j) {
      int32_t k = acol[j];
      s += brpt[k + 1] - brpt[k];
    }
    if (row_ip) row_ip[i] = s;
    total += s;
  }
  return total;
}

/* Symbolic pass: crpt[0..n] = exclusive scan of the distinct-column counts.
 * Returns nnz(C) or a negative error. Rows [r0, r1) only when r1 > r0 > -1
 * (crpt is then indexed from r0: crpt[0] = 0, crpt[r1-r0] = block nnz). */
static int64_t symbolic_rows(int32_t r0, int32_t r1, int32_t ncols,
                             const int32_t *arpt, const int32_t *acol,
                             const int32_t *brpt, const int32_t *bcol,
                             int32_t *crpt) {
  const int32_t nr = r1 - r0;
  int32_t *cnt = (int32_t *)malloc(sizeof(int32_t) * (size_t)(nr > 0 ? nr : 1));
  if (!cnt) return ORACLE_ERR_ALLOC;
  int failed = 0;
#pragma omp parallel
  {
    int32_t *mark = (int32_t *)malloc(sizeof(int32_t) * (size_t)(ncols > 0 ? ncols : 1));
    if (!mark) {
#pragma omp atomic write
      failed = 1;
    } else {
      for (int32_t c = 0; c < ncols; ++c) mark[c] = -1;
#pragma omp for schedule(dynamic, 256)
      for (int32_t i = r0; i < r1; ++i) {
        int32_t c = 0;
        for (int32_t j = arpt[i]; j < arpt[i + 1]; ++j) {
          int32_t k = acol[j];
          for (int32_t e = brpt[k]; e < brpt[k + 1]; ++e) {
            int32_t key = bcol[e];
            if (mark[key] != i) {
              mark[key] = i;
              ++c;
            }
          }
        }
        cnt[i - r0] = c;
      }
      free(mark);
    }
  }
  if (failed) {
    free(cnt);
    return ORACLE_ERR_ALLOC;
  }
  int64_t acc = 0;
  crpt[0] = 0;
  for (int32_t q = 0; q < nr; ++q) {
    acc += cnt[q];
    crpt[q + 1] = acc > INT32_MAX ? INT32_MAX : (int32_t)acc;
  }
  free(cnt);
  return acc > INT32_MAX ? ORACLE_ERR_OVERFLOW : acc;
}

int64_t oracle_symbolic(int32_t n, int32_t ncols, const int32_t *arpt,
                        const int32_t *acol, const int32_t *brpt,
                        const int32_t *bcol, int32_t *crpt, int nthreads) {
  if (n < 0 || ncols < 0 || !crpt) return ORACLE_ERR_INVALID;
  set_threads(nthreads);
  return symbolic_rows(0, n, ncols, arpt, acol, brpt, bcol, crpt);
}

int64_t oracle_symbolic_rows(int32_t r0, int32_t r1, int32_t ncols,
                             const int32_t *arpt, const int32_t *acol,
                             const int32_t *brpt, const int32_t *bcol,
                             int32_t *crpt, int nthreads) {
  if (r0 < 0 || r1 < r0 || ncols < 0 || !crpt) return ORACLE_ERR_INVALID;
  set_threads(nthreads);
  return symbolic_rows(r0, r1, ncols, arpt, acol, brpt, bcol, crpt);
}

static int cmp_i32(const void *a, const void *b) {
  int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
  return (x > y) - (x < y);
}

static void sort_i32(int32_t *v, int32_t len) {
  if (len <= 32) {
    for (int32_t p = 1; p < len; ++p) {
      int32_t x = v[p], q = p - 1;
      while (q >= 0 && v[q] > x) {
        v[q + 1] = v[q];
        --q;
      }
      v[q + 1] = x;
    }
  } else {
    qsort(v, (size_t)len, sizeof(int32_t), cmp_i32);
  }
}

/* Numeric pass for rows [r0, r1): crpt indexed from r0 (crpt[0] = 0).
 * ccol/cval receive the block's entries from position 0. */
static int numeric_rows(int32_t r0, int32_t r1, int32_t ncols,
                        const int32_t *arpt, const int32_t *acol,
                        const double *aval, const int32_t *brpt,
                        const int32_t *bcol, const double *bval,
                        const int32_t *crpt, int32_t *ccol, double *cval) {
  int failed = 0;
#pragma omp parallel
  {
    int32_t *mark = (int32_t *)malloc(sizeof(int32_t) * (size_t)(ncols > 0 ? ncols : 1));
    double *acc = (double *)malloc(sizeof(double) * (size_t)(ncols > 0 ? ncols : 1));
    if (!mark || !acc) {
#pragma omp atomic write
      failed = 1;
    } else {
      for (int32_t c = 0; c < ncols; ++c) mark[c] = -1;
#pragma omp for schedule(dynamic, 256)
      for (int32_t i = r0; i < r1; ++i) {
        int32_t *list = ccol + crpt[i - r0];
        int32_t len = 0;
        for (int32_t j = arpt[i]; j < arpt[i + 1]; ++j) {
          const int32_t k = acol[j];
          const double a = aval[j];
          for (int32_t e = brpt[k]; e < brpt[k + 1]; ++e) {
            const int32_t key = bcol[e];
            const double p = a * bval[e];
            if (mark[key] != i) {
              mark[key] = i;
              acc[key] = 0.0;
              list[len++] = key;
            }
            acc[key] = acc[key] + p;
          }
        }
        sort_i32(list, len);
        double *out = cval + crpt[i - r0];
        for (int32_t q = 0; q < len; ++q) out[q] = acc[list[q]];
      }
    }
    free(mark);
    free(acc);
  }
  return failed ? ORACLE_ERR_ALLOC : ORACLE_OK;
}

int oracle_numeric(int32_t n, int32_t ncols, const int32_t *arpt,
                   const int32_t *acol, const double *aval,
                   const int32_t *brpt, const int32_t *bcol,
                   const double *bval, const int32_t *crpt, int32_t *ccol,
                   double *cval, int nthreads) {
  if (n < 0 || ncols < 0 || !crpt || !ccol || !cval) return ORACLE_ERR_INVALID;
  set_threads(nthreads);
  return numeric_rows(0, n, ncols, arpt, acol, aval, brpt, bcol, bval, crpt,
                      ccol, cval);
}

int oracle_numeric_rows(int32_t r0, int32_t r1, int32_t ncols,
                        const int32_t *arpt, const int32_t *acol,
                        const double *aval, const int32_t *brpt,
                        const int32_t *bcol, const double *bval,
                        const int32_t *crpt, int32_t *ccol, double *cval,
                        int nthreads) {
  if (r0 < 0 || r1 < r0 || ncols < 0) return ORACLE_ERR_INVALID;
  set_threads(nthreads);
  return numeric_rows(r0, r1, ncols, arpt, acol, aval, brpt, bcol, bval, crpt,
                      ccol, cval);
}

/* Per-entry magnitude bound sum_k |a_ik * b_kj| in the same layout as C,
 * for the cancellation-safe tolerance |c - c*| <= tol * bound. */
int oracle_absbound(int32_t n, int32_t ncols, const int32_t *arpt,
                    const int32_t *acol, const double *aval,
                    const int32_t *brpt, const int32_t *bcol,
                    const double *bval, const int32_t *crpt,
                    const int32_t *ccol, double *bound, int nthreads) {
  if (n < 0 || ncols < 0) return ORACLE_ERR_INVALID;
  set_threads(nthreads);
  int failed = 0;
#pragma omp parallel
  {
    double *acc = (double *)calloc((size_t)(ncols > 0 ? ncols : 1), sizeof(double));
    if (!acc) {
#pragma omp atomic write
      failed = 1;
    } else {
#pragma omp for schedule(dynamic, 256)
      for (int32_t i = 0; i < n; ++i) {
        for (int32_t j = arpt[i]; j < arpt[i + 1]; ++j) {
          const int32_t k = acol[j];
          const double a = aval[j] < 0 ? -aval[j] : aval[j];
          for (int32_t e = brpt[k]; e < brpt[k + 1]; ++e) {
            const double b = bval[e] < 0 ? -bval[e] : bval[e];
            acc[bcol[e]] += a * b;
          }
        }
        for (int32_t q = crpt[i]; q < crpt[i + 1]; ++q) {
          bound[q] = acc[ccol[q]];
          acc[ccol[q]] = 0.0;
        }
      }
      free(acc);
    }
  }
  return failed ? ORACLE_ERR_ALLOC : ORACLE_OK;
}

/* getmct (src/getmct.cu:41-92): sorted unique column indices outside the
 * local row range [first, last]; with first > last every column counts.
 * Returns the count written to out (out must hold nnz entries). */
int64_t oracle_getmct(const int32_t *col, int64_t nnz, int32_t first,
                      int32_t last, int32_t *out) {
  int64_t w = 0;
  for (int64_t q = 0; q < nnz; ++q) {
    int32_t c = col[q];
    if (first > last || c < first || c > last) out[w++] = c;
  }
  if (w > 1) qsort(out, (size_t)w, sizeof(int32_t), cmp_i32);
  int64_t u = 0;
  for (int64_t q = 0; q < w; ++q)
    if (u == 0 || out[u - 1] != out[q]) out[u++] = out[q];
  return u;
}

/* compactcol (src/compactcol.cu:160-163 with cuCompactor.cuh:34-154): keep
 * the entries with c < lo || c > hi, in order. */
int64_t oracle_compactcol(const int32_t *in, int64_t n, int32_t lo, int32_t hi,
                          int32_t *out) {
  int64_t w = 0;
  for (int64_t q = 0; q < n; ++q)
    if (in[q] < lo || in[q] > hi) out[w++] = in[q];
  return w;
}

/* apply_mask_permut_GPU_noSideEffects (src/spspmpi.cu:58-84): position of
 * each column in the sorted list by binary search, -1 when absent. */
void oracle_shrink_col(const int32_t *col, int64_t nnz, const int32_t *cols,
                       int64_t ncols, int32_t *out) {
  for (int64_t q = 0; q < nnz; ++q) {
    int64_t lo = 0, hi = ncols;
    while (lo < hi) {
      int64_t mid = (lo + hi) >> 1;
      if (cols[mid] < col[q]) lo = mid + 1; else hi = mid;
    }
    out[q] = (lo < ncols && cols[lo] == col[q]) ? (int32_t)lo : -1;
  }
}
