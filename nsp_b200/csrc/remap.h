// Device-side column remap helpers shared by the C ABI and the row-blocked
// product (stream-ordered; each returns an nspb_status).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace nspb {
int compactcol_dev(const int *d_in, int64_t n, int lo, int hi, int *d_out, int64_t *nout,
                   cudaStream_t s);
int getmct_dev(const int *d_col, int64_t nnz, int first, int last, int *d_out, int64_t *nout,
               cudaStream_t s);
int shrink_col_dev(const int *d_col, int64_t nnz, const int *d_cols, int64_t ncols, int *d_out,
                   cudaStream_t s);
}  // namespace nspb
