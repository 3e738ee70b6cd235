// TEST INFRASTRUCTURE — a C entry to the reference's own product
// nsp_spgemm_kernel_hash (nsp/inc/nsp.h:105, nsp/src/nsp.cu:2448-2488),
// compiled together with the reference sources (oracle/Makefile, target
// `ref`) into oracle/_ref/libnsp_ref.so. Used only by tests and the golden
// fixture script to pin the CPU oracle against the reference on a B200.
#include <cuda_runtime.h>

#include <cstdlib>
#include <cstring>

#include "nsp.h"

namespace {

template <typename T>
T *dev_copy(const T *h, size_t n) {
  T *d = nullptr;
  if (cudaMalloc(&d, (n ? n : 1) * sizeof(T)) != cudaSuccess) return nullptr;
  if (n) cudaMemcpy(d, h, n * sizeof(T), cudaMemcpyHostToDevice);
  return d;
}

}  // namespace

// C = A·B with host inputs; outputs are malloc'ed host arrays (ref_free).
// Returns 0, or a cudaError_t value.
extern "C" int ref_nsp_spgemm_host(int M, int K, int N, const int *a_rpt, const int *a_col,
                                   const double *a_val, const int *b_rpt, const int *b_col,
                                   const double *b_val, int *nnz_out, int **c_rpt, int **c_col,
                                   double **c_val) {
  const int annz = a_rpt[M], bnnz = b_rpt[K];
  sfCSR a, b, c;
  std::memset(&a, 0, sizeof(a));
  std::memset(&b, 0, sizeof(b));
  std::memset(&c, 0, sizeof(c));
  a.M = (unsigned)M;
  a.N = (unsigned)K;
  a.nnz = annz;
  b.M = (unsigned)K;
  b.N = (unsigned)N;
  b.nnz = bnnz;
  a.d_rpt = dev_copy(a_rpt, (size_t)M + 1);
  a.d_col = dev_copy(a_col, (size_t)annz);
  a.d_val = dev_copy(a_val, (size_t)annz);
  b.d_rpt = dev_copy(b_rpt, (size_t)K + 1);
  b.d_col = dev_copy(b_col, (size_t)bnnz);
  b.d_val = dev_copy(b_val, (size_t)bnnz);
  if (!a.d_rpt || !a.d_col || !a.d_val || !b.d_rpt || !b.d_col || !b.d_val) return (int)cudaErrorMemoryAllocation;
  nsp_spgemm_kernel_hash(&a, &b, &c);
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) {
    *nnz_out = c.nnz;
    *c_rpt = (int *)std::malloc(sizeof(int) * ((size_t)M + 1));
    *c_col = (int *)std::malloc(sizeof(int) * (size_t)(c.nnz ? c.nnz : 1));
    *c_val = (double *)std::malloc(sizeof(double) * (size_t)(c.nnz ? c.nnz : 1));
    cudaMemcpy(*c_rpt, c.d_rpt, sizeof(int) * ((size_t)M + 1), cudaMemcpyDeviceToHost);
    if (c.nnz) {
      cudaMemcpy(*c_col, c.d_col, sizeof(int) * (size_t)c.nnz, cudaMemcpyDeviceToHost);
      cudaMemcpy(*c_val, c.d_val, sizeof(double) * (size_t)c.nnz, cudaMemcpyDeviceToHost);
    }
    e = cudaGetLastError();
  }
  cudaFree(a.d_rpt);
  cudaFree(a.d_col);
  cudaFree(a.d_val);
  cudaFree(b.d_rpt);
  cudaFree(b.d_col);
  cudaFree(b.d_val);
  cudaFree(c.d_rpt);
  cudaFree(c.d_col);
  cudaFree(c.d_val);
  return (int)e;
}

extern "C" void ref_free(void *p) { std::free(p); }

// Milliseconds per call of nsp_spgemm_kernel_hash on device inputs (C is
// allocated inside each call, as in the reference, and freed after it),
// mean over `reps` calls after `warm` untimed calls, CUDA events on the
// default stream; times_out (may be NULL) receives every timed call's ms.
// *nnz_out receives nnz(C).
extern "C" float ref_nsp_time_device(int M, int K, int N, int *a_rpt, int *a_col, double *a_val,
                                     int annz, int *b_rpt, int *b_col, double *b_val, int bnnz,
                                     int warm, int reps, int *nnz_out, float *times_out) {
  sfCSR a, b;
  std::memset(&a, 0, sizeof(a));
  std::memset(&b, 0, sizeof(b));
  a.M = (unsigned)M;
  a.N = (unsigned)K;
  a.nnz = annz;
  a.d_rpt = a_rpt;
  a.d_col = a_col;
  a.d_val = a_val;
  b.M = (unsigned)K;
  b.N = (unsigned)N;
  b.nnz = bnnz;
  b.d_rpt = b_rpt;
  b.d_col = b_col;
  b.d_val = b_val;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float total = 0.f;
  for (int r = 0; r < warm + reps; ++r) {
    sfCSR c;
    std::memset(&c, 0, sizeof(c));
    cudaDeviceSynchronize();
    cudaEventRecord(e0, 0);
    nsp_spgemm_kernel_hash(&a, &b, &c);
    cudaEventRecord(e1, 0);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (r >= warm) {
      total += ms;
      if (times_out) times_out[r - warm] = ms;
    }
    *nnz_out = c.nnz;
    cudaFree(c.d_rpt);
    cudaFree(c.d_col);
    cudaFree(c.d_val);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return reps > 0 ? total / (float)reps : 0.f;
}
