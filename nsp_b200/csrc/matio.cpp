// Matrix files in the reference's formats (host code): binary and text COO
// readers with the one-rank semantics of load_MatrixMPI
// (src/distribute.cu:1071-1125 over src/READ_MATRIX_MPI.cpp:146-356 and :365),
// the binary writer of main.cu:468-512 and the MatrixMarket writer of
// src/matrixIO.cu:299-339.
#include <algorithm>
#include <cerrno>
#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <vector>

#include "../../include/nspb.h"

namespace {

struct File {
  FILE *f = nullptr;
  File(const char *path, const char *mode) : f(path ? std::fopen(path, mode) : nullptr) {}
  ~File() {
    if (f) std::fclose(f);
  }
};

// COO triplets (1-based file indices) -> the library's host CSR, following
// the reference: rows relative to the first stored row, columns minus one,
// out-of-order rows stably sorted by column.
int coo_to_csr(int64_t nr, int64_t nc, const std::vector<int64_t> &ii,
               const std::vector<int64_t> &jj, std::vector<double> &aa, nspb_host_csr *out) {
  const int64_t nt = (int64_t)ii.size();
  *out = nspb_host_csr{};
  out->full_nrows = nr;
  out->ncols = nc;
  if (nt > INT32_MAX || nc > INT32_MAX || nr < 0 || nc < 0) return NSPB_ERR_OVERFLOW;
  for (int64_t t = 1; t < nt; ++t)
    if (ii[t] < ii[t - 1]) return NSPB_ERR_INVALID;  // records must be sorted by row
  for (int64_t t = 0; t < nt; ++t)
    if (jj[t] < 1 || jj[t] > nc) return NSPB_ERR_INVALID;
  const int64_t first = nt ? ii[0] : 1;
  const int64_t n = nt ? ii[nt - 1] - first + 1 : 0;
  if (n > INT32_MAX) return NSPB_ERR_OVERFLOW;
  out->nrows = n;
  out->nnz = nt;
  out->first_row = first - 1;
  out->rowptr = static_cast<int32_t *>(std::malloc((size_t)(n + 1) * sizeof(int32_t)));
  out->col = static_cast<int32_t *>(std::malloc((size_t)std::max<int64_t>(nt, 1) * sizeof(int32_t)));
  out->val = static_cast<double *>(std::malloc((size_t)std::max<int64_t>(nt, 1) * sizeof(double)));
  if (!out->rowptr || !out->col || !out->val) {
    nspb_host_csr_free(out);
    return NSPB_ERR_ALLOC;
  }
  std::fill(out->rowptr, out->rowptr + n + 1, 0);
  for (int64_t t = 0; t < nt; ++t) ++out->rowptr[ii[t] - first + 1];
  for (int64_t r = 0; r < n; ++r) out->rowptr[r + 1] += out->rowptr[r];
  std::vector<int64_t> order;
  for (int64_t r = 0; r < n; ++r) {
    const int64_t s = out->rowptr[r], e = out->rowptr[r + 1];
    bool sorted = true;
    for (int64_t t = s + 1; t < e && sorted; ++t) sorted = jj[t] >= jj[t - 1];
    if (sorted) {
      for (int64_t t = s; t < e; ++t) {
        out->col[t] = (int32_t)(jj[t] - 1);
        out->val[t] = aa[t];
      }
      continue;
    }
    order.resize(e - s);
    std::iota(order.begin(), order.end(), s);
    std::stable_sort(order.begin(), order.end(),
                     [&](int64_t x, int64_t y) { return jj[x] < jj[y]; });
    for (int64_t t = s; t < e; ++t) {
      out->col[t] = (int32_t)(jj[order[t - s]] - 1);
      out->val[t] = aa[order[t - s]];
    }
  }
  return NSPB_OK;
}

}  // namespace

extern "C" {

int nspb_read_coo_bin(const char *path, int header_type, int index_bytes, nspb_host_csr *out) {
  if (!out || (index_bytes != 4 && index_bytes != 8)) return NSPB_ERR_INVALID;
  *out = nspb_host_csr{};
  File fh(path, "rb");
  if (!fh.f) return NSPB_ERR_IO;
  int64_t hdr[3] = {0, 0, 0};
  const size_t nh = header_type ? 3 : 2;
  if (std::fread(hdr, sizeof(int64_t), nh, fh.f) != nh) return NSPB_ERR_IO;
  const int64_t nr = hdr[0];
  const int64_t nc = header_type ? hdr[1] : hdr[0];
  const int64_t nt = header_type ? hdr[2] : hdr[1];
  if (nr < 0 || nc < 0 || nt < 0) return NSPB_ERR_INVALID;
  if (nt > INT32_MAX) return NSPB_ERR_OVERFLOW;
  // records {ii, jj, aa} with the C struct layout of the writer: no padding
  // for either index width (4+4+8 and 8+8+8 bytes)
  const size_t rec = (size_t)index_bytes * 2 + sizeof(double);
  std::vector<unsigned char> buf((size_t)nt * rec);
  if (nt && std::fread(buf.data(), rec, (size_t)nt, fh.f) != (size_t)nt) return NSPB_ERR_IO;
  std::vector<int64_t> ii((size_t)nt), jj((size_t)nt);
  std::vector<double> aa((size_t)nt);
  for (int64_t t = 0; t < nt; ++t) {
    const unsigned char *p = buf.data() + (size_t)t * rec;
    if (index_bytes == 8) {
      std::memcpy(&ii[t], p, 8);
      std::memcpy(&jj[t], p + 8, 8);
    } else {
      int32_t a, b;
      std::memcpy(&a, p, 4);
      std::memcpy(&b, p + 4, 4);
      ii[t] = a;
      jj[t] = b;
    }
    std::memcpy(&aa[t], p + 2 * index_bytes, 8);
  }
  return coo_to_csr(nr, nc, ii, jj, aa, out);
}

int nspb_read_coo_ascii(const char *path, nspb_host_csr *out) {
  if (!out) return NSPB_ERR_INVALID;
  *out = nspb_host_csr{};
  File fh(path, "r");
  if (!fh.f) return NSPB_ERR_IO;
  std::vector<char> line(1 << 16);
  // header: the first line that does not start with '%'
  int64_t nr = 0, nc = 0, nt = 0;
  for (;;) {
    if (!std::fgets(line.data(), (int)line.size(), fh.f)) return NSPB_ERR_IO;
    if (line[0] != '%') break;
  }
  const int got = std::sscanf(line.data(), "%" SCNd64 " %" SCNd64 " %" SCNd64, &nr, &nc, &nt);
  if (got == 2) {
    nt = nc;
    nc = nr;
  } else if (got != 3) {
    return NSPB_ERR_INVALID;
  }
  if (nr < 0 || nc < 0 || nt < 0) return NSPB_ERR_INVALID;
  if (nt > INT32_MAX) return NSPB_ERR_OVERFLOW;
  std::vector<int64_t> ii((size_t)nt), jj((size_t)nt);
  std::vector<double> aa((size_t)nt);
  for (int64_t t = 0; t < nt; ++t) {
    if (std::fscanf(fh.f, "%" SCNd64 " %" SCNd64 " %lf", &ii[t], &jj[t], &aa[t]) != 3)
      return NSPB_ERR_IO;
  }
  return coo_to_csr(nr, nc, ii, jj, aa, out);
}

void nspb_host_csr_free(nspb_host_csr *m) {
  if (!m) return;
  std::free(m->rowptr);
  std::free(m->col);
  std::free(m->val);
  m->rowptr = nullptr;
  m->col = nullptr;
  m->val = nullptr;
}

int nspb_write_coo_bin(const char *path, const int32_t *rowptr, const int32_t *col,
                       const double *val, int64_t nrows, int64_t ncols, int index_bytes) {
  if (nrows < 0 || ncols < 0 || !rowptr || (index_bytes != 4 && index_bytes != 8))
    return NSPB_ERR_INVALID;
  const int64_t nt = rowptr[nrows] - rowptr[0];
  if (nt < 0 || (nt > 0 && (!col || !val))) return NSPB_ERR_INVALID;
  File fh(path, "wb");
  if (!fh.f) return NSPB_ERR_IO;
  // header {nr, nc} in the index width, then nt as int64 (struct hdr of the
  // writer: 4+4+8 or 8+8+8 bytes, no padding)
  unsigned char hdr[24];
  size_t hn;
  if (index_bytes == 4) {
    const int32_t a = (int32_t)nrows, b = (int32_t)ncols;
    std::memcpy(hdr, &a, 4);
    std::memcpy(hdr + 4, &b, 4);
    std::memcpy(hdr + 8, &nt, 8);
    hn = 16;
  } else {
    std::memcpy(hdr, &nrows, 8);
    std::memcpy(hdr + 8, &ncols, 8);
    std::memcpy(hdr + 16, &nt, 8);
    hn = 24;
  }
  if (std::fwrite(hdr, 1, hn, fh.f) != hn) return NSPB_ERR_IO;
  const size_t rec = (size_t)index_bytes * 2 + sizeof(double);
  std::vector<unsigned char> buf;
  const int64_t chunk = 1 << 16;
  for (int64_t r0 = 0; r0 < nrows; r0 += chunk) {
    const int64_t r1 = std::min(nrows, r0 + chunk);
    buf.resize((size_t)(rowptr[r1] - rowptr[r0]) * rec);
    unsigned char *p = buf.data();
    for (int64_t r = r0; r < r1; ++r) {
      for (int64_t t = rowptr[r]; t < rowptr[r + 1]; ++t, p += rec) {
        if (index_bytes == 4) {
          const int32_t a = (int32_t)(r + 1), b = col[t] + 1;
          std::memcpy(p, &a, 4);
          std::memcpy(p + 4, &b, 4);
        } else {
          const int64_t a = r + 1, b = (int64_t)col[t] + 1;
          std::memcpy(p, &a, 8);
          std::memcpy(p + 8, &b, 8);
        }
        std::memcpy(p + 2 * index_bytes, &val[t], 8);
      }
    }
    if (!buf.empty() && std::fwrite(buf.data(), 1, buf.size(), fh.f) != buf.size())
      return NSPB_ERR_IO;
  }
  return std::fflush(fh.f) == 0 ? NSPB_OK : NSPB_ERR_IO;
}

int nspb_write_mtx(const char *path, const int32_t *rowptr, const int32_t *col,
                   const double *val, int64_t nrows, int64_t ncols) {
  if (nrows < 0 || ncols < 0 || !rowptr) return NSPB_ERR_INVALID;
  const int64_t nt = rowptr[nrows] - rowptr[0];
  if (nt < 0 || (nt > 0 && (!col || !val))) return NSPB_ERR_INVALID;
  File fh(path, "w");
  if (!fh.f) return NSPB_ERR_IO;
  // the reference's layout, spacing included
  if (std::fprintf(fh.f, "%s\n", "%%MatrixMarket matrix coordinate real general") < 0)
    return NSPB_ERR_IO;
  if (std::fprintf(fh.f, "%" PRId64 "  %" PRId64 " %" PRId64 " \n", nrows, ncols, nt) < 0)
    return NSPB_ERR_IO;
  for (int64_t r = 0; r < nrows; ++r)
    for (int64_t t = rowptr[r]; t < rowptr[r + 1]; ++t)
      if (std::fprintf(fh.f, "%" PRId64 "   %d  %lg\n", r + 1, col[t] + 1, val[t]) < 0)
        return NSPB_ERR_IO;
  return std::fflush(fh.f) == 0 ? NSPB_OK : NSPB_ERR_IO;
}

}  // extern "C"
