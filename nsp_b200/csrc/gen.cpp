// Seeded CSR input generators (host). Every value depends only on
// (seed, stream, row, slot) through a counter-based mixer, so the output is
// identical for any OpenMP thread count and on any machine with the same libm.
//
// The reference reads its matrices from binary COO files
// (src/READ_MATRIX_MPI.cpp:146-356); there is no generator there. These
// produce the workloads named by the benchmark configurations: 3-D 7-point
// and 27-point stencils, power-law rows and uniform random rows. Rows are
// emitted column-sorted, which is the precondition the reference's loader
// establishes with check_and_fix_order (src/distribute.cu:1050-1069).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/nspb.h"

namespace {

inline uint64_t mix64(uint64_t z) {
  z += 0x9e3779b97f4a7c15ULL;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

// One 64-bit draw keyed by (seed, stream, row, slot).
inline uint64_t draw(uint64_t seed, uint64_t stream, uint64_t row, uint64_t slot) {
  return mix64(mix64(mix64(seed ^ (stream * 0x632be59bd9b4e019ULL)) + row) + slot);
}

inline double unit01(uint64_t r) { return (double)(r >> 11) * 0x1.0p-53; }
inline double unit_pm1(uint64_t r) { return 2.0 * unit01(r) - 1.0; }
// Uniform integer in [0, m) by the high half of a 64x64 product.
inline uint64_t below(uint64_t r, uint64_t m) {
  return (uint64_t)(((unsigned __int128)r * m) >> 64);
}
inline double maybe_f32(double v, int fp32) { return fp32 ? (double)(float)v : v; }

// Stream ids keep the draws of different generators independent.
enum : uint64_t {
  S_STENCIL = 27,
  S_PL_DEG = 101,
  S_PL_COL = 102,
  S_PL_VAL = 103,
  S_RND_DEG = 201,
  S_RND_COL = 202,
  S_RND_VAL = 203
};

// Floyd's sampling of d distinct columns from [0, n), sorted into out.
void floyd_sorted(uint64_t seed, uint64_t stream, uint64_t row, int32_t d,
                  int32_t n, std::vector<uint64_t> &bits, int32_t *out) {
  int32_t w = 0;
  for (int64_t j = (int64_t)n - d; j < n; ++j) {
    uint64_t t = below(draw(seed, stream, row, (uint64_t)w), (uint64_t)j + 1);
    uint64_t pick = (bits[t >> 6] >> (t & 63)) & 1ULL ? (uint64_t)j : t;
    bits[pick >> 6] |= 1ULL << (pick & 63);
    out[w++] = (int32_t)pick;
  }
  std::sort(out, out + d);
  for (int32_t q = 0; q < d; ++q) bits[(uint32_t)out[q] >> 6] = 0;
}

}  // namespace

extern "C" int64_t nspb_gen_stencil(int32_t nx, int32_t ny, int32_t nz,
                                    int32_t npts, uint64_t seed,
                                    int32_t fp32_values, int32_t *rowptr,
                                    int32_t *col, double *val) {
  return nspb_gen_stencil_slab(nx, ny, nz, 0, nz, npts, seed, fp32_values, rowptr, col, val);
}

extern "C" int64_t nspb_gen_stencil_slab(int32_t nx, int32_t ny, int32_t nz,
                                         int32_t z0, int32_t z1, int32_t npts,
                                         uint64_t seed, int32_t fp32_values,
                                         int32_t *rowptr, int32_t *col, double *val) {
  if (nx < 0 || ny < 0 || nz < 0 || (npts != 7 && npts != 27) || !rowptr)
    return NSPB_ERR_INVALID;
  if (z0 < 0 || z1 < z0 || z1 > nz) return NSPB_ERR_INVALID;
  if ((int64_t)nx * ny * nz > INT32_MAX - 1) return NSPB_ERR_OVERFLOW;
  const int64_t first = (int64_t)nx * ny * z0;  // global id of the slab's first row
  const int64_t n = (int64_t)nx * ny * (z1 - z0);
  auto count = [&](int64_t i) -> int32_t {
    int32_t x = (int32_t)(i % nx), y = (int32_t)((i / nx) % ny), z = (int32_t)(i / ((int64_t)nx * ny));
    int32_t cx = 1 + (x > 0) + (x < nx - 1);
    int32_t cy = 1 + (y > 0) + (y < ny - 1);
    int32_t cz = 1 + (z > 0) + (z < nz - 1);
    return npts == 27 ? cx * cy * cz : 1 + (cx - 1) + (cy - 1) + (cz - 1);
  };
  std::vector<int32_t> cnt((size_t)n);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) cnt[(size_t)i] = count(first + i);
  int64_t acc = 0;
  rowptr[0] = 0;
  for (int64_t i = 0; i < n; ++i) {
    acc += cnt[(size_t)i];
    if (acc > INT32_MAX) return NSPB_ERR_OVERFLOW;
    rowptr[i + 1] = (int32_t)acc;
  }
  if (!col && !val) return acc;
  const int64_t sxy = (int64_t)nx * ny;
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < n; ++r) {
    const int64_t i = first + r;  // global row id
    int32_t x = (int32_t)(i % nx), y = (int32_t)((i / nx) % ny), z = (int32_t)(i / sxy);
    int64_t w = rowptr[r];
    int64_t diag_pos = -1;
    double asum = 0.0;
    for (int dz = -1; dz <= 1; ++dz) {
      if (z + dz < 0 || z + dz >= nz) continue;
      for (int dy = -1; dy <= 1; ++dy) {
        if (y + dy < 0 || y + dy >= ny) continue;
        for (int dx = -1; dx <= 1; ++dx) {
          if (x + dx < 0 || x + dx >= nx) continue;
          int nonzero_axes = (dx != 0) + (dy != 0) + (dz != 0);
          if (npts == 7 && nonzero_axes > 1) continue;
          int64_t j = i + dx + (int64_t)nx * dy + sxy * dz;
          if (col) col[w] = (int32_t)j;
          if (j == i) {
            diag_pos = w;
          } else if (val) {
            double v;
            if (npts == 7) {
              v = -1.0;
            } else {
              // symmetric: the pair {i,j} shares one draw
              int64_t lo = std::min(i, j), hi = std::max(i, j);
              v = maybe_f32(unit_pm1(draw(seed, S_STENCIL, (uint64_t)lo, (uint64_t)hi)), fp32_values);
            }
            val[w] = v;
            asum += std::fabs(v);
          }
          ++w;
        }
      }
    }
    if (val && diag_pos >= 0)
      val[diag_pos] = npts == 7 ? 6.0 : maybe_f32(asum + 1.0, fp32_values);
  }
  return acc;
}

// Mean of floor(X) for X ~ Pareto(alpha, xmin) truncated at xmax, with
// floor(X) >= 1: E = sum_{k=1..xmax} P(X >= k).
static double powerlaw_mean(double alpha, double xmin, double xmax) {
  const double a = alpha - 1.0;
  const double r = std::pow(xmin / xmax, a);
  double m = 0.0;
  for (int64_t k = 1; k <= (int64_t)xmax; ++k) {
    if ((double)k <= xmin) {
      m += 1.0;
    } else {
      m += (std::pow(xmin / (double)k, a) - r) / (1.0 - r);
    }
  }
  return m;
}

extern "C" double nspb_powerlaw_xmin(double alpha, double mean_deg, int32_t max_deg) {
  double lo = 1.0, hi = std::max(1.0, mean_deg);
  for (int it = 0; it < 100; ++it) {
    double mid = 0.5 * (lo + hi);
    if (powerlaw_mean(alpha, mid, (double)max_deg) < mean_deg) lo = mid; else hi = mid;
  }
  // fixed precision so every host derives the same degrees
  return std::round(0.5 * (lo + hi) * 1e9) / 1e9;
}

extern "C" int64_t nspb_gen_powerlaw(int32_t nrows, int32_t ncols, double alpha,
                                     double mean_deg, int32_t max_deg,
                                     uint64_t seed, int32_t fp32_values,
                                     int32_t *rowptr, int32_t *col, double *val) {
  if (nrows < 0 || ncols < 0 || !(alpha > 1.0) || max_deg < 1 || !rowptr)
    return NSPB_ERR_INVALID;
  const double xmin = nspb_powerlaw_xmin(alpha, mean_deg, max_deg);
  const double a = alpha - 1.0;
  const double r = std::pow(xmin / (double)max_deg, a);
  std::vector<int32_t> deg((size_t)nrows);
#pragma omp parallel for schedule(static)
  for (int32_t i = 0; i < nrows; ++i) {
    double u = unit01(draw(seed, S_PL_DEG, (uint64_t)i, 0));
    double x = xmin * std::pow(1.0 - u * (1.0 - r), -1.0 / a);
    int64_t d = (int64_t)std::floor(x);
    d = std::max<int64_t>(1, std::min<int64_t>(d, max_deg));
    d = std::min<int64_t>(d, ncols);
    deg[(size_t)i] = (int32_t)d;
  }
  int64_t acc = 0;
  rowptr[0] = 0;
  for (int32_t i = 0; i < nrows; ++i) {
    acc += deg[(size_t)i];
    if (acc > INT32_MAX) return NSPB_ERR_OVERFLOW;
    rowptr[i + 1] = (int32_t)acc;
  }
  if (!col && !val) return acc;
#pragma omp parallel
  {
    std::vector<uint64_t> bits(((size_t)ncols + 63) / 64 + 1, 0);
    std::vector<int32_t> tmp;
#pragma omp for schedule(dynamic, 256)
    for (int32_t i = 0; i < nrows; ++i) {
      int32_t d = deg[(size_t)i];
      int64_t w = rowptr[i];
      tmp.resize((size_t)d);
      floyd_sorted(seed, S_PL_COL, (uint64_t)i, d, ncols, bits, tmp.data());
      for (int32_t q = 0; q < d; ++q) {
        if (col) col[w + q] = tmp[(size_t)q];
        if (val) val[w + q] = maybe_f32(unit_pm1(draw(seed, S_PL_VAL, (uint64_t)i, (uint64_t)q)), fp32_values);
      }
    }
  }
  return acc;
}

extern "C" int64_t nspb_gen_random(int32_t nrows, int32_t ncols, int32_t dmin,
                                   int32_t dmax, uint64_t seed,
                                   int32_t fp32_values, int32_t *rowptr,
                                   int32_t *col, double *val) {
  if (nrows < 0 || ncols < 0 || dmin < 0 || dmax < dmin || !rowptr)
    return NSPB_ERR_INVALID;
  std::vector<int32_t> deg((size_t)nrows);
#pragma omp parallel for schedule(static)
  for (int32_t i = 0; i < nrows; ++i) {
    int64_t d = dmin + (int64_t)below(draw(seed, S_RND_DEG, (uint64_t)i, 0), (uint64_t)(dmax - dmin + 1));
    deg[(size_t)i] = (int32_t)std::min<int64_t>(d, ncols);
  }
  int64_t acc = 0;
  rowptr[0] = 0;
  for (int32_t i = 0; i < nrows; ++i) {
    acc += deg[(size_t)i];
    if (acc > INT32_MAX) return NSPB_ERR_OVERFLOW;
    rowptr[i + 1] = (int32_t)acc;
  }
  if (!col && !val) return acc;
#pragma omp parallel
  {
    std::vector<uint64_t> bits(((size_t)ncols + 63) / 64 + 1, 0);
    std::vector<int32_t> tmp;
#pragma omp for schedule(dynamic, 256)
    for (int32_t i = 0; i < nrows; ++i) {
      int32_t d = deg[(size_t)i];
      int64_t w = rowptr[i];
      tmp.resize((size_t)d);
      floyd_sorted(seed, S_RND_COL, (uint64_t)i, d, ncols, bits, tmp.data());
      for (int32_t q = 0; q < d; ++q) {
        if (col) col[w + q] = tmp[(size_t)q];
        if (val) val[w + q] = maybe_f32(unit_pm1(draw(seed, S_RND_VAL, (uint64_t)i, (uint64_t)q)), fp32_values);
      }
    }
  }
  return acc;
}
