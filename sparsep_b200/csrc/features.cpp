// features.cpp -- the cheap sparsity features the learned variant selector
// reads: one O(nnz) pass over a CSR structure plus its right-hand-side count.
// No counterpart in the reference (its variants are chosen at compile time).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "sparsep.h"

namespace {

// Distinct b x b blocks touched by the nonzeros (one stamp array over the
// block columns, reset per block row by generation number).
uint64_t count_blocks(uint32_t nrows, uint32_t ncols, const uint32_t *rowptr, const uint32_t *colind, uint32_t b) {
  const uint32_t nbc = (ncols + b - 1) / b;
  std::vector<uint32_t> stamp(nbc + 1, 0);
  uint64_t blocks = 0;
  uint32_t gen = 0;
  for (uint32_t r0 = 0; r0 < nrows; r0 += b) {
    ++gen;
    const uint32_t r1 = std::min(nrows, r0 + b);
    for (uint32_t q = rowptr[r0]; q < rowptr[r1]; ++q) {
      const uint32_t bc = colind[q] / b;
      if (stamp[bc] != gen) {
        stamp[bc] = gen;
        ++blocks;
      }
    }
  }
  return blocks;
}

}  // namespace

extern "C" int sparsep_features(uint32_t nrows, uint32_t ncols, const uint32_t *rowptr, const uint32_t *colind,
                                uint32_t k, float *out) {
  if (!rowptr || !out || k == 0 || (rowptr[nrows] && !colind)) return SPARSEP_EINVAL;
  const uint64_t nnz = rowptr[nrows];
  double f[SPARSEP_NFEATURES] = {};
  const double n = std::max<uint32_t>(nrows, 1);
  const double mean = nnz / n;
  double var = 0, maxlen = 0, long_nnz = 0, short_rows = 0;
  double band = 0, near = 0, gaps = 0, gap_n = 0;
  for (uint32_t r = 0; r < nrows; ++r) {
    const uint32_t a = rowptr[r], e = rowptr[r + 1];
    const double len = e - a;
    var += (len - mean) * (len - mean);
    maxlen = std::max(maxlen, len);
    if (len > 4096) long_nnz += len;
    if (len < 4) short_rows += 1;
    for (uint32_t q = a; q < e; ++q) {
      const double d = std::fabs((double)colind[q] - (double)r);
      band += d;
      near += d <= 64;
      if (q > a) {
        gaps += std::fabs((double)colind[q] - (double)colind[q - 1]);
        gap_n += 1;
      }
    }
  }
  const double nz = std::max<uint64_t>(nnz, 1);
  const double nc = std::max<uint32_t>(ncols, 1);
  f[0] = std::log2(n + 1);
  f[1] = std::log2((double)nnz + 1);
  f[2] = std::log2((double)k);
  f[3] = k % 4 == 0;
  f[4] = k % 2 == 0;
  f[5] = std::log2(mean + 1);
  f[6] = mean > 0 ? std::sqrt(var / n) / mean : 0;  // row-length coefficient of variation
  f[7] = std::log2(maxlen + 1);
  f[8] = long_nnz / nz;                               // share of nonzeros in rows > 4096
  f[9] = short_rows / n;                              // rows with < 4 nonzeros
  f[10] = band / nz / nc;                             // mean |col - row| / ncols
  f[11] = near / nz;                                  // nonzeros within 64 of the diagonal
  f[12] = nnz ? nz / (16.0 * count_blocks(nrows, ncols, rowptr, colind, 4)) : 0;  // 4x4 block fill
  f[13] = nnz ? nz / (64.0 * count_blocks(nrows, ncols, rowptr, colind, 8)) : 0;  // 8x8 block fill
  f[14] = std::log2(nc * k * 4.0);                    // bytes of x
  f[15] = std::log2((gap_n ? gaps / gap_n : 0) + 1);  // mean column step inside a row
  for (int i = 0; i < SPARSEP_NFEATURES; ++i) out[i] = (float)f[i];
  return SPARSEP_OK;
}
