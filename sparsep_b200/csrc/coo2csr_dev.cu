// coo2csr_dev.cu -- COO -> CSR on the device, with the arrays the host
// converter coo2csr (formats.cpp; the reference's counting sort,
// spmv/1D/CSR-row/support/matrix.h:113-152) produces: rows in order, and
// inside a row the input order kept (a stable sort by row).
//
// Stable LSD radix sort (radix.cuh) of (row, input index) pairs, 4 bits per
// pass, only as many passes as the row count needs (20 bits -> 5 passes for
// 1M rows).  Then rowptr[r] = first sorted position with row >= r (a binary search per
// row), and columns / values are gathered through the sorted input indices.
#include <algorithm>
#include <cstdio>
#include <new>

#include "fault.hpp"
#include "internal.hpp"
#include "radix.cuh"
#include "sparsep.h"

namespace sparsep {
namespace c2c {

// rowptr[r] = number of sorted rows < r (lower bound), r = 0 .. nrows
__global__ void rowptr_kernel(const uint32_t *__restrict__ key, uint32_t n, uint32_t nrows,
                              uint32_t *__restrict__ rowptr) {
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r > nrows) return;
  uint32_t lo = 0, hi = n;
  while (lo < hi) {
    const uint32_t mid = lo + ((hi - lo) >> 1);
    if (key[mid] < r) lo = mid + 1;
    else hi = mid;
  }
  rowptr[r] = lo;
}

template <int ES>
__global__ void gather(const uint32_t *__restrict__ idx, uint32_t n, const uint32_t *__restrict__ cols,
                       const unsigned char *__restrict__ vals, uint32_t *__restrict__ cols_out,
                       unsigned char *__restrict__ vals_out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t s = idx[i];
    cols_out[i] = cols[s];
    for (int b = 0; b < ES; ++b) vals_out[(size_t)i * ES + b] = vals[(size_t)s * ES + b];
  }
}

}  // namespace c2c
}  // namespace sparsep

using namespace sparsep::c2c;

static int c2c_err(cudaError_t e) {
  if (e == cudaSuccess) return SPARSEP_OK;
  char msg[160];
  std::snprintf(msg, sizeof msg, "%s (%d)", cudaGetErrorString(e), (int)e);
  sparsep::record_error(msg);
  return e == cudaErrorMemoryAllocation ? SPARSEP_ENOMEM : SPARSEP_EIO;
}

// Device COO (rows, cols, vals of es bytes each) -> device CSR.
static int coo2csr_device(const uint32_t *rows, const uint32_t *cols, const void *vals, size_t es, uint32_t nnz,
                          uint32_t nrows, uint32_t *rowptr, uint32_t *colind, void *vals_out, cudaStream_t s) {
  if (!rowptr || nrows == 0xFFFFFFFFu || (nnz && (!rows || !cols || !vals || !colind || !vals_out)))
    return SPARSEP_EINVAL;
  int bits = 0;
  while (bits < 32 && (nrows - 1) >> bits) ++bits;  // bits of the largest row index
  if (nrows <= 1) bits = 0;
  uint32_t *buf = nullptr;
  int *bad = nullptr;
  const size_t words = 2 * (size_t)nnz + sparsep::radix::radix_scratch_words(nnz);
  int st = c2c_err(sparsep::dev_malloc((void **)&buf, words * 4));
  if (!st) st = c2c_err(sparsep::dev_malloc((void **)&bad, sizeof(int)));
  if (st) {
    sparsep::dev_free(buf);
    sparsep::dev_free(bad);
    return st;
  }
  const uint32_t *key = nullptr, *idx = nullptr;
  int h_bad = 0;
  st = c2c_err(cudaMemsetAsync(bad, 0, sizeof(int), s));
  if (!st)
    st = c2c_err(sparsep::radix::radix_sort<uint32_t>(rows, nnz, bits, buf, buf + nnz, buf + 2 * (size_t)nnz, &key,
                                                        &idx, s, bad, nrows));
  if (!st) st = c2c_err(cudaMemcpyAsync(&h_bad, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
  if (!st) st = c2c_err(cudaStreamSynchronize(s));
  if (!st && h_bad) st = SPARSEP_EINVAL;  // a row index >= nrows
  if (!st) {
    rowptr_kernel<<<(nrows + 1 + 255) / 256, 256, 0, s>>>(nnz ? key : nullptr, nnz, nrows, rowptr);
    if (nnz) {
      const unsigned grid = (unsigned)std::min<uint32_t>(4096, (nnz + 255) / 256);
      const auto *v = static_cast<const unsigned char *>(vals);
      auto *vo = static_cast<unsigned char *>(vals_out);
      switch (es) {
        case 1: gather<1><<<grid, 256, 0, s>>>(idx, nnz, cols, v, colind, vo); break;
        case 2: gather<2><<<grid, 256, 0, s>>>(idx, nnz, cols, v, colind, vo); break;
        case 4: gather<4><<<grid, 256, 0, s>>>(idx, nnz, cols, v, colind, vo); break;
        default: gather<8><<<grid, 256, 0, s>>>(idx, nnz, cols, v, colind, vo); break;
      }
    }
    st = c2c_err(cudaGetLastError());
    if (!st) st = c2c_err(cudaStreamSynchronize(s));
  }
  sparsep::dev_free(buf);
  sparsep::dev_free(bad);
  return st;
}

#define SPARSEP_C2C_ENTRY(T, S)                                                                                 \
  int sparsep_coo2csr_device_##S(const uint32_t *d_rows, const uint32_t *d_cols, const T *d_vals, uint32_t nnz, \
                                 uint32_t nrows, uint32_t *d_rowptr, uint32_t *d_colind, T *d_vals_out,         \
                                 void *stream) {                                                                \
    return coo2csr_device(d_rows, d_cols, d_vals, sizeof(T), nnz, nrows, d_rowptr, d_colind, d_vals_out,       \
                          static_cast<cudaStream_t>(stream));                                                   \
  }

extern "C" {
SPARSEP_C2C_ENTRY(int8_t, i8)
SPARSEP_C2C_ENTRY(int16_t, i16)
SPARSEP_C2C_ENTRY(int32_t, i32)
SPARSEP_C2C_ENTRY(int64_t, i64)
SPARSEP_C2C_ENTRY(float, f32)
SPARSEP_C2C_ENTRY(double, f64)
}
