// coo2csr_dev.cu -- COO -> CSR on the device, with the arrays the host
// converter coo2csr (formats.cpp; the reference's counting sort,
// spmv/1D/CSR-row/support/matrix.h:113-152) produces: rows in order, and
// inside a row the input order kept (a stable sort by row).
//
// Stable LSD radix sort of (row, input index) pairs, 4 bits per pass, only as
// many passes as the row count needs (20 bits -> 5 passes for 1M rows):
//   hist     per 1024-element tile, counts of each digit  -> hist[d][tile]
//   scan     exclusive scan of hist in digit-major order (three launches)
//   scatter  each element to scan[d][tile] + (earlier elements of its tile
//            with digit d): the tile is walked in four 256-element rounds;
//            inside a round, __match_any_sync gives the rank among the warp's
//            lanes with the same digit, a prefix over the warps and a running
//            count per digit over the rounds do the rest -- input order kept.
// Then rowptr[r] = first sorted position with row >= r (a binary search per
// row), and columns / values are gathered through the sorted input indices.
#include <algorithm>
#include <cstdio>
#include <new>

#include "internal.hpp"
#include "sparsep.h"

namespace sparsep {
namespace c2c {

constexpr int NT = 256;         // threads per CTA
constexpr int ROUNDS = 4;       // elements per thread per tile
constexpr int TILE = NT * ROUNDS;
constexpr int RADIX = 16;       // 4-bit digits

__global__ void __launch_bounds__(NT) hist(const uint32_t *__restrict__ key, uint32_t n, int shift, uint32_t nt,
                                           uint32_t *__restrict__ h, uint32_t nrows, int *__restrict__ bad) {
  __shared__ uint32_t c[RADIX];
  if (threadIdx.x < RADIX) c[threadIdx.x] = 0;
  __syncthreads();
  const uint32_t base = blockIdx.x * TILE;
  for (int r = 0; r < ROUNDS; ++r) {
    const uint32_t i = base + r * NT + threadIdx.x;
    if (i < n) {
      const uint32_t k = key[i];
      if (bad && k >= nrows) atomicExch(bad, 1);  // first pass only: rows must be < nrows
      atomicAdd(&c[(k >> shift) & (RADIX - 1)], 1u);
    }
  }
  __syncthreads();
  if (threadIdx.x < RADIX) h[(size_t)threadIdx.x * nt + blockIdx.x] = c[threadIdx.x];
}

// Exclusive scan of the m digit counts in place, in three launches:
//   scan_reduce  CTA b sums its chunk h[b*SCAN_CHUNK, ...)        -> sums[b]
//   scan_top     one CTA scans sums[0, nb) (exclusive), in chunks
//   scan_down    CTA b scans its chunk and adds sums[b]
// A chunk is SCAN_CHUNK = 4 counts per thread; a thread scans its 4 serially
// and the CTA scans the thread totals with warp shuffles.
constexpr int SCAN_CHUNK = 4 * NT;

// exclusive scan of v over the CTA; *total gets the sum of all v
__device__ __forceinline__ uint32_t block_scan(uint32_t v, uint32_t *total) {
  __shared__ uint32_t ws[NT / 32 + 1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) ws[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    const uint32_t w = lane < NT / 32 ? ws[lane] : 0u;
    uint32_t wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += t;
    }
    if (lane < NT / 32) ws[lane] = wi - w;
    if (lane == NT / 32 - 1) ws[NT / 32] = wi;
  }
  __syncthreads();
  const uint32_t r = ws[warp] + inc - v;
  *total = ws[NT / 32];
  __syncthreads();  // ws is reused by the next call
  return r;
}

// exclusive scan of a[base, base + SCAN_CHUNK) (clipped to m) plus offset; returns the chunk's sum
__device__ __forceinline__ uint32_t scan_chunk(uint32_t *__restrict__ a, uint32_t m, uint32_t base, uint32_t offset) {
  const uint32_t i0 = base + 4 * threadIdx.x;
  uint32_t v[4], t = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    v[k] = i0 + k < m ? a[i0 + k] : 0u;
    t += v[k];
  }
  uint32_t total;
  uint32_t run = offset + block_scan(t, &total);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (i0 + k < m) a[i0 + k] = run;
    run += v[k];
  }
  return total;
}

__global__ void __launch_bounds__(NT) scan_reduce(const uint32_t *__restrict__ h, uint32_t m,
                                                  uint32_t *__restrict__ sums) {
  const uint32_t i0 = blockIdx.x * SCAN_CHUNK + 4 * threadIdx.x;
  uint32_t t = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) t += i0 + k < m ? h[i0 + k] : 0u;
  uint32_t total;
  block_scan(t, &total);
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(NT) scan_top(uint32_t *__restrict__ sums, uint32_t nb) {
  uint32_t carry = 0;
  for (uint32_t b = 0; b < nb; b += SCAN_CHUNK) carry += scan_chunk(sums, nb, b, carry);
}

__global__ void __launch_bounds__(NT) scan_down(uint32_t *__restrict__ h, uint32_t m,
                                                const uint32_t *__restrict__ sums) {
  scan_chunk(h, m, blockIdx.x * SCAN_CHUNK, sums[blockIdx.x]);
}

__global__ void __launch_bounds__(NT) scatter(const uint32_t *__restrict__ key, const uint32_t *__restrict__ idx,
                                              uint32_t n, int shift, uint32_t nt, const uint32_t *__restrict__ off,
                                              uint32_t *__restrict__ key_out, uint32_t *__restrict__ idx_out) {
  __shared__ uint32_t warp_cnt[NT / 32][RADIX];
  __shared__ uint32_t running[RADIX];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x < RADIX) running[threadIdx.x] = 0;
  const uint32_t base = blockIdx.x * TILE;
  for (int r = 0; r < ROUNDS; ++r) {
    const uint32_t i = base + r * NT + threadIdx.x;
    const bool in = i < n;
    const uint32_t k = in ? key[i] : 0;
    const uint32_t d = in ? (k >> shift) & (RADIX - 1) : RADIX;  // out-of-range lanes form their own group
    const unsigned same = __match_any_sync(0xffffffffu, d);
    const uint32_t rank = __popc(same & ((1u << lane) - 1u));
    __syncthreads();  // the previous round's readers of warp_cnt / running are done
    if (lane < RADIX) warp_cnt[warp][lane] = 0;
    __syncwarp();
    if (in && rank == 0) warp_cnt[warp][d] = __popc(same);  // the group's first lane
    __syncthreads();
    if (in) {
      uint32_t before = running[d];
      for (int w = 0; w < warp; ++w) before += warp_cnt[w][d];
      const uint32_t pos = off[(size_t)d * nt + blockIdx.x] + before + rank;
      key_out[pos] = k;
      idx_out[pos] = idx ? idx[i] : i;
    }
    __syncthreads();
    if (threadIdx.x < RADIX) {
      uint32_t t = 0;
      for (int w = 0; w < NT / 32; ++w) t += warp_cnt[w][threadIdx.x];
      running[threadIdx.x] += t;
    }
  }
}

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
  const uint32_t nt = (nnz + TILE - 1) / TILE;
  uint32_t *buf = nullptr;
  int *bad = nullptr;
  const uint32_t m = RADIX * nt, nb = (m + SCAN_CHUNK - 1) / SCAN_CHUNK;  // digit counts, scan chunks
  const size_t words = 4 * (size_t)nnz + (size_t)m + nb + 8;
  int st = c2c_err(cudaMalloc(&buf, words * 4));
  if (!st) st = c2c_err(cudaMalloc(&bad, sizeof(int)));
  if (st) {
    cudaFree(buf);
    cudaFree(bad);
    return st;
  }
  uint32_t *k0 = buf, *i0 = k0 + nnz, *k1 = i0 + nnz, *i1 = k1 + nnz, *h = i1 + nnz, *sums = h + m;
  const uint32_t *key = rows, *idx = nullptr;
  int h_bad = 0;
  st = c2c_err(cudaMemsetAsync(bad, 0, sizeof(int), s));
  for (int shift = 0; !st && nnz && shift < (bits ? bits : 1); shift += 4) {
    uint32_t *ko = (shift / 4) % 2 ? k1 : k0, *io = (shift / 4) % 2 ? i1 : i0;
    hist<<<nt, NT, 0, s>>>(key, nnz, shift, nt, h, nrows, shift == 0 ? bad : nullptr);
    scan_reduce<<<nb, NT, 0, s>>>(h, m, sums);
    scan_top<<<1, NT, 0, s>>>(sums, nb);
    scan_down<<<nb, NT, 0, s>>>(h, m, sums);
    scatter<<<nt, NT, 0, s>>>(key, idx, nnz, shift, nt, h, ko, io);
    st = c2c_err(cudaGetLastError());
    key = ko;
    idx = io;
  }
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
  cudaFree(buf);
  cudaFree(bad);
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
