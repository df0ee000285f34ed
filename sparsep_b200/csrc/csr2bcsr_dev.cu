// csr2bcsr_dev.cu -- CSR -> BCSR on the device, with the arrays the host
// converter csr2bcsr produces (formats.cpp; the reference's csr2bcsr +
// sortBCSRMatrix + countNNZperBlockBCSRMatrix,
// spmv/1D/BCSR-nnz/support/matrix.h:202-485): per block row the blocks sorted
// by block column, each block a row-major rb x cb array in which a later
// duplicate entry of a position overwrites an earlier one, and
// nnz_per_block[b] = the block's entries != 0.
//
// layout (type-independent, sparsep_bcsr_layout_device):
//   keys   per nonzero k: its row r (binary search in rowptr) and the key
//          (r / rb) << jbits | colind[k] / cb; rowptr and columns checked
//   sort   stable radix sort of the keys (radix.cuh) carrying k, so that the
//          entries of one block stay in input order
//   heads  a block starts where the sorted key changes: exclusive scan of the
//          head flags -> block start positions and block keys
// fill (per element type, sparsep_csr2bcsr_device_<t>):
//   browptr  lower bound of each block row among the block keys
//   blocks   one thread per block: zero it, write its entries in input order,
//            count the nonzero values; bcolind from the key
#include <algorithm>
#include <cstdio>
#include <new>

#include "fault.hpp"
#include "internal.hpp"
#include "radix.cuh"
#include "sparsep.h"

namespace sparsep {
namespace c2b {

constexpr int NT = 256;

// rowptr[0] == 0, non-decreasing, rowptr[nrows] == nnz
__global__ void check_rowptr(const uint32_t *__restrict__ rowptr, uint32_t nrows, uint32_t nnz, int *__restrict__ bad) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < nrows; r += gridDim.x * blockDim.x)
    if (rowptr[r] > rowptr[r + 1]) atomicExch(bad, 1);
  if (blockIdx.x == 0 && threadIdx.x == 0 && (rowptr[0] != 0 || rowptr[nrows] != nnz)) atomicExch(bad, 1);
}

__global__ void __launch_bounds__(NT) keys(const uint32_t *__restrict__ rowptr, uint32_t nrows,
                                           const uint32_t *__restrict__ colind, uint32_t nnz, uint32_t ncols,
                                           uint32_t rb, uint32_t cb, int jbits, uint64_t *__restrict__ key,
                                           uint32_t *__restrict__ row, int *__restrict__ bad) {
  for (uint32_t k = blockIdx.x * NT + threadIdx.x; k < nnz; k += gridDim.x * NT) {
    uint32_t lo = 0, hi = nrows - 1;  // last row whose start is <= k
    while (lo < hi) {
      const uint32_t mid = lo + ((hi - lo + 1) >> 1);
      if (rowptr[mid] <= k) lo = mid;
      else hi = mid - 1;
    }
    uint32_t c = colind[k];
    if (c >= ncols) {
      atomicExch(bad, 1);
      c = 0;
    }
    row[k] = lo;
    key[k] = ((uint64_t)(lo / rb) << jbits) | (c / cb);
  }
}

__global__ void __launch_bounds__(NT) head_flags(const uint64_t *__restrict__ skey, uint32_t n,
                                                 uint32_t *__restrict__ flag) {
  for (uint32_t i = blockIdx.x * NT + threadIdx.x; i < n; i += gridDim.x * NT)
    flag[i] = (i == 0 || skey[i] != skey[i - 1]) ? 1u : 0u;
}

// excl = exclusive scan of the head flags: block excl[i] starts at sorted position i
__global__ void __launch_bounds__(NT) block_starts(const uint64_t *__restrict__ skey, uint32_t n,
                                                   const uint32_t *__restrict__ excl, uint32_t *__restrict__ bstart,
                                                   uint64_t *__restrict__ bkey, uint32_t *__restrict__ nblocks) {
  for (uint32_t i = blockIdx.x * NT + threadIdx.x; i < n; i += gridDim.x * NT) {
    const bool head = i == 0 || skey[i] != skey[i - 1];
    if (head) {
      bstart[excl[i]] = i;
      bkey[excl[i]] = skey[i];
    }
    if (i == n - 1) {
      const uint32_t nb = excl[i] + (head ? 1u : 0u);
      bstart[nb] = n;
      *nblocks = nb;
    }
  }
}

// browptr[I] = number of blocks in block rows < I, I = 0 .. nbr
__global__ void browptr_kernel(const uint64_t *__restrict__ bkey, uint32_t nblocks, uint32_t nbr, int jbits,
                               uint32_t *__restrict__ browptr) {
  const uint32_t I = blockIdx.x * blockDim.x + threadIdx.x;
  if (I > nbr) return;
  const uint64_t want = (uint64_t)I << jbits;
  uint32_t lo = 0, hi = nblocks;
  while (lo < hi) {
    const uint32_t mid = lo + ((hi - lo) >> 1);
    if (bkey[mid] < want) lo = mid + 1;
    else hi = mid;
  }
  browptr[I] = lo;
}

template <typename T>
__global__ void __launch_bounds__(NT) fill_blocks(const uint64_t *__restrict__ bkey,
                                                  const uint32_t *__restrict__ bstart, uint32_t nblocks,
                                                  const uint32_t *__restrict__ sidx, const uint32_t *__restrict__ row,
                                                  const uint32_t *__restrict__ colind, const T *__restrict__ values,
                                                  uint32_t rb, uint32_t cb, int jbits, uint32_t *__restrict__ bcolind,
                                                  T *__restrict__ bval, uint32_t *__restrict__ nnz_per_block) {
  const uint64_t jmask = (1ull << jbits) - 1;
  const size_t bs = (size_t)rb * cb;
  for (uint32_t b = blockIdx.x * NT + threadIdx.x; b < nblocks; b += gridDim.x * NT) {
    const uint64_t k = bkey[b];
    const uint32_t J = (uint32_t)(k & jmask), r0 = (uint32_t)(k >> jbits) * rb, c0 = J * cb;
    bcolind[b] = J;
    T *blk = bval + (size_t)b * bs;
    for (size_t q = 0; q < bs; ++q) blk[q] = T(0);
    for (uint32_t i = bstart[b]; i < bstart[b + 1]; ++i) {  // input order: a later duplicate wins
      const uint32_t e = sidx[i], dc = colind[e] - c0;
      if (dc < cb) blk[(size_t)(row[e] - r0) * cb + dc] = values[e];  // columns as checked by the layout
    }
    uint32_t cnt = 0;
    for (size_t q = 0; q < bs; ++q) cnt += blk[q] != T(0);
    nnz_per_block[b] = cnt;
  }
}

}  // namespace c2b
}  // namespace sparsep

using namespace sparsep::c2b;

struct sparsep_bcsr_layout {
  uint32_t nrows = 0, ncols = 0, nnz = 0, rb = 0, cb = 0, nbr = 0, nblocks = 0;
  int jbits = 0;
  const uint32_t *colind = nullptr;  // the caller's column indices (read again by the fill)
  uint32_t *row = nullptr;           // row of each nonzero
  uint32_t *sidx = nullptr;          // nonzeros in block order (input order inside a block)
  uint32_t *bstart = nullptr;        // nblocks + 1 start positions in sidx
  uint64_t *bkey = nullptr;          // block keys (block row << jbits | block column)
};

static int c2b_err(cudaError_t e) {
  if (e == cudaSuccess) return SPARSEP_OK;
  char msg[160];
  std::snprintf(msg, sizeof msg, "%s (%d)", cudaGetErrorString(e), (int)e);
  sparsep::record_error(msg);
  return e == cudaErrorMemoryAllocation ? SPARSEP_ENOMEM : SPARSEP_EIO;
}

static int bits_for(uint64_t v) {  // bits of the largest value < v
  int b = 0;
  while (b < 64 && v > 1 && ((v - 1) >> b)) ++b;
  return b;
}

static unsigned grid_for(uint64_t n) { return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(16384, (n + NT - 1) / NT)); }

static int layout(const uint32_t *rowptr, const uint32_t *colind, uint32_t nrows, uint32_t ncols, uint32_t nnz,
                  uint32_t rb, uint32_t cb, sparsep_bcsr_layout *L, cudaStream_t s) {
  using sparsep::radix::radix_scratch_words;
  L->nrows = nrows;
  L->ncols = ncols;
  L->nnz = nnz;
  L->rb = rb;
  L->cb = cb;
  L->colind = colind;
  L->nbr = (uint32_t)(((uint64_t)nrows + rb - 1) / rb);
  const uint64_t nbc = ((uint64_t)ncols + cb - 1) / cb;
  L->jbits = bits_for(nbc);
  const int bits = L->jbits + bits_for(L->nbr);
  int *bad = nullptr;
  uint32_t *dnb = nullptr;
  int st = c2b_err(sparsep::dev_malloc((void **)&bad, 2 * sizeof(int)));
  if (st) return st;
  dnb = reinterpret_cast<uint32_t *>(bad + 1);
  int h_bad = 0;
  st = c2b_err(cudaMemsetAsync(bad, 0, 2 * sizeof(int), s));
  if (!st && nrows) check_rowptr<<<grid_for(nrows), NT, 0, s>>>(rowptr, nrows, nnz, bad);
  if (!st && nnz) {
    // scratch, in 32-bit words: input keys (2n), two key buffers (2n each), the
    // radix scratch, the head flags (n) with their scan sums (nbs + 8), and
    // the block starts (n + 1).  After the sort the input-key buffer holds the
    // block keys.
    const uint32_t nbs = (nnz + sparsep::radix::SCAN_CHUNK - 1) / sparsep::radix::SCAN_CHUNK;
    const size_t rsw = radix_scratch_words(nnz);
    const size_t words = 6 * (size_t)nnz + rsw + ((size_t)nnz + nbs + 8) + ((size_t)nnz + 1) + 8;
    uint32_t *buf = nullptr;
    st = c2b_err(sparsep::dev_malloc((void **)&buf, words * 4));
    if (!st) st = c2b_err(sparsep::dev_malloc((void **)&L->row, (size_t)nnz * 4));
    if (!st) {
      uint64_t *key = reinterpret_cast<uint64_t *>(buf), *k0 = key + nnz, *k1 = k0 + nnz;
      uint32_t *scratch = reinterpret_cast<uint32_t *>(k1 + nnz);
      uint32_t *flag = scratch + rsw, *sums = flag + nnz, *bstart_tmp = sums + nbs + 8;
      uint64_t *bkey_tmp = key;
      keys<<<grid_for(nnz), NT, 0, s>>>(rowptr, nrows, colind, nnz, ncols, rb, cb, L->jbits, key, L->row, bad);
      const uint64_t *skey = nullptr;
      const uint32_t *sidx = nullptr;
      st = c2b_err(sparsep::radix::radix_sort<uint64_t>(key, nnz, bits, k0, k1, scratch, &skey, &sidx, s));
      if (!st) {
        head_flags<<<grid_for(nnz), NT, 0, s>>>(skey, nnz, flag);
        sparsep::radix::scan_reduce<<<nbs, sparsep::radix::NT, 0, s>>>(flag, nnz, sums);
        sparsep::radix::scan_top<<<1, sparsep::radix::NT, 0, s>>>(sums, nbs);
        sparsep::radix::scan_down<<<nbs, sparsep::radix::NT, 0, s>>>(flag, nnz, sums);
        block_starts<<<grid_for(nnz), NT, 0, s>>>(skey, nnz, flag, bstart_tmp, bkey_tmp, dnb);
        st = c2b_err(cudaGetLastError());
      }
      if (!st) st = c2b_err(cudaMemcpyAsync(&h_bad, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
      if (!st) st = c2b_err(cudaMemcpyAsync(&L->nblocks, dnb, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
      if (!st) st = c2b_err(cudaStreamSynchronize(s));
      if (!st && h_bad) st = SPARSEP_EINVAL;
      if (!st) st = c2b_err(sparsep::dev_malloc((void **)&L->sidx, (size_t)nnz * 4));
      if (!st) st = c2b_err(sparsep::dev_malloc((void **)&L->bstart, ((size_t)L->nblocks + 1) * 4));
      if (!st) st = c2b_err(sparsep::dev_malloc((void **)&L->bkey, (size_t)std::max<uint32_t>(L->nblocks, 1) * 8));
      if (!st) st = c2b_err(cudaMemcpyAsync(L->sidx, sidx, (size_t)nnz * 4, cudaMemcpyDeviceToDevice, s));
      if (!st)
        st = c2b_err(cudaMemcpyAsync(L->bstart, bstart_tmp, ((size_t)L->nblocks + 1) * 4, cudaMemcpyDeviceToDevice, s));
      if (!st) st = c2b_err(cudaMemcpyAsync(L->bkey, bkey_tmp, (size_t)L->nblocks * 8, cudaMemcpyDeviceToDevice, s));
      if (!st) st = c2b_err(cudaStreamSynchronize(s));
    }
    sparsep::dev_free(buf);
  } else if (!st) {
    st = c2b_err(cudaMemcpyAsync(&h_bad, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
    if (!st) st = c2b_err(cudaStreamSynchronize(s));
    if (!st && h_bad) st = SPARSEP_EINVAL;
    L->nblocks = 0;
  }
  sparsep::dev_free(bad);
  return st;
}

template <typename T>
static int fill(const sparsep_bcsr_layout *L, const T *values, uint32_t *browptr, uint32_t *bcolind, T *bval,
                uint32_t *nnz_per_block, cudaStream_t s) {
  if (!L || !browptr || (L->nblocks && (!values || !bcolind || !bval || !nnz_per_block))) return SPARSEP_EINVAL;
  browptr_kernel<<<(L->nbr + 1 + 255) / 256, 256, 0, s>>>(L->bkey, L->nblocks, L->nbr, L->jbits, browptr);
  if (L->nblocks)
    fill_blocks<T><<<grid_for(L->nblocks), NT, 0, s>>>(L->bkey, L->bstart, L->nblocks, L->sidx, L->row, L->colind,
                                                        values, L->rb, L->cb, L->jbits, bcolind, bval, nnz_per_block);
  int st = c2b_err(cudaGetLastError());
  if (!st) st = c2b_err(cudaStreamSynchronize(s));
  return st;
}

extern "C" {

int sparsep_bcsr_layout_device(const uint32_t *d_rowptr, const uint32_t *d_colind, uint32_t nrows, uint32_t ncols,
                               uint32_t nnz, uint32_t rb, uint32_t cb, sparsep_bcsr_layout **out, uint64_t *nblocks,
                               void *stream) {
  if (!out) return SPARSEP_EINVAL;
  *out = nullptr;
  if (!d_rowptr || (nnz && !d_colind) || rb == 0 || cb == 0 || (nnz && nrows == 0)) return SPARSEP_EINVAL;
  auto *L = new (std::nothrow) sparsep_bcsr_layout();
  if (!L) return SPARSEP_ENOMEM;
  const int st = layout(d_rowptr, d_colind, nrows, ncols, nnz, rb, cb, L, static_cast<cudaStream_t>(stream));
  if (st) {
    sparsep_bcsr_layout_free(L);
    return st;
  }
  if (nblocks) *nblocks = L->nblocks;
  *out = L;
  return SPARSEP_OK;
}

void sparsep_bcsr_layout_free(sparsep_bcsr_layout *L) {
  if (!L) return;
  for (void *d : {(void *)L->row, (void *)L->sidx, (void *)L->bstart, (void *)L->bkey})
    if (d) sparsep::dev_free(d);
  delete L;
}

#define SPARSEP_C2B_ENTRY(T, S)                                                                                   \
  int sparsep_csr2bcsr_device_##S(const sparsep_bcsr_layout *L, const T *d_values, uint32_t *d_browptr,          \
                                  uint32_t *d_bcolind, T *d_bval, uint32_t *d_nnz_per_block, void *stream) {      \
    return fill<T>(L, d_values, d_browptr, d_bcolind, d_bval, d_nnz_per_block, static_cast<cudaStream_t>(stream)); \
  }
SPARSEP_C2B_ENTRY(int8_t, i8)
SPARSEP_C2B_ENTRY(int16_t, i16)
SPARSEP_C2B_ENTRY(int32_t, i32)
SPARSEP_C2B_ENTRY(int64_t, i64)
SPARSEP_C2B_ENTRY(float, f32)
SPARSEP_C2B_ENTRY(double, f64)

}  // extern "C"
