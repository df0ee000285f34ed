// radix.cuh -- stable LSD radix sort of (key, index) pairs on the device,
// 4 bits per pass, used by the device format builders (COO -> CSR sorts by
// row; CSR -> BCSR by (block row, block column)).
//   hist     per 1024-element tile, counts of each digit  -> hist[d][tile]
//   scan     exclusive scan of hist in digit-major order (three launches)
//   scatter  each element to scan[d][tile] + (earlier elements of its tile
//            with digit d): the tile is walked in four 256-element rounds;
//            inside a round, __match_any_sync gives the rank among the warp's
//            lanes with the same digit, a prefix over the warps and a running
//            count per digit over the rounds do the rest -- input order kept.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace sparsep {
namespace radix {
namespace {  // internal linkage: every translation unit that sorts gets its own kernels

constexpr int NT = 256;         // threads per CTA
constexpr int ROUNDS = 4;       // elements per thread per tile
constexpr int TILE = NT * ROUNDS;
constexpr int RADIX = 16;       // 4-bit digits

template <typename K>
__global__ void __launch_bounds__(NT) hist(const K *__restrict__ key, uint32_t n, int shift, uint32_t nt,
                                           uint32_t *__restrict__ h, K bound, int *__restrict__ bad) {
  __shared__ uint32_t c[RADIX];
  if (threadIdx.x < RADIX) c[threadIdx.x] = 0;
  __syncthreads();
  const uint32_t base = blockIdx.x * TILE;
  for (int r = 0; r < ROUNDS; ++r) {
    const uint32_t i = base + r * NT + threadIdx.x;
    if (i < n) {
      const K k = key[i];
      if (bad && k >= bound) atomicExch(bad, 1);  // first pass only: keys must be < bound
      atomicAdd(&c[(uint32_t)(k >> shift) & (RADIX - 1)], 1u);
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

template <typename K>
__global__ void __launch_bounds__(NT) scatter(const K *__restrict__ key, const uint32_t *__restrict__ idx,
                                              uint32_t n, int shift, uint32_t nt, const uint32_t *__restrict__ off,
                                              K *__restrict__ key_out, uint32_t *__restrict__ idx_out) {
  __shared__ uint32_t warp_cnt[NT / 32][RADIX];
  __shared__ uint32_t running[RADIX];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x < RADIX) running[threadIdx.x] = 0;
  const uint32_t base = blockIdx.x * TILE;
  for (int r = 0; r < ROUNDS; ++r) {
    const uint32_t i = base + r * NT + threadIdx.x;
    const bool in = i < n;
    const K k = in ? key[i] : K(0);
    const uint32_t d = in ? (uint32_t)(k >> shift) & (RADIX - 1) : RADIX;  // out-of-range lanes form their own group
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


// Scratch words (32-bit) radix_sort needs for n elements besides the key buffers.
inline size_t radix_scratch_words(uint32_t n) {
  const uint32_t nt = (n + TILE - 1) / TILE, m = RADIX * nt, nb = (m + SCAN_CHUNK - 1) / SCAN_CHUNK;
  return 2 * (size_t)n + m + nb + 8;
}

// Stable sort of keys[0, n) by their low `bits` bits (at least one pass, so
// that the index array is produced even for bits = 0), carrying the input
// index.  k0/k1: two key buffers of n; scratch: radix_scratch_words(n) words.
// On return *ks / *is point at the sorted keys and input indices (inside k0/k1
// and scratch).  bad/bound: when bad is set, the first pass flags a key >= bound.
template <typename K>
cudaError_t radix_sort(const K *keys, uint32_t n, int bits, K *k0, K *k1, uint32_t *scratch, const K **ks,
                       const uint32_t **is, cudaStream_t s, int *bad = nullptr, K bound = K(0)) {
  const uint32_t nt = (n + TILE - 1) / TILE, m = RADIX * nt, nb = (m + SCAN_CHUNK - 1) / SCAN_CHUNK;
  uint32_t *i0 = scratch, *i1 = i0 + n, *h = i1 + n, *sums = h + m;
  const K *key = keys;
  const uint32_t *idx = nullptr;
  for (int shift = 0; n && shift < (bits ? bits : 1); shift += 4) {
    const bool odd = (shift / 4) % 2;
    K *ko = odd ? k1 : k0;
    uint32_t *io = odd ? i1 : i0;
    hist<K><<<nt, NT, 0, s>>>(key, n, shift, nt, h, bound, shift == 0 ? bad : nullptr);
    scan_reduce<<<nb, NT, 0, s>>>(h, m, sums);
    scan_top<<<1, NT, 0, s>>>(sums, nb);
    scan_down<<<nb, NT, 0, s>>>(h, m, sums);
    scatter<K><<<nt, NT, 0, s>>>(key, idx, n, shift, nt, h, ko, io);
    if (cudaError_t e = cudaGetLastError()) return e;
    key = ko;
    idx = io;
  }
  *ks = key;
  *is = idx;
  return cudaSuccess;
}

}  // namespace
}  // namespace radix
}  // namespace sparsep
