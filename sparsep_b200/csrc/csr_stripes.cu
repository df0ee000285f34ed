// csr_stripes.cu -- the heavy rows of a split 1D CSR plan: column stripes whose
// x segment sits in shared memory (sm_100a).
//
// A CSR SpMV over a matrix whose columns are spread over all of a large x is
// bound by the x gathers: every nonzero is one random read of x through L1
// and L2.  A split plan moves the rows with many nonzeros ("heavy rows") out
// of the row kernels and re-lays them out stripe-major: stripe row
// v = s * nH + k holds heavy row k's nonzeros whose columns fall in stripe s,
// with 16-bit stripe-local columns.  This kernel runs persistent CTAs (one per
// SM: the stripe takes most of shared memory), each over a contiguous list of
// chunks (<= CAP nonzeros, <= RCAP stripe rows, one stripe).  Per CTA:
//   - when the chunk's stripe changes, the stripe's x columns are brought into
//     shared memory by one bulk (TMA) copy of the 16-byte aligned body plus
//     plain loads of the ragged ends (no read past x);
//   - thread 0 keeps NS-1 chunks in flight ahead of the consumers: bulk copies
//     of the chunk's stripe-row offsets, columns and values into a ring of
//     stages, each tracked by a transaction-count mbarrier (bounded waits);
//   - the consumers multiply each staged value by x read from shared memory,
//     then sum stripe rows from shared memory: a thread per short row, a warp
//     per longer one, consecutive threads storing consecutive partials.  A
//     stripe row longer than a chunk is cut into pieces added in order.
// launch_heavy_merge then writes y[hrow[k]] = sum over stripes of the partials,
// in stripe order (the reference's 2D merge order, spmv/2D/BDCSR/host/app.c:
// 437-447, applied to the heavy rows' stripes).
//
// The products and sums are the reference's (spmv/1D/CSR-row/host/app.c:66-77)
// in another order: integers wrap exactly as there, floating point stays within
// the per-row gamma bound.
#include <atomic>

#include "device.cuh"
#include "kernels.hpp"

namespace sparsep {
namespace stripes {

constexpr int NT = 1024;                 // threads per CTA
constexpr size_t X_BUDGET = 128 * 1024;  // shared memory for the x stripe
constexpr size_t SMEM_MAX = 227 * 1024;  // opt-in limit per CTA on sm_100a

constexpr size_t up16(size_t v) { return (v + 15) & ~(size_t)15; }
constexpr size_t up128(size_t v) { return (v + 127) & ~(size_t)127; }

template <typename T> struct Layout {
  static constexpr uint32_t W = (X_BUDGET / sizeof(T)) > 65536 ? 65536 : (uint32_t)(X_BUDGET / sizeof(T));
  static constexpr int CAP = sizeof(T) == 8 ? 2048 : 4096;  // nonzeros per chunk
  static constexpr int RCAP = CAP / 4;                      // stripe rows per chunk
  // columns and values are staged from one aligned nonzero index: 16 bytes of
  // both arrays (columns are 2 bytes)
  static constexpr int AL = (16 / (int)sizeof(T)) > 8 ? (16 / (int)sizeof(T)) : 8;
  static constexpr size_t XBYTES = up128((size_t)W * sizeof(T) + 32);
  static constexpr size_t RB = (size_t)(RCAP + 8) * 4;
  static constexpr size_t CB = up16((size_t)(CAP + 2 * AL) * 2);
  static constexpr size_t VB = up16((size_t)(CAP + 2 * AL) * sizeof(T));
  static constexpr size_t STAGE = RB + CB + VB;
  static constexpr bool IN_PLACE = sizeof(T) == sizeof(Acc<T>);
  static constexpr size_t PB = IN_PLACE ? 0 : (size_t)CAP * sizeof(Acc<T>);
  static constexpr size_t STATIC = 8 * 1024;  // barriers, reduction slots, long-row list
  static constexpr int NS = (XBYTES + 3 * STAGE + PB + STATIC <= SMEM_MAX) ? 3 : 2;
  static constexpr size_t BYTES = XBYTES + NS * STAGE + PB;
  static_assert(XBYTES + 2 * STAGE + PB + STATIC <= SMEM_MAX, "stripe kernel does not fit shared memory");
};

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// bounded wait for the phase of parity `parity` to complete
__device__ __forceinline__ bool wait_bar(uint64_t *bar, uint32_t parity) {
  uint32_t done = 0;
  for (uint32_t i = 0; i < (1u << 24) && !done; ++i) {
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
  }
  return done != 0;
}

// 16-byte aligned copy windows of a chunk
struct Win {
  uint32_t r_lo, r_n;  // stripe-row offsets [r_lo, r_lo + r_n)
  uint32_t n_lo, n_n;  // columns and values [n_lo, n_lo + n_n)
};

template <typename T>
__device__ __forceinline__ Win window(const StripeChunk &c) {
  constexpr uint32_t AL = Layout<T>::AL;
  Win w;
  w.r_lo = c.v0 & ~3u;
  w.r_n = ((c.v1 + 1 + 3) & ~3u) - w.r_lo;
  w.n_lo = c.n0 / AL * AL;
  w.n_n = c.n1 > c.n0 ? (c.n1 + AL - 1) / AL * AL - w.n_lo : 0u;
  return w;
}

// Stage x[lo, lo + w) into xsm: the 16-byte aligned body by one bulk copy on
// `bar`, the ragged head and tail (< 16 bytes each) by plain loads.  Returns
// the shared pointer to element lo.  Every thread calls it; the caller waits
// on `bar` and then synchronises the CTA.
template <typename T>
__device__ const T *stage_stripe(const T *x, uint32_t lo, uint32_t w, unsigned char *xsm, uint64_t *bar) {
  const uintptr_t g_lo = reinterpret_cast<uintptr_t>(x + lo), g_hi = g_lo + (uintptr_t)w * sizeof(T);
  const uintptr_t g0 = g_lo & ~(uintptr_t)15;
  uintptr_t a0 = (g_lo + 15) & ~(uintptr_t)15, a1 = g_hi & ~(uintptr_t)15;
  if (a0 > g_hi) a0 = g_hi;
  if (a1 < a0) a1 = a0;
  if (threadIdx.x == 0) {
    // earlier generic reads of the previous stripe are ordered before the copy
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    expect_tx(bar, (uint32_t)(a1 - a0));
    const uint32_t CH = 32768;
    for (uintptr_t off = a0; off < a1; off += CH) {
      const uint32_t n = (uint32_t)((a1 - off) < CH ? (a1 - off) : CH);
      bulk_g2s(xsm + (off - g0), reinterpret_cast<const void *>(off), n, bar);
    }
  }
  T *xs = reinterpret_cast<T *>(xsm + (g_lo - g0));
  const uint32_t nhead = (uint32_t)((a0 - g_lo) / sizeof(T)), ntail = (uint32_t)((g_hi - a1) / sizeof(T));
  if (threadIdx.x < nhead) xs[threadIdx.x] = x[lo + threadIdx.x];
  if (threadIdx.x >= 32 && threadIdx.x - 32 < ntail) {
    const uint32_t c = w - ntail + (threadIdx.x - 32);
    xs[c] = x[lo + c];
  }
  return xs;
}

template <typename T>
__global__ void __launch_bounds__(NT, 1) stripe_rows(StripeParams<T> P) {
  using A = Acc<T>;
  using L = Layout<T>;
  constexpr int CAP = L::CAP, RCAP = L::RCAP, NS = L::NS;
  constexpr int PER = (CAP + NT - 1) / NT;
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ uint64_t full[NS];
  __shared__ uint64_t xbar;
  __shared__ A red[NT / 32];
  __shared__ uint32_t longs[RCAP];
  __shared__ uint32_t nlong;
  __shared__ int abort_flag;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t c0 = P.cta_first[blockIdx.x], c1 = P.cta_first[blockIdx.x + 1];
  unsigned char *xsm = sm;
  auto stage_ptr = [&](uint32_t s) { return sm + L::XBYTES + (size_t)s * L::STAGE; };
  A *prs = reinterpret_cast<A *>(sm + L::XBYTES + (size_t)NS * L::STAGE);

  if (threadIdx.x == 0) {
    for (int s = 0; s < NS; ++s)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&full[s])) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&xbar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    abort_flag = 0;
  }
  __syncthreads();

  // producer: stage local chunk k into ring slot k % NS
  auto issue = [&](uint32_t k) {
    if (c0 + k >= c1) return;
    const StripeChunk c = P.chunks[c0 + k];
    const Win w = window<T>(c);
    const uint32_t s = k % NS;
    unsigned char *st = stage_ptr(s);
    const uint32_t bytes = w.r_n * 4 + w.n_n * 2 + w.n_n * (uint32_t)sizeof(T);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (SP_BAD(P, w.r_n <= (uint32_t)RCAP + 8 && w.n_n <= (uint32_t)(CAP + 2 * L::AL) &&
                      (uint64_t)w.r_lo + w.r_n <= P.n_vptr && (uint64_t)w.n_lo + w.n_n <= P.n_h,
               -1030)) {
      asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&full[s])) : "memory");
      return;
    }
    expect_tx(&full[s], bytes);
    bulk_g2s(st, P.vptr + w.r_lo, w.r_n * 4, &full[s]);
    if (w.n_n) {
      bulk_g2s(st + L::RB, P.hcol + w.n_lo, w.n_n * 2, &full[s]);
      bulk_g2s(st + L::RB + L::CB, P.hval + w.n_lo, w.n_n * (uint32_t)sizeof(T), &full[s]);
    }
  };

  if (threadIdx.x == 0)
    for (int k = 0; k < NS - 1; ++k) issue(k);

  uint32_t cur = 0xFFFFFFFFu, xphase = 0;
  bool x_pending = false;
  const T *xs = nullptr;
  A carry = A(0);  // running sum of a stripe row cut into pieces (thread 0)
  uint32_t k = 0;
  for (; c0 + k < c1; ++k) {
    const StripeChunk c = P.chunks[c0 + k];
    if (threadIdx.x == 0) issue(k + NS - 1);  // into the slot chunk k-1 released
    if (c.stripe != cur) {
      // every thread is past its reads of the previous stripe (loop-end barrier)
      const uint32_t lo = c.stripe * P.W;
      const uint32_t w = P.ncols - lo < P.W ? P.ncols - lo : P.W;
      xs = stage_stripe<T>(P.x, lo, w, xsm, &xbar);
      x_pending = true;
      if (!wait_bar(&xbar, xphase)) {
        if (P.err) atomicCAS(P.err, 0, SPARSEP_ETIMEDOUT);
        abort_flag = 1;
      } else {
        x_pending = false;
      }
      xphase ^= 1u;
      cur = c.stripe;
    }
    const Win w = window<T>(c);
    const uint32_t s = k % NS;
    unsigned char *st = stage_ptr(s);
    if (!wait_bar(&full[s], (k / NS) & 1u)) {
      if (P.err) atomicCAS(P.err, 0, SPARSEP_ETIMEDOUT);
      abort_flag = 1;
    }
    if (threadIdx.x == 0) nlong = 0;
    __syncthreads();
    if (abort_flag) break;
    const uint32_t *srp = reinterpret_cast<const uint32_t *>(st) + (c.v0 - w.r_lo);
    const uint16_t *cb = reinterpret_cast<const uint16_t *>(st + L::RB) + (c.n0 - w.n_lo);
    T *vb = reinterpret_cast<T *>(st + L::RB + L::CB) + (c.n0 - w.n_lo);
    A *pr = L::IN_PLACE ? reinterpret_cast<A *>(vb) : prs;
    const uint32_t n = c.n1 - c.n0;
    const uint32_t sw = P.ncols - cur * P.W < P.W ? P.ncols - cur * P.W : P.W;  // stripe width
    if (SP_BAD(P, n <= (uint32_t)CAP && c.v1 > c.v0 && (c.piece || c.v1 - c.v0 <= (uint32_t)RCAP), -1031)) {
      __syncthreads();
      continue;
    }

    // products: every x read of a thread issued before any use
    A acc = A(0);
    {
      uint32_t col[PER];
#pragma unroll
      for (int u = 0; u < PER; ++u) {
        const uint32_t j = threadIdx.x + u * NT;
        col[u] = j < n ? cb[j] : 0u;
        if (SP_BAD(P, col[u] < sw, -1032)) col[u] = 0;
      }
      T xv[PER];
#pragma unroll
      for (int u = 0; u < PER; ++u) xv[u] = xs[col[u]];
#pragma unroll
      for (int u = 0; u < PER; ++u) {
        const uint32_t j = threadIdx.x + u * NT;
        if (j < n) {
          const A p = mul<T>(vb[j], xv[u]);
          if (c.piece) acc += p;
          else pr[j] = p;
        }
      }
    }
    if (c.piece) {
      // a piece of one long stripe row: block sum, added in chunk order
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (lane == 0) red[warp] = acc;
      __syncthreads();
      if (threadIdx.x == 0) {
        A tot = A(0);
        for (int q = 0; q < NT / 32; ++q) tot += red[q];
        carry = (c.piece & 1u) ? tot : carry + tot;
        if ((c.piece & 2u) && !SP_BAD(P, c.v0 < P.n_part, -1033)) P.part[c.v0] = from_acc<T>(carry);
      }
    } else {
      __syncthreads();
      // stripe rows [v0, v1): short ones summed by one thread, longer by a warp
      const uint32_t nr = c.v1 - c.v0, base = srp[0];
      for (uint32_t i = threadIdx.x; i < nr; i += NT) {
        // rows of a whole-rows chunk end inside it; the clamp keeps a
        // malformed chunk inside the staged products
        const uint32_t b = min(srp[i + 1] - base, n), a = min(srp[i] - base, b);
        if (b - a <= 32u) {
          A sum = A(0);
          for (uint32_t q = a; q < b; ++q) sum += pr[q];
          if (!SP_BAD(P, c.v0 + i < P.n_part && b <= n, -1033)) P.part[c.v0 + i] = from_acc<T>(sum);
        } else {
          longs[atomicAdd(&nlong, 1u)] = i;
        }
      }
      __syncthreads();
      for (uint32_t li = warp; li < nlong; li += NT / 32) {
        const uint32_t i = longs[li];
        const uint32_t b = min(srp[i + 1] - base, n), a = min(srp[i] - base, b);
        A sum = A(0);
        for (uint32_t q = a + lane; q < b; q += 32) sum += pr[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        if (lane == 0 && !SP_BAD(P, c.v0 + i < P.n_part && b <= n, -1033)) P.part[c.v0 + i] = from_acc<T>(sum);
      }
    }
    __syncthreads();  // the slot may be refilled and the stripe replaced after this point
  }

  // after an abort, wait (bounded) for the copies this CTA still has in flight
  if (threadIdx.x == 0 && abort_flag) {
    if (x_pending) wait_bar(&xbar, xphase ^ 1u);
    for (uint32_t q = k; q < k + NS; ++q) {
      if (c0 + q >= c1) break;
      wait_bar(&full[q % NS], (q / NS) & 1u);
    }
  }
}

// y[hrow[k]] = part[k] + part[nH + k] + ... in stripe order
template <typename T>
__global__ void heavy_merge(const T *__restrict__ part, const uint32_t *__restrict__ hrow, uint32_t nH, uint32_t nS,
                            T *__restrict__ y) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nH; k += gridDim.x * blockDim.x) {
    Acc<T> s = to_acc<T>(part[k]);
    uint32_t st = 1;
    for (; st + 8 <= nS; st += 8) {  // eight loads in flight, added in stripe order
      T v[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) v[q] = __ldcg(part + (uint64_t)(st + q) * nH + k);
#pragma unroll
      for (int q = 0; q < 8; ++q) s += to_acc<T>(v[q]);
    }
    for (; st < nS; ++st) s += to_acc<T>(__ldcg(part + (uint64_t)st * nH + k));
    y[hrow[k]] = from_acc<T>(s);
  }
}

}  // namespace stripes

template <typename T>
void stripe_geometry(uint32_t *width, size_t *smem, uint32_t *chunk_nnz, uint32_t *chunk_rows) {
  using L = stripes::Layout<T>;
  if (width) *width = L::W;
  if (smem) *smem = L::BYTES;
  if (chunk_nnz) *chunk_nnz = L::CAP;
  if (chunk_rows) *chunk_rows = L::RCAP;
}

template <typename T>
cudaError_t launch_stripes(const StripeParams<T> &P, uint32_t ctas, cudaStream_t st) {
  if (ctas == 0) return cudaSuccess;
  auto k = stripes::stripe_rows<T>;
  const size_t smem = stripes::Layout<T>::BYTES;
  static std::atomic<unsigned long long> set_on{0};  // attribute set once per device
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = 1ull << (dev & 63);
  if (!(set_on.load() & bit)) {
    e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    set_on.fetch_or(bit);
  }
  k<<<ctas, stripes::NT, smem, st>>>(P);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_heavy_merge(const T *part, const uint32_t *hrow, uint32_t nH, uint32_t nS, T *y, int sms,
                               cudaStream_t st) {
  if (nH == 0) return cudaSuccess;
  uint32_t blocks = (nH + 255) / 256, cap = (uint32_t)sms * 4;
  stripes::heavy_merge<T><<<blocks < cap ? blocks : cap, 256, 0, st>>>(part, hrow, nH, nS, y);
  return cudaGetLastError();
}

#ifndef SPARSEP_KT
#define SPARSEP_KT float
#endif
template void stripe_geometry<SPARSEP_KT>(uint32_t *, size_t *, uint32_t *, uint32_t *);
template cudaError_t launch_stripes<SPARSEP_KT>(const StripeParams<SPARSEP_KT> &, uint32_t, cudaStream_t);
template cudaError_t launch_heavy_merge<SPARSEP_KT>(const SPARSEP_KT *, const uint32_t *, uint32_t, uint32_t,
                                                    SPARSEP_KT *, int, cudaStream_t);

}  // namespace sparsep
