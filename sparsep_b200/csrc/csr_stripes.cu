// csr_stripes.cu -- the persistent kernel of a split 1D CSR plan (sm_100a).
//
// A CSR SpMV over a matrix whose columns spread over all of a large x is bound
// by the x gathers: every nonzero is one random read of x through L1 and L2.
// A split plan moves the rows with many nonzeros ("heavy rows") into column
// stripes: stripe row v = s * nH + k holds heavy row k's nonzeros whose
// columns fall in stripe s, with 16-bit stripe-local columns, so their x is
// read from shared memory.  The other rows ("light rows") stay CSR rows whose
// x is gathered from global memory.  One persistent CTA per SM walks its own
// list of chunks, heavy and light interleaved so that one chunk's x gathers
// overlap another's streaming:
//   - the producer warp keeps NS chunks in flight: bulk (TMA) copies of a
//     chunk's row offsets, columns and values into a ring slot, tracked by a
//     transaction-count mbarrier ("full"); it refills a slot once every
//     consumer warp has released it ("empty" mbarrier), and before the first
//     chunk of a new stripe it brings the stripe's x columns into shared
//     memory (bulk copy of the 16-byte aligned body, plain loads of the ragged
//     ends: nothing past x is read);
//   - each of the 31 consumer warps takes the rows of a chunk whose first
//     nonzero falls in its share of the chunk's nonzeros: it multiplies their
//     values by x (shared-memory stripe or global gathers, several in flight
//     per lane), then sums rows from shared memory, a lane per short row and
//     the whole warp per longer one, and stores stripe partials (heavy) or y
//     (light).  Warps synchronise only within themselves, so one warp's
//     gathers overlap another's sums.  A row longer than a chunk is cut into
//     pieces that warp 0 adds in order.
// launch_heavy_merge then writes y[hrow[k]] = sum over stripes of the
// partials, in stripe order (the reference's 2D merge order, spmv/2D/BDCSR/
// host/app.c:437-447, applied to the heavy rows' stripes); the light chunks
// wrote zero for the heavy rows, which carry no light nonzeros.
//
// The products and sums are the reference's (spmv/1D/CSR-row/host/app.c:66-77)
// in another order: integers wrap exactly as there, floating point stays within
// the per-row gamma bound.  Every wait is bounded; one that runs out records
// SPARSEP_ETIMEDOUT and the CTA waits (bounded) for its copies before leaving.
#include <atomic>

#include "device.cuh"
#include "kernels.hpp"

namespace sparsep {
namespace stripes {

constexpr int NT = 1024;                 // threads per CTA
constexpr int NCW = SPLIT_WARPS;         // consumer warps; warp NCW is the producer
constexpr size_t X_BUDGET = 128 * 1024;  // shared memory for the x stripe
constexpr size_t SMEM_MAX = 227 * 1024;  // opt-in limit per CTA on sm_100a

constexpr size_t up16(size_t v) { return (v + 15) & ~(size_t)15; }
constexpr size_t up128(size_t v) { return (v + 127) & ~(size_t)127; }
constexpr size_t max2(size_t a, size_t b) { return a > b ? a : b; }

template <typename T> struct Layout {
  static constexpr uint32_t W = (X_BUDGET / sizeof(T)) > 65536 ? 65536 : (uint32_t)(X_BUDGET / sizeof(T));
  static constexpr int CAP = sizeof(T) == 8 ? 2048 : 4096;  // heavy nonzeros per chunk (16-bit columns)
  static constexpr int CAP_L = CAP / 2;                     // light nonzeros per chunk (32-bit columns)
  static constexpr int RCAP = NCW * 32;                     // rows per chunk
  // columns and values are staged from one aligned nonzero index
  static constexpr int AL = (16 / (int)sizeof(T)) > 8 ? (16 / (int)sizeof(T)) : 8;
  static constexpr size_t XBYTES = up128((size_t)W * sizeof(T) + 32);
  static constexpr size_t RB = up16((size_t)(RCAP + 8) * 4);
  static constexpr size_t CB = up16(max2((size_t)(CAP + 2 * AL) * 2, (size_t)(CAP_L + 2 * AL) * 4));
  static constexpr size_t VB = up16((size_t)(CAP + 2 * AL) * sizeof(T));
  static constexpr size_t STAGE = RB + CB + VB;
  static constexpr bool IN_PLACE = sizeof(T) == sizeof(Acc<T>);
  static constexpr size_t PB = IN_PLACE ? 0 : (size_t)CAP * sizeof(Acc<T>);  // products, per slot
  static constexpr size_t STATIC = 2 * 1024;  // barriers and flags
  static constexpr size_t fits(int ns) { return XBYTES + ns * (STAGE + PB) + STATIC; }
  static constexpr int NS = fits(4) <= SMEM_MAX ? 4 : (fits(3) <= SMEM_MAX ? 3 : 2);
  static constexpr size_t BYTES = XBYTES + NS * (STAGE + PB);
  static_assert(fits(2) <= SMEM_MAX, "split kernel does not fit shared memory");
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

__device__ __forceinline__ void arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Bounded wait for the phase of parity `parity` to complete.  Each try
// suspends the warp for up to 20 us (or until the phase completes) instead of
// spinning, so waiting warps take no issue slots; 2^16 tries bound the wait at
// about 1.3 s.
__device__ __forceinline__ bool wait_bar(uint64_t *bar, uint32_t parity) {
  uint32_t done = 0;
  for (uint32_t i = 0; i < (1u << 16) && !done; ++i) {
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3; selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity), "r"(20000)
        : "memory");
  }
  return done != 0;
}

// 16-byte aligned copy windows of a chunk: row offsets [r_lo, r_lo + r_n),
// columns and values [n_lo, n_lo + n_n)
struct Win {
  uint32_t r_lo, r_n, n_lo, n_n;
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

// Shared-memory address of x element lo of the stripe staged from x + lo (the
// copy keeps x's offset within its 16-byte line).
template <typename T>
__device__ __forceinline__ T *stripe_base(const T *x, uint32_t lo, unsigned char *xsm) {
  const uintptr_t g_lo = reinterpret_cast<uintptr_t>(x + lo);
  return reinterpret_cast<T *>(xsm + (g_lo & 15));
}

// Stage x[lo, lo + w) into xsm, run by the producer warp: the ragged head and
// tail (under 16 bytes each) by plain loads of its lanes, then lane 0 arrives
// on `bar` expecting the 16-byte aligned body and issues its bulk copies.
template <typename T>
__device__ void stage_stripe(const T *x, uint32_t lo, uint32_t w, unsigned char *xsm, uint64_t *bar, int lane) {
  const uintptr_t g_lo = reinterpret_cast<uintptr_t>(x + lo), g_hi = g_lo + (uintptr_t)w * sizeof(T);
  const uintptr_t g0 = g_lo & ~(uintptr_t)15;
  uintptr_t a0 = (g_lo + 15) & ~(uintptr_t)15, a1 = g_hi & ~(uintptr_t)15;
  if (a0 > g_hi) a0 = g_hi;
  if (a1 < a0) a1 = a0;
  T *xs = stripe_base(x, lo, xsm);
  const uint32_t nhead = (uint32_t)((a0 - g_lo) / sizeof(T)), ntail = (uint32_t)((g_hi - a1) / sizeof(T));
  if ((uint32_t)lane < nhead) xs[lane] = x[lo + lane];
  if ((uint32_t)lane < ntail) xs[w - ntail + lane] = x[lo + w - ntail + lane];
  __syncwarp();
  if (lane == 0) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    expect_tx(bar, (uint32_t)(a1 - a0));
    const uint32_t CH = 32768;
    for (uintptr_t off = a0; off < a1; off += CH) {
      const uint32_t n = (uint32_t)((a1 - off) < CH ? (a1 - off) : CH);
      bulk_g2s(xsm + (off - g0), reinterpret_cast<const void *>(off), n, bar);
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(NT, 1) split_rows(StripeParams<T> P) {
  using A = Acc<T>;
  using L = Layout<T>;
  constexpr int NS = L::NS;
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ uint64_t full[NS], empty[NS];
  __shared__ uint64_t xbar;
  __shared__ volatile int abort_flag;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t c0 = P.cta_first[blockIdx.x], nk = P.cta_first[blockIdx.x + 1] - c0;
  unsigned char *xsm = sm;
  auto slot = [&](uint32_t s) { return sm + L::XBYTES + (size_t)s * L::STAGE; };
  auto prod = [&](uint32_t s) {
    return reinterpret_cast<A *>(sm + L::XBYTES + (size_t)NS * L::STAGE + (size_t)s * L::PB);
  };

  if (threadIdx.x == 0) {
    for (int s = 0; s < NS; ++s) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&full[s])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&empty[s])), "r"(NCW) : "memory");
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&xbar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    abort_flag = 0;
  }
  __syncthreads();

  if (warp == NCW) {
    // ---------------- producer ----------------
    uint32_t cur = STRIPE_LIGHT, nx = 0, k = 0;
    for (; k < nk; ++k) {
      if (abort_flag) break;
      const StripeChunk c = P.chunks[c0 + k];
      const uint32_t s = k % NS;
      bool ok = true;
      if (lane == 0 && k >= NS) ok = wait_bar(&empty[s], ((k / NS) - 1) & 1u);  // chunk k - NS released
      if (c.stripe != STRIPE_LIGHT && c.stripe != cur) {
        // a new stripe replaces x once every consumer has released chunk k - 1
        if (lane == 0 && ok && k >= 1) ok = wait_bar(&empty[(k - 1) % NS], ((k - 1) / NS) & 1u);
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (ok) {
          const uint32_t lo = c.stripe * P.W, w = P.ncols - lo < P.W ? P.ncols - lo : P.W;
          stage_stripe<T>(P.x, lo, w, xsm, &xbar, lane);
          cur = c.stripe;
          ++nx;
        }
      }
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) {
        if (lane == 0) {
          if (P.err) atomicCAS(P.err, 0, SPARSEP_ETIMEDOUT);
          abort_flag = 1;
        }
        break;
      }
      if (lane == 0) {
        const bool heavy = c.stripe != STRIPE_LIGHT;
        const Win w = window<T>(c);
        unsigned char *st = slot(s);
        const uint32_t cbytes = heavy ? 2u : 4u;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        if (SP_BAD(P, w.r_n <= (uint32_t)L::RCAP + 8 && w.n_n * cbytes <= (uint32_t)L::CB &&
                          w.n_n * (uint32_t)sizeof(T) <= (uint32_t)L::VB &&
                          (uint64_t)w.r_lo + w.r_n <= (heavy ? P.n_vptr : P.n_lptr) &&
                          (uint64_t)w.n_lo + w.n_n <= (heavy ? P.n_h : P.n_l),
                   -1030)) {
          arrive(&full[s]);  // checked build: the phase completes without copies
        } else {
          expect_tx(&full[s], w.r_n * 4 + w.n_n * (cbytes + (uint32_t)sizeof(T)));
          bulk_g2s(st, (heavy ? P.vptr : P.lptr) + w.r_lo, w.r_n * 4, &full[s]);
          if (w.n_n) {
            if (heavy) bulk_g2s(st + L::RB, P.hcol + w.n_lo, w.n_n * 2, &full[s]);
            else bulk_g2s(st + L::RB, P.lcol + w.n_lo, w.n_n * 4, &full[s]);
            bulk_g2s(st + L::RB + L::CB, (heavy ? P.hval : P.lval) + w.n_lo, w.n_n * (uint32_t)sizeof(T), &full[s]);
          }
        }
      }
    }
    // the copies still in flight land (bounded) before the CTA may leave
    if (lane == 0) {
      for (uint32_t q = k > (uint32_t)NS ? k - NS : 0u; q < k; ++q) wait_bar(&full[q % NS], (q / NS) & 1u);
      if (nx) wait_bar(&xbar, (nx - 1) & 1u);
    }
    return;
  }

  // ---------------- consumers ----------------
  uint32_t cur = STRIPE_LIGHT, xph = 0;
  const T *xs = nullptr;
  // running sums of a row cut into pieces (warp 0): at most one heavy and one
  // light row are open at a time, the two chunk lists being interleaved
  A carry_h = A(0), carry_l = A(0);
  for (uint32_t k = 0; k < nk; ++k) {
    if (abort_flag) break;
    const StripeChunk c = P.chunks[c0 + k];
    const uint32_t s = k % NS;
    const bool heavy = c.stripe != STRIPE_LIGHT;
    bool ok = true;
    if (heavy && c.stripe != cur) {
      ok = wait_bar(&xbar, xph);
      xph ^= 1u;
      cur = c.stripe;
      xs = stripe_base(P.x, cur * P.W, xsm);
    }
    if (ok) ok = wait_bar(&full[s], (k / NS) & 1u);
    if (!__all_sync(0xffffffffu, ok)) {
      if (lane == 0) {
        if (P.err) atomicCAS(P.err, 0, SPARSEP_ETIMEDOUT);
        abort_flag = 1;
      }
      break;
    }
    const Win wn = window<T>(c);
    unsigned char *st = slot(s);
    const uint32_t off = c.n0 - wn.n_lo;
    const uint16_t *hc = reinterpret_cast<const uint16_t *>(st + L::RB) + off;
    const uint32_t *lc = reinterpret_cast<const uint32_t *>(st + L::RB) + off;
    T *vb = reinterpret_cast<T *>(st + L::RB + L::CB) + off;
    const uint32_t n = c.n1 - c.n0;
    const uint32_t sw = heavy ? (P.ncols - cur * P.W < P.W ? P.ncols - cur * P.W : P.W) : P.ncols;
    T *out = heavy ? P.part : P.y;
    const uint64_t out_n = heavy ? P.n_part : P.nrows;
    if (c.piece) {
      // one piece of a long row: warp 0 sums it and adds it in chunk order
      if (warp == 0) {
        A acc = A(0);
        for (uint32_t j = lane; j < n; j += 32) {
          uint32_t col = heavy ? hc[j] : lc[j];
          if (SP_BAD(P, col < sw, -1032)) col = 0;
          acc += mul<T>(vb[j], heavy ? xs[col] : __ldg(P.x + col));
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) {
          A &carry = heavy ? carry_h : carry_l;
          carry = (c.piece & 1u) ? acc : carry + acc;
          if ((c.piece & 2u) && !SP_BAD(P, c.v0 < out_n, -1033)) out[c.v0] = from_acc<T>(carry);
        }
      }
    } else {
      const uint32_t *srp = reinterpret_cast<const uint32_t *>(st) + (c.v0 - wn.r_lo);
      const uint32_t nr = c.v1 - c.v0, base = srp[0];
      // this warp's rows (those whose first nonzero is in its share of the
      // chunk's nonzeros), split on the host: rows [wsplit[w], wsplit[w+1])
      const uint16_t *ws = P.wsplit + (size_t)(c0 + k) * (NCW + 1);
      const uint32_t rb = min((uint32_t)ws[warp], nr), re = min((uint32_t)ws[warp + 1], nr);
      A *pr = L::IN_PLACE ? reinterpret_cast<A *>(vb) : prod(s);  // indexed from the chunk's first nonzero
      if (rb < re) {
        const uint32_t a = srp[rb] - base, b = min(srp[re] - base, n);
        // products, every x read of a lane issued before any use
        if (heavy) {
          constexpr int U = 4;
          for (uint32_t j0 = a + lane; j0 < b; j0 += 32 * U) {
            uint32_t cc[U];
            T xv[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
              const uint32_t j = j0 + 32 * u;
              cc[u] = j < b ? hc[j] : 0u;
              if (SP_BAD(P, cc[u] < sw, -1032)) cc[u] = 0;
            }
#pragma unroll
            for (int u = 0; u < U; ++u) xv[u] = xs[cc[u]];
#pragma unroll
            for (int u = 0; u < U; ++u)
              if (j0 + 32 * u < b) pr[j0 + 32 * u] = mul<T>(vb[j0 + 32 * u], xv[u]);
          }
        } else {
          constexpr int U = 8;
          for (uint32_t j0 = a + lane; j0 < b; j0 += 32 * U) {
            uint32_t cc[U];
            T xv[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
              const uint32_t j = j0 + 32 * u;
              cc[u] = j < b ? lc[j] : 0u;
              if (SP_BAD(P, cc[u] < sw, -1032)) cc[u] = 0;
            }
#pragma unroll
            for (int u = 0; u < U; ++u) xv[u] = __ldg(P.x + cc[u]);
#pragma unroll
            for (int u = 0; u < U; ++u)
              if (j0 + 32 * u < b) pr[j0 + 32 * u] = mul<T>(vb[j0 + 32 * u], xv[u]);
          }
        }
        __syncwarp();
        // row sums: a lane per short row, the warp per row longer than 32
        for (uint32_t i0 = rb; i0 < re; i0 += 32) {
          const uint32_t i = i0 + lane;
          const bool mine = i < re;
          const uint32_t rhi = mine ? min(srp[i + 1] - base, n) : 0u, rlo = mine ? min(srp[i] - base, rhi) : 0u;
          const bool lng = rhi - rlo > 32u;
          if (mine && !lng) {
            A sum = A(0);
            for (uint32_t q = rlo; q < rhi; ++q) sum += pr[q];
            if (!SP_BAD(P, c.v0 + i < out_n, -1033)) out[c.v0 + i] = from_acc<T>(sum);
          }
          unsigned m = __ballot_sync(0xffffffffu, lng);
          while (m) {
            const int src = __ffs(m) - 1;
            m &= m - 1;
            const uint32_t la = __shfl_sync(0xffffffffu, rlo, src), lb = __shfl_sync(0xffffffffu, rhi, src);
            A sum = A(0);
            for (uint32_t q = la + lane; q < lb; q += 32) sum += pr[q];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
            if (lane == 0 && !SP_BAD(P, c.v0 + i0 + src < out_n, -1033)) out[c.v0 + i0 + src] = from_acc<T>(sum);
          }
        }
      }
    }
    __syncwarp();
    if (lane == 0) arrive(&empty[s]);  // this warp is done with the slot
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
void stripe_geometry(uint32_t *width, size_t *smem, uint32_t *chunk_nnz, uint32_t *light_nnz, uint32_t *chunk_rows) {
  using L = stripes::Layout<T>;
  if (width) *width = L::W;
  if (smem) *smem = L::BYTES;
  if (chunk_nnz) *chunk_nnz = L::CAP;
  if (light_nnz) *light_nnz = L::CAP_L;
  if (chunk_rows) *chunk_rows = L::RCAP;
}

template <typename T>
cudaError_t launch_stripes(const StripeParams<T> &P, uint32_t ctas, cudaStream_t st) {
  if (ctas == 0) return cudaSuccess;
  auto k = stripes::split_rows<T>;
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
template void stripe_geometry<SPARSEP_KT>(uint32_t *, size_t *, uint32_t *, uint32_t *, uint32_t *);
template cudaError_t launch_stripes<SPARSEP_KT>(const StripeParams<SPARSEP_KT> &, uint32_t, cudaStream_t);
template cudaError_t launch_heavy_merge<SPARSEP_KT>(const SPARSEP_KT *, const uint32_t *, uint32_t, uint32_t,
                                                    SPARSEP_KT *, int, cudaStream_t);

}  // namespace sparsep
