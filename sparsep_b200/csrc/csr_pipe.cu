// csr_pipe.cu -- persistent, TMA-pipelined CSR SpMV for sm_100a (the 1D CSR
// path with automatic work items).
//
// Each CTA walks the items blockIdx.x, blockIdx.x + gridDim.x, ...  Thread 0 is
// the producer: for an item it issues bulk (TMA) copies of the item's rowptr
// slice, colind range and value range into one stage of an S-deep ring in
// shared memory, S-1 items ahead of the consumers; one transaction-count
// mbarrier per stage tracks completion.  The consumers (all threads) gather x
// for the staged nonzeros -- CAP / blockDim independent loads per thread in
// flight -- multiply into a product array, then sum rows from shared memory:
// a thread per short row, a warp per long row, consecutive threads writing
// consecutive rows of y.  Chunks of a row longer than CAP (ITEM_LONG) are
// block-reduced; chunk 0 stores the row and the others leave carries that the
// last CTA to finish adds in chunk order (deterministic).
//
// Same arithmetic as the reference (spmv/1D/CSR-row/host/app.c:66-77).  The
// planner sizes items so each fits one stage (<= CAP nonzeros, <= RCAP rows).
// Waits are bounded: one that runs out records SPARSEP_ETIMEDOUT, and the CTA
// waits (bounded) for its copies in flight before it returns.
#include <atomic>
#include "device.cuh"
#include "kernels.hpp"

namespace sparsep {
namespace pipe {

constexpr int NT = 256;  // threads per CTA
constexpr unsigned long long NO_CARRY = ~0ull;

// CAP nonzeros / CAP/4 rows per stage; the smaller stage fits six CTAs per SM
template <typename T, int CAP_> struct Layout {
  static constexpr int CAP = CAP_;
  static constexpr int RCAP = CAP_ / 4;
  static constexpr int PER = CAP_ / NT;
  // colind and values are staged from the same element index, aligned so both
  // copies start on 16 bytes: ALIGN = max(4, 16 / sizeof(T)) elements
  static constexpr int ALIGN = (16 / (int)sizeof(T)) > 4 ? (16 / (int)sizeof(T)) : 4;
  static constexpr int RBUF = RCAP + 8;        // rowptr slots (+ alignment slack)
  static constexpr int CBUF = CAP + 2 * ALIGN;  // colind slots
  static constexpr int VBUF = CAP + 2 * ALIGN;  // value slots
  static constexpr size_t RBYTES = RBUF * 4;
  static constexpr size_t CBYTES = CBUF * 4;
  static constexpr size_t VBYTES = ((size_t)VBUF * sizeof(T) + 15) & ~(size_t)15;
  static constexpr size_t STAGE = RBYTES + CBYTES + VBYTES;
  // narrow element types keep their 32-bit products in a separate array
  static constexpr bool IN_PLACE = sizeof(T) == sizeof(Acc<T>);
  static constexpr size_t PBYTES = IN_PLACE ? 0 : (size_t)CAP * sizeof(Acc<T>);
  static size_t bytes(int S) { return STAGE * S + PBYTES; }
};

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

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

// 16-byte aligned copy windows of an item: rowptr [a0, a1] of the tile,
// colind / values [n0, n1).  lo = first copied index, n = copied count.
struct Win {
  uint64_t r_lo, c_lo, v_lo;
  uint32_t r_n, c_n, v_n;
};

template <typename T>
__device__ __forceinline__ Win window(const Item &it) {
  constexpr uint64_t VA = Layout<T, 2048>::ALIGN;
  Win w;
  if (it.kind == ITEM_LONG) {
    w.r_lo = 0;
    w.r_n = 0;
  } else {
    const uint64_t p0 = it.ptr_base + it.a0, p1 = it.ptr_base + it.a1 + 1;
    w.r_lo = p0 & ~3ull;
    w.r_n = (uint32_t)(((p1 + 3) & ~3ull) - w.r_lo);
  }
  w.c_lo = w.v_lo = it.n0 / VA * VA;
  w.c_n = w.v_n = it.n1 > it.n0 ? (uint32_t)((it.n1 + VA - 1) / VA * VA - w.c_lo) : 0;
  return w;
}

template <typename T, int S, int CAP_>
__global__ void __launch_bounds__(NT, CAP_ <= 2048 ? 5 : 3) csr_pipe(Params<T> P) {
  using A = Acc<T>;
  using L = Layout<T, CAP_>;
  constexpr int CAP = L::CAP, RCAP = L::RCAP, PER = L::PER;
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ uint64_t full[S];
  __shared__ A red[NT / 32];
  __shared__ KV<Acc<T>, 1> scan[NT / 32];
  __shared__ int abort_flag;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t stride = gridDim.x;
  auto stage_ptr = [&](uint32_t s) { return sm + (size_t)s * L::STAGE; };
  // products: in place of the staged values when the widths match
  A *prs = reinterpret_cast<A *>(sm + (size_t)S * L::STAGE);

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&full[s])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    abort_flag = 0;
  }
  __syncthreads();

  // producer: stage local item k (global id blockIdx.x + k*stride)
  auto issue = [&](uint32_t k) {
    const uint64_t g = blockIdx.x + (uint64_t)k * stride;
    if (g >= P.nitems) return;
    const Item it = P.items[g];
    const Win w = window<T>(it);
    const uint32_t s = k % S;
    unsigned char *st = stage_ptr(s);
    const uint32_t bytes = w.r_n * 4 + w.c_n * 4 + w.v_n * (uint32_t)sizeof(T);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (SP_BAD(P, w.r_n <= (uint32_t)L::RBUF && w.c_n <= (uint32_t)L::CBUF && w.v_n <= (uint32_t)L::VBUF, -1019)) {
      // an oversized item is skipped: complete the phase without copies
      asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&full[s])) : "memory");
      return;
    }
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(&full[s])), "r"(bytes)
                 : "memory");
    if (w.r_n) bulk_g2s(st, P.rowptr + w.r_lo, w.r_n * 4, &full[s]);
    if (w.c_n) bulk_g2s(st + L::RBYTES, P.colind + w.c_lo, w.c_n * 4, &full[s]);
    if (w.v_n) bulk_g2s(st + L::RBYTES + L::CBYTES, P.val + w.v_lo, w.v_n * (uint32_t)sizeof(T), &full[s]);
  };

  if (threadIdx.x == 0)
    for (int k = 0; k < S - 1; ++k) issue(k);

  uint32_t k = 0;
  for (;; ++k) {
    const uint64_t g = blockIdx.x + (uint64_t)k * stride;
    if (g >= P.nitems) break;
    const Item it = P.items[g];
    if (threadIdx.x == 0) issue(k + S - 1);  // into the stage item k-1 released
    const Win w = window<T>(it);
    const uint32_t s = k % S;
    unsigned char *st = stage_ptr(s);
    if (!wait_bar(&full[s], (k / S) & 1u)) {
      if (P.err) atomicCAS(P.err, 0, SPARSEP_ETIMEDOUT);
      abort_flag = 1;
    }
    __syncthreads();
    if (abort_flag) break;
    const uint32_t *srp = reinterpret_cast<const uint32_t *>(st) + (it.ptr_base + it.a0 - w.r_lo);
    const uint32_t *cb = reinterpret_cast<const uint32_t *>(st + L::RBYTES) + (it.n0 - w.c_lo);
    T *vb = reinterpret_cast<T *>(st + L::RBYTES + L::CBYTES) + (it.n0 - w.v_lo);
    A *pr = L::IN_PLACE ? reinterpret_cast<A *>(vb) : prs;
    const uint32_t n = (uint32_t)(it.n1 - it.n0);
    if (SP_BAD(P, n <= (uint32_t)CAP && (it.kind == ITEM_LONG || (it.a1 > it.a0 && it.a1 - it.a0 <= RCAP)), -1019)) {
      __syncthreads();
      continue;
    }

    // products of the staged nonzeros: all x gathers of a thread in flight
    // before any use; consecutive threads on consecutive slots
    A acc = A(0);
    {
      uint32_t col[PER];
      T xv[PER];
#pragma unroll
      for (int u = 0; u < PER; ++u) {
        const uint32_t j = threadIdx.x + u * NT;
        col[u] = j < n ? cb[j] : 0u;
      }
#pragma unroll
      for (int u = 0; u < PER; ++u) {
        const uint32_t j = threadIdx.x + u * NT;
        const uint64_t c = (uint64_t)it.col_off + col[u];
        xv[u] = (j < n && !SP_BAD(P, c < P.n_x, -1003)) ? __ldg(P.x + c) : T(0);
      }
#pragma unroll
      for (int u = 0; u < PER; ++u) {
        const uint32_t j = threadIdx.x + u * NT;
        if (j < n) {
          const A p = mul<T>(vb[j], xv[u]);
          if (it.kind == ITEM_LONG) acc += p;
          else pr[j] = p;
        }
      }
    }
    T *out = P.y;
    if (it.kind == ITEM_LONG) {
      // one chunk of a long row: block reduction; the last chunk to arrive sums
      // the row's chunk partials in chunk order
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (lane == 0) red[warp] = acc;
      __syncthreads();
      if (threadIdx.x == 0) {
        A tot = A(0);
        for (int q = 0; q < NT / 32; ++q) tot += red[q];
        if (!SP_BAD(P, it.crow < P.nrows && it.first + it.nchunk <= P.nitems && g < P.n_carry, -1007)) {
          P.carry_val[g] = acc_bits(tot);
          __threadfence();
          const unsigned int prev = atomicAdd(P.row_cnt + it.cslot, 1u);
          if (prev == it.nchunk - 1) {
            __threadfence();
            A sum = A(0);
            for (uint32_t c = 0; c < it.nchunk; ++c) sum += bits_acc<A>(__ldcg(P.carry_val + it.first + c));
            out[it.crow] = from_acc<T>(sum);
            P.row_cnt[it.cslot] = 0;  // ready for the next launch
          }
        }
      }
    } else {
      // rows [a0, a1): merge path over the nr row ends and n nonzeros; every
      // thread takes the same number of steps, a step either adds a product
      // or closes a row.  Runs crossing threads are completed by the block
      // segmented scan.
      __syncthreads();
      const uint32_t nr = (uint32_t)(it.a1 - it.a0), base = srp[0];
      const uint32_t M = nr + n, ipt = (M + NT - 1) / NT;
      const uint32_t d0 = min(threadIdx.x * ipt, M), d1 = min(d0 + ipt, M);
      uint32_t lo = d0 > n ? d0 - n : 0u, hi = d0 < nr ? d0 : nr;
      while (lo < hi) {  // first row whose end is past the nonzero index on this diagonal
        const uint32_t m = (lo + hi) >> 1;
        if (srp[m + 1] - base <= d0 - m - 1) lo = m + 1; else hi = m;
      }
      uint32_t i = lo, j = d0 - lo;
      uint32_t rend = i < nr ? srp[i + 1] - base : 0xFFFFFFFFu;
      const uint64_t orow = (uint64_t)it.row_off + it.a0;
      const uint32_t head = i;
      bool closed = false;
      A head_acc = A(0);
      A run = A(0);
      for (uint32_t d = d0; d < d1; ++d) {
        if (j < rend) {
          run += pr[j];
          ++j;
        } else {
          if (!closed) {
            head_acc = run;
            closed = true;
          } else {
            out[orow + i] = from_acc<T>(run);
          }
          run = A(0);
          ++i;
          rend = i < nr ? srp[i + 1] - base : 0xFFFFFFFFu;
        }
      }
      KV<A, 1> mine, init, ex, in;
      mine.k = i;  // the open row at the end of the thread's steps (nr = none)
      mine.v[0] = run;
      init.k = -1;
      init.v[0] = A(0);
      block_seg_scan<A, 1>(mine, init, ex, in, scan);
      (void)in;
      if (closed) out[orow + head] = from_acc<T>(head_acc + (ex.k == (long long)head ? ex.v[0] : A(0)));
      if (P.carry_idx && threadIdx.x == 0 && !SP_BAD(P, g < P.n_carry, -1018)) P.carry_idx[g] = NO_CARRY;
    }
    __syncthreads();  // the stage may be refilled after this point
  }

  // after an abort, wait (bounded) for copies this CTA still has in flight
  if (threadIdx.x == 0 && abort_flag) {
    for (uint32_t q = k; q < k + S; ++q) {
      const uint64_t g = blockIdx.x + (uint64_t)q * stride;
      if (g >= P.nitems) break;
      wait_bar(&full[q % S], (q / S) & 1u);
    }
  }
}

}  // namespace pipe

// Stages per element type: as many as fit with 3 CTAs per SM for the 4-byte
// types (2 stages), 2 CTAs for the 8-byte types.
template <typename T> constexpr int pipe_stages() { return 2; }

template <typename T, int CAP>
static cudaError_t launch_cap(const Params<T> &P, int sms, cudaStream_t st, int *grid_out) {
  constexpr int S = pipe_stages<T>();
  auto k = pipe::csr_pipe<T, S, CAP>;
  const size_t smem = pipe::Layout<T, CAP>::bytes(S);
  // the shared-memory attribute, set once per device (concurrent host threads allowed)
  static std::atomic<unsigned long long> set_on{0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = 1ull << (dev & 63);
  if (!(set_on.load() & bit)) {
    e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    set_on.fetch_or(bit);
  }
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, pipe::NT, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) per_sm = 1;
  uint64_t grid = (uint64_t)sms * per_sm;
  if (grid > P.nitems) grid = P.nitems;
  if (grid_out) *grid_out = (int)grid;
  k<<<(unsigned)grid, pipe::NT, smem, st>>>(P);
  return cudaGetLastError();
}

// items of at most 2048 nonzeros (and 512 rows) take the small-stage kernel
template <typename T>
cudaError_t launch_csr_pipe(const Params<T> &P, int sms, cudaStream_t st, int *grid_out, uint32_t max_item_nnz) {
  if (P.nitems == 0) return cudaSuccess;
  if (max_item_nnz <= 2048) return launch_cap<T, 2048>(P, sms, st, grid_out);
  return launch_cap<T, 4096>(P, sms, st, grid_out);
}

#ifndef SPARSEP_KT
#define SPARSEP_KT float
#endif
template cudaError_t launch_csr_pipe<SPARSEP_KT>(const Params<SPARSEP_KT> &, int, cudaStream_t, int *, uint32_t);

}  // namespace sparsep
