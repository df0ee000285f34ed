// device.cuh -- device-side building blocks of the sparsep_b200 SpMV kernels:
// accumulator types with the reference's wrap-around semantics, streaming
// loads, typed atomics, the work-item descriptor and the block-wide
// segmented (reduce-by-key) scan used by the lock-free COO / BCOO paths.
#pragma once
#include <cstdint>
#include <type_traits>
#include <cuda_runtime.h>

#include "sparsep.h"

namespace sparsep {

// ---------------------------------------------------------------------------
// Accumulators.  The reference sums `val_dt sum += x * val` in the element type
// (spmv/1D/CSR-row/host/app.c:66-77), so integer results are the exact sum
// modulo 2^w.  Summing in a wider unsigned type and truncating once is the same
// value modulo 2^w in every order, which makes every GPU order bit-exact.
// ---------------------------------------------------------------------------
template <typename T> struct AccOf;
template <> struct AccOf<int8_t> { using type = uint32_t; };
template <> struct AccOf<int16_t> { using type = uint32_t; };
template <> struct AccOf<int32_t> { using type = uint32_t; };
template <> struct AccOf<int64_t> { using type = unsigned long long; };
template <> struct AccOf<float> { using type = float; };
template <> struct AccOf<double> { using type = double; };
template <typename T> using Acc = typename AccOf<T>::type;

template <typename T> __device__ __forceinline__ Acc<T> to_acc(T v) {
  if constexpr (std::is_integral<T>::value) {
    using S = typename std::conditional<sizeof(T) == 8, long long, int>::type;
    return (Acc<T>)(S)v;  // sign-extend, then reinterpret as unsigned
  } else {
    return v;
  }
}
template <typename T> __device__ __forceinline__ T from_acc(Acc<T> a) { return (T)a; }
template <typename T> __device__ __forceinline__ Acc<T> mul(T a, T b) { return to_acc(a) * to_acc(b); }

// Carries are kept in a 64-bit slot whatever the accumulator.
template <typename A> __device__ __forceinline__ unsigned long long acc_bits(A a) {
  if constexpr (sizeof(A) == 8) return *reinterpret_cast<unsigned long long *>(&a);
  else return (unsigned long long)*reinterpret_cast<uint32_t *>(&a);
}
template <typename A> __device__ __forceinline__ A bits_acc(unsigned long long b) {
  if constexpr (sizeof(A) == 8) return *reinterpret_cast<A *>(&b);
  else { uint32_t u = (uint32_t)b; return *reinterpret_cast<A *>(&u); }
}

// ---------------------------------------------------------------------------
// Loads: matrix arrays are streamed once (evict-first), x is reused (default).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint4 ld_stream4(const void *p) {
  return __ldcs(reinterpret_cast<const uint4 *>(p));
}
__device__ __forceinline__ uint32_t ld_stream1(const uint32_t *p) { return __ldcs(p); }

// Four consecutive elements starting at a 4-element-aligned index.
template <typename T> struct Vec4 { T v[4]; };
template <typename T> __device__ __forceinline__ Vec4<T> ld_vals4(const T *p) {
  Vec4<T> r;
  if constexpr (sizeof(T) == 1) {
    uint32_t w = __ldcs(reinterpret_cast<const unsigned int *>(p));
    for (int k = 0; k < 4; ++k) r.v[k] = (T)(int8_t)(w >> (8 * k));
  } else if constexpr (sizeof(T) == 2) {
    uint2 w = __ldcs(reinterpret_cast<const uint2 *>(p));
    r.v[0] = (T)(int16_t)(w.x & 0xFFFF);
    r.v[1] = (T)(int16_t)(w.x >> 16);
    r.v[2] = (T)(int16_t)(w.y & 0xFFFF);
    r.v[3] = (T)(int16_t)(w.y >> 16);
  } else if constexpr (sizeof(T) == 4) {
    uint4 w = ld_stream4(p);
    r.v[0] = __builtin_bit_cast(T, w.x);
    r.v[1] = __builtin_bit_cast(T, w.y);
    r.v[2] = __builtin_bit_cast(T, w.z);
    r.v[3] = __builtin_bit_cast(T, w.w);
  } else {
    uint4 a = ld_stream4(p), b = ld_stream4(reinterpret_cast<const char *>(p) + 16);
    r.v[0] = __builtin_bit_cast(T, ((unsigned long long)a.y << 32) | a.x);
    r.v[1] = __builtin_bit_cast(T, ((unsigned long long)a.w << 32) | a.z);
    r.v[2] = __builtin_bit_cast(T, ((unsigned long long)b.y << 32) | b.x);
    r.v[3] = __builtin_bit_cast(T, ((unsigned long long)b.w << 32) | b.z);
  }
  return r;
}

template <typename T> __device__ __forceinline__ T ldx(const T *p) { return __ldg(p); }

// ---------------------------------------------------------------------------
// Typed atomic add (red.global) with wrap-around for integers.  int8 / int16
// have no native form: a CAS loop on the containing 32-bit word updates only
// the addressed lane, which is exact because integer addition modulo 2^w does
// not depend on order.
// ---------------------------------------------------------------------------
template <typename T> __device__ __forceinline__ void atomic_add_out(T *p, Acc<T> v) {
  if constexpr (std::is_same<T, float>::value) {
    atomicAdd(p, v);
  } else if constexpr (std::is_same<T, double>::value) {
    atomicAdd(p, v);
  } else if constexpr (sizeof(T) == 4) {
    atomicAdd(reinterpret_cast<unsigned int *>(p), (unsigned int)v);
  } else if constexpr (sizeof(T) == 8) {
    atomicAdd(reinterpret_cast<unsigned long long *>(p), (unsigned long long)v);
  } else {
    uintptr_t a = reinterpret_cast<uintptr_t>(p);
    unsigned int *w = reinterpret_cast<unsigned int *>(a & ~(uintptr_t)3);
    int shift = (int)(a & 3) * 8;
    unsigned int mask = (sizeof(T) == 1 ? 0xFFu : 0xFFFFu) << shift;
    unsigned int old = *w, assumed;
    do {
      assumed = old;
      unsigned int lane = (assumed & mask) >> shift;
      unsigned int nl = ((lane + (unsigned int)v) << shift) & mask;
      old = atomicCAS(w, assumed, (assumed & ~mask) | nl);
    } while (old != assumed);
  }
}

// ---------------------------------------------------------------------------
// Work items.  One CTA executes one item (or a persistent CTA a sequence).
// ---------------------------------------------------------------------------
enum ItemKind : uint16_t {
  ITEM_ROWS = 0,   // CSR rows / BCSR block rows [a0, a1) of a tile
  ITEM_LONG = 1,   // CSR: elements [a0, a1) of one long row `crow` (chunk `chunk`)
  ITEM_ELEMS = 2,  // COO elements / BCOO blocks [a0, a1), owning output rows [own0, own1)
};

enum OutMode : int { OUT_DIRECT = 0, OUT_PARTIAL = 1, OUT_ATOMIC = 2 };

struct Item {
  uint64_t a0, a1;      // see ItemKind
  uint64_t ptr_base;    // CSR/BCSR: (b)rowptr index of the tile's local row 0
  uint64_t nnz_base;    // CSR/BCSR: added to local (b)rowptr values
  uint32_t row_off;     // output row of tile-local row 0 (BCSR/BCOO: of local block row 0, in rows)
  uint32_t col_off;     // x column of tile-local column 0
  uint32_t own0, own1;  // ITEM_ELEMS: owned output rows (BCOO: block rows relative to row_off/rb)
  uint32_t xlo, xw;     // stage x[xlo, xlo+xw) in shared memory when xw > 0
  uint32_t slot;        // partial-y slice (2D lock-free)
  uint16_t kind, lanes;
  uint32_t crow;        // ITEM_LONG: output row
  uint32_t chunk;       // ITEM_LONG: chunk index within the row (0 owns the row)
  uint32_t worker_bal;  // ITEM_ROWS: sparsep_balance across warps
  uint32_t row_end;     // exclusive bound on output rows this item may write
  uint64_t n0, n1;      // CSR: absolute nonzero range of the item (for bulk prefetch)
  uint32_t nchunk;      // ITEM_LONG: chunks of the row
  uint32_t first;       // ITEM_LONG: item index of the row's chunk 0
  uint32_t cslot;       // ITEM_LONG: the row's arrival counter
  uint32_t band;        // row band of y the item writes (host-buffer path, see Params::band_cnt)
};

// Per-launch parameters shared by all kernels.
template <typename T> struct Params {
  const Item *items;
  uint32_t nitems;
  uint32_t nrows;        // rows of y (and of each partial slice)
  uint32_t ncols;        // columns of x (block columns past it read as zero)
  // CSR / 2D CSR
  const uint32_t *rowptr;
  const uint32_t *colind;
  const T *val;
  // COO (AoS, reference elem_t layout)
  const void *elems;
  // BCSR / BCOO
  const uint32_t *bcolind;
  const sparsep_bind *bind;
  const T *bval;
  uint32_t rb, cb;
  // vectors
  const T *x;
  T *y;
  T *part;               // OUT_PARTIAL: slices of nrows
  int out_mode;
  // scratch (lock-free carries)
  unsigned long long *carry_val;
  unsigned long long *carry_idx;  // output index or ~0ull
  unsigned int *done;             // completion counter, reset by the last CTA
  unsigned int *row_cnt;          // per long row arrival counters (pipelined CSR)
  unsigned int *band_cnt;         // when set: items finished per row band of y (one counter per band)
  int *err;                       // device error word (bounded waits, checked builds)
  // array extents, used by the bounds-checked build (-DSPARSEP_CHECK)
  uint64_t n_rowptr, n_idx, n_val, n_elems, n_x, n_xalloc, n_carry;
  uint32_t nslots, smem_bytes;
  int fault_wait;  // test support: add a staging wait that nothing completes (after the copy)
};

// ---------------------------------------------------------------------------
// Split CSR plans (csr_stripes.cu).  The heavy rows (nH of them) are laid out
// stripe-major: stripe row v = s * nH + k holds the nonzeros of heavy row k
// whose columns fall in stripe s (columns [s*W, s*W + W)), with 16-bit
// stripe-local columns; its sum is the partial part[v], and
// y[hrow[k]] = sum over s of part[s*nH + k].  The light rows stay a CSR
// (heavy rows empty there) whose chunks write y directly.
// ---------------------------------------------------------------------------
constexpr uint32_t STRIPE_LIGHT = 0xFFFFFFFFu;  // StripeChunk::stripe of a light chunk
constexpr uint32_t SPLIT_WARPS = 31;            // consumer warps of the split kernel (one more produces)

struct StripeChunk {
  uint32_t n0, n1;  // nonzeros [n0, n1) of the heavy (stripe-major) or light arrays
  uint32_t v0, v1;  // stripe rows (heavy) or rows (light) [v0, v1); a piece has v1 = v0 + 1
  uint32_t stripe;  // x columns [stripe * W, stripe * W + W); STRIPE_LIGHT for light rows
  uint32_t piece;   // 0: whole rows; a piece of row v0 has bit 2 set, bit 0 on its
                    // first piece and bit 1 on its last
};

template <typename T> struct StripeParams {
  const StripeChunk *chunks;
  const uint32_t *cta_first;  // chunks [cta_first[b], cta_first[b+1]) run on CTA b, in order
  const uint16_t *wsplit;     // per chunk 32 row boundaries: consumer warp w takes rows [w, w+1)
  const uint32_t *vptr;       // heavy: nS * nH + 1 offsets into hcol / hval
  const uint16_t *hcol;       // heavy: stripe-local columns
  const T *hval;
  const uint32_t *lptr;       // light: nrows + 1 offsets into lcol / lval
  const uint32_t *lcol;
  const T *lval;
  const T *x;
  T *y;
  T *part;                    // nS * nH partial sums
  uint32_t ncols, nrows, W;
  int *err;
  uint64_t n_vptr, n_h, n_lptr, n_l, n_part;  // allocated extents (checked build)
};

// Bounds checks of the checked build: a failed check records `code` in the
// error word (first failure wins) and the caller skips the access.  The
// release build compiles them away.
__device__ __forceinline__ bool sp_flag(int *err, int code) {
  if (err) atomicCAS(err, 0, code);
  return true;
}
#ifdef SPARSEP_CHECK
#define SP_BAD(P, cond, code) (!(cond) && ::sparsep::sp_flag((P).err, (code)))
#else
#define SP_BAD(P, cond, code) false
#endif

template <typename T> __device__ __forceinline__ T *out_base(const Params<T> &P, const Item &it) {
  return P.out_mode == OUT_PARTIAL ? P.part + (size_t)it.slot * P.nrows : P.y;
}

// ---------------------------------------------------------------------------
// Shared-memory staging of an x-segment with a bulk (TMA) copy.
// The global range is widened to 16-byte boundaries (the copy's alignment
// rule); callers pass a buffer with >= 16 bytes of slack past its last column.
// Returns the shared pointer p such that p[c] is x[c] for c in [lo, lo+w).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Test support (sparsep_test_wait_fault): once the CTA's own copies have
// landed, thread 0 arms one more phase of `mbar` for 16 bytes that no copy
// brings; the CTA's bounded wait on it (1024 tries) runs out and records
// SPARSEP_ETIMEDOUT, then thread 0 completes the phase itself, so the barrier
// is left clean and nothing is in flight.
__device__ __forceinline__ void inject_wait_timeout(uint64_t *mbar, uint32_t &phase, int *err) {
  __syncthreads();
  if (threadIdx.x == 0)
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(mbar)), "r"(16u)
                 : "memory");
  uint32_t done = 0;
  for (uint32_t it = 0; it < (1u << 10) && !done; ++it) {
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(smem_u32(mbar)), "r"(phase)
        : "memory");
  }
  if (!__syncthreads_or(done) && threadIdx.x == 0 && err) atomicExch(err, SPARSEP_ETIMEDOUT);
  if (threadIdx.x == 0)
    asm volatile("mbarrier.complete_tx.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(16u) : "memory");
  __syncthreads();
  phase ^= 1u;
}

template <typename T>
__device__ const T *stage_x(const T *x, uint32_t lo, uint32_t w, unsigned char *smem, uint64_t *mbar,
                            uint32_t &phase, int *err, uint32_t smem_cap, uintptr_t x_end, int fault = 0) {
  (void)smem_cap;
  (void)x_end;
  uintptr_t gb = reinterpret_cast<uintptr_t>(x) + (uintptr_t)lo * sizeof(T);
  uintptr_t g0 = gb & ~(uintptr_t)15;
  uintptr_t g1 = (gb + (uintptr_t)w * sizeof(T) + 15) & ~(uintptr_t)15;
  uint32_t bytes = (uint32_t)(g1 - g0);
#ifdef SPARSEP_CHECK
  if (bytes > smem_cap || g1 > x_end) {
    if (threadIdx.x == 0 && err) atomicCAS(err, 0, -1017);
    phase ^= 1u;
    return x;
  }
#endif
  if (threadIdx.x == 0) {
    // order earlier generic-proxy reads of this buffer before the async writes
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(mbar)), "r"(bytes)
                 : "memory");
    const uint32_t CH = 32768;
    for (uint32_t off = 0; off < bytes; off += CH) {
      uint32_t n = bytes - off < CH ? bytes - off : CH;
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
              smem_u32(smem + off)),
          "l"(g0 + off), "r"(n), "r"(smem_u32(mbar))
          : "memory");
    }
  }
  // bounded wait on the barrier phase
  uint32_t done = 0;
  for (uint32_t it = 0; it < (1u << 24) && !done; ++it) {
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(smem_u32(mbar)), "r"(phase)
        : "memory");
  }
  if (!done && err) atomicExch(err, SPARSEP_ETIMEDOUT);
  phase ^= 1u;
  if (fault && done) inject_wait_timeout(mbar, phase, err);
  return reinterpret_cast<const T *>(smem + (gb - g0)) - lo;
}

__device__ __forceinline__ void mbar_init(uint64_t *mbar) {
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Block-wide segmented scan over (key, W values) with keys non-decreasing in
// thread order:  (k1,v1) o (k2,v2) = (k2, v2 + [k1 == k2] v1).  Associative
// for sorted keys.  Returns each thread's exclusive prefix (the sum of the
// run of equal keys that ends just before the thread) and its inclusive one.
// `init` seeds thread 0 (the previous chunk's tail).
// ---------------------------------------------------------------------------
template <typename A, int W> struct KV {
  long long k;
  A v[W];
};

template <typename A, int W>
__device__ __forceinline__ KV<A, W> kv_op(const KV<A, W> &l, const KV<A, W> &r) {
  KV<A, W> o;
  o.k = r.k;
  bool same = (l.k == r.k);
#pragma unroll
  for (int i = 0; i < W; ++i) o.v[i] = r.v[i] + (same ? l.v[i] : A(0));
  return o;
}

template <typename A, int W>
__device__ __forceinline__ KV<A, W> kv_shfl_up(const KV<A, W> &a, int d) {
  KV<A, W> o;
  o.k = __shfl_up_sync(0xffffffffu, a.k, d);
#pragma unroll
  for (int i = 0; i < W; ++i) o.v[i] = __shfl_up_sync(0xffffffffu, a.v[i], d);
  return o;
}

// smem: at least (blockDim.x/32) KV entries.
template <typename A, int W>
__device__ void block_seg_scan(const KV<A, W> &mine, const KV<A, W> &init, KV<A, W> &excl, KV<A, W> &incl,
                               KV<A, W> *smem) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  KV<A, W> x = mine;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    KV<A, W> y = kv_shfl_up(x, d);
    if (lane >= d) x = kv_op(y, x);
  }
  if (lane == 31) smem[warp] = x;
  __syncthreads();
  KV<A, W> wpre = init;
  for (int w = 0; w < warp; ++w) wpre = kv_op(wpre, smem[w]);
  KV<A, W> up = kv_shfl_up(x, 1);
  excl = (lane == 0) ? wpre : kv_op(wpre, up);
  incl = kv_op(wpre, x);
  __syncthreads();
  (void)nw;
}

}  // namespace sparsep
