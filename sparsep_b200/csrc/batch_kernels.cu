// batch_kernels.cu -- the kernel of the batched multi-RHS SpMV: many CSR
// matrices with 1..256 right-hand sides each, one launch per batch.
//
// A work item is a row range of one matrix holding at most BCAP nonzeros (or
// one longer row, processed in BCAP-sized chunks), and carries that matrix's
// array pointers.  A CTA runs one item: one thread issues TMA bulk copies of
// the item's rowptr slice, column indices and values into shared memory
// (16-byte aligned windows, completion on an mbarrier with a bounded wait),
// so the whole item arrives in one memory round trip; afterwards only the x
// gathers go to memory.  In the batch launch, CTAs claim items from a global
// counter (atomicAdd, no waiting) in queue order -- long rows first -- so
// matrices of very different sizes share the GPU without per-matrix launch
// gaps or tails.
//
// Row routines, chosen per matrix (the autotuner picks among them).  The CTA
// is cut into groups of G lanes; lane l of a group reads right-hand sides
// [(l + aG)V, (l + aG)V + V) of each nonzero's x row with one V-wide load
// (V in 1, 2, 4; k % V == 0), a < ACC, V * ACC <= 8 accumulators.
//   Rows mode: the item's rows dealt round-robin to the groups.
//   Merge mode: the item's row ends and nonzeros split evenly over the groups
//     along the merge path; rows cut by a split are finished from the
//     groups' carries, in group order.
//   Long rows (> BCAP nonzeros): the whole CTA, groups of G lanes striding
//     over each staged chunk, then a fixed-order reduction over the groups.
// Same arithmetic as the single-vector path: integers accumulate in 32-bit
// unsigned and wrap exactly; FP in the element type, each row's products
// summed in a fixed order (deterministic from run to run).
#include "batch.hpp"
#include "device.cuh"

namespace sparsep {
namespace batch {

constexpr uint32_t RP_N = BRCAP + 16;  // staged rowptr window (+ alignment lead and tail)
constexpr uint32_t NZ_N = BCAP + 8;    // staged colind / values window

template <typename T> struct BShared {
  alignas(16) uint32_t rp[RP_N];
  alignas(16) uint32_t col[NZ_N];  // after the compute: carries / long-row partials (<= BCAP accumulators)
  alignas(16) T val[NZ_N];
  alignas(8) uint64_t bar;
  unsigned next;
};

// The item's matrix, typed.
template <typename T> struct View {
  const T *x;
  T *y;
  uint32_t k;
  uint32_t ncols;
};

// The staged arrays, indexed from the item's first row / nonzero.
template <typename T> struct Staged {
  const uint32_t *rp;  // rp[i] = rowptr[r0 + i]
  const uint32_t *col; // col[q] = colind[p0 + q]
  const T *val;
  uint32_t n;          // staged nonzeros
  int *err;
};

// Index guards: a failed check records its site code in the error word
// (read by sparsep_batch_status) and the guarded work is skipped, so a
// corrupted item or column index cannot take the GPU down.  The per-item ones
// (staging windows, staged rowptr ends, every staged column inside x) are
// always on; the checked build (-DSPARSEP_CHECK) adds a full scan of each
// staged rowptr slice.
__device__ __forceinline__ bool bchk(bool ok, int *err, int code) {
  if (!ok && err) atomicCAS(err, 0, code);
  return ok;
}

template <typename T, int V> struct VecT;
template <typename T> struct VecT<T, 1> {
  T v[1];
  static __device__ __forceinline__ VecT load(const T *p) {
    VecT r;
    r.v[0] = __ldg(p);
    return r;
  }
};
template <typename T> struct VecT<T, 2> {
  T v[2];
  static __device__ __forceinline__ VecT load(const T *p) {
    VecT r;
    if constexpr (std::is_same<T, float>::value) {
      const float2 q = __ldg(reinterpret_cast<const float2 *>(p));
      r.v[0] = q.x, r.v[1] = q.y;
    } else {
      const int2 q = __ldg(reinterpret_cast<const int2 *>(p));
      r.v[0] = (T)q.x, r.v[1] = (T)q.y;
    }
    return r;
  }
};
template <typename T> struct VecT<T, 4> {
  T v[4];
  static __device__ __forceinline__ VecT load(const T *p) {
    VecT r;
    if constexpr (std::is_same<T, float>::value) {
      const float4 q = __ldg(reinterpret_cast<const float4 *>(p));
      r.v[0] = q.x, r.v[1] = q.y, r.v[2] = q.z, r.v[3] = q.w;
    } else {
      const int4 q = __ldg(reinterpret_cast<const int4 *>(p));
      r.v[0] = (T)q.x, r.v[1] = (T)q.y, r.v[2] = (T)q.z, r.v[3] = (T)q.w;
    }
    return r;
  }
};

template <typename T, int V> __device__ __forceinline__ void store_vec(T *p, const Acc<T> *a) {
  if constexpr (V == 4 && std::is_same<T, float>::value) {
    *reinterpret_cast<float4 *>(p) = make_float4(a[0], a[1], a[2], a[3]);
  } else if constexpr (V == 2 && std::is_same<T, float>::value) {
    *reinterpret_cast<float2 *>(p) = make_float2(a[0], a[1]);
  } else if constexpr (V == 4) {
    *reinterpret_cast<int4 *>(p) = make_int4((int)a[0], (int)a[1], (int)a[2], (int)a[3]);
  } else if constexpr (V == 2) {
    *reinterpret_cast<int2 *>(p) = make_int2((int)a[0], (int)a[1]);
  } else {
    p[0] = from_acc<T>(a[0]);
  }
}

// ---------------------------------------------------------------------------
// Staging: TMA bulk copies of 16-byte aligned windows, one mbarrier.
// ---------------------------------------------------------------------------
struct Window {
  uintptr_t g0;    // first copied byte (16-byte aligned)
  uint32_t bytes;  // multiple of 16
  uint32_t lead;   // elements copied before the requested first one
};

__device__ __forceinline__ Window window(const void *base, uint64_t lo, uint64_t hi, uint32_t es) {
  const uintptr_t a = reinterpret_cast<uintptr_t>(base) + lo * es;
  const uintptr_t b = reinterpret_cast<uintptr_t>(base) + hi * es;
  Window w;
  w.g0 = a & ~(uintptr_t)15;
  w.bytes = (uint32_t)(((b + 15) & ~(uintptr_t)15) - w.g0);
  w.lead = (uint32_t)((a - w.g0) / es);
  return w;
}

__device__ __forceinline__ void bulk_copy(void *dst, uintptr_t src, uint32_t bytes, uint64_t *bar) {
  if (!bytes) return;
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Thread 0 arms the barrier for the windows' bytes and issues the copies.
__device__ __forceinline__ void issue(uint64_t *bar, void *d0, const Window &w0, void *d1, const Window &w1,
                                      void *d2, const Window &w2) {
  // order earlier generic reads of the buffers before the async writes
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(w0.bytes + w1.bytes + w2.bytes)
               : "memory");
  bulk_copy(d0, w0.g0, w0.bytes, bar);
  bulk_copy(d1, w1.g0, w1.bytes, bar);
  bulk_copy(d2, w2.g0, w2.bytes, bar);
}

// Bounded wait for the barrier phase; true (for every thread of the CTA) if
// it completed.  On a timeout the error word is set and the copies get one
// more bounded wait before the CTA gives up on the item.
__device__ __forceinline__ bool landed(uint64_t *bar, uint32_t parity, int *err) {
  auto spin = [&]() {
    uint32_t done = 0;
    for (uint32_t i = 0; i < (1u << 22) && !done; ++i)
      asm volatile(
          "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
          : "=r"(done)
          : "r"(smem_u32(bar)), "r"(parity)
          : "memory");
    return done != 0;
  };
  const bool ok = spin();
  if (__syncthreads_or(!ok)) {
    if (threadIdx.x == 0 && err) atomicExch(err, SPARSEP_ETIMEDOUT);
    spin();
    return false;
  }
  // test support: err[1] set (sparsep_test_wait_fault) adds a wait that runs
  // out once the copies above have landed; the item is then given up as on a
  // real timeout
  if (err && *reinterpret_cast<volatile int *>(err + 1)) {
    uint32_t ph = parity ^ 1u;
    inject_wait_timeout(bar, ph, err);
    return false;
  }
  return true;
}

// Every staged column index below ncols (and `ok` on every thread): the gather
// loops read x without per-load checks.  One pass over the staged chunk, shared
// by all lanes; the result is the same on every thread of the CTA.
__device__ __forceinline__ bool staged_ok(const uint32_t *col, uint32_t n, uint32_t ncols, bool ok, int *err,
                                          int code) {
  bool cols = true;
  for (uint32_t q = threadIdx.x; q < n; q += BT) cols &= col[q] < ncols;
  ok = ok && bchk(cols, err, code);
  return !__syncthreads_or(!ok);
}

// ---------------------------------------------------------------------------
// Row arithmetic
// ---------------------------------------------------------------------------
template <typename T, int V, int ACC> __device__ __forceinline__ void zero_acc(Acc<T> (&acc)[ACC][V]) {
#pragma unroll
  for (int a = 0; a < ACC; ++a)
#pragma unroll
    for (int u = 0; u < V; ++u) acc[a][u] = Acc<T>(0);
}

// Staged nonzeros [q, e) into the accumulators, in index order.  U nonzeros
// per step, U * V * ACC = 16 registers of x in flight per lane.
template <typename T, int G, int V, int ACC>
__device__ __forceinline__ void acc_range(Acc<T> (&acc)[ACC][V], const View<T> &m, const Staged<T> &s, uint32_t q,
                                          uint32_t e, int gl) {
  constexpr int U = 16 / (V * ACC) > 2 ? 16 / (V * ACC) : 2;
  const uint32_t k = m.k;
  if (!bchk(q <= e && e <= s.n, s.err, -2101)) return;  // staged columns were checked against x once
  for (; q + U <= e; q += U) {
    uint32_t c[U];
    T v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) c[u] = s.col[q + u], v[u] = s.val[q + u];
    VecT<T, V> xv[U][ACC];
#pragma unroll
    for (int a = 0; a < ACC; ++a) {
      const uint32_t j = (uint32_t)(gl + a * G) * V;
      if (j < k)
#pragma unroll
        for (int u = 0; u < U; ++u) xv[u][a] = VecT<T, V>::load(m.x + (size_t)c[u] * k + j);
    }
#pragma unroll
    for (int a = 0; a < ACC; ++a) {
      const uint32_t j = (uint32_t)(gl + a * G) * V;
      if (j < k)
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
          for (int w = 0; w < V; ++w) acc[a][w] += mul<T>(v[u], xv[u][a].v[w]);
    }
  }
  for (; q < e; ++q) {
    const T *xr = m.x + (size_t)s.col[q] * k;
    const T v = s.val[q];
#pragma unroll
    for (int a = 0; a < ACC; ++a) {
      const uint32_t j = (uint32_t)(gl + a * G) * V;
      if (j < k) {
        const VecT<T, V> xv = VecT<T, V>::load(xr + j);
#pragma unroll
        for (int w = 0; w < V; ++w) acc[a][w] += mul<T>(v, xv.v[w]);
      }
    }
  }
}

template <typename T, int G, int V, int ACC>
__device__ __forceinline__ void store_row(const View<T> &m, uint32_t row, Acc<T> (&acc)[ACC][V], int gl) {
  T *yr = m.y + (size_t)row * m.k;
#pragma unroll
  for (int a = 0; a < ACC; ++a) {
    const uint32_t j = (uint32_t)(gl + a * G) * V;
    if (j < m.k) store_vec<T, V>(yr + j, acc[a]);
  }
}

// Rows mode: the item's rows dealt round-robin to groups of G lanes.
template <typename T, int G, int V, int ACC>
__device__ __forceinline__ void item_rows(const View<T> &m, const Staged<T> &s, const BItem &it, BShared<T> &,
                                          int tid) {
  using A = Acc<T>;
  constexpr int NG = BT / G;
  const int gi = tid / G, gl = tid % G;
  const uint32_t nr = it.nr;
  for (uint32_t lr = gi; lr < nr; lr += NG) {
    A acc[ACC][V];
    zero_acc<T, V, ACC>(acc);
    acc_range<T, G, V, ACC>(acc, m, s, s.rp[lr] - it.p0, s.rp[lr + 1] - it.p0, gl);
    store_row<T, G, V, ACC>(m, it.r0 + lr, acc, gl);
  }
}

// Rows completed before merge-path diagonal d of the item's row ends
// (rp[i + 1] - p0, i < nr) merged with its nonzero indices (0 .. n - 1): the
// largest i with rp[i] - p0 <= d - i, i.e. every nonzero of rows < i is
// consumed and d - i nonzeros in all.
__device__ __forceinline__ uint32_t merge_search(const uint32_t *rp, uint32_t p0, uint32_t nr, uint32_t n, uint32_t d) {
  uint32_t lo = d > n ? d - n : 0, hi = d < nr ? d : nr;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (rp[mid + 1] - p0 + mid + 1 <= d) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// Merge mode: the item's row ends and nonzeros, as one merged sequence, split
// evenly over the groups (rows of any length cost every group the same).  A
// group writes the rows that start and end in its share; the first row it
// ends may have begun in earlier groups, so it waits for their carries (the
// partial sums of the row each group left open) and adds them, earliest
// first, to its own part.
template <typename T, int G, int V, int ACC>
__device__ __forceinline__ void item_merge(const View<T> &m, const Staged<T> &s, const BItem &it, BShared<T> &sh,
                                           int tid) {
  using A = Acc<T>;
  constexpr int NG = BT / G;
  const int gi = tid / G, gl = tid % G;
  const uint32_t k = m.k, nr = it.nr, n = it.p1 - it.p0, total = nr + n;
  const uint32_t d0 = (uint32_t)((uint64_t)total * gi / NG), d1 = (uint32_t)((uint64_t)total * (gi + 1) / NG);
  const uint32_t i0 = merge_search(s.rp, it.p0, nr, n, d0), i1 = merge_search(s.rp, it.p0, nr, n, d1);
  const uint32_t j1 = d1 - i1;
  uint32_t j = d0 - i0;
  bchk(i0 <= i1 && i1 <= nr && j <= j1 && j1 <= n, s.err, -2102);
  A head[ACC][V], acc[ACC][V];
  zero_acc<T, V, ACC>(head);
  for (uint32_t r = i0; r < i1; ++r) {
    const uint32_t e = s.rp[r + 1] - it.p0;
    zero_acc<T, V, ACC>(acc);
    acc_range<T, G, V, ACC>(acc, m, s, j, e, gl);
    j = e;
    if (r == i0) {
#pragma unroll
      for (int a = 0; a < ACC; ++a)
#pragma unroll
        for (int u = 0; u < V; ++u) head[a][u] = acc[a][u];
    } else {
      store_row<T, G, V, ACC>(m, it.r0 + r, acc, gl);
    }
  }
  zero_acc<T, V, ACC>(acc);
  acc_range<T, G, V, ACC>(acc, m, s, j, j1, gl);  // this group's part of row i1
  __syncthreads();                                 // every group is done with the staged arrays
  A *cbuf = reinterpret_cast<A *>(sh.col);         // NG * k <= BT * V * ACC <= BCAP partials
  uint32_t *crow = sh.rp;                          // NG <= RP_N carry rows
  if (gl == 0) crow[gi] = i1;
#pragma unroll
  for (int a = 0; a < ACC; ++a) {
    const uint32_t jj = (uint32_t)(gl + a * G) * V;
    if (jj < k)
#pragma unroll
      for (int u = 0; u < V; ++u) cbuf[gi * k + jj + u] = acc[a][u];
  }
  __syncthreads();
  if (i0 < i1) {
    int g0 = gi;
    while (g0 > 0 && crow[g0 - 1] == i0) --g0;
#pragma unroll
    for (int a = 0; a < ACC; ++a) {
      const uint32_t jj = (uint32_t)(gl + a * G) * V;
      if (jj < k) {
#pragma unroll
        for (int u = 0; u < V; ++u) {
          A t = A(0);
          for (int g = g0; g < gi; ++g) t += cbuf[g * k + jj + u];
          head[a][u] = t + head[a][u];
        }
      }
    }
    store_row<T, G, V, ACC>(m, it.r0 + i0, head, gl);
  }
}

// One row longer than BCAP: chunks staged in turn, groups of G lanes stride
// over each chunk's nonzeros, then the NG partial vectors are summed in group
// order.  NG * k <= BT * ACC <= BCAP partials fit in the column buffer.
template <typename T, int G, int ACC>
__device__ __forceinline__ void item_long(const View<T> &m, const BItem &it, BShared<T> &sh, int tid, int *err) {
  using A = Acc<T>;
  constexpr int NG = BT / G;
  const int gi = tid / G, gl = tid % G;
  const uint32_t k = m.k;
  A acc[ACC][1];
  zero_acc<T, 1, ACC>(acc);
  uint32_t parity = 0;
  for (uint32_t c0 = it.p0; c0 < it.p1; c0 += BCAP, parity ^= 1u) {
    const uint32_t n = min(BCAP, it.p1 - c0);
    const Window wc = window(it.colind, c0, c0 + n, 4), wv = window(it.val, c0, c0 + n, sizeof(T));
    if (!bchk(wc.bytes <= sizeof(sh.col) && wv.bytes <= sizeof(sh.val), err, -2103)) return;
    __syncthreads();  // the previous chunk is consumed
    if (tid == 0) issue(&sh.bar, sh.col, wc, sh.val, wv, nullptr, Window{0, 0, 0});
    if (!landed(&sh.bar, parity, err)) return;
    const Staged<T> s{nullptr, sh.col + wc.lead, sh.val + wv.lead, n, err};
    if (!staged_ok(s.col, n, m.ncols, true, err, -2107)) return;
    for (uint32_t q = gi; q < n; q += NG) {
      const T *xr = m.x + (size_t)s.col[q] * k;
      const T v = s.val[q];
#pragma unroll
      for (int a = 0; a < ACC; ++a) {
        const uint32_t j = (uint32_t)(gl + a * G);
        if (j < k) acc[a][0] += mul<T>(v, __ldg(xr + j));
      }
    }
  }
  __syncthreads();
  A *red = reinterpret_cast<A *>(sh.col);
#pragma unroll
  for (int a = 0; a < ACC; ++a) {
    const uint32_t j = (uint32_t)(gl + a * G);
    if (j < k) red[gi * k + j] = acc[a][0];
  }
  __syncthreads();
  T *yr = m.y + (size_t)it.r0 * k;
  for (uint32_t j = tid; j < k; j += BT) {
    A t = A(0);
    for (int g = 0; g < NG; ++g) t += red[g * k + j];
    yr[j] = from_acc<T>(t);
  }
}

// ---------------------------------------------------------------------------
// Dispatch on the item's (mode, lanes, vec, acc)
// ---------------------------------------------------------------------------
template <typename T, int MODE, int G, int V, int ACC>
__device__ __forceinline__ void body(const View<T> &m, const Staged<T> &s, const BItem &it, BShared<T> &sh, int tid) {
  if constexpr (MODE == MODE_ROWS) item_rows<T, G, V, ACC>(m, s, it, sh, tid);
  else item_merge<T, G, V, ACC>(m, s, it, sh, tid);
}

template <typename T, int MODE, int G, int V>
__device__ __forceinline__ void by_acc(const View<T> &m, const Staged<T> &s, const BItem &it, BShared<T> &sh,
                                       int tid) {
  switch (it.acc) {
    case 1: body<T, MODE, G, V, 1>(m, s, it, sh, tid); break;
    case 2: if constexpr (V <= 4) body<T, MODE, G, V, 2>(m, s, it, sh, tid); break;
    case 4: if constexpr (V <= 2) body<T, MODE, G, V, 4>(m, s, it, sh, tid); break;
    default: if constexpr (V == 1) body<T, MODE, G, V, 8>(m, s, it, sh, tid); break;
  }
}

template <typename T, int MODE, int G>
__device__ __forceinline__ void by_vec(const View<T> &m, const Staged<T> &s, const BItem &it, BShared<T> &sh,
                                       int tid) {
  switch (it.vec) {
    case 4: by_acc<T, MODE, G, 4>(m, s, it, sh, tid); break;
    case 2: by_acc<T, MODE, G, 2>(m, s, it, sh, tid); break;
    default: by_acc<T, MODE, G, 1>(m, s, it, sh, tid); break;
  }
}

template <typename T, int MODE>
__device__ __forceinline__ void by_lanes(const View<T> &m, const Staged<T> &s, const BItem &it, BShared<T> &sh,
                                         int tid) {
  switch (it.lanes) {
    case 1: by_vec<T, MODE, 1>(m, s, it, sh, tid); break;
    case 2: by_vec<T, MODE, 2>(m, s, it, sh, tid); break;
    case 4: by_vec<T, MODE, 4>(m, s, it, sh, tid); break;
    case 8: by_vec<T, MODE, 8>(m, s, it, sh, tid); break;
    case 16: by_vec<T, MODE, 16>(m, s, it, sh, tid); break;
    default: by_vec<T, MODE, 32>(m, s, it, sh, tid); break;
  }
}

template <typename T, int G>
__device__ __forceinline__ void long_acc(const View<T> &m, const BItem &it, BShared<T> &sh, int tid, int *err) {
  switch (it.acc) {
    case 1: item_long<T, G, 1>(m, it, sh, tid, err); break;
    case 2: item_long<T, G, 2>(m, it, sh, tid, err); break;
    case 4: item_long<T, G, 4>(m, it, sh, tid, err); break;
    default: item_long<T, G, 8>(m, it, sh, tid, err); break;
  }
}

// One CTA per item.  The whole batch is one launch of n = #items CTAs, each
// claiming the next item of the queue with an atomic ticket, so items start in
// queue order (long rows first) whatever order the hardware schedules CTAs
// in, and the block scheduler refills every SM as its CTAs finish.  (A loop
// over items inside each CTA would keep the same order; it costs 128+
// registers and spills across the ~100 inlined row routines, so each CTA
// runs one.)  Without a ticket counter, CTA b runs item i0 + b (one matrix's
// items: the per-matrix launches and the autotuner's timing runs).
template <typename T>
__global__ void __launch_bounds__(BT, 4) batch_items(const BItem *items, uint32_t i0, unsigned int *head, int *err) {
  __shared__ BShared<T> sh;
  const int tid = threadIdx.x;
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&sh.bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    if (head) sh.next = atomicAdd(head, 1u);
  }
  __syncthreads();
  const BItem it = items[head ? sh.next : i0 + blockIdx.x];
  const View<T> m{static_cast<const T *>(it.x), static_cast<T *>(it.y), it.k, it.ncols};
  if (it.mode == MODE_LONG) {
    switch (it.lanes) {
      case 1: long_acc<T, 1>(m, it, sh, tid, err); break;
      case 2: long_acc<T, 2>(m, it, sh, tid, err); break;
      case 4: long_acc<T, 4>(m, it, sh, tid, err); break;
      case 8: long_acc<T, 8>(m, it, sh, tid, err); break;
      case 16: long_acc<T, 16>(m, it, sh, tid, err); break;
      default: long_acc<T, 32>(m, it, sh, tid, err); break;
    }
    return;
  }
  const Window wr = window(it.rowptr, it.r0, it.r0 + it.nr + 1, 4);
  const Window wc = window(it.colind, it.p0, it.p1, 4);
  const Window wv = window(it.val, it.p0, it.p1, sizeof(T));
  if (!bchk(wr.bytes <= sizeof(sh.rp) && wc.bytes <= sizeof(sh.col) && wv.bytes <= sizeof(sh.val) &&
                it.nr <= BRCAP && it.p1 - it.p0 <= BCAP,
            err, -2104))
    return;
  if (tid == 0) issue(&sh.bar, sh.rp, wr, sh.col, wc, sh.val, wv);
  if (!landed(&sh.bar, 0, err)) return;
  const Staged<T> s{sh.rp + wr.lead, sh.col + wc.lead, sh.val + wv.lead, it.p1 - it.p0, err};
  {
    // the staged rowptr must run from p0 to p1 (checked build: non-decreasing),
    // and every staged column must lie inside x
    bool rp_ok = s.rp[0] == it.p0 && s.rp[it.nr] == it.p1;
#ifdef SPARSEP_CHECK
    for (uint32_t i = tid; i < it.nr; i += BT) rp_ok = rp_ok && s.rp[i] <= s.rp[i + 1];
#endif
    if (!staged_ok(s.col, it.p1 - it.p0, it.ncols, bchk(rp_ok, err, -2105), err, -2106)) return;
  }
  if (it.mode == MODE_ROWS) by_lanes<T, MODE_ROWS>(m, s, it, sh, tid);
  else by_lanes<T, MODE_MERGE>(m, s, it, sh, tid);
}

template <typename T>
cudaError_t batch_launch(const BItem *items, uint32_t i0, uint32_t n, unsigned int *head, int *err, cudaStream_t s) {
  if (!n) return cudaSuccess;
  batch_items<T><<<n, BT, 0, s>>>(items, i0, head, err);
  return cudaGetLastError();
}

// The build compiles this file once per element type (-DSPARSEP_BT=<type>).
#ifndef SPARSEP_BT
#define SPARSEP_BT float
#endif
template cudaError_t batch_launch<SPARSEP_BT>(const BItem *, uint32_t, uint32_t, unsigned int *, int *, cudaStream_t);

}  // namespace batch
}  // namespace sparsep
