// batch_kernels.cu -- the kernel of the batched multi-RHS SpMV: many CSR
// matrices with 1..256 right-hand sides each, one launch per batch.
//
// A work item is a row range of one matrix holding at most BCAP nonzeros (or
// one longer row, processed in BCAP-sized chunks), and carries that matrix's
// array pointers.  A CTA runs one item: one thread issues TMA bulk copies of
// the item's rowptr slice, column indices and values into the CTA's staging
// arena (16-byte aligned windows, completion on an mbarrier with a bounded
// wait), so the whole item arrives in one memory round trip; afterwards only
// the x gathers go to memory.  A window item (a 2D tile: a row range whose
// columns all fall in a narrow range [c0, c0 + cw), as in banded matrices)
// also stages those rows of x by the same bulk copy, and every gather of the
// item is a shared-memory load.  In the batch launch, CTAs claim items from a
// global counter (atomicAdd, no waiting) in queue order -- long rows first --
// so matrices of very different sizes share the GPU without per-matrix launch
// gaps or tails.
//
// x and y rows are `pitch` elements apart (k rounded up to a multiple of 4
// for k >= 3), so every row starts on a 16-byte boundary and 4-wide loads
// serve any k; the routines compute the whole padded row.
//
// Row routines, chosen per matrix (the autotuner picks among them).  The CTA
// is cut into groups of G lanes; lane l of a group reads right-hand sides
// [(l + aG)V, (l + aG)V + V) of each nonzero's x row with one V-wide load
// (V in 1, 2, 4; pitch % V == 0), a < ACC, V * ACC <= 8 accumulators.
//   Rows mode: the item's rows dealt round-robin to the groups.
//   Merge mode: the item's row ends and nonzeros split evenly over the groups
//     along the merge path; rows cut by a split are finished from the
//     groups' carries, in group order.
//   A merge-mode group streams its nonzeros in steps of U across row ends,
//   so its loads stay U deep in flight rather than draining at every row;
//   a rows-mode row ends with one masked step.
//   Block items: a 4 x 4 BCSR copy of the matrix, block rows dealt to groups.
//   Long rows (> BCAP nonzeros): one item per BCAP-nonzero chunk, the CTA's
//     groups on contiguous parts of it; partial rows summed in chunk order
//     by the row's last chunk to arrive.
// Same arithmetic as the single-vector path: integers accumulate in 32-bit
// unsigned and wrap exactly; FP in the element type, each row's products
// summed in a fixed order (deterministic from run to run).
#include "batch.hpp"
#include "device.cuh"

// Registers of x in flight per lane (U nonzeros x V x ACC per step), with the
// register budget of MINB CTAs per SM.  Measured on the 512-matrix FP32
// batch (autotuned queue, one run each): 16 / 4 CTAs 7.74 ms; 32 / 4 CTAs
// 7.79 ms (spills); 32 / 3 CTAs 8.77 ms; 16 / 5 CTAs (48 registers) 7.60 ms;
// the next step's loads issued before the current step's products (software
// pipelining) 10.1-10.3 ms (spills).
#ifndef SPARSEP_BATCH_XREGS
#define SPARSEP_BATCH_XREGS 16
#endif

namespace sparsep {
namespace batch {

template <typename T> struct BShared {
  alignas(16) unsigned char arena[ARENA];  // staged item (carve); after the compute: carries / partials
  uint32_t crow[BT];                       // merge mode: the row each group left open
  alignas(8) uint64_t bar;
  unsigned next;
};

// The item's matrix, typed.  x is global memory, or the staged window of a
// window item (rows rebased to c0).
template <typename T> struct View {
  const T *x;
  T *y;
  uint32_t k;  // row pitch of x and y, all computed
  uint32_t ncols;
};

// The staged arrays, indexed from the item's first row / nonzero.
template <typename T> struct Staged {
  const uint32_t *rp;  // rp[i] = rowptr[r0 + i]
  const uint32_t *col; // col[q] = colind[p0 + q] (window items: - c0)
  const T *val;
  uint32_t n;          // staged nonzeros
  int *err;
};

// Index guards: a failed check records its site code in the error word
// (read by sparsep_batch_status) and the guarded work is skipped, so a
// corrupted item or column index cannot take the GPU down.  The per-item ones
// (staging windows, staged rowptr ends, every staged column inside x or the
// window) are always on; the checked build (-DSPARSEP_CHECK) adds a full scan
// of each staged rowptr slice.
__device__ __forceinline__ bool bchk(bool ok, int *err, int code) {
  if (!ok && err) atomicCAS(err, 0, code);
  return ok;
}

template <typename T> __device__ __forceinline__ T bits_as(int v);
template <> __device__ __forceinline__ float bits_as<float>(int v) { return __int_as_float(v); }
template <> __device__ __forceinline__ int32_t bits_as<int32_t>(int v) { return v; }

// V consecutive elements of x: read-only cache loads from global memory, or
// shared-memory loads from a staged window (XS).
template <typename T, int V> struct VecT {
  T v[V];
};
template <typename T, int V, bool XS> __device__ __forceinline__ VecT<T, V> ldx(const T *p) {
  VecT<T, V> r;
  if constexpr (V == 4) {
    int4 q;
    if constexpr (XS) q = *reinterpret_cast<const int4 *>(p);
    else q = __ldg(reinterpret_cast<const int4 *>(p));
    r.v[0] = bits_as<T>(q.x), r.v[1] = bits_as<T>(q.y), r.v[2] = bits_as<T>(q.z),
    r.v[3] = bits_as<T>(q.w);
  } else if constexpr (V == 2) {
    int2 q;
    if constexpr (XS) q = *reinterpret_cast<const int2 *>(p);
    else q = __ldg(reinterpret_cast<const int2 *>(p));
    r.v[0] = bits_as<T>(q.x), r.v[1] = bits_as<T>(q.y);
  } else {
    if constexpr (XS) r.v[0] = *p;
    else r.v[0] = __ldg(p);
  }
  return r;
}

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
  w.bytes = lo < hi ? (uint32_t)(((b + 15) & ~(uintptr_t)15) - w.g0) : 0;
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

// Thread 0 arms the barrier for the windows' bytes and issues the copies
// (up to four: rowptr, columns, values, x window).
__device__ __forceinline__ void issue(uint64_t *bar, void *const (&dst)[4], const Window (&w)[4]) {
  // order earlier generic reads of the buffers before the async writes
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(w[0].bytes + w[1].bytes + w[2].bytes + w[3].bytes)
               : "memory");
#pragma unroll
  for (int i = 0; i < 4; ++i) bulk_copy(dst[i], w[i].g0, w[i].bytes, bar);
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

// Every staged column index inside x (below ncols), or for a window item
// inside the window, rebased to it (col - c0 < cw, written back); and `ok` on
// every thread.  The gather loops then read x without per-load checks.  One
// pass over the staged chunk, shared by all lanes; the result is the same on
// every thread of the CTA.
__device__ __forceinline__ bool staged_ok(uint32_t *col, uint32_t n, uint32_t c0, uint32_t bound, bool rebase,
                                          bool ok, int *err, int code) {
  bool cols = true;
  if (rebase) {
    for (uint32_t q = threadIdx.x; q < n; q += BT) {
      const uint32_t c = col[q] - c0;
      cols &= c < bound;
      col[q] = c;
    }
  } else {
    for (uint32_t q = threadIdx.x; q < n; q += BT) cols &= col[q] < bound;
  }
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

// Accumulators of lane gl that fall inside the row: (gl + a G) V < k for a < na.
template <int G, int V, int ACC> __device__ __forceinline__ int active_acc(int gl, uint32_t k) {
  int na = 0;
#pragma unroll
  for (int a = 0; a < ACC; ++a) na += (uint32_t)(gl + a * G) * V < k;
  return na;
}

// x row c of the view, from the lane's first column on: 64-bit offsets into
// global memory, 32-bit into a staged window.
template <typename T, bool XS> __device__ __forceinline__ const T *xrow(const T *xl, uint32_t c, uint32_t k) {
  if constexpr (XS) return xl + c * k;
  else return xl + (size_t)c * k;
}

// Staged nonzeros [q, e) into the accumulators, in index order.  xl is x plus
// the lane's first column (gl V); accumulator a reads columns a G V further.
// U nonzeros per step, U * V * ACC = SPARSEP_BATCH_XREGS registers of x in
// flight per lane; the last e - q < U nonzeros as one masked step (one round
// trip), products added in index order either way.
template <typename T, int G, int V, int ACC, bool XS>
__device__ __forceinline__ void acc_range(Acc<T> (&acc)[ACC][V], const T *xl, uint32_t k, int na,
                                          const Staged<T> &s, uint32_t q, uint32_t e) {
  constexpr int U = SPARSEP_BATCH_XREGS / (V * ACC) > 2 ? SPARSEP_BATCH_XREGS / (V * ACC) : 2;
  if (!bchk(q <= e && e <= s.n, s.err, -2101)) return;  // staged columns were checked against x once
  for (; q < e; q += U) {
    uint32_t c[U];
    T v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const bool in = q + u < e;
      c[u] = in ? s.col[q + u] : 0u;
      v[u] = in ? s.val[q + u] : T(0);
    }
    VecT<T, V> xv[U][ACC];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const T *p = xrow<T, XS>(xl, c[u], k);
#pragma unroll
      for (int a = 0; a < ACC; ++a)
        if (a < na && q + u < e) xv[u][a] = ldx<T, V, XS>(p + a * G * V);
    }
#pragma unroll
    for (int a = 0; a < ACC; ++a)
      if (a < na)
#pragma unroll
        for (int u = 0; u < U; ++u)
          if (q + u < e)
#pragma unroll
            for (int w = 0; w < V; ++w) acc[a][w] += mul<T>(v[u], xv[u][a].v[w]);
  }
}

template <typename T, int G, int V, int ACC>
__device__ __forceinline__ void store_row(T *yl, uint32_t row, uint32_t k, int na, Acc<T> (&acc)[ACC][V]) {
  T *yr = yl + (size_t)row * k;
#pragma unroll
  for (int a = 0; a < ACC; ++a)
    if (a < na) store_vec<T, V>(yr + a * G * V, acc[a]);
}

// Item-local nonzeros [j, j1) of rows r .. i1 - 1 (row r may have begun
// before j) and the start of row i1, in steps of U across row ends, so that U
// loads stay in flight all along (a merge-mode group's share).  Each row is
// summed from zero in index order; with keep_first, row r's sum goes to head
// (its earlier part is in other groups' carries), every other finished row to
// y.  Returns with acc
// holding this range's part of row i1 (zero when [j, j1) ends with row i1 - 1).
template <typename T, int G, int V, int ACC, bool XS>
__device__ __forceinline__ void stream_rows(Acc<T> (&acc)[ACC][V], Acc<T> (&head)[ACC][V], bool keep_first,
                                            const T *xl, T *yl, uint32_t k, int na, const Staged<T> &s,
                                            const BItem &it, uint32_t r, uint32_t i1, uint32_t j, uint32_t j1) {
  const uint32_t first = r;
  uint32_t rend = r < i1 ? s.rp[r + 1] - it.p0 : j1;
  zero_acc<T, V, ACC>(acc);
  auto finish = [&]() {
    if (keep_first && r == first) {
#pragma unroll
      for (int a = 0; a < ACC; ++a)
#pragma unroll
        for (int u = 0; u < V; ++u) head[a][u] = acc[a][u];
    } else {
      store_row<T, G, V, ACC>(yl, it.r0 + r, k, na, acc);
    }
    zero_acc<T, V, ACC>(acc);
    ++r;
    rend = r < i1 ? s.rp[r + 1] - it.p0 : j1;
  };
  constexpr int U = SPARSEP_BATCH_XREGS / (V * ACC) > 2 ? SPARSEP_BATCH_XREGS / (V * ACC) : 2;
  for (uint32_t q = j; q < j1; q += U) {
    uint32_t c[U];
    T v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const bool in = q + u < j1;
      c[u] = in ? s.col[q + u] : 0u;
      v[u] = in ? s.val[q + u] : T(0);
    }
    VecT<T, V> xv[U][ACC];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const T *p = xrow<T, XS>(xl, c[u], k);
#pragma unroll
      for (int a = 0; a < ACC; ++a)
        if (a < na && q + u < j1) xv[u][a] = ldx<T, V, XS>(p + a * G * V);
    }
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (q + u < j1) {
        while (r < i1 && rend == q + u) finish();  // rows ending here (empty ones too)
#pragma unroll
        for (int a = 0; a < ACC; ++a)
          if (a < na)
#pragma unroll
            for (int w = 0; w < V; ++w) acc[a][w] += mul<T>(v[u], xv[u][a].v[w]);
      }
  }
  while (r < i1) finish();  // rows ending at j1, all their nonzeros consumed
}

// Rows mode: the item's rows dealt round-robin to groups of G lanes, so that
// the groups of a warp work on consecutive rows (their y stores coalesce and,
// in banded matrices, their x rows overlap).  Measured against contiguous
// blocks of rows streamed per group on the 512-matrix FP32 batch: the blocks
// were slower on the uniform (+5.6 %) and banded (+9.4 %) matrices.
template <typename T, int G, int V, int ACC, bool XS>
__device__ __forceinline__ void item_rows(const View<T> &m, const Staged<T> &s, const BItem &it, BShared<T> &,
                                          int tid) {
  using A = Acc<T>;
  constexpr int NG = BT / G;
  const int gi = tid / G, gl = tid % G;
  const int na = active_acc<G, V, ACC>(gl, m.k);
  const T *xl = m.x + gl * V;
  T *yl = m.y + gl * V;
  const uint32_t nr = it.nr;
  for (uint32_t lr = gi; lr < nr; lr += NG) {
    A acc[ACC][V];
    zero_acc<T, V, ACC>(acc);
    acc_range<T, G, V, ACC, XS>(acc, xl, m.k, na, s, s.rp[lr] - it.p0, s.rp[lr + 1] - it.p0);
    store_row<T, G, V, ACC>(yl, it.r0 + lr, m.k, na, acc);
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
template <typename T, int G, int V, int ACC, bool XS>
__device__ __forceinline__ void item_merge(const View<T> &m, const Staged<T> &s, const BItem &it, BShared<T> &sh,
                                           int tid) {
  using A = Acc<T>;
  constexpr int NG = BT / G;
  const int gi = tid / G, gl = tid % G;
  const uint32_t k = m.k, nr = it.nr, n = it.p1 - it.p0, total = nr + n;
  const int na = active_acc<G, V, ACC>(gl, k);
  const T *xl = m.x + gl * V;
  T *yl = m.y + gl * V;
  const uint32_t d0 = (uint32_t)((uint64_t)total * gi / NG), d1 = (uint32_t)((uint64_t)total * (gi + 1) / NG);
  const uint32_t i0 = merge_search(s.rp, it.p0, nr, n, d0);
  uint32_t i1 = merge_search(s.rp, it.p0, nr, n, d1);
  const uint32_t j = d0 - i0;
  uint32_t j1 = d1 - i1;
  // a failed check leaves the group's range empty (the error is recorded); the
  // group still takes part in the barriers below
  if (!bchk(i0 <= i1 && i1 <= nr && j <= j1 && j1 <= n, s.err, -2102)) i1 = i0, j1 = j;
  A head[ACC][V], acc[ACC][V];
  zero_acc<T, V, ACC>(head);
  stream_rows<T, G, V, ACC, XS>(acc, head, true, xl, yl, k, na, s, it, i0, i1, j, j1);
  // acc: this group's part of row i1
  __syncthreads();  // every group is done with the staged arrays
  A *cbuf = reinterpret_cast<A *>(sh.arena);               // NG * k <= BT * V * ACC partials
  uint32_t *crow = sh.crow;
  if (gl == 0) crow[gi] = i1;
#pragma unroll
  for (int a = 0; a < ACC; ++a)
    if (a < na)
#pragma unroll
      for (int u = 0; u < V; ++u) cbuf[gi * k + (gl + a * G) * V + u] = acc[a][u];
  __syncthreads();
  if (i0 < i1) {
    int g0 = gi;
    while (g0 > 0 && crow[g0 - 1] == i0) --g0;
#pragma unroll
    for (int a = 0; a < ACC; ++a)
      if (a < na) {
        const uint32_t jj = (uint32_t)(gl + a * G) * V;
#pragma unroll
        for (int u = 0; u < V; ++u) {
          A t = A(0);
          for (int g = g0; g < gi; ++g) t += cbuf[g * k + jj + u];
          head[a][u] = t + head[a][u];
        }
      }
    store_row<T, G, V, ACC>(yl, it.r0 + i0, k, na, head);
  }
}

// Block items (4 x 4 BCSR copy): block rows dealt round-robin to groups of G
// lanes, each lane 4 consecutive right-hand sides (pitch <= 4 G).  A block's
// 4 x rows are loaded once for its 4 rows -- a quarter of the x gathers of the
// same nonzeros in CSR -- two blocks per step; the block's values come from
// shared memory 4 per load.  Each row's sum runs over its block row's blocks
// in block-column order and within a block in column order.
template <typename T, int G>
__device__ __forceinline__ void item_bcsr(const BItem &it, const Staged<T> &s, int tid) {
  using A = Acc<T>;
  constexpr int NG = BT / G, V = 4;
  const int gi = tid / G, gl = tid % G;
  const uint32_t k = it.k;
  if ((uint32_t)gl * V >= k) return;  // no barrier follows: idle lanes may leave
  const T *xl = static_cast<const T *>(it.x) + gl * V;
  T *yl = static_cast<T *>(it.y) + gl * V;
  for (uint32_t lb = gi; lb < it.nr; lb += NG) {
    A acc[4][V];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int w = 0; w < V; ++w) acc[r][w] = A(0);
    const uint32_t q0 = s.rp[lb] - it.p0, q1 = s.rp[lb + 1] - it.p0;
    for (uint32_t q = q0; q < q1; q += 2) {
      const bool two = q + 1 < q1;
      VecT<T, V> xv[2][4];
#pragma unroll
      for (int b = 0; b < 2; ++b)
        if (b == 0 || two) {
          const T *xb = xl + (size_t)s.col[q + b] * 4 * k;
#pragma unroll
          for (int c = 0; c < 4; ++c) xv[b][c] = ldx<T, V, false>(xb + c * k);
        }
#pragma unroll
      for (int b = 0; b < 2; ++b)
        if (b == 0 || two) {
          const T *bv = s.val + (size_t)(q + b) * 16;
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            const VecT<T, 4> a4 = ldx<T, 4, true>(bv + r * 4);
#pragma unroll
            for (int c = 0; c < 4; ++c)
#pragma unroll
              for (int w = 0; w < V; ++w) acc[r][w] += mul<T>(a4.v[c], xv[b][c].v[w]);
          }
        }
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const uint32_t row = 4 * (it.r0 + lb) + r;
      if (row < it.nrows) store_vec<T, V>(yl + (size_t)row * k, acc[r]);
    }
  }
}

// One chunk (<= BCAP nonzeros) of a row longer than BCAP; the row's chunks
// are separate items, so a long row spreads over many SMs.  The CTA's groups
// split the chunk's nonzeros into contiguous ranges (the row routines' vector
// loads), their partial vectors are summed in group order into the chunk's
// partial row, and the last of the row's chunks to arrive sums the partials
// in chunk order into y (deterministic) and resets the row's counter.  Every
// chunk arrives -- after a failed staging or check with a zero partial, the
// error word set -- so the counter is zero again after every launch.
template <typename T, int G, int V, int ACC>
__device__ __forceinline__ void item_chunk(const BItem &it, BShared<T> &sh, int tid, int *err) {
  using A = Acc<T>;
  constexpr int NG = BT / G;
  constexpr Carve cv = carve(0, BCAP, sizeof(T), 0);
  const uint32_t k = it.k, n = it.p1 - it.p0;
  const int gi = tid / G, gl = tid % G;
  const int na = active_acc<G, V, ACC>(gl, k);
  const Window w[4] = {window(it.colind, it.p0, it.p1, 4), window(it.val, it.p0, it.p1, sizeof(T)),
                       Window{0, 0, 0}, Window{0, 0, 0}};
  bool ok = bchk(n <= BCAP && it.c0 < it.cw && w[0].bytes <= cv.val - cv.col && w[1].bytes <= cv.xw - cv.val &&
                     (uint32_t)NG * k * (uint32_t)sizeof(A) <= ARENA,
                 err, -2103);
  if (ok) {
    void *const dst[4] = {sh.arena + cv.col, sh.arena + cv.val, nullptr, nullptr};
    if (tid == 0) issue(&sh.bar, dst, w);
    ok = landed(&sh.bar, 0, err);
  }
  uint32_t *col = reinterpret_cast<uint32_t *>(sh.arena + cv.col) + w[0].lead;
  if (ok) ok = staged_ok(col, n, 0, it.ncols, false, true, err, -2107);
  A acc[ACC][V];
  zero_acc<T, V, ACC>(acc);
  if (ok) {
    const Staged<T> s{nullptr, col, reinterpret_cast<const T *>(sh.arena + cv.val) + w[1].lead, n, err};
    const uint32_t q0 = (uint32_t)((uint64_t)n * gi / NG), q1 = (uint32_t)((uint64_t)n * (gi + 1) / NG);
    acc_range<T, G, V, ACC, false>(acc, static_cast<const T *>(it.x) + gl * V, k, na, s, q0, q1);
  }
  __syncthreads();  // the staged chunk is consumed
  A *red = reinterpret_cast<A *>(sh.arena);
  if (ok)
#pragma unroll
    for (int a = 0; a < ACC; ++a)
      if (a < na)
#pragma unroll
        for (int u = 0; u < V; ++u) red[gi * k + (gl + a * G) * V + u] = acc[a][u];
  __syncthreads();
  T *part = static_cast<T *>(it.part);
  for (uint32_t j = tid; j < k; j += BT) {
    A t = A(0);
    if (ok)
      for (int g = 0; g < NG; ++g) t += red[g * k + j];
    part[(size_t)it.c0 * k + j] = from_acc<T>(t);
  }
  __threadfence();  // the partial is visible before the arrival
  __syncthreads();
  if (tid == 0) sh.next = atomicAdd(it.cnt, 1u) == it.cw - 1;
  __syncthreads();
  if (!sh.next) return;
  __threadfence();
  T *yr = static_cast<T *>(it.y) + (size_t)it.r0 * k;
  for (uint32_t j = tid; j < k; j += BT) {
    A t = A(0);
    for (uint32_t c = 0; c < it.cw; ++c) t += A(__ldcg(part + (size_t)c * k + j));
    yr[j] = from_acc<T>(t);
  }
  if (tid == 0) atomicExch(it.cnt, 0u);
}

template <typename T, int G>
__device__ __forceinline__ void chunk_by_vec(const BItem &it, BShared<T> &sh, int tid, int *err) {
  switch (it.vec) {
    case 4:
      if (it.acc == 2) item_chunk<T, G, 4, 2>(it, sh, tid, err);
      else item_chunk<T, G, 4, 1>(it, sh, tid, err);
      break;
    case 2: item_chunk<T, G, 2, 1>(it, sh, tid, err); break;
    default: item_chunk<T, G, 1, 1>(it, sh, tid, err); break;
  }
}

// ---------------------------------------------------------------------------
// Dispatch on the item's (mode, lanes, vec, acc) and whether x is staged.
// Window items come from 4-wide variants only.
// ---------------------------------------------------------------------------
template <typename T, int MODE, int G, int V, int ACC, bool XS>
__device__ __forceinline__ void body(const View<T> &m, const Staged<T> &s, const BItem &it, BShared<T> &sh, int tid) {
  if constexpr (MODE == MODE_ROWS) item_rows<T, G, V, ACC, XS>(m, s, it, sh, tid);
  else item_merge<T, G, V, ACC, XS>(m, s, it, sh, tid);
}

template <typename T, int MODE, int G, int V, bool XS>
__device__ __forceinline__ void by_acc(const View<T> &m, const Staged<T> &s, const BItem &it, BShared<T> &sh,
                                       int tid) {
  switch (it.acc) {
    case 1: body<T, MODE, G, V, 1, XS>(m, s, it, sh, tid); break;
    case 2: if constexpr (V <= 4) body<T, MODE, G, V, 2, XS>(m, s, it, sh, tid); break;
    case 4: if constexpr (V <= 2) body<T, MODE, G, V, 4, XS>(m, s, it, sh, tid); break;
    default: if constexpr (V == 1) body<T, MODE, G, V, 8, XS>(m, s, it, sh, tid); break;
  }
}

template <typename T, int MODE, int G, bool XS>
__device__ __forceinline__ void by_vec(const View<T> &m, const Staged<T> &s, const BItem &it, BShared<T> &sh,
                                       int tid) {
  if constexpr (XS) {
    by_acc<T, MODE, G, 4, XS>(m, s, it, sh, tid);
  } else {
    switch (it.vec) {
      case 4: by_acc<T, MODE, G, 4, XS>(m, s, it, sh, tid); break;
      case 2: by_acc<T, MODE, G, 2, XS>(m, s, it, sh, tid); break;
      default: by_acc<T, MODE, G, 1, XS>(m, s, it, sh, tid); break;
    }
  }
}

template <typename T, int MODE, bool XS>
__device__ __forceinline__ void by_lanes(const View<T> &m, const Staged<T> &s, const BItem &it, BShared<T> &sh,
                                         int tid) {
  switch (it.lanes) {
    case 1: by_vec<T, MODE, 1, XS>(m, s, it, sh, tid); break;
    case 2: by_vec<T, MODE, 2, XS>(m, s, it, sh, tid); break;
    case 4: by_vec<T, MODE, 4, XS>(m, s, it, sh, tid); break;
    case 8: by_vec<T, MODE, 8, XS>(m, s, it, sh, tid); break;
    case 16: by_vec<T, MODE, 16, XS>(m, s, it, sh, tid); break;
    default: by_vec<T, MODE, 32, XS>(m, s, it, sh, tid); break;
  }
}

// One CTA per item.  The whole batch is one launch of n = #items CTAs, each
// claiming the next item of the queue with an atomic ticket, so items start in
// queue order (long rows first) whatever order the hardware schedules CTAs
// in, and the block scheduler refills every SM as its CTAs finish.  (A loop
// over items inside each CTA would keep the same order; it costs 128+
// registers and spills across the inlined row routines, so each CTA runs
// one.)  Without a ticket counter, CTA b runs item i0 + b (one matrix's
// items: the per-matrix launches and the autotuner's timing runs).
template <typename T>
__global__ void __launch_bounds__(BT, MINB)
    batch_items(const BItem *items, uint32_t i0, unsigned int *head, int *err) {
  __shared__ BShared<T> sh;
  const int tid = threadIdx.x;
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&sh.bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    if (head) sh.next = atomicAdd(head, 1u);
  }
  __syncthreads();
  const BItem it = items[head ? sh.next : i0 + blockIdx.x];
  if (it.mode == MODE_LONG) {
    switch (it.lanes) {
      case 1: chunk_by_vec<T, 1>(it, sh, tid, err); break;
      case 2: chunk_by_vec<T, 2>(it, sh, tid, err); break;
      case 4: chunk_by_vec<T, 4>(it, sh, tid, err); break;
      case 8: chunk_by_vec<T, 8>(it, sh, tid, err); break;
      case 16: chunk_by_vec<T, 16>(it, sh, tid, err); break;
      default: chunk_by_vec<T, 32>(it, sh, tid, err); break;
    }
    return;
  }
  const uint32_t n = it.p1 - it.p0;
  const bool blocks = it.mode == MODE_BCSR;
  const uint32_t vpe = blocks ? 16 : 1;  // values per staged entry
  const bool win = !blocks && it.cw != 0;
  const Carve cv = carve(it.nr, n, vpe * (uint32_t)sizeof(T), win ? it.cw * it.k * (uint32_t)sizeof(T) : 0);
  const Window w[4] = {window(it.rowptr, it.r0, it.r0 + it.nr + 1, 4), window(it.colind, it.p0, it.p1, 4),
                       window(it.val, (uint64_t)it.p0 * vpe, (uint64_t)it.p1 * vpe, sizeof(T)),
                       win ? window(it.x, (uint64_t)it.c0 * it.k, (uint64_t)(it.c0 + it.cw) * it.k, sizeof(T))
                           : Window{0, 0, 0}};
  if (!bchk(it.nr <= BRCAP && n <= (blocks ? BBCAP : BCAP) && cv.end <= ARENA && w[0].bytes <= cv.col &&
                (!blocks || (w[2].lead == 0 && it.vec == 4 && (uint32_t)it.lanes * 4 >= it.k)) &&
                w[1].bytes <= cv.val - cv.col && w[2].bytes <= cv.xw - cv.val &&
                (!win || (w[3].bytes <= cv.end - cv.xw && w[3].lead == 0 && it.vec == 4 &&
                          (uint64_t)it.c0 + it.cw <= it.ncols)),
            err, -2104))
    return;
  void *const dst[4] = {sh.arena, sh.arena + cv.col, sh.arena + cv.val, sh.arena + cv.xw};
  if (tid == 0) issue(&sh.bar, dst, w);
  if (!landed(&sh.bar, 0, err)) return;
  uint32_t *col = reinterpret_cast<uint32_t *>(sh.arena + cv.col) + w[1].lead;
  const Staged<T> s{reinterpret_cast<const uint32_t *>(sh.arena) + w[0].lead, col,
                    reinterpret_cast<const T *>(sh.arena + cv.val) + w[2].lead, n, err};
  {
    // the staged rowptr must run from p0 to p1 (checked build: non-decreasing),
    // and every staged column must lie inside x (window items: inside the
    // window, rebased to it)
    bool rp_ok = s.rp[0] == it.p0 && s.rp[it.nr] == it.p1;
#ifdef SPARSEP_CHECK
    for (uint32_t i = tid; i < it.nr; i += BT) rp_ok = rp_ok && s.rp[i] <= s.rp[i + 1];
#endif
    const uint32_t bound = blocks ? (it.ncols + 3) / 4 : win ? it.cw : it.ncols;  // block columns, or columns
    if (!staged_ok(col, n, it.c0, bound, win, bchk(rp_ok, err, -2105), err, -2106)) return;
  }
  if (blocks) {
    switch (it.lanes) {
      case 1: item_bcsr<T, 1>(it, s, tid); break;
      case 2: item_bcsr<T, 2>(it, s, tid); break;
      case 4: item_bcsr<T, 4>(it, s, tid); break;
      case 8: item_bcsr<T, 8>(it, s, tid); break;
      case 16: item_bcsr<T, 16>(it, s, tid); break;
      default: item_bcsr<T, 32>(it, s, tid); break;
    }
    return;
  }
  if (win) {
    const View<T> m{reinterpret_cast<const T *>(sh.arena + cv.xw), static_cast<T *>(it.y), it.k, it.cw};
    if (it.mode == MODE_ROWS) by_lanes<T, MODE_ROWS, true>(m, s, it, sh, tid);
    else by_lanes<T, MODE_MERGE, true>(m, s, it, sh, tid);
  } else {
    const View<T> m{static_cast<const T *>(it.x), static_cast<T *>(it.y), it.k, it.ncols};
    if (it.mode == MODE_ROWS) by_lanes<T, MODE_ROWS, false>(m, s, it, sh, tid);
    else by_lanes<T, MODE_MERGE, false>(m, s, it, sh, tid);
  }
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
