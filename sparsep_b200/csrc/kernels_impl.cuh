// kernels_impl.cuh -- the sm_100a SpMV kernels of sparsep_b200 (device code,
// included by kernels.cu and by the allocation-free entry point).
//
// One kernel template executes a list of work items (device.cuh: Item); one
// CTA runs one item.  The item kinds cover every reference kernel family:
//   CSR rows  (spmv/1D/CSR-*/dpu/task.c:31-215, spmv/2D/*DCSR/dpu/task.c)
//       -> L lanes per row (L = 1..32), 128-bit loads of colind / values
//   CSR long-row chunks (no reference counterpart; the nnz balance remedy of
//       partition_by_nnz pushed below row granularity) -> CTA-wide reduction
//   COO elements (spmv/1D/COO-nnz/dpu/task.c lf :21-679, lb-fg :686-1338)
//       -> lock-free: block segmented scan + carries fixed up by the last CTA
//       -> atomic:    warp segmented scan + red.global per row run
//   BCSR block rows (spmv/1D/BCSR-nnz/dpu/task.c:231-380) -> dense block in
//       registers, L lanes per block row
//   BCOO blocks (spmv/1D/BCOO-nnz/dpu/task.c:22-894) -> as COO with a
//       row-block-wide payload
// 2D tiles are items whose x-segment is staged into shared memory by bulk
// (TMA) copies; their partial y goes to per-stripe slices merged on the device.
#pragma once
#include <cstdio>

#include "device.cuh"

namespace sparsep {

constexpr unsigned long long NO_CARRY = ~0ull;
constexpr int COO_K = 4;  // elements per thread per chunk

// ---------------------------------------------------------------------------
// output helpers
// ---------------------------------------------------------------------------
// Carry targets are indices into the mode's output array: y, or the partial
// slices (slot * nrows + row).
template <typename T>
__device__ __forceinline__ uint64_t out_index(const Params<T> &P, const Item &it, uint64_t row) {
  return P.out_mode == OUT_PARTIAL ? (uint64_t)it.slot * P.nrows + row : row;
}

// x element: the staged segment lives in shared memory and must be read with
// generic loads; the non-coherent read-only path (ld.global.nc) is for x in
// global memory only.
template <typename T>
__device__ __forceinline__ T xload(const T *__restrict__ xb, uint64_t i, bool staged) {
  return staged ? xb[i] : __ldg(xb + i);
}

// checked build: x index valid for the staged segment or the whole vector
template <typename T>
__device__ __forceinline__ bool x_ok(const Params<T> &P, const Item &it, uint64_t col) {
  return it.xw > 0 ? (col >= it.xlo && col - it.xlo < it.xw) : col < P.n_x;
}

template <typename T>
__device__ __forceinline__ void put(const Params<T> &P, T *out, uint64_t r, Acc<T> v) {
  if (SP_BAD(P, r < P.nrows, -1004)) return;
  if (P.out_mode == OUT_ATOMIC) atomic_add_out<T>(out + r, v);
  else out[r] = from_acc<T>(v);
}

// ---------------------------------------------------------------------------
// CSR rows, L lanes per row
// ---------------------------------------------------------------------------
template <typename T, int L>
__device__ void csr_rows(const Params<T> &P, const Item &it, const T *__restrict__ xb) {
  using A = Acc<T>;
  constexpr int G = 32 / L;
  T *out = out_base(P, it);
  const int nw = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane / L, gl = lane % L;
  const uint32_t *rp = P.rowptr + it.ptr_base;
  const uint64_t r0 = it.a0, r1 = it.a1;
  const uint32_t xoff = it.col_off;

  auto do_row = [&](uint64_t r, bool valid_in) {
    bool valid = valid_in;
    A acc = A(0);
    if (valid && SP_BAD(P, it.ptr_base + r + 1 < P.n_rowptr, -1001)) valid = false;
    if (valid) {
      const uint64_t s = (uint64_t)rp[r] + it.nnz_base, e = (uint64_t)rp[r + 1] + it.nnz_base;
#pragma unroll 2
      for (uint64_t j = (s & ~3ull) + 4 * gl; j < e; j += 4 * L) {
        if (SP_BAD(P, j + 3 < P.n_idx && j + 3 < P.n_val, -1002)) break;
        const uint4 c4 = ld_stream4(P.colind + j);
        const Vec4<T> v4 = ld_vals4<T>(P.val + j);
        const uint32_t cc[4] = {c4.x, c4.y, c4.z, c4.w};
#pragma unroll
        for (int k = 0; k < 4; ++k)
          if (j + k >= s && j + k < e && !SP_BAD(P, x_ok(P, it, (uint64_t)xoff + cc[k]), -1003))
            acc += mul<T>(v4.v[k], xload(xb, (uint64_t)xoff + cc[k], it.xw > 0));
      }
    }
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (valid && gl == 0) put<T>(P, out, it.row_off + r, acc);
  };

  if (it.worker_bal == SPARSEP_BAL_INTERLEAVE) {
    for (uint64_t k = 0;; ++k) {
      uint64_t base = r0 + (k * nw + warp) * G;
      if (base >= r1) break;
      do_row(base + g, base + g < r1);
    }
    return;
  }
  // contiguous row range per warp (reference tasklet split, partition_tsklt_by_row /
  // partition_tsklt_by_nnz, spmv/1D/CSR-row/support/partition.h:66-131)
  uint64_t wb, we;
  if (it.worker_bal == SPARSEP_BAL_NNZ) {
    const uint64_t lo = rp[r0], hi = rp[r1];
    auto find = [&](uint64_t target) {  // first row whose start >= target
      uint64_t a = r0, b = r1;
      while (a < b) {
        uint64_t m = (a + b) >> 1;
        if (rp[m] < target) a = m + 1; else b = m;
      }
      return a;
    };
    wb = warp == 0 ? r0 : find(lo + (hi - lo) * warp / nw);
    we = warp == nw - 1 ? r1 : find(lo + (hi - lo) * (warp + 1) / nw);
  } else {
    const uint64_t n = r1 - r0, q = n / nw, rem = n % nw;
    wb = r0 + q * warp + (warp < (int)rem ? warp : rem);
    we = wb + q + (warp < (int)rem ? 1 : 0);
  }
  for (uint64_t base = wb; base < we; base += G) do_row(base + g, base + g < we);
}

// ---------------------------------------------------------------------------
// CSR rows, staged ("stream") form used when lanes = auto.  A chunk of up to
// CSR_RCAP rows / CSR_CAP nonzeros is moved in three coalesced sweeps: its
// rowptr slice into shared memory, then every nonzero (128-bit loads of colind
// and values) times its gathered x into a shared product array; rows are then
// summed from shared memory (a thread per short row, a warp per long row) and
// written with consecutive threads on consecutive rows.  A row longer than the
// chunk capacity is reduced by the whole CTA straight from global memory.
// ---------------------------------------------------------------------------
// x gathers each thread keeps in flight in the chunk's product pass: 4 x this.
// On the 1M-row Zipf FP32 matrix: 1 (40 registers, 6 CTAs/SM) 93.2 us; 2 (62
// registers, 4 CTAs/SM) 99.4 us -- occupancy buys more than depth here.
#ifndef SPARSEP_CSR_GATHER
#define SPARSEP_CSR_GATHER 1
#endif
#ifndef SPARSEP_CSR_CAP
#define SPARSEP_CSR_CAP 4096
#endif
#ifndef SPARSEP_CSR_SHORT
#define SPARSEP_CSR_SHORT 48
#endif
constexpr int CSR_CAP = SPARSEP_CSR_CAP;      // nonzeros per chunk
constexpr int CSR_RCAP = 1024;                // rows per chunk
constexpr int CSR_SHORT = SPARSEP_CSR_SHORT;  // rows up to this length are summed by one thread

// sum of a[s, e) x over the whole CTA (thread 0 gets the total)
template <typename T>
__device__ Acc<T> cta_range_sum(const Params<T> &P, const Item &it, const T *__restrict__ xb, uint64_t s,
                                uint64_t e, Acc<T> *red) {
  using A = Acc<T>;
  A acc = A(0);
#pragma unroll 2
  for (uint64_t j = (s & ~3ull) + 4 * threadIdx.x; j < e; j += 4 * blockDim.x) {
    if (SP_BAD(P, j + 3 < P.n_idx && j + 3 < P.n_val, -1005)) break;
    const uint4 c4 = ld_stream4(P.colind + j);
    const Vec4<T> v4 = ld_vals4<T>(P.val + j);
    const uint32_t cc[4] = {c4.x, c4.y, c4.z, c4.w};
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (j + k >= s && j + k < e && !SP_BAD(P, x_ok(P, it, (uint64_t)it.col_off + cc[k]), -1006))
        acc += mul<T>(v4.v[k], xload(xb, (uint64_t)it.col_off + cc[k], it.xw > 0));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  __syncthreads();  // red may still be read from a previous call
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  A tot = A(0);
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += red[w];
  return tot;
}

template <typename T>
__device__ void csr_stream(const Params<T> &P, const Item &it, const T *__restrict__ xb) {
  using A = Acc<T>;
  __shared__ A prods[CSR_CAP];
  __shared__ uint32_t srp[CSR_RCAP + 1];
  __shared__ uint32_t longs[CSR_RCAP];
  __shared__ uint32_t nlong;
  __shared__ A red[32];
  T *out = out_base(P, it);
  const uint32_t *rp = P.rowptr + it.ptr_base;
  const int nw = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool staged = it.xw > 0;
  uint64_t r = it.a0;
  while (r < it.a1) {
    const uint32_t nr = (uint32_t)((it.a1 - r) < CSR_RCAP ? (it.a1 - r) : CSR_RCAP);
    if (SP_BAD(P, it.ptr_base + r + nr < P.n_rowptr, -1001)) return;
    for (uint32_t i = threadIdx.x; i <= nr; i += blockDim.x) srp[i] = __ldcs(rp + r + i);
    if (threadIdx.x == 0) nlong = 0;
    __syncthreads();
    // rows [r, r+k) form the chunk: the longest prefix within CSR_CAP nonzeros
    const uint32_t base = srp[0];
    uint32_t k = nr;
    if (srp[nr] - base > (uint32_t)CSR_CAP) {
      uint32_t lo = 0, hi = nr;  // largest k with srp[k] - base <= CAP
      while (lo < hi) {
        const uint32_t m = (lo + hi + 1) >> 1;
        if (srp[m] - base <= (uint32_t)CSR_CAP) lo = m; else hi = m - 1;
      }
      k = lo;
    }
    if (k == 0) {  // one row longer than the chunk: whole-CTA reduction from global
      const A tot = cta_range_sum<T>(P, it, xb, (uint64_t)base + it.nnz_base, (uint64_t)srp[1] + it.nnz_base, red);
      if (threadIdx.x == 0) put<T>(P, out, it.row_off + r, tot);
      __syncthreads();
      r += 1;
      continue;
    }
    const uint64_t s0 = (uint64_t)base + it.nnz_base, e0 = (uint64_t)srp[k] + it.nnz_base;
    // R groups of 4 nonzeros per thread per pass: their index and value loads,
    // then all 4R x gathers in flight at once, then the products
    constexpr int R = SPARSEP_CSR_GATHER;
    for (uint64_t g0 = (s0 >> 2) + threadIdx.x; 4 * g0 < e0; g0 += (uint64_t)R * blockDim.x) {
      uint32_t cc[R][4];
      Vec4<T> v4[R];
      bool live[R];
#pragma unroll
      for (int i = 0; i < R; ++i) {
        const uint64_t j = 4 * (g0 + (uint64_t)i * blockDim.x);
        live[i] = j < e0 && !SP_BAD(P, j + 3 < P.n_idx && j + 3 < P.n_val, -1002);
        if (live[i]) {
          const uint4 c4 = ld_stream4(P.colind + j);
          v4[i] = ld_vals4<T>(P.val + j);
          cc[i][0] = c4.x, cc[i][1] = c4.y, cc[i][2] = c4.z, cc[i][3] = c4.w;
        }
      }
      T xv[R][4];
      uint32_t bad = 0;
#pragma unroll
      for (int i = 0; i < R; ++i)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const uint64_t j = 4 * (g0 + (uint64_t)i * blockDim.x) + q;
          if (live[i] && j >= s0 && j < e0) {
            const uint64_t col = (uint64_t)it.col_off + cc[i][q];
            if (SP_BAD(P, x_ok(P, it, col), -1003)) bad |= 1u << (4 * i + q);
            else xv[i][q] = xload(xb, col, staged);
          }
        }
#pragma unroll
      for (int i = 0; i < R; ++i)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const uint64_t j = 4 * (g0 + (uint64_t)i * blockDim.x) + q;
          if (live[i] && j >= s0 && j < e0)
            prods[j - s0] = (bad >> (4 * i + q)) & 1u ? A(0) : mul<T>(v4[i].v[q], xv[i][q]);
        }
    }
    __syncthreads();
    // short rows: one thread each; long rows are queued for the warps
    for (uint32_t i = threadIdx.x; i < k; i += blockDim.x) {
      const uint32_t a = srp[i] - base, b = srp[i + 1] - base;
      if (b - a <= (uint32_t)CSR_SHORT) {
        A acc = A(0);
        for (uint32_t q = a; q < b; ++q) acc += prods[q];
        put<T>(P, out, it.row_off + r + i, acc);
      } else {
        longs[atomicAdd(&nlong, 1u)] = i;
      }
    }
    __syncthreads();
    for (uint32_t li = warp; li < nlong; li += nw) {
      const uint32_t i = longs[li];
      const uint32_t a = srp[i] - base, b = srp[i + 1] - base;
      A acc = A(0);
      for (uint32_t q = a + lane; q < b; q += 32) acc += prods[q];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (lane == 0) put<T>(P, out, it.row_off + r + i, acc);
    }
    __syncthreads();
    r += k;
  }
}

// ---------------------------------------------------------------------------
// CSR long-row chunk: all threads reduce elements [a0, a1) of row crow.
// ---------------------------------------------------------------------------
template <typename T>
__device__ void csr_long(const Params<T> &P, const Item &it, const T *__restrict__ xb, uint32_t item_id) {
  using A = Acc<T>;
  __shared__ A red[32];
  const uint64_t s = it.a0, e = it.a1;
  A acc = A(0);
#pragma unroll 2
  for (uint64_t j = (s & ~3ull) + 4 * threadIdx.x; j < e; j += 4 * blockDim.x) {
    if (SP_BAD(P, j + 3 < P.n_idx && j + 3 < P.n_val, -1005)) break;
    const uint4 c4 = ld_stream4(P.colind + j);
    const Vec4<T> v4 = ld_vals4<T>(P.val + j);
    const uint32_t cc[4] = {c4.x, c4.y, c4.z, c4.w};
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (j + k >= s && j + k < e && !SP_BAD(P, x_ok(P, it, (uint64_t)it.col_off + cc[k]), -1006))
        acc += mul<T>(v4.v[k], xload(xb, (uint64_t)it.col_off + cc[k], it.xw > 0));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    A tot = A(0);
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += red[w];
    T *out = out_base(P, it);
    if (SP_BAD(P, it.crow < P.nrows && (P.out_mode == OUT_ATOMIC || item_id < P.n_carry), -1007)) return;
    if (P.out_mode == OUT_ATOMIC) {
      atomic_add_out<T>(out + it.crow, tot);
    } else {
      // the last chunk of the row to arrive sums the row's partials in chunk order
      P.carry_val[item_id] = acc_bits(tot);
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
}

// ---------------------------------------------------------------------------
// Units of the element-wise paths: COO elements (W = 1) and BCOO blocks
// (W = rb).  A unit has a key (output row / block row) and W products.
// ---------------------------------------------------------------------------
// the reference's AoS nonzero for element type T
template <typename T> struct ElemOf;
template <> struct ElemOf<int8_t> { using type = sparsep_elem_i8; };
template <> struct ElemOf<int16_t> { using type = sparsep_elem_i16; };
template <> struct ElemOf<int32_t> { using type = sparsep_elem_i32; };
template <> struct ElemOf<int64_t> { using type = sparsep_elem_i64; };
template <> struct ElemOf<float> { using type = sparsep_elem_f32; };
template <> struct ElemOf<double> { using type = sparsep_elem_f64; };

template <typename T, int W>
struct Unit {
  long long key;
  Acc<T> v[W];
};

// Load the 4 COO elements of aligned group g (reference elem_t layout:
// {u32 rowind, u32 colind, val_dt val}, 12 bytes for types up to 4 bytes and
// 16 bytes for 8-byte types).
template <typename T>
__device__ __forceinline__ void load_coo4(const Params<T> &P, const Item &it, const T *__restrict__ xb,
                                          uint64_t g, Unit<T, 1> (&u)[4], uint64_t lo, uint64_t hi) {
  if (4 * g + 3 >= P.n_elems) {
    // last group of an array without padding: load only the elements that exist
    for (int k = 0; k < 4; ++k) {
      const uint64_t e = 4 * g + k;
      u[k].key = LLONG_MAX;
      u[k].v[0] = Acc<T>(0);
      if (e < P.n_elems && e >= lo && e < hi) {
        const auto *el = reinterpret_cast<const typename ElemOf<T>::type *>(P.elems) + e;
        u[k].key = (long long)it.row_off + el->rowind;
        u[k].v[0] = mul<T>(el->val, xload(xb, (uint64_t)it.col_off + el->colind, it.xw > 0));
      }
    }
    return;
  }
  if constexpr (sizeof(T) <= 4) {
    const char *base = reinterpret_cast<const char *>(P.elems) + g * 48;
    uint4 w0 = ld_stream4(base), w1 = ld_stream4(base + 16), w2 = ld_stream4(base + 32);
    uint32_t w[12] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w, w2.x, w2.y, w2.z, w2.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      uint64_t e = 4 * g + k;
      bool ok = e >= lo && e < hi && !SP_BAD(P, !(e >= lo && e < hi) || x_ok(P, it, (uint64_t)it.col_off + w[3 * k + 1]), -1009);
      T val;
      if constexpr (sizeof(T) == 1) val = (T)(int8_t)(w[3 * k + 2] & 0xFF);
      else if constexpr (sizeof(T) == 2) val = (T)(int16_t)(w[3 * k + 2] & 0xFFFF);
      else val = __builtin_bit_cast(T, w[3 * k + 2]);
      u[k].key = ok ? (long long)it.row_off + w[3 * k] : LLONG_MAX;
      u[k].v[0] = ok ? mul<T>(val, xload(xb, (uint64_t)it.col_off + w[3 * k + 1], it.xw > 0)) : Acc<T>(0);
    }
  } else {
    const char *base = reinterpret_cast<const char *>(P.elems) + g * 64;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      uint4 w = ld_stream4(base + 16 * k);
      uint64_t e = 4 * g + k;
      bool ok = e >= lo && e < hi && !SP_BAD(P, !(e >= lo && e < hi) || x_ok(P, it, (uint64_t)it.col_off + w.y), -1009);
      T val = __builtin_bit_cast(T, ((unsigned long long)w.w << 32) | w.z);
      u[k].key = ok ? (long long)it.row_off + w.x : LLONG_MAX;
      u[k].v[0] = ok ? mul<T>(val, xload(xb, (uint64_t)it.col_off + w.y, it.xw > 0)) : Acc<T>(0);
    }
  }
}

// Row-vector of CB elements of a dense block row, at an address aligned to CB*sizeof(T).
template <typename T, int CB>
__device__ __forceinline__ void load_brow(const T *p, T (&v)[CB]) {
  constexpr int BYTES = CB * (int)sizeof(T);
  if constexpr (BYTES >= 16) {
#pragma unroll
    for (int q = 0; q < BYTES / 16; ++q) {
      uint4 w = ld_stream4(reinterpret_cast<const char *>(p) + 16 * q);
      const T *t = reinterpret_cast<const T *>(&w);
#pragma unroll
      for (int i = 0; i < 16 / (int)sizeof(T); ++i) v[q * (16 / sizeof(T)) + i] = t[i];
    }
  } else if constexpr (BYTES == 8) {
    uint2 w = __ldcs(reinterpret_cast<const uint2 *>(p));
    const T *t = reinterpret_cast<const T *>(&w);
#pragma unroll
    for (int i = 0; i < CB; ++i) v[i] = t[i];
  } else if constexpr (BYTES == 4) {
    unsigned int w = __ldcs(reinterpret_cast<const unsigned int *>(p));
    const T *t = reinterpret_cast<const T *>(&w);
#pragma unroll
    for (int i = 0; i < CB; ++i) v[i] = t[i];
  } else {
#pragma unroll
    for (int i = 0; i < CB; ++i) v[i] = p[i];
  }
}

// One dense RB x CB block times its x-segment, accumulated into acc[RB].
// RB = CB = 0 selects the runtime-size path (rb <= 16).
template <typename T, int RB, int CB>
__device__ __forceinline__ void block_mv(const Params<T> &P, const T *__restrict__ xb, uint64_t b, uint32_t J,
                                         uint32_t col_off, Acc<T> *acc, const Item &it) {
  if (SP_BAD(P, (b + 1) * P.rb * P.cb <= P.n_val, -1010)) return;
  if constexpr (RB > 0) {
    const uint64_t c0 = (uint64_t)col_off + (uint64_t)J * CB;
    T xv[CB];
#pragma unroll
    for (int c = 0; c < CB; ++c)
      xv[c] = (c0 + c < P.ncols && !SP_BAD(P, x_ok(P, it, c0 + c), -1011)) ? xload(xb, c0 + c, it.xw > 0) : T(0);
    const T *bp = P.bval + b * (RB * CB);
#pragma unroll
    for (int r = 0; r < RB; ++r) {
      T v[CB];
      load_brow<T, CB>(bp + r * CB, v);
#pragma unroll
      for (int c = 0; c < CB; ++c) acc[r] += mul<T>(v[c], xv[c]);
    }
  } else {
    const uint32_t rb = P.rb, cb = P.cb;
    const uint64_t c0 = (uint64_t)col_off + (uint64_t)J * cb;
    const T *bp = P.bval + b * rb * cb;
    for (uint32_t c = 0; c < cb; ++c) {
      if (c0 + c >= P.ncols) break;
      if (SP_BAD(P, x_ok(P, it, c0 + c), -1011)) break;
      T xv = xload(xb, c0 + c, it.xw > 0);
      for (uint32_t r = 0; r < rb; ++r) acc[r] += mul<T>(bp[r * cb + c], xv);
    }
  }
}

// ---------------------------------------------------------------------------
// BCSR block rows, L lanes per block row
// ---------------------------------------------------------------------------
template <typename T, int RB, int CB, int L>
__device__ void bcsr_rows(const Params<T> &P, const Item &it, const T *__restrict__ xb) {
  using A = Acc<T>;
  constexpr int RMAX = RB > 0 ? RB : 16;
  constexpr int G = 32 / L;
  T *out = out_base(P, it);
  const int nw = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane / L, gl = lane % L;
  const uint32_t rb = RB > 0 ? RB : P.rb;
  const uint32_t *bp = P.rowptr + it.ptr_base;  // browptr
  for (uint64_t k = 0;; ++k) {
    const uint64_t base = it.a0 + (k * nw + warp) * G;
    if (base >= it.a1) break;
    const uint64_t br = base + g;
    const bool valid = br < it.a1;
    A acc[RMAX];
#pragma unroll
    for (int r = 0; r < RMAX; ++r) acc[r] = A(0);
    if (valid && !SP_BAD(P, it.ptr_base + br + 1 < P.n_rowptr, -1012)) {
      const uint64_t s = (uint64_t)bp[br] + it.nnz_base, e = (uint64_t)bp[br + 1] + it.nnz_base;
      for (uint64_t b = s + gl; b < e; b += L) {
        if (SP_BAD(P, b < P.n_idx, -1013)) break;
        block_mv<T, RB, CB>(P, xb, b, __ldcs(P.bcolind + b), it.col_off, acc, it);
      }
    }
#pragma unroll
    for (int r = 0; r < RMAX; ++r) {
#pragma unroll
      for (int o = L / 2; o > 0; o >>= 1) acc[r] += __shfl_xor_sync(0xffffffffu, acc[r], o);
    }
    if (valid) {
#pragma unroll
      for (int r = 0; r < RMAX; ++r) {
        if (r < (int)rb && gl == (r % L)) {
          const uint64_t row = (uint64_t)it.row_off + br * rb + r;
          if (row < it.row_end) put<T>(P, out, row, acc[r]);
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Element-wise lock-free path (COO W=1, BCOO W=rb): block segmented scan.
// Keys are output rows (COO) or output block rows (BCOO, row = key*rb + r).
// The item writes every row in [own0, own1): sums of complete row runs, zeros
// for rows without units; a run reaching own1 is a carry for the fix-up.
// ---------------------------------------------------------------------------
// Output row of key k, lane r: COO keys are output rows; BCOO keys are
// tile-local block rows (row = row_off + k*rb + r).
template <typename T, int W>
__device__ __forceinline__ uint64_t key_row(const Item &it, long long k, uint32_t r, uint32_t rb) {
  if constexpr (W == 1) return (uint64_t)k;
  else return (uint64_t)it.row_off + (uint64_t)k * rb + r;
}

template <typename T, int W>
__device__ __forceinline__ void zero_rows(const Params<T> &P, const Item &it, T *out, long long k0, long long k1,
                                          uint32_t rb) {
  // keys strictly inside (k0, k1)
  for (long long k = k0 + 1; k < k1; ++k)
    for (uint32_t r = 0; r < (W == 1 ? 1u : rb); ++r) {
      const uint64_t row = key_row<T, W>(it, k, r, rb);
      if (row < it.row_end && !SP_BAD(P, row < P.nrows, -1015)) out[row] = T(0);
    }
}

template <typename T, int W>
__device__ __forceinline__ void write_run(const Params<T> &P, const Item &it, T *out, long long key,
                                          const Acc<T> (&v)[W], uint32_t rb, bool atomic) {
#pragma unroll
  for (int r = 0; r < W; ++r) {
    if (r >= (int)rb) break;
    const uint64_t row = key_row<T, W>(it, key, r, rb);
    if (row >= it.row_end) continue;
    if (SP_BAD(P, row < P.nrows, -1015)) continue;
    if (atomic) atomic_add_out<T>(out + row, v[r]);
    else out[row] = from_acc<T>(v[r]);
  }
}

// Units per thread per chunk: COO 4 elements, BCOO 1 block.
template <typename T, int W, int RB, int CB>
__device__ __forceinline__ void load_units(const Params<T> &P, const Item &it, const T *__restrict__ xb,
                                           uint64_t t0, Unit<T, W> (&u)[W == 1 ? COO_K : 1], uint64_t lo,
                                           uint64_t hi) {
  if constexpr (W == 1) {
    load_coo4<T>(P, it, xb, t0, u, lo, hi);
  } else {
    const uint64_t b = t0;
    const bool ok = b >= lo && b < hi;
#pragma unroll
    for (int r = 0; r < W; ++r) u[0].v[r] = Acc<T>(0);
    u[0].key = LLONG_MAX;
    if (ok && !SP_BAD(P, b < P.n_elems, -1014)) {
      const sparsep_bind bi = P.bind[b];
      u[0].key = (long long)bi.rowind;
      block_mv<T, RB, CB>(P, xb, b, bi.colind, it.col_off, u[0].v, it);
    }
  }
}

template <typename T, int W, int RB, int CB>
__device__ void elems_lf(const Params<T> &P, const Item &it, const T *__restrict__ xb, uint32_t item_id,
                         uint32_t cw) {
  // cw = carry slots per item (1 for COO, rb for BCOO), the scratch stride
  using A = Acc<T>;
  using KVT = KV<A, W>;
  constexpr int K = (W == 1) ? COO_K : 1;
  __shared__ KVT scan_smem[32];
  __shared__ KVT tail_smem;
  __shared__ long long heads_smem[512];
  T *out = out_base(P, it);
  const uint32_t rb = W == 1 ? 1u : (RB > 0 ? RB : P.rb);
  const uint64_t lo = it.a0, hi = it.a1;
  const bool atomic = P.out_mode == OUT_ATOMIC;

  if (SP_BAD(P, (uint64_t)(item_id + 1) * cw <= P.n_carry || atomic, -1018)) return;
  if (lo >= hi) {  // empty: only zero the owned rows
    if (!atomic && threadIdx.x == 0) zero_rows<T, W>(P, it, out, (long long)it.own0 - 1, it.own1, rb);
    if (!atomic && threadIdx.x < cw) P.carry_idx[(uint64_t)item_id * cw + threadIdx.x] = NO_CARRY;
    return;
  }
  // thread groups: COO aligned 4-element groups, BCOO single blocks
  const uint64_t g_first = (W == 1) ? lo / 4 : lo;
  const uint64_t g_last = (W == 1) ? (hi + 3) / 4 : hi;  // exclusive
  KVT carry;
  carry.k = (long long)it.own0 - 1;
#pragma unroll
  for (int i = 0; i < W; ++i) carry.v[i] = A(0);

  for (uint64_t cg = g_first; cg < g_last; cg += blockDim.x) {
    const uint64_t g = cg + threadIdx.x;
    Unit<T, W> u[K];
    if (g < g_last) {
      load_units<T, W, RB, CB>(P, it, xb, g, u, lo, hi);
    } else {
#pragma unroll
      for (int k = 0; k < K; ++k) {
        u[k].key = LLONG_MAX;
#pragma unroll
        for (int i = 0; i < W; ++i) u[k].v[i] = A(0);
      }
    }
    // thread-local runs
    long long head = LLONG_MAX, tail = LLONG_MAX;
    A head_acc[W], run[W];
#pragma unroll
    for (int i = 0; i < W; ++i) head_acc[i] = run[i] = A(0);
    bool first = true, any = false;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (u[k].key == LLONG_MAX) continue;
      if (!any) {
        head = tail = u[k].key;
        any = true;
      } else if (u[k].key != tail) {
        if (first) {
#pragma unroll
          for (int i = 0; i < W; ++i) head_acc[i] = run[i];
          first = false;
        } else {
          write_run<T, W>(P, it, out, tail, run, rb, atomic);
        }
        if (!atomic) zero_rows<T, W>(P, it, out, tail, u[k].key, rb);
        tail = u[k].key;
#pragma unroll
        for (int i = 0; i < W; ++i) run[i] = A(0);
      }
#pragma unroll
      for (int i = 0; i < W; ++i) run[i] += u[k].v[i];
    }
    KVT mine;
    mine.k = tail;
#pragma unroll
    for (int i = 0; i < W; ++i) mine.v[i] = run[i];
    heads_smem[threadIdx.x] = any ? head : LLONG_MAX;  // read after the scan's barriers
    KVT ex, in;
    block_seg_scan<A, W>(mine, carry, ex, in, scan_smem);
    const uint64_t last_g = (g_last < cg + blockDim.x ? g_last : cg + blockDim.x) - 1;
    // a tail run is complete when the next thread starts another key; the
    // chunk's last thread hands its tail on instead
    if (any && g != last_g && heads_smem[threadIdx.x + 1] != tail) write_run<T, W>(P, it, out, tail, in.v, rb, atomic);
    // likewise the run handed over by the previous chunk
    if (threadIdx.x == 0 && carry.k >= (long long)it.own0 && head != carry.k)
      write_run<T, W>(P, it, out, carry.k, carry.v, rb, atomic);
    if (any) {
      if (!atomic) zero_rows<T, W>(P, it, out, ex.k, head, rb);
      if (head != tail) {
        A h[W];
#pragma unroll
        for (int i = 0; i < W; ++i) h[i] = head_acc[i] + (ex.k == head ? ex.v[i] : A(0));
        write_run<T, W>(P, it, out, head, h, rb, atomic);
      }
    }
    // the chunk's last thread with units hands its tail to the next chunk
    if (g == last_g) tail_smem = in;
    __syncthreads();
    carry = tail_smem;
    __syncthreads();
  }
  // final tail of the item
  if (threadIdx.x == 0) {
    if (atomic) {
      write_run<T, W>(P, it, out, carry.k, carry.v, rb, true);
    } else if (carry.k < (long long)it.own1) {
      write_run<T, W>(P, it, out, carry.k, carry.v, rb, false);
      zero_rows<T, W>(P, it, out, carry.k, it.own1, rb);
      for (uint32_t i = 0; i < cw; ++i) P.carry_idx[(uint64_t)item_id * cw + i] = NO_CARRY;
    } else {
      for (uint32_t i = 0; i < cw && i < (uint32_t)W; ++i) {
        const uint64_t row = key_row<T, W>(it, carry.k, i, rb);
        const bool ok = i < rb && row < it.row_end;
        P.carry_idx[(uint64_t)item_id * cw + i] = ok ? out_index(P, it, row) : NO_CARRY;
        P.carry_val[(uint64_t)item_id * cw + i] = acc_bits(carry.v[i]);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Carry fix-up, run by the last CTA to finish: slot runs with the same target
// are summed in item order, then added once (deterministic).
// ---------------------------------------------------------------------------
template <typename T>
__device__ void carry_fixup(const Params<T> &P, uint32_t nslots, uint32_t W) {
  using A = Acc<T>;
  for (uint32_t s = threadIdx.x; s < nslots; s += blockDim.x) {
    const unsigned long long idx = __ldcg(P.carry_idx + s);
    if (idx == NO_CARRY) continue;
    if (SP_BAD(P, idx < (uint64_t)P.nslots * P.nrows, -1016)) continue;
    if (s >= W && __ldcg(P.carry_idx + s - W) == idx) continue;  // not the first of its run
    A sum = bits_acc<A>(__ldcg(P.carry_val + s));
    for (uint32_t t = s + W; t < nslots && __ldcg(P.carry_idx + t) == idx; t += W)
      sum += bits_acc<A>(__ldcg(P.carry_val + t));
    T *p = (P.out_mode == OUT_PARTIAL ? P.part : P.y) + idx;
    T cur = __ldcg(p);
    *p = from_acc<T>(to_acc<T>(cur) + sum);
  }
}

// ---------------------------------------------------------------------------
// The item kernel
// ---------------------------------------------------------------------------
template <typename T, int FMT, int RB, int CB>
__global__ void __launch_bounds__(512) spmv_items(Params<T> P, uint32_t carry_w) {
  extern __shared__ __align__(128) unsigned char dyn_smem[];
  __shared__ uint64_t mbar;
  __shared__ uint32_t is_last;
  const uint32_t item_id = blockIdx.x;
  const Item it = P.items[item_id];
  const T *xb = P.x;
  if (it.xw > 0) {
    uint32_t phase = 0;
    mbar_init(&mbar);
    xb = stage_x<T>(P.x, it.xlo, it.xw, dyn_smem, &mbar, phase, P.err, P.smem_bytes,
                    reinterpret_cast<uintptr_t>(P.x + P.n_xalloc), P.fault_wait);
  }

  if constexpr (FMT == SPARSEP_FMT_CSR) {
    if (it.kind == ITEM_LONG) {
      csr_long<T>(P, it, xb, item_id);
    } else {
      switch (it.lanes) {
        case 0: csr_stream<T>(P, it, xb); break;
        case 1: csr_rows<T, 1>(P, it, xb); break;
        case 2: csr_rows<T, 2>(P, it, xb); break;
        case 4: csr_rows<T, 4>(P, it, xb); break;
        case 8: csr_rows<T, 8>(P, it, xb); break;
        case 16: csr_rows<T, 16>(P, it, xb); break;
        default: csr_rows<T, 32>(P, it, xb); break;
      }
    }
  } else if constexpr (FMT == SPARSEP_FMT_COO) {
    elems_lf<T, 1, 0, 0>(P, it, xb, item_id, carry_w);
  } else if constexpr (FMT == SPARSEP_FMT_BCSR) {
    switch (it.lanes) {
      case 1: bcsr_rows<T, RB, CB, 1>(P, it, xb); break;
      case 2: bcsr_rows<T, RB, CB, 2>(P, it, xb); break;
      case 4: bcsr_rows<T, RB, CB, 4>(P, it, xb); break;
      case 8: bcsr_rows<T, RB, CB, 8>(P, it, xb); break;
      case 16: bcsr_rows<T, RB, CB, 16>(P, it, xb); break;
      default: bcsr_rows<T, RB, CB, 32>(P, it, xb); break;
    }
  } else {
    elems_lf<T, (RB > 0 ? RB : 16), RB, CB>(P, it, xb, item_id, carry_w);
  }

  // lock-free carries: the last CTA to finish adds them (threadfence reduction)
  if (P.carry_idx != nullptr && P.out_mode != OUT_ATOMIC) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      const unsigned int ticket = atomicAdd(P.done, 1u);
      is_last = (ticket == P.nitems - 1);
    }
    __syncthreads();
    if (is_last) {
      __threadfence();
      carry_fixup<T>(P, P.nitems * carry_w, carry_w);
      if (threadIdx.x == 0) *P.done = 0;
    }
  }

  // Host-buffer path: the item is counted in its row band once all of its
  // writes to y are visible device-wide (barrier, then one fence before the
  // count: the fence is cumulative over the writes the barrier ordered before
  // it); a copy stream waiting on the band's count moves those rows to the
  // host while later items still run.
  if (P.band_cnt != nullptr) {
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      atomicAdd(P.band_cnt + P.items[item_id].band, 1u);  // re-read: keeps the band out of the body's registers
    }
  }
}

// ---------------------------------------------------------------------------
// 2D merge of per-stripe partial y, in stripe order like the reference's host
// merge (spmv/2D/BDCSR/host/app.c:437-447, spmv/2D/DCSR/host/app.c:340-351).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void merge_partials(const T *__restrict__ part, T *__restrict__ y, uint32_t nrows, uint32_t V) {
  for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nrows; r += (uint64_t)gridDim.x * blockDim.x) {
    Acc<T> s = to_acc<T>(__ldcs(part + r));
    for (uint32_t c = 1; c < V; ++c) {
      if constexpr (std::is_floating_point<T>::value) s = (T)(s + __ldcs(part + (uint64_t)c * nrows + r));
      else s += to_acc<T>(__ldcs(part + (uint64_t)c * nrows + r));
    }
    y[r] = from_acc<T>(s);
  }
}


}  // namespace sparsep
