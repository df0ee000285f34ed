// kernels.cu -- host launchers of the sm_100a SpMV kernels (kernels_impl.cuh).
#include <atomic>

#include "kernels_impl.cuh"
#include "kernels.hpp"

namespace sparsep {

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
template <typename T, int FMT, int RB, int CB>
static cudaError_t launch_t(const Params<T> &P, uint32_t carry_w, int threads, size_t smem, cudaStream_t st) {
  auto k = spmv_items<T, FMT, RB, CB>;
  // the default dynamic limit is 48 KB minus the kernel's static shared
  // memory; the largest size set so far is kept per device (host threads may
  // plan concurrently, on different devices)
  static std::atomic<int> configured[64];
  if (smem > 0) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::atomic<int> &c = configured[dev & 63];
    if ((int)smem > c.load()) {
      e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
      int cur = c.load();
      while ((int)smem > cur && !c.compare_exchange_weak(cur, (int)smem)) {
      }
    }
  }
  k<<<P.nitems, threads, smem, st>>>(P, carry_w);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_items(const Params<T> &P, int fmt, uint32_t carry_w, int threads, size_t smem,
                         cudaStream_t st) {
  if (P.nitems == 0) return cudaSuccess;
  const uint32_t rb = P.rb, cb = P.cb;
  switch (fmt) {
    case SPARSEP_FMT_CSR: return launch_t<T, SPARSEP_FMT_CSR, 0, 0>(P, carry_w, threads, smem, st);
    case SPARSEP_FMT_COO: return launch_t<T, SPARSEP_FMT_COO, 0, 0>(P, carry_w, threads, smem, st);
    case SPARSEP_FMT_BCSR:
      if (rb == 4 && cb == 4) return launch_t<T, SPARSEP_FMT_BCSR, 4, 4>(P, carry_w, threads, smem, st);
      if (rb == 8 && cb == 8) return launch_t<T, SPARSEP_FMT_BCSR, 8, 8>(P, carry_w, threads, smem, st);
      if (rb == 2 && cb == 2) return launch_t<T, SPARSEP_FMT_BCSR, 2, 2>(P, carry_w, threads, smem, st);
      return launch_t<T, SPARSEP_FMT_BCSR, 0, 0>(P, carry_w, threads, smem, st);
    case SPARSEP_FMT_BCOO:
      if (rb == 4 && cb == 4) return launch_t<T, SPARSEP_FMT_BCOO, 4, 4>(P, carry_w, threads, smem, st);
      if (rb == 8 && cb == 8) return launch_t<T, SPARSEP_FMT_BCOO, 8, 8>(P, carry_w, threads, smem, st);
      if (rb == 2 && cb == 2) return launch_t<T, SPARSEP_FMT_BCOO, 2, 2>(P, carry_w, threads, smem, st);
      return launch_t<T, SPARSEP_FMT_BCOO, 0, 0>(P, carry_w, threads, smem, st);
  }
  return cudaErrorInvalidValue;
}

template <typename T>
cudaError_t launch_merge(const T *part, T *y, uint32_t nrows, uint32_t V, int sms, cudaStream_t st) {
  if (nrows == 0) return cudaSuccess;
  uint32_t blocks = (nrows + 255) / 256;
  uint32_t cap = (uint32_t)sms * 8;
  if (blocks > cap) blocks = cap;
  merge_partials<T><<<blocks, 256, 0, st>>>(part, y, nrows, V);
  return cudaGetLastError();
}

// The build compiles this file once per element type (-DSPARSEP_KT=<type>) so
// the instantiations build in parallel.
#ifndef SPARSEP_KT
#define SPARSEP_KT float
#endif
template cudaError_t launch_items<SPARSEP_KT>(const Params<SPARSEP_KT> &, int, uint32_t, int, size_t, cudaStream_t);
template cudaError_t launch_merge<SPARSEP_KT>(const SPARSEP_KT *, SPARSEP_KT *, uint32_t, uint32_t, int, cudaStream_t);

}  // namespace sparsep
