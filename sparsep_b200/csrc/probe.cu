// probe.cu -- the gather floor of an SpMV: the time to read x at a matrix's
// column indices and nothing else (no values, row pointers, sums per row or
// stores of y).  Measurement support with no reference counterpart: a CSR
// SpMV over uniformly random columns is bound by this random-gather rate,
// not by HBM bandwidth, and this kernel measures that bound on the device.
#include <cstdint>

#include "sparsep.h"

namespace sparsep {
namespace probe {

constexpr int NT = 512;

// Every thread strides over the indices and sums x at them (the sum is
// stored so that the loads are not optimised away).
__global__ void __launch_bounds__(NT) gather_sum(const uint32_t *__restrict__ idx, uint64_t n,
                                                 const float *__restrict__ x, float *__restrict__ out) {
  const uint64_t tid = (uint64_t)blockIdx.x * NT + threadIdx.x, nth = (uint64_t)gridDim.x * NT;
  float s = 0.f;
  for (uint64_t i = tid; i < n; i += nth) s += __ldg(x + __ldcs(idx + i));
  out[tid] = s;
}

}  // namespace probe
}  // namespace sparsep

extern "C" int sparsep_probe_gather_f32(const uint32_t *d_idx, uint64_t n, const float *d_x, float *d_out,
                                        int ctas, void *stream) {
  if (!d_idx || !d_x || !d_out || ctas < 1) return SPARSEP_EINVAL;
  sparsep::probe::gather_sum<<<ctas, sparsep::probe::NT, 0, static_cast<cudaStream_t>(stream)>>>(d_idx, n, d_x,
                                                                                               d_out);
  return cudaGetLastError() == cudaSuccess ? SPARSEP_OK : SPARSEP_EIO;
}
