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

// Every thread strides over the indices, four at a time (one 16-byte load),
// two groups per step: eight independent x reads in flight per thread, each
// summed into its own accumulator (the sums are stored so that the loads are
// not optimised away).  idx must be 16-byte aligned.
__global__ void __launch_bounds__(NT) gather_sum(const uint32_t *__restrict__ idx, uint64_t n,
                                                 const float *__restrict__ x, float *__restrict__ out) {
  const uint64_t tid = (uint64_t)blockIdx.x * NT + threadIdx.x, nth = (uint64_t)gridDim.x * NT;
  const uint64_t n4 = n / 4;
  const uint4 *idx4 = reinterpret_cast<const uint4 *>(idx);
  float s[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  uint64_t i = tid;
  for (; i + nth < n4; i += 2 * nth) {
    const uint4 a = __ldcs(idx4 + i), b = __ldcs(idx4 + i + nth);
    s[0] += __ldg(x + a.x);
    s[1] += __ldg(x + a.y);
    s[2] += __ldg(x + a.z);
    s[3] += __ldg(x + a.w);
    s[4] += __ldg(x + b.x);
    s[5] += __ldg(x + b.y);
    s[6] += __ldg(x + b.z);
    s[7] += __ldg(x + b.w);
  }
  for (; i < n4; i += nth) {
    const uint4 a = __ldcs(idx4 + i);
    s[0] += __ldg(x + a.x);
    s[1] += __ldg(x + a.y);
    s[2] += __ldg(x + a.z);
    s[3] += __ldg(x + a.w);
  }
  for (uint64_t j = n4 * 4 + tid; j < n; j += nth) s[0] += __ldg(x + __ldcs(idx + j));
  out[tid] = ((s[0] + s[1]) + (s[2] + s[3])) + ((s[4] + s[5]) + (s[6] + s[7]));
}

}  // namespace probe
}  // namespace sparsep

extern "C" int sparsep_probe_gather_f32(const uint32_t *d_idx, uint64_t n, const float *d_x, float *d_out,
                                        int ctas, void *stream) {
  if (!d_idx || !d_x || !d_out || ctas < 1 || (reinterpret_cast<uintptr_t>(d_idx) & 15)) return SPARSEP_EINVAL;
  sparsep::probe::gather_sum<<<ctas, sparsep::probe::NT, 0, static_cast<cudaStream_t>(stream)>>>(d_idx, n, d_x,
                                                                                               d_out);
  return cudaGetLastError() == cudaSuccess ? SPARSEP_OK : SPARSEP_EIO;
}
