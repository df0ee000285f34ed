// kernels.hpp -- host-side declarations of the kernel launchers (kernels.cu).
#pragma once
#include <cuda_runtime.h>

#include "device.cuh"

namespace sparsep {

// Launch the work-item kernel for format `fmt` (sparsep_format) with one CTA
// per item.  carry_w = carry slots per item (1 for CSR/COO, rb for BCOO).
template <typename T>
cudaError_t launch_items(const Params<T> &P, int fmt, uint32_t carry_w, int threads, size_t smem,
                         cudaStream_t st);

// y[r] = sum over the V partial slices of row r, in slice order.
template <typename T>
cudaError_t launch_merge(const T *part, T *y, uint32_t nrows, uint32_t V, int sms, cudaStream_t st);

// Persistent TMA-pipelined CSR kernel (csr_pipe.cu) for 1D items built by the
// automatic planner; grid = SMs x resident CTAs (capped at the item count).
template <typename T>
cudaError_t launch_csr_pipe(const Params<T> &P, int sms, cudaStream_t st, int *grid_out, uint32_t max_item_nnz);

// Split CSR plans (csr_stripes.cu).  stripe_geometry gives, for element type
// T, the stripe width (columns), the kernel's dynamic shared memory, the
// nonzeros of a heavy and of a light chunk and the rows of a chunk;
// launch_stripes runs `ctas` persistent CTAs over their chunk lists;
// launch_heavy_merge writes y[hrow[k]] = sum over stripes of the partials.
template <typename T>
void stripe_geometry(uint32_t *width, size_t *smem, uint32_t *chunk_nnz, uint32_t *light_nnz, uint32_t *chunk_rows);
template <typename T>
cudaError_t launch_stripes(const StripeParams<T> &P, uint32_t ctas, cudaStream_t st);
template <typename T>
cudaError_t launch_heavy_merge(const T *part, const uint32_t *hrow, uint32_t nH, uint32_t nS, T *y, int sms,
                               cudaStream_t st);

}  // namespace sparsep
