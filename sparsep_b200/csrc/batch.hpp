// batch.hpp -- work items and matrix descriptors of the batched multi-RHS
// SpMV, shared by the host planner (batch.cu) and the kernels
// (batch_kernels.cu, compiled once per element type).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace sparsep {
namespace batch {

// Device arrays of one matrix of the batch (host-side record).
template <typename T> struct Mat {
  const uint32_t *rowptr;
  const uint32_t *colind;
  const T *val;
  const T *x;
  T *y;
  uint32_t nrows, ncols, k, pad;
};

constexpr int BT = 256;            // threads per CTA
constexpr uint32_t BCAP = 4096;    // nonzeros staged per item (and per long-row chunk)
constexpr uint32_t BRCAP = 1024;   // rows per item
constexpr int ACC_REGS = 8;        // V * ACC accumulators per lane

enum : uint8_t { MODE_ROWS = 0, MODE_MERGE = 1, MODE_LONG = 2 };

// A work item carries its matrix's arrays, so a CTA needs one load to start.
struct BItem {
  const uint32_t *rowptr;
  const uint32_t *colind;
  const void *val;
  const void *x;
  void *y;
  uint32_t r0;      // rows [r0, r0 + nr)
  uint32_t p0, p1;  // nonzeros [p0, p1) = rowptr[r0] .. rowptr[r0 + nr]
  uint32_t ncols;   // columns of the matrix (bounds of x)
  uint16_t nr;      // rows (<= BRCAP)
  uint16_t k;       // right-hand sides (x: ncols x k, y: nrows x k, row-major)
  uint8_t mode, lanes, vec, acc;
};
static_assert(sizeof(BItem) == 64, "item layout");

// One kernel launch over items: with `head`, n CTAs claim items
// items[0 .. n) in queue order by atomic ticket (head must be 0 at launch);
// without it, CTA b runs items[i0 + b].  A staging copy that never lands
// (bounded wait) sets *err to SPARSEP_ETIMEDOUT and its item is skipped.
// Device arrays need 16 elements of slack past their end (rowptr included):
// staging copies 16-byte aligned windows.
template <typename T>
cudaError_t batch_launch(const BItem *items, uint32_t i0, uint32_t n, unsigned int *head, int *err,
                         cudaStream_t s);

}  // namespace batch
}  // namespace sparsep
