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
  T *part;         // rows longer than BCAP: their chunks' partial rows (chunks x pitch each)
  unsigned *cnt;   // and one arrival counter per such row (zero between launches)
  const uint32_t *browptr;  // 4 x 4 BCSR copy (block variants), or null: block-row pointers,
  const uint32_t *bcol;     // block columns,
  const T *bval;            // 16 values per block, row-major
  uint32_t nrows, ncols, k;
  uint32_t pitch;  // x / y row pitch in elements: k rounded up to a multiple of 4 (k >= 3)
};

// Row pitch of x and y on the device: k for k <= 2, else k rounded up to a
// multiple of 4, so that every row starts on a 16-byte boundary and 4-wide
// loads serve any k.  Column j of y depends on column j of x only, so the
// pad columns never reach a result.
constexpr uint32_t row_pitch(uint32_t k) { return k <= 2 ? k : (k + 3) & ~3u; }

constexpr int BT = 256;            // threads per CTA
#ifndef SPARSEP_BATCH_BCAP
#define SPARSEP_BATCH_BCAP 5120
#endif
#ifndef SPARSEP_BATCH_ARENA
#define SPARSEP_BATCH_ARENA 48000
#endif
#ifndef SPARSEP_BATCH_MINB
#define SPARSEP_BATCH_MINB 4
#endif
constexpr uint32_t MINB = SPARSEP_BATCH_MINB;  // CTAs per SM the kernel's registers are budgeted for
constexpr uint32_t BCAP = SPARSEP_BATCH_BCAP;  // nonzeros staged per item (and per long-row chunk)
constexpr uint32_t BRCAP = 1024;   // rows per item
constexpr int ACC_REGS = 8;        // V * ACC accumulators per lane

enum : uint8_t { MODE_ROWS = 0, MODE_MERGE = 1, MODE_LONG = 2, MODE_BCSR = 3 };
constexpr uint32_t BBCAP = 512;   // 4 x 4 blocks staged per block item

// Per-CTA staging arena (static shared memory, under the 48 KB static limit
// with the carry rows and the barrier).  A work item's staged arrays are
// carved from it in this order, each region 16-byte aligned with room for the
// alignment lead and tail of its copy: rowptr slice, column indices, values,
// and for a window item the rows [c0, c0 + cw) of x.  The host cuts items so
// that the carve fits; the kernel recomputes it from the item.
constexpr uint32_t ARENA = SPARSEP_BATCH_ARENA;
struct Carve {
  uint32_t col, val, xw, end;  // byte offsets (the rowptr slice starts at 0)
};
__host__ __device__ constexpr uint32_t align16(uint32_t v) { return (v + 15u) & ~15u; }
__host__ __device__ constexpr Carve carve(uint32_t nr, uint32_t n, uint32_t es, uint32_t xbytes) {
  return Carve{align16((nr + 1) * 4 + 32), align16((nr + 1) * 4 + 32) + align16(n * 4 + 32),
               align16((nr + 1) * 4 + 32) + align16(n * 4 + 32) + align16(n * es + 32),
               align16((nr + 1) * 4 + 32) + align16(n * 4 + 32) + align16(n * es + 32) +
                   (xbytes ? align16(xbytes + 32) : 0)};
}
static_assert(carve(BRCAP, BCAP, 4, 0).end <= ARENA, "a full item of 4-byte values fits the arena");

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
  uint16_t k;       // row pitch of x (ncols x k) and y (nrows x k), row-major: the
                    // right-hand sides rounded up (row_pitch), all computed
  uint8_t mode, lanes, vec, acc;
  uint32_t c0;      // window item: x rows [c0, c0 + cw) staged in shared memory
  uint32_t cw;      // and every column of the item inside them; 0: x read from memory.
                    // MODE_LONG (one chunk of a row longer than BCAP): chunk c0 of cw
  void *part;       // MODE_LONG: the row's chunk partials (cw x k elements)
  unsigned *cnt;    // MODE_LONG: the row's arrival counter (the last chunk sums, resets)
  uint32_t nrows;   // rows of the matrix (MODE_BCSR: the last block row's rows past it are not stored)
  uint32_t pad;
};
// MODE_BCSR items: rowptr / colind / val are the 4 x 4 BCSR copy's block-row
// pointers, block columns and values; r0, nr count block rows and p0, p1 blocks.
static_assert(sizeof(BItem) == 96, "item layout");
static_assert(carve(BRCAP / 4, BBCAP, 64, 0).end <= ARENA, "a full block item fits the arena");

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
