/*
 * sparsep_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of SparseP's host-side CPU SpMV (`spmv_host`), one
 * function per reference struct and element type, used as the checker of the
 * sparsep_b200 CUDA path.  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg may load this library; the product never does.
 *
 * Each function follows the reference loop order and arithmetic exactly:
 * the accumulator is the element type (`val_dt sum = 0; sum += x * val`), so
 * integer results wrap at the element width (built with -fwrapv, which pins the
 * int32/int64 wrap-around the reference relies on) and FP sums are sequential
 * in the reference order (built with -ffp-contract=off, as the reference's
 * -std=c11 build).  Pinned against the reference itself: tests compare these
 * functions with the reference's own spmv_host compiled from its sources
 * (oracle/build_ref.sh -> oracle/_ref) and with committed golden vectors
 * (tests/golden/).
 *
 * y-length conventions follow the reference's allocation of y_host:
 *   CSR / COO / RBD / BD CSR-COO: nrows;  BCSR / BCOO: num_block_rows*rb;
 *   D tiles: horz_partitions*tile_height (+ rb for block tiles);
 *   2D block stripes: nrows + rb.
 * x must hold every column the reference reads (block formats read whole
 * blocks; the reference pads x, e.g. spmv/2D/DBCSR/host/app.c:151-169).
 * Functions that the reference calls on a calloc'd y zero y first.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

#include "sparsep.h"

#define ORACLE_DEFINE(T, S)                                                                          \
  /* spmv/1D/CSR-row/host/app.c:66-77 */                                                             \
  void oracle_spmv_csr_##S(T *y, const sparsep_csr_##S *A, const T *x) {                            \
    for (uint32_t r = 0; r < A->nrows; ++r) {                                                        \
      T sum = 0;                                                                                     \
      for (uint32_t i = A->rowptr[r]; i < A->rowptr[r + 1]; ++i) sum += x[A->colind[i]] * A->values[i]; \
      y[r] = sum;                                                                                    \
    }                                                                                                \
  }                                                                                                  \
  /* spmv/1D/COO-nnz/host/app.c:69-74 (y calloc'd by the caller there) */                           \
  void oracle_spmv_cooe_##S(T *y, const sparsep_cooe_##S *A, const T *x) {                          \
    memset(y, 0, sizeof(T) * A->nrows);                                                              \
    for (uint32_t n = 0; n < A->nnz; n++) y[A->nnzs[n].rowind] += x[A->nnzs[n].colind] * A->nnzs[n].val; \
  }                                                                                                  \
  /* spmv/1D/BCSR-nnz/host/app.c:71-86 */                                                            \
  void oracle_spmv_bcsr_##S(T *y, const sparsep_bcsr_##S *A, const T *x) {                          \
    const uint64_t rb = A->row_block_size, cb = A->col_block_size;                                   \
    memset(y, 0, sizeof(T) * (size_t)A->num_block_rows * rb);                                        \
    for (uint64_t n = 0; n < A->num_block_rows; n++)                                                 \
      for (uint64_t i = A->browptr[n]; i < A->browptr[n + 1]; i++) {                                 \
        uint64_t j = A->bcolind[i];                                                                  \
        for (uint64_t r = 0; r < rb; r++) {                                                          \
          T acc = 0;                                                                                 \
          for (uint64_t c = 0; c < cb; c++)                                                          \
            if ((n * rb + r < A->nrows) && (j * cb + c < A->ncols))                                  \
              acc += A->bval[i * cb * rb + r * cb + c] * x[j * cb + c];                              \
          y[n * rb + r] += acc;                                                                      \
        }                                                                                            \
      }                                                                                              \
  }                                                                                                  \
  /* spmv/1D/BCOO-nnz/host/app.c:72-86 */                                                            \
  void oracle_spmv_bcoo_##S(T *y, const sparsep_bcoo_##S *A, const T *x) {                          \
    const uint64_t rb = A->row_block_size, cb = A->col_block_size;                                   \
    memset(y, 0, sizeof(T) * (size_t)A->num_block_rows * rb);                                        \
    for (uint64_t n = 0; n < A->num_blocks; n++) {                                                   \
      uint64_t i = A->bind[n].rowind, j = A->bind[n].colind;                                         \
      for (uint64_t r = 0; r < rb; r++) {                                                            \
        T acc = 0;                                                                                   \
        for (uint64_t c = 0; c < cb; c++)                                                            \
          if ((i * rb + r < A->nrows) && (j * cb + c < A->ncols))                                    \
            acc += A->bval[n * cb * rb + r * cb + c] * x[j * cb + c];                                \
        y[i * rb + r] += acc;                                                                        \
      }                                                                                              \
    }                                                                                                \
  }                                                                                                  \
  /* spmv/2D/DCSR/host/app.c:84-103 */                                                               \
  void oracle_spmv_dcsr_##S(T *y, const sparsep_dcsr_##S *A, const T *x) {                          \
    memset(y, 0, sizeof(T) * (size_t)A->horz_partitions * A->tile_height);                          \
    uint64_t tot = 0;                                                                                \
    for (uint32_t r = 0; r < A->horz_partitions; r++)                                                \
      for (uint32_t c = 0; c < A->vert_partitions; c++)                                              \
        for (uint32_t row = 0; row < A->tile_height; ++row) {                                        \
          T sum = 0;                                                                                 \
          uint64_t po = (uint64_t)(r * A->vert_partitions + c) * (A->tile_height + 1);               \
          for (uint32_t n = A->drowptr[po + row]; n < A->drowptr[po + row + 1]; n++) {               \
            uint32_t col = A->dcolind[tot];                                                          \
            T v = A->dval[tot++];                                                                    \
            sum += x[c * A->tile_width + col] * v;                                                   \
          }                                                                                          \
          y[r * A->tile_height + row] += sum;                                                        \
        }                                                                                            \
  }                                                                                                  \
  /* spmv/2D/RBDCSR/host/app.c:88-103 */                                                             \
  void oracle_spmv_rbdcsr_##S(T *y, const sparsep_rbdcsr_##S *A, const T *x) {                      \
    memset(y, 0, sizeof(T) * A->nrows);                                                              \
    uint64_t tot = 0;                                                                                \
    for (uint32_t c = 0; c < A->vert_partitions; c++)                                                \
      for (uint32_t row = 0; row < A->nrows; ++row) {                                                \
        T sum = 0;                                                                                   \
        uint64_t po = (uint64_t)c * (A->nrows + 1);                                                  \
        for (uint32_t n = A->drowptr[po + row]; n < A->drowptr[po + row + 1]; n++) {                 \
          uint32_t col = A->dcolind[tot];                                                            \
          T v = A->dval[tot++];                                                                      \
          sum += x[c * A->tile_width + col] * v;                                                     \
        }                                                                                            \
        y[row] += sum;                                                                               \
      }                                                                                              \
  }                                                                                                  \
  /* spmv/2D/BDCSR/host/app.c:88-103 */                                                              \
  void oracle_spmv_bdcsr_##S(T *y, const sparsep_bdcsr_##S *A, const T *x) {                        \
    memset(y, 0, sizeof(T) * A->nrows);                                                              \
    uint64_t tot = 0;                                                                                \
    for (uint32_t c = 0; c < A->vert_partitions; c++)                                                \
      for (uint32_t row = 0; row < A->nrows; ++row) {                                                \
        T sum = 0;                                                                                   \
        uint64_t po = (uint64_t)c * (A->nrows + 1);                                                  \
        for (uint32_t n = A->drowptr[po + row]; n < A->drowptr[po + row + 1]; n++) {                 \
          uint32_t col = A->dcolind[tot];                                                            \
          T v = A->dval[tot++];                                                                      \
          sum += x[A->vert_tile_widths[c] + col] * v;                                                \
        }                                                                                            \
        y[row] += sum;                                                                               \
      }                                                                                              \
  }                                                                                                  \
  /* spmv/2D/DCOO/host/app.c:80-95 */                                                                \
  void oracle_spmv_dcoo_##S(T *y, const sparsep_dcoo_##S *A, const T *x) {                          \
    memset(y, 0, sizeof(T) * (size_t)A->horz_partitions * A->tile_height);                          \
    uint64_t tot = 0;                                                                                \
    for (uint32_t r = 0; r < A->horz_partitions; r++)                                                \
      for (uint32_t c = 0; c < A->vert_partitions; c++) {                                            \
        uint32_t p = r * A->vert_partitions + c;                                                     \
        for (uint32_t n = 0; n < A->nnzs_per_partition[p]; n++) {                                    \
          uint32_t row = A->nnzs[tot].rowind, col = A->nnzs[tot].colind;                             \
          T v = A->nnzs[tot++].val;                                                                  \
          y[r * A->tile_height + row] += (v * x[c * A->tile_width + col]);                           \
        }                                                                                            \
      }                                                                                              \
  }                                                                                                  \
  /* spmv/2D/RBDCOO/host/app.c (spmv_host) */                                                        \
  void oracle_spmv_rbdcoo_##S(T *y, const sparsep_rbdcoo_##S *A, const T *x) {                      \
    memset(y, 0, sizeof(T) * A->nrows);                                                              \
    uint64_t tot = 0;                                                                                \
    for (uint32_t c = 0; c < A->vert_partitions; c++)                                                \
      for (uint32_t n = 0; n < A->nnzs_per_vert_partition[c]; n++) {                                 \
        uint32_t row = A->nnzs[tot].rowind, col = A->nnzs[tot].colind;                               \
        T v = A->nnzs[tot++].val;                                                                    \
        y[row] += (v * x[c * A->tile_width + col]);                                                  \
      }                                                                                              \
  }                                                                                                  \
  /* spmv/2D/BDCOO/host/app.c:88-100 */                                                              \
  void oracle_spmv_bdcoo_##S(T *y, const sparsep_bdcoo_##S *A, const T *x) {                        \
    memset(y, 0, sizeof(T) * A->nrows);                                                              \
    uint64_t tot = 0;                                                                                \
    for (uint32_t c = 0; c < A->vert_partitions; c++)                                                \
      for (uint32_t n = 0; n < A->nnzs_per_vert_partition[c]; n++) {                                 \
        uint32_t row = A->nnzs[tot].rowind, col = A->nnzs[tot].colind;                               \
        T v = A->nnzs[tot++].val;                                                                    \
        y[row] += (v * x[A->vert_tile_widths[c] + col]);                                             \
      }                                                                                              \
  }                                                                                                  \
  /* spmv/2D/DBCSR/host/app.c:86-110 */                                                              \
  void oracle_spmv_dbcsr_##S(T *y, const sparsep_dbcsr_##S *A, const T *x) {                        \
    const uint64_t rb = A->row_block_size, cb = A->col_block_size;                                   \
    memset(y, 0, sizeof(T) * ((size_t)A->horz_partitions * A->tile_height + rb));                   \
    uint64_t tb = 0;                                                                                 \
    for (uint32_t r = 0; r < A->horz_partitions; r++)                                                \
      for (uint32_t c = 0; c < A->vert_partitions; c++) {                                            \
        uint64_t po = (uint64_t)(r * A->vert_partitions + c) * (A->num_block_rows + 1);              \
        for (uint64_t n = 0; n < A->num_block_rows; n++)                                             \
          for (uint64_t i = A->browptr[po + n]; i < A->browptr[po + n + 1]; i++) {                   \
            uint64_t j = A->bcolind[tb + i];                                                         \
            for (uint64_t br = 0; br < rb; br++) {                                                   \
              T acc = 0;                                                                             \
              for (uint64_t bc = 0; bc < cb; bc++)                                                   \
                acc += A->bval[(tb + i) * cb * rb + br * cb + bc] * x[c * A->tile_width + j * cb + bc]; \
              y[r * A->tile_height + n * rb + br] += acc;                                            \
            }                                                                                        \
          }                                                                                          \
        tb += A->blocks_per_partition[r * A->vert_partitions + c];                                   \
      }                                                                                              \
  }                                                                                                  \
  /* spmv/2D/DBCOO/host/app.c:88 */                                                                  \
  void oracle_spmv_dbcoo_##S(T *y, const sparsep_dbcoo_##S *A, const T *x) {                        \
    const uint64_t rb = A->row_block_size, cb = A->col_block_size;                                   \
    memset(y, 0, sizeof(T) * ((size_t)A->horz_partitions * A->tile_height + rb));                   \
    uint64_t tb = 0;                                                                                 \
    for (uint32_t r = 0; r < A->horz_partitions; r++)                                                \
      for (uint32_t c = 0; c < A->vert_partitions; c++) {                                            \
        uint32_t p = r * A->vert_partitions + c;                                                     \
        for (uint64_t n = 0; n < A->blocks_per_partition[p]; n++) {                                  \
          uint64_t i = A->bind[tb + n].rowind, j = A->bind[tb + n].colind;                           \
          for (uint64_t br = 0; br < rb; br++) {                                                     \
            T acc = 0;                                                                               \
            for (uint64_t bc = 0; bc < cb; bc++)                                                     \
              acc += A->bval[tb * rb * cb + n * cb * rb + br * cb + bc] * x[c * A->tile_width + j * cb + bc]; \
            y[r * A->tile_height + i * rb + br] += acc;                                              \
          }                                                                                          \
        }                                                                                            \
        tb += A->blocks_per_partition[p];                                                            \
      }                                                                                              \
  }                                                                                                  \
  /* spmv/2D/RBDBCSR-nnz/host/app.c:91 */                                                            \
  void oracle_spmv_rbdbcsr_##S(T *y, const sparsep_rbdbcsr_##S *A, const T *x) {                    \
    const uint64_t rb = A->row_block_size, cb = A->col_block_size;                                   \
    memset(y, 0, sizeof(T) * ((size_t)A->nrows + rb));                                               \
    uint64_t tb = 0;                                                                                 \
    for (uint32_t c = 0; c < A->vert_partitions; c++) {                                              \
      uint64_t po = (uint64_t)c * (A->num_block_rows + 1);                                           \
      for (uint64_t n = 0; n < A->num_block_rows; n++)                                               \
        for (uint64_t i = A->browptr[po + n]; i < A->browptr[po + n + 1]; i++) {                     \
          uint64_t j = A->bcolind[tb + i];                                                           \
          for (uint64_t br = 0; br < rb; br++) {                                                     \
            T acc = 0;                                                                               \
            for (uint64_t bc = 0; bc < cb; bc++)                                                     \
              acc += A->bval[(tb + i) * cb * rb + br * cb + bc] * x[c * A->tile_width + j * cb + bc]; \
            y[n * rb + br] += acc;                                                                   \
          }                                                                                          \
        }                                                                                            \
      tb += A->blocks_per_vert_partition[c];                                                         \
    }                                                                                                \
  }                                                                                                  \
  /* spmv/2D/RBDBCOO-nnz/host/app.c:94 */                                                            \
  void oracle_spmv_rbdbcoo_##S(T *y, const sparsep_rbdbcoo_##S *A, const T *x) {                    \
    const uint64_t rb = A->row_block_size, cb = A->col_block_size;                                   \
    memset(y, 0, sizeof(T) * ((size_t)A->nrows + rb));                                               \
    uint64_t tb = 0;                                                                                 \
    for (uint32_t c = 0; c < A->vert_partitions; c++) {                                              \
      for (uint64_t n = 0; n < A->blocks_per_vert_partition[c]; n++) {                               \
        uint64_t i = A->bind[tb + n].rowind, j = A->bind[tb + n].colind;                             \
        for (uint64_t br = 0; br < rb; br++) {                                                       \
          T acc = 0;                                                                                 \
          for (uint64_t bc = 0; bc < cb; bc++)                                                       \
            acc += A->bval[tb * rb * cb + n * cb * rb + br * cb + bc] * x[c * A->tile_width + j * cb + bc]; \
          y[i * rb + br] += acc;                                                                     \
        }                                                                                            \
      }                                                                                              \
      tb += A->blocks_per_vert_partition[c];                                                         \
    }                                                                                                \
  }                                                                                                  \
  /* spmv/2D/BDBCSR-nnz/host/app.c:91 */                                                             \
  void oracle_spmv_bdbcsr_##S(T *y, const sparsep_bdbcsr_##S *A, const T *x) {                      \
    const uint64_t rb = A->row_block_size, cb = A->col_block_size;                                   \
    memset(y, 0, sizeof(T) * ((size_t)A->nrows + rb));                                               \
    uint64_t tb = 0;                                                                                 \
    for (uint32_t c = 0; c < A->vert_partitions; c++) {                                              \
      uint64_t po = (uint64_t)c * (A->num_block_rows + 1);                                           \
      for (uint64_t n = 0; n < A->num_block_rows; n++)                                               \
        for (uint64_t i = A->browptr[po + n]; i < A->browptr[po + n + 1]; i++) {                     \
          uint64_t j = A->bcolind[tb + i];                                                           \
          for (uint64_t br = 0; br < rb; br++) {                                                     \
            T acc = 0;                                                                               \
            for (uint64_t bc = 0; bc < cb; bc++)                                                     \
              acc += A->bval[(tb + i) * cb * rb + br * cb + bc] * x[A->vert_tile_widths[c] + j * cb + bc]; \
            y[n * rb + br] += acc;                                                                   \
          }                                                                                          \
        }                                                                                            \
      tb += A->blocks_per_vert_partition[c];                                                         \
    }                                                                                                \
  }                                                                                                  \
  /* spmv/2D/BDBCOO-nnz/host/app.c:91 */                                                             \
  void oracle_spmv_bdbcoo_##S(T *y, const sparsep_bdbcoo_##S *A, const T *x) {                      \
    const uint64_t rb = A->row_block_size, cb = A->col_block_size;                                   \
    memset(y, 0, sizeof(T) * ((size_t)A->nrows + rb));                                               \
    uint64_t tb = 0;                                                                                 \
    for (uint32_t c = 0; c < A->vert_partitions; c++) {                                              \
      for (uint64_t n = 0; n < A->blocks_per_vert_partition[c]; n++) {                               \
        uint64_t i = A->bind[tb + n].rowind, j = A->bind[tb + n].colind;                             \
        for (uint64_t br = 0; br < rb; br++) {                                                       \
          T acc = 0;                                                                                 \
          for (uint64_t bc = 0; bc < cb; bc++)                                                       \
            acc += A->bval[tb * rb * cb + n * cb * rb + br * cb + bc] * x[A->vert_tile_widths[c] + j * cb + bc]; \
          y[i * rb + br] += acc;                                                                     \
        }                                                                                            \
      }                                                                                              \
      tb += A->blocks_per_vert_partition[c];                                                         \
    }                                                                                                \
  }

ORACLE_DEFINE(int8_t, i8)
ORACLE_DEFINE(int16_t, i16)
ORACLE_DEFINE(int32_t, i32)
ORACLE_DEFINE(int64_t, i64)
ORACLE_DEFINE(float, f32)
ORACLE_DEFINE(double, f64)

/*
 * High-precision reference for the FP error bound: from (row, col, value)
 * triplets, y_hi[r] = sum a_rj x_j accumulated in long double with Neumaier
 * compensation, abs[r] = sum |a_rj x_j|, cnt[r] = terms in row r.  Tests then
 * check |y_gpu - y_hi| <= gamma_{cnt} * abs (+ the rounding of y_hi itself).
 */
void oracle_ref_triplets(uint64_t n, const uint32_t *rows, const uint32_t *cols, const double *vals,
                         const double *x, uint32_t nrows, double *y_hi, double *abs_sum, uint32_t *cnt) {
  long double *s = (long double *)calloc(nrows ? nrows : 1, sizeof(long double));
  long double *c = (long double *)calloc(nrows ? nrows : 1, sizeof(long double));
  long double *a = (long double *)calloc(nrows ? nrows : 1, sizeof(long double));
  memset(cnt, 0, sizeof(uint32_t) * nrows);
  for (uint64_t k = 0; k < n; ++k) {
    uint32_t r = rows[k];
    long double p = (long double)vals[k] * (long double)x[cols[k]];
    long double t = s[r] + p;
    if (fabsl(s[r]) >= fabsl(p)) c[r] += (s[r] - t) + p;
    else c[r] += (p - t) + s[r];
    s[r] = t;
    a[r] += fabsl(p);
    cnt[r]++;
  }
  for (uint32_t r = 0; r < nrows; ++r) {
    y_hi[r] = (double)(s[r] + c[r]);
    abs_sum[r] = (double)a[r];
  }
  free(s);
  free(c);
  free(a);
}

/* Threaded CPU baseline over row slices of the reference CSR loop: each
 * thread runs oracle_spmv_csr on a view of rows [r0, r1) (same rowptr
 * values, y offset), which is the reference's loop unchanged. */
#include <pthread.h>
typedef struct {
  const sparsep_csr_f32 *A;
  const float *x;
  float *y;
  uint32_t r0, r1;
} csr_slice_f32;

static void *csr_slice_run(void *arg) {
  csr_slice_f32 *s = (csr_slice_f32 *)arg;
  sparsep_csr_f32 v = *s->A;
  v.nrows = s->r1 - s->r0;
  v.rowptr = s->A->rowptr + s->r0;
  oracle_spmv_csr_f32(s->y + s->r0, &v, s->x);
  return NULL;
}

int oracle_spmv_csr_f32_threads(float *y, const sparsep_csr_f32 *A, const float *x, int threads) {
  if (threads < 1) threads = 1;
  if (threads > 256) threads = 256;
  pthread_t tid[256];
  csr_slice_f32 sl[256];
  uint64_t nnz = A->rowptr[A->nrows];
  uint32_t r = 0;
  for (int t = 0; t < threads; ++t) {
    uint64_t target = nnz * (uint64_t)(t + 1) / threads;
    uint32_t r1 = r;
    while (r1 < A->nrows && A->rowptr[r1] < target) ++r1;
    if (t == threads - 1) r1 = A->nrows;
    sl[t].A = A;
    sl[t].x = x;
    sl[t].y = y;
    sl[t].r0 = r;
    sl[t].r1 = r1;
    r = r1;
  }
  for (int t = 0; t < threads; ++t) pthread_create(&tid[t], NULL, csr_slice_run, &sl[t]);
  for (int t = 0; t < threads; ++t) pthread_join(tid[t], NULL);
  return 0;
}
