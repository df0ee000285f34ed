/*
 * sparsep.h -- C-ABI of sparsep_b200, a B200 (sm_100a) SpMV library.
 *
 * The library replaces the UPMEM segment of each SparseP host program
 * (spmv/<1D|2D>/<kernel>/host/app.c: dpu_alloc .. dpu_push_xfer .. dpu_launch ..
 * gather .. host merge) with one call over CUDA, while keeping the reference's
 * matrix structs, .mtx reader, converters and partition/balance options.
 *
 * Every struct below is byte-compatible with the reference struct of the same
 * role for the element type named by the suffix:
 *     _i8 int8_t   _i16 int16_t   _i32 int32_t   _i64 int64_t   _f32 float   _f64 double
 * (reference: spmv/1D/CSR-row/support/utils.h:12-34, `val_dt`).  Include
 * "sparsep_compat.h" instead to get the reference's own names (struct CSRMatrix,
 * val_dt, ...) selected by -DINT8 ... -DFP64 exactly as the reference does.
 *
 * Arithmetic contract (reference: spmv/1D/CSR-row/host/app.c:66-77):
 *   y[r] = sum_j A[r][j] * x[j] with the sum taken in the element type.
 *   Integer results wrap at the element width and are bit-exact against the
 *   reference host SpMV for every format, scheme, balance and sync option.
 *   FP32/FP64 results satisfy |dy_r| <= gamma_{n_r} * sum_j |A[r][j] x[j]|.
 *
 * Errors: every entry point returns an int status (0 = OK, negative errno-style
 * code otherwise); nothing aborts.  Ownership: host structs stay owned by the
 * caller; a plan owns its device copies.  A plan is not thread-safe; use one
 * plan per host thread / stream.
 */
#ifndef SPARSEP_H_
#define SPARSEP_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* Status codes                                                              */
/* ------------------------------------------------------------------------ */
#define SPARSEP_OK 0
#define SPARSEP_EIO (-5)         /* CUDA runtime error                        */
#define SPARSEP_ENOMEM (-12)     /* host or device allocation failed          */
#define SPARSEP_ENODEV (-19)     /* no CUDA device / kernel image not loadable*/
#define SPARSEP_EINVAL (-22)     /* invalid argument, struct or option        */
#define SPARSEP_ENOSYS (-38)     /* option combination not provided           */
#define SPARSEP_ERANGE (-34)     /* size beyond a documented limit            */
#define SPARSEP_ETIMEDOUT (-110) /* bounded device wait ran out               */
#define SPARSEP_EBADF (-9)       /* .mtx file missing or malformed            */

const char *sparsep_strerror(int status);

/* Text of the last CUDA runtime error the calling thread's library calls saw
 * ("" if none); SPARSEP_EIO results carry their cause here. */
const char *sparsep_last_error(void);

/* ------------------------------------------------------------------------ */
/* Element types (reference: -DINT8/INT16/INT32/INT64/FP32/FP64)             */
/* ------------------------------------------------------------------------ */
typedef enum {
  SPARSEP_INT8 = 0,
  SPARSEP_INT16 = 1,
  SPARSEP_INT32 = 2,
  SPARSEP_INT64 = 3,
  SPARSEP_FP32 = 4,
  SPARSEP_FP64 = 5
} sparsep_dtype;

/* ------------------------------------------------------------------------ */
/* Options (reference: Makefile -D macros + getopt flags, see                 */
/* spmv/1D/CSR-row/Makefile:4-8, spmv/1D/COO-nnz/Makefile:7-9,                */
/* spmv/1D/BCSR-nnz/support/params.h:8-67, spmv/2D/BDCSR/support/params.h)    */
/* ------------------------------------------------------------------------ */
typedef enum {
  SPARSEP_FMT_CSR = 0,
  SPARSEP_FMT_COO = 1,
  SPARSEP_FMT_BCSR = 2,
  SPARSEP_FMT_BCOO = 3
} sparsep_format;

typedef enum {
  SPARSEP_1D = 0,         /* row partitions, whole x per partition (spmv/1D)     */
  SPARSEP_2D_EQUAL = 1,   /* D:   equal-sized tiles        (spmv/2D/D*)          */
  SPARSEP_2D_EQUAL_W = 2, /* RBD: equal-width stripes x nnz-balanced row ranges */
  SPARSEP_2D_VAR = 3      /* BD:  nnz-balanced stripes x nnz-balanced row ranges */
} sparsep_scheme;

typedef enum {
  SPARSEP_BAL_ROW = 0,       /* equal rows (CSR-row, COO-row, partition_by_row)     */
  SPARSEP_BAL_NNZ = 1,       /* equal nnz at row / block-row granularity            */
  SPARSEP_BAL_BLOCK = 2,     /* equal blocks at block-row granularity (BCSR-block)  */
  SPARSEP_BAL_NNZ_ELEM = 3,  /* equal nnz at element / block granularity; rows may
                                straddle parts (COO-nnz, BCOO-nnz)                  */
  SPARSEP_BAL_INTERLEAVE = 4 /* workers only: rows dealt round-robin to lane groups */
} sparsep_balance;

typedef enum {
  SPARSEP_SYNC_LF = 0,     /* lock-free: partial sums merged without atomics (lf)  */
  SPARSEP_SYNC_ATOMIC = 1, /* fine-grained: red.global per row segment (lb-fg)     */
  SPARSEP_SYNC_CG = 2      /* coarse-grained lock (lb-cg); executed as ATOMIC       */
} sparsep_sync;

typedef struct sparsep_opts {
  int32_t format;          /* sparsep_format (informational for typed entry points) */
  int32_t scheme;          /* sparsep_scheme (informational for typed entry points) */
  int32_t part_balance;    /* sparsep_balance across parts (reference: DPUs)     */
  int32_t worker_balance;  /* sparsep_balance across workers (reference: tasklets)*/
  int32_t sync;            /* sparsep_sync                                       */
  int32_t nr_parts;        /* reference NR_DPUS: parts = CTAs; 0 = auto          */
  int32_t nr_workers;      /* reference NR_TASKLETS: warps per part; 0 = auto    */
  int32_t vert_partitions; /* reference -v (2D schemes built from COO)           */
  int32_t row_block_size;  /* reference -r (BCSR/BCOO built from CSR)            */
  int32_t col_block_size;  /* reference -c                                       */
  int32_t lanes;           /* lanes per row / block row: 1,2,4,8,16,32; 0 = auto */
  int32_t nrhs;            /* right-hand sides (x is ncols x nrhs row-major)     */
  int32_t stage_x;         /* 2D: stage the x-segment in shared memory (1/0/-1=auto) */
  int32_t item_nnz;        /* auto plans: target nonzeros per CTA work item (0 = auto) */
  int32_t pipeline;        /* 1D CSR auto plans: 1 = persistent TMA-pipelined kernel */
  int32_t autotune;        /* 0 = the options as given; 1 = learned choice of the
                              plan variant with exhaustive fallback; 2 = exhaustive */
  int32_t heavy_rows;      /* 1D CSR auto plans: rows with at least this many
                              nonzeros run in column stripes whose x segment is
                              staged in shared memory (0 = planner's choice,
                              -1 = never) */
  int32_t reserved[2];
} sparsep_opts;

/* Defaults: 1D, nnz balance, auto parts/workers/lanes, LF, nrhs = 1. */
void sparsep_opts_default(sparsep_opts *o);

/* ------------------------------------------------------------------------ */
/* Reference structs, byte-compatible per element type                       */
/* ------------------------------------------------------------------------ */
/* spmv/1D/BCOO-nnz/support/utils.h:39-42 */
typedef struct sparsep_bind {
  uint32_t rowind;
  uint32_t colind;
} sparsep_bind;

#define SPARSEP_DEFINE_TYPES(T, S)                                                  \
  /* AoS nonzero, spmv/1D/COO-nnz/support/utils.h:39-43 */                          \
  typedef struct sparsep_elem_##S {                                                 \
    uint32_t rowind;                                                                \
    uint32_t colind;                                                                \
    T val;                                                                          \
  } sparsep_elem_##S;                                                               \
  /* SoA COO, spmv/1D/CSR-row/support/matrix.h:19-26 */                             \
  typedef struct sparsep_coo_##S {                                                  \
    uint32_t nrows, ncols, nnz;                                                     \
    uint32_t *rowindx;                                                              \
    uint32_t *colind;                                                               \
    T *values;                                                                      \
  } sparsep_coo_##S;                                                                \
  /* AoS COO with per-row counts, spmv/1D/COO-nnz/support/matrix.h:19-25 */         \
  typedef struct sparsep_cooe_##S {                                                 \
    uint32_t nrows, ncols, nnz;                                                     \
    uint32_t *rows;                                                                 \
    sparsep_elem_##S *nnzs;                                                         \
  } sparsep_cooe_##S;                                                               \
  /* spmv/1D/CSR-row/support/matrix.h:31-38 */                                      \
  typedef struct sparsep_csr_##S {                                                  \
    uint32_t nrows, ncols, nnz;                                                     \
    uint32_t *rowptr;                                                               \
    uint32_t *colind;                                                               \
    T *values;                                                                      \
  } sparsep_csr_##S;                                                                \
  /* spmv/1D/BCSR-nnz/support/matrix.h:43-57 */                                     \
  typedef struct sparsep_bcsr_##S {                                                 \
    uint64_t row_block_size, col_block_size;                                        \
    uint32_t num_block_rows, num_block_cols;                                        \
    uint64_t num_blocks;                                                            \
    uint32_t num_rows_left, nrows, ncols, nnz;                                      \
    uint32_t *browptr;                                                              \
    uint32_t *bcolind;                                                              \
    T *bval;                                                                        \
    uint32_t *nnz_per_block;                                                        \
  } sparsep_bcsr_##S;                                                               \
  /* spmv/1D/BCOO-nnz/support/matrix.h:62-76 */                                     \
  typedef struct sparsep_bcoo_##S {                                                 \
    uint64_t row_block_size, col_block_size;                                        \
    uint32_t num_block_rows, num_block_cols;                                        \
    uint64_t num_blocks;                                                            \
    uint32_t num_rows_left, nrows, ncols, nnz;                                      \
    sparsep_bind *bind;                                                             \
    T *bval;                                                                        \
    uint32_t *nnz_per_block;                                                        \
  } sparsep_bcoo_##S;                                                               \
  /* spmv/2D/DCSR/support/matrix.h:31-44 */                                         \
  typedef struct sparsep_dcsr_##S {                                                 \
    uint32_t nrows, ncols, nnz, npartitions, horz_partitions, vert_partitions;      \
    uint32_t tile_height, tile_width;                                               \
    uint32_t *nnzs_per_partition;                                                   \
    uint32_t *drowptr;                                                              \
    uint32_t *dcolind;                                                              \
    T *dval;                                                                        \
  } sparsep_dcsr_##S;                                                               \
  /* spmv/2D/RBDCSR/support/matrix.h:31-43 */                                       \
  typedef struct sparsep_rbdcsr_##S {                                               \
    uint32_t nrows, ncols, nnz, npartitions, horz_partitions, vert_partitions;      \
    uint32_t tile_width;                                                            \
    uint32_t *nnzs_per_vert_partition;                                              \
    uint32_t *drowptr;                                                              \
    uint32_t *dcolind;                                                              \
    T *dval;                                                                        \
  } sparsep_rbdcsr_##S;                                                             \
  /* spmv/2D/BDCSR/support/matrix.h:31-45 */                                        \
  typedef struct sparsep_bdcsr_##S {                                                \
    uint32_t nrows, ncols, nnz, npartitions, horz_partitions, vert_partitions;      \
    uint32_t max_tile_width;                                                        \
    uint32_t *vert_tile_widths;                                                     \
    uint32_t *nnzs_per_column;                                                      \
    uint32_t *nnzs_per_vert_partition;                                              \
    uint32_t *drowptr;                                                              \
    uint32_t *dcolind;                                                              \
    T *dval;                                                                        \
  } sparsep_bdcsr_##S;                                                              \
  /* spmv/2D/DCOO/support/matrix.h:30-42 */                                         \
  typedef struct sparsep_dcoo_##S {                                                 \
    uint32_t nrows, ncols, nnz, npartitions, horz_partitions, vert_partitions;      \
    uint32_t tile_height, tile_width;                                               \
    uint32_t *nnzs_per_partition;                                                   \
    sparsep_elem_##S *nnzs;                                                         \
  } sparsep_dcoo_##S;                                                               \
  /* spmv/2D/RBDCOO/support/matrix.h:31 */                                          \
  typedef struct sparsep_rbdcoo_##S {                                               \
    uint32_t nrows, ncols, nnz, npartitions, horz_partitions, vert_partitions;      \
    uint32_t tile_width;                                                            \
    uint32_t *nnzs_per_vert_partition;                                              \
    sparsep_elem_##S *nnzs;                                                         \
  } sparsep_rbdcoo_##S;                                                             \
  /* spmv/2D/BDCOO/support/matrix.h:30 */                                           \
  typedef struct sparsep_bdcoo_##S {                                                \
    uint32_t nrows, ncols, nnz, npartitions, horz_partitions, vert_partitions;      \
    uint32_t max_tile_width;                                                        \
    uint32_t *vert_tile_widths;                                                     \
    uint32_t *nnzs_per_vert_partition;                                              \
    uint32_t *nnzs_per_column;                                                      \
    sparsep_elem_##S *nnzs;                                                         \
  } sparsep_bdcoo_##S;                                                              \
  /* spmv/2D/DBCSR/support/matrix.h:50-71 */                                        \
  typedef struct sparsep_dbcsr_##S {                                                \
    uint32_t nrows, ncols, nnz, npartitions, horz_partitions, vert_partitions;      \
    uint32_t nblocks;                                                               \
    uint64_t tile_height, tile_width;                                               \
    uint32_t *nnzs_per_partition;                                                   \
    uint32_t *blocks_per_partition;                                                 \
    uint64_t row_block_size, col_block_size;                                        \
    uint32_t num_block_rows, num_block_cols, num_rows_left;                         \
    uint32_t *browptr;                                                              \
    uint32_t *bcolind;                                                              \
    T *bval;                                                                        \
    uint32_t *nnz_per_block;                                                        \
  } sparsep_dbcsr_##S;                                                              \
  /* spmv/2D/DBCOO/support/matrix.h:77 */                                           \
  typedef struct sparsep_dbcoo_##S {                                                \
    uint32_t nrows, ncols, nnz, npartitions, horz_partitions, vert_partitions;      \
    uint32_t nblocks;                                                               \
    uint64_t tile_height, tile_width;                                               \
    uint32_t *nnzs_per_partition;                                                   \
    uint32_t *blocks_per_partition;                                                 \
    uint64_t row_block_size, col_block_size;                                        \
    uint32_t num_block_rows, num_block_cols, num_rows_left;                         \
    sparsep_bind *bind;                                                             \
    T *bval;                                                                        \
    uint32_t *nnz_per_block;                                                        \
  } sparsep_dbcoo_##S;                                                              \
  /* spmv/2D/RBDBCSR-nnz/support/matrix.h:50 */                                     \
  typedef struct sparsep_rbdbcsr_##S {                                              \
    uint32_t nrows, ncols, nnz, npartitions, horz_partitions, vert_partitions;      \
    uint32_t nblocks;                                                               \
    uint32_t tile_width;                                                            \
    uint32_t *nnzs_per_vert_partition;                                              \
    uint32_t *blocks_per_vert_partition;                                            \
    uint64_t row_block_size, col_block_size;                                        \
    uint32_t num_block_rows, num_block_cols, num_rows_left;                         \
    uint32_t *browptr;                                                              \
    uint32_t *bcolind;                                                              \
    T *bval;                                                                        \
    uint32_t *nnz_per_block;                                                        \
  } sparsep_rbdbcsr_##S;                                                            \
  /* spmv/2D/RBDBCOO-nnz/support/matrix.h:76 */                                     \
  typedef struct sparsep_rbdbcoo_##S {                                              \
    uint32_t nrows, ncols, nnz, npartitions, horz_partitions, vert_partitions;      \
    uint32_t nblocks;                                                               \
    uint32_t tile_width;                                                            \
    uint32_t *nnzs_per_vert_partition;                                              \
    uint32_t *blocks_per_vert_partition;                                            \
    uint64_t row_block_size, col_block_size;                                        \
    uint32_t num_block_rows, num_block_cols, num_rows_left;                         \
    sparsep_bind *bind;                                                             \
    T *bval;                                                                        \
    uint32_t *nnz_per_block;                                                        \
  } sparsep_rbdbcoo_##S;                                                            \
  /* spmv/2D/BDBCSR-nnz/support/matrix.h:51 */                                      \
  typedef struct sparsep_bdbcsr_##S {                                               \
    uint32_t nrows, ncols, nnz, npartitions, horz_partitions, vert_partitions;      \
    uint32_t nblocks;                                                               \
    uint32_t max_tile_width;                                                        \
    uint32_t *nnzs_per_vert_partition;                                              \
    uint32_t *nnzs_per_column;                                                      \
    uint32_t *blocks_per_vert_partition;                                            \
    uint32_t *vert_tile_widths;                                                     \
    uint32_t *nnz_per_block;                                                        \
    uint64_t row_block_size, col_block_size;                                        \
    uint32_t num_block_rows, num_block_cols, num_rows_left;                         \
    uint32_t *browptr;                                                              \
    uint32_t *bcolind;                                                              \
    T *bval;                                                                        \
  } sparsep_bdbcsr_##S;                                                             \
  /* spmv/2D/BDBCOO-nnz/support/matrix.h:79 */                                      \
  typedef struct sparsep_bdbcoo_##S {                                               \
    uint32_t nrows, ncols, nnz, npartitions, horz_partitions, vert_partitions;      \
    uint32_t nblocks;                                                               \
    uint32_t max_tile_width;                                                        \
    uint32_t *nnzs_per_column;                                                      \
    uint32_t *nnzs_per_vert_partition;                                              \
    uint32_t *blocks_per_vert_partition;                                            \
    uint32_t *vert_tile_widths;                                                     \
    uint32_t *nnz_per_block;                                                        \
    uint64_t row_block_size, col_block_size;                                        \
    uint32_t num_block_rows, num_block_cols, num_rows_left;                         \
    sparsep_bind *bind;                                                             \
    T *bval;                                                                        \
  } sparsep_bdbcoo_##S;

SPARSEP_DEFINE_TYPES(int8_t, i8)
SPARSEP_DEFINE_TYPES(int16_t, i16)
SPARSEP_DEFINE_TYPES(int32_t, i32)
SPARSEP_DEFINE_TYPES(int64_t, i64)
SPARSEP_DEFINE_TYPES(float, f32)
SPARSEP_DEFINE_TYPES(double, f64)

/* ------------------------------------------------------------------------ */
/* Plans: the reference's Load Matrix phase done once, executed many times  */
/* ------------------------------------------------------------------------ */
typedef struct sparsep_plan sparsep_plan;

/* Reference timer slots (spmv/1D/CSR-row/host/app.c:291-300), milliseconds of
 * the most recent call: 0 Load Matrix, 1 Load Input Vector, 2 Kernel,
 * 3 Retrieve Output Vector, 4 Merge Partial Results. */
int sparsep_timings(const sparsep_plan *plan, double ms[5]);

typedef struct sparsep_plan_info {
  int32_t dtype, format, scheme, nrhs;
  uint32_t nrows, ncols;
  uint64_t nnz;           /* stored nonzeros (blocks: stored entries)          */
  uint64_t nblocks;       /* BCSR/BCOO                                          */
  uint64_t items;         /* CTA work items per execution                      */
  uint64_t tiles;         /* tiles (parts) per execution                       */
  uint64_t compulsory_bytes; /* bytes one SpMV must move (values, indices, x, y) */
  uint64_t device_bytes;  /* device memory held by the plan                    */
  uint64_t scratch_bytes; /* of which scratch (partials, carries, counters)   */
  int32_t kernel_launches; /* kernels launched per execution                   */
  int32_t lanes, workers, stage_x;
  char variant[96];       /* human-readable variant name                      */
  int32_t y_bands;        /* host-buffer path: row bands of y copied back while
                             the kernel runs (0: one copy after the kernel)     */
} sparsep_plan_info;

int sparsep_plan_get_info(const sparsep_plan *plan, sparsep_plan_info *info);
void sparsep_plan_free(sparsep_plan *plan);

/* Execute with DEVICE pointers on a CUDA stream (cudaStream_t as void*, NULL =
 * legacy default stream).  x holds ncols*nrhs elements, y receives nrows*nrhs.
 * Stream-ordered; nothing synchronises.  Safe for CUDA graph capture after the
 * first call on that plan. */
int sparsep_execute_device(sparsep_plan *plan, const void *d_x, void *d_y, void *stream);

/* Execute with HOST pointers: H2D x, kernel(s), D2H y, synchronous.  Fills the
 * timer slots 1..4.  1D CSR plans with at least 1 MB of y copy y back in up to
 * 4 row bands (info.y_bands), each as soon as the kernel has finished the
 * items writing it; slot 3 is then the part of the copy left after the
 * kernel.  A pinned y buffer lets the band copies run without host waits. */
int sparsep_execute_host(sparsep_plan *plan, const void *h_x, void *h_y);

/* Device-resident x / y buffers owned by the plan (ncols*nrhs, nrows*nrhs). */
void *sparsep_plan_x(sparsep_plan *plan);
void *sparsep_plan_y(sparsep_plan *plan);

/* ------------------------------------------------------------------------ */
/* Per-dtype entry points                                                    */
/* ------------------------------------------------------------------------ */
/* For each struct kind K in {csr, coo, cooe, bcsr, bcoo, dcsr, rbdcsr, bdcsr,
 * dcoo, rbdcoo, bdcoo, dbcsr, dbcoo, rbdbcsr, rbdbcoo, bdbcsr, bdbcoo}:
 *   sparsep_plan_K_S(const sparsep_K_S *A, const sparsep_opts *o, sparsep_plan **out)
 *   sparsep_spmv_K_S(const sparsep_K_S *A, const T *x, T *y, const sparsep_opts *o)
 * The one-shot form plans, executes on host buffers and frees (the whole
 * reference main() between reading the matrix and printing the timers).
 *
 * Lengths: x has ncols elements (BCSR/BCOO: ncols; 2D: ncols), y has nrows
 * elements; entries of y past nrows are never written.  cooe / 2D COO inputs
 * must be sorted by (row, col) as the reference's sortCOOMatrix leaves them
 * (spmv/1D/COO-nnz/support/matrix.h:88-125); 2D tiles as the reference
 * converters produce them.
 *
 * Readers and converters (host, reference support/matrix.h semantics):
 *   sparsep_read_coo_S(file, &coo)      readCOOMatrix, SoA, pads nrows/ncols to 8/sizeof(T)
 *                                       (spmv/1D/CSR-row/support/matrix.h:44-96)
 *   sparsep_read_coo_nopad_S(file, &coo) same without padding (spmv/1D/BCSR-nnz/support/matrix.h:63-110)
 *   sparsep_read_mtx_values_S(file, &coo) no reference counterpart: the file's
 *     own values (real / integer / pattern = 1), symmetric and skew-symmetric
 *     files expanded, no padding; ENOSYS for complex, hermitian or array files
 *   sparsep_read_cooe_S(file, &cooe)    readCOOMatrix, AoS (spmv/1D/COO-nnz/support/matrix.h:31-83)
 *   sparsep_sort_cooe_S(cooe)           sortCOOMatrix (spmv/1D/COO-nnz/support/matrix.h:88-125)
 *   sparsep_coo2csr_S(coo, &csr)        coo2csr (spmv/1D/CSR-row/support/matrix.h:113-152)
 *   sparsep_csr2bcsr_S(csr, rb, cb, &b) csr2bcsr + sortBCSRMatrix + countNNZperBlockBCSRMatrix
 *                                       (spmv/1D/BCSR-nnz/support/matrix.h:202-485)
 *   sparsep_bcsr2bcoo_S(bcsr, &bcoo)    bcsr2bcoo (spmv/1D/BCOO-nnz/support/matrix.h:549-578)
 *   sparsep_cooe2dcsr_S(cooe, H, V, &d)   coo2dcsr   (spmv/2D/DCSR/support/matrix.h:159-230)
 *   sparsep_cooe2rbdcsr_S(cooe, H, V, &d) coo2rbdcsr (spmv/2D/RBDCSR/support/matrix.h:159-223)
 *   sparsep_cooe2bdcsr_S(cooe, H, V, &d)  coo2bdcsr  (spmv/2D/BDCSR/support/matrix.h:161-282)
 *   sparsep_cooe2dcoo_S / rbdcoo / bdcoo  coo2dcoo etc. (spmv/2D/DCOO/support/matrix.h:158-217)
 *   sparsep_dcsr2dbcsr_S(d, rb, cb, &b)   dcsr2dbcsr + countNNZperBlock (spmv/2D/DBCSR/support/matrix.h:278-557)
 *   sparsep_dcsr2dbcoo_S, sparsep_rbdcsr2rbdbcsr_S, sparsep_rbdcsr2rbdbcoo_S,
 *   sparsep_bdcsr2bdbcsr_S, sparsep_bdcsr2bdbcoo_S   (the other 2D block converters)
 *   sparsep_free_K_S(ptr)               frees a struct returned by the library
 */
#define SPARSEP_DECLARE_KIND(T, S, K)                                                    \
  int sparsep_plan_##K##_##S(const sparsep_##K##_##S *A, const sparsep_opts *o,          \
                             sparsep_plan **out);                                        \
  int sparsep_spmv_##K##_##S(const sparsep_##K##_##S *A, const T *x, T *y,               \
                             const sparsep_opts *o);                                     \
  void sparsep_free_##K##_##S(sparsep_##K##_##S *A);

#define SPARSEP_DECLARE_DTYPE(T, S)                                                      \
  SPARSEP_DECLARE_KIND(T, S, csr)                                                        \
  SPARSEP_DECLARE_KIND(T, S, coo)                                                        \
  SPARSEP_DECLARE_KIND(T, S, cooe)                                                       \
  SPARSEP_DECLARE_KIND(T, S, bcsr)                                                       \
  SPARSEP_DECLARE_KIND(T, S, bcoo)                                                       \
  SPARSEP_DECLARE_KIND(T, S, dcsr)                                                       \
  SPARSEP_DECLARE_KIND(T, S, rbdcsr)                                                     \
  SPARSEP_DECLARE_KIND(T, S, bdcsr)                                                      \
  SPARSEP_DECLARE_KIND(T, S, dcoo)                                                       \
  SPARSEP_DECLARE_KIND(T, S, rbdcoo)                                                     \
  SPARSEP_DECLARE_KIND(T, S, bdcoo)                                                      \
  SPARSEP_DECLARE_KIND(T, S, dbcsr)                                                      \
  SPARSEP_DECLARE_KIND(T, S, dbcoo)                                                      \
  SPARSEP_DECLARE_KIND(T, S, rbdbcsr)                                                    \
  SPARSEP_DECLARE_KIND(T, S, rbdbcoo)                                                    \
  SPARSEP_DECLARE_KIND(T, S, bdbcsr)                                                     \
  SPARSEP_DECLARE_KIND(T, S, bdbcoo)                                                     \
  int sparsep_read_coo_##S(const char *file, sparsep_coo_##S **out);                     \
  int sparsep_read_coo_nopad_##S(const char *file, sparsep_coo_##S **out);               \
  int sparsep_read_mtx_values_##S(const char *file, sparsep_coo_##S **out);             \
  int sparsep_read_cooe_##S(const char *file, sparsep_cooe_##S **out);                   \
  int sparsep_sort_cooe_##S(sparsep_cooe_##S *A);                                        \
  int sparsep_coo2csr_##S(const sparsep_coo_##S *A, sparsep_csr_##S **out);              \
  int sparsep_csr2bcsr_##S(const sparsep_csr_##S *A, uint32_t rb, uint32_t cb,           \
                           sparsep_bcsr_##S **out);                                      \
  int sparsep_bcsr2bcoo_##S(const sparsep_bcsr_##S *A, sparsep_bcoo_##S **out);          \
  int sparsep_cooe2dcsr_##S(const sparsep_cooe_##S *A, uint32_t h, uint32_t v,           \
                            sparsep_dcsr_##S **out);                                     \
  int sparsep_cooe2rbdcsr_##S(const sparsep_cooe_##S *A, uint32_t h, uint32_t v,         \
                              sparsep_rbdcsr_##S **out);                                 \
  int sparsep_cooe2bdcsr_##S(const sparsep_cooe_##S *A, uint32_t h, uint32_t v,          \
                             sparsep_bdcsr_##S **out);                                   \
  int sparsep_cooe2dcoo_##S(const sparsep_cooe_##S *A, uint32_t h, uint32_t v,           \
                            sparsep_dcoo_##S **out);                                     \
  int sparsep_cooe2rbdcoo_##S(const sparsep_cooe_##S *A, uint32_t h, uint32_t v,         \
                              sparsep_rbdcoo_##S **out);                                 \
  int sparsep_cooe2bdcoo_##S(const sparsep_cooe_##S *A, uint32_t h, uint32_t v,          \
                             sparsep_bdcoo_##S **out);                                   \
  int sparsep_dcsr2dbcsr_##S(const sparsep_dcsr_##S *A, uint32_t rb, uint32_t cb,        \
                             sparsep_dbcsr_##S **out);                                   \
  int sparsep_dcsr2dbcoo_##S(const sparsep_dcsr_##S *A, uint32_t rb, uint32_t cb,        \
                             sparsep_dbcoo_##S **out);                                   \
  int sparsep_rbdcsr2rbdbcsr_##S(const sparsep_rbdcsr_##S *A, uint32_t rb, uint32_t cb,  \
                                 sparsep_rbdbcsr_##S **out);                             \
  int sparsep_rbdcsr2rbdbcoo_##S(const sparsep_rbdcsr_##S *A, uint32_t rb, uint32_t cb,  \
                                 sparsep_rbdbcoo_##S **out);                             \
  int sparsep_bdcsr2bdbcsr_##S(const sparsep_bdcsr_##S *A, uint32_t rb, uint32_t cb,     \
                               sparsep_bdbcsr_##S **out);                                \
  int sparsep_bdcsr2bdbcoo_##S(const sparsep_bdcsr_##S *A, uint32_t rb, uint32_t cb,     \
                               sparsep_bdbcoo_##S **out);

SPARSEP_DECLARE_DTYPE(int8_t, i8)
SPARSEP_DECLARE_DTYPE(int16_t, i16)
SPARSEP_DECLARE_DTYPE(int32_t, i32)
SPARSEP_DECLARE_DTYPE(int64_t, i64)
SPARSEP_DECLARE_DTYPE(float, f32)
SPARSEP_DECLARE_DTYPE(double, f64)

/* ------------------------------------------------------------------------ */
/* Partitioners (reference semantics, host).  `split` receives parts+1      */
/* boundaries.  Exposed so callers can reproduce the reference's DPU split; */
/* the plans use the same code for nr_parts > 0.                            */
/* ------------------------------------------------------------------------ */
/* partition_by_row, spmv/1D/CSR-row/support/partition.h:35-60 */
int sparsep_partition_by_row(uint32_t nrows, uint32_t parts, uint32_t *split);
/* partition_by_nnz (row granularity), spmv/1D/CSR-nnz/support/partition.h:35-77 */
int sparsep_partition_by_nnz(const uint32_t *rowptr, uint32_t nrows, uint32_t parts,
                             uint32_t *split);
/* element-granular equal-nnz split, spmv/1D/COO-nnz/host/app.c:118-156:
 * split[i] = first nnz of part i (rows may straddle parts). */
int sparsep_partition_by_elem(uint64_t nnz, uint32_t parts, uint64_t *split);
/* BCSR partition_by_nnz / partition_by_blocks at block-row granularity,
 * spmv/1D/BCSR-nnz/support/partition.h:39-112, spmv/1D/BCSR-block/support/partition.h:39.
 * weights[b] = nnz_per_block[b] (by nnz) or NULL (by blocks). */
int sparsep_partition_block_rows(const uint32_t *browptr, uint32_t num_block_rows,
                                 const uint32_t *weights, uint32_t parts, uint32_t *split);

/* ------------------------------------------------------------------------ */
/* Batched multi-RHS SpMV (no reference counterpart)                         */
/* ------------------------------------------------------------------------ */
/* Many CSR matrices, each with its own k = 1..256 right-hand sides (x is
 * ncols x k and y nrows x k, row-major; on the device their rows are `pitch`
 * elements apart, k rounded up to a multiple of 4 for k >= 3, so that 4-wide
 * loads serve every k), multiplied by ONE kernel launch:
 * its CTAs claim work items (row ranges of any matrix, at most 5120 nonzeros,
 * or one longer row) from a device work queue by atomic ticket, replayed as a
 * CUDA graph (queue reset + kernel).  The row routine of each matrix is a
 * variant: the CTA is cut into groups of `lanes` (1..32, power of two) lanes,
 * each lane reading `vec` (1, 2, 4; pitch % vec == 0) consecutive
 * right-hand sides per load, pitch <= 8 * lanes;
 *   mode 0: the rows of a work item dealt round-robin to the groups;
 *   mode 1: the rows and nonzeros of a work item split evenly over the groups
 *           (merge path), rows cut by a split finished from carries;
 *   mode 2, 3: as 0, 1, with window items (2D tiles): a work item whose
 *           columns span few enough rows of x has that x tile staged in
 *           shared memory with its nonzeros, and gathers from there (vec 4);
 *   mode 4: block items on a 4 x 4 BCSR copy of the matrix (built at create
 *           for matrices whose 4 x 4 blocks are at least a quarter full and
 *           no block row holds more than 512 blocks): block rows dealt to the
 *           groups, a block's 4 x rows loaded once for its 4 rows (vec 4,
 *           pitch <= 4 * lanes); sparsep_batch_variant_applies says where;
 *   item_work: nonzero x right-hand-side products per item (0 = 163840).
 * A row longer than 5120 nonzeros runs as one work item per 5120-nonzero
 * chunk; the last chunk to finish sums the chunks' partial rows in order.
 * FP32 and INT32 (integers wrap exactly, as the single-vector path).  Status
 * ENOSYS: the variant does not apply to that k. */
typedef struct sparsep_batch sparsep_batch;
typedef struct sparsep_batch_variant {
  int32_t mode, lanes, item_work, vec;
} sparsep_batch_variant;

void sparsep_batch_variant_default(uint32_t k, sparsep_batch_variant *v);
int sparsep_batch_create_f32(uint32_t nmats, const sparsep_csr_f32 *const *A, const uint32_t *nrhs,
                             const sparsep_batch_variant *variants, sparsep_batch **out);
int sparsep_batch_create_i32(uint32_t nmats, const sparsep_csr_i32 *const *A, const uint32_t *nrhs,
                             const sparsep_batch_variant *variants, sparsep_batch **out);
void sparsep_batch_free(sparsep_batch *b);
/* x / y of matrix m: device pointers (rows `pitch` elements apart; the pad
 * columns never reach a result), or host copies in and out (dense rows of k) */
int sparsep_batch_x(sparsep_batch *b, uint32_t m, void **d_x, void **d_y);
int sparsep_batch_pitch(const sparsep_batch *b, uint32_t m, uint32_t *pitch);
int sparsep_batch_set_x(sparsep_batch *b, uint32_t m, const void *h_x);
int sparsep_batch_get_y(sparsep_batch *b, uint32_t m, void *h_y);
/* change a matrix's variant; sparsep_batch_commit rebuilds the work queue */
int sparsep_batch_set_variant(sparsep_batch *b, uint32_t m, const sparsep_batch_variant *v);
/* OK if variant v can run matrix m (its k; for mode 4 a BCSR copy), else ENOSYS */
int sparsep_batch_variant_applies(const sparsep_batch *b, uint32_t m, const sparsep_batch_variant *v);
int sparsep_batch_get_variant(const sparsep_batch *b, uint32_t m, sparsep_batch_variant *v);
int sparsep_batch_commit(sparsep_batch *b);
/* the whole batch as one graph launch (NULL stream: synchronous, and the
 * status of sparsep_batch_status is returned) */
int sparsep_batch_execute(sparsep_batch *b, void *stream);
/* SPARSEP_ETIMEDOUT if a work item's staging copy did not land within its
 * bounded wait since the last call (that item's rows were not written), else
 * OK; waits for the batch's work */
int sparsep_batch_status(sparsep_batch *b);
/* 1 (default): the batch launch's CTAs claim work items by atomic ticket, so
 * items start in queue order (long rows first); 0: CTA b runs item b */
int sparsep_batch_set_ticket(sparsep_batch *b, int on);
/* baseline: one plain launch per matrix, in order, each with the default
 * variant for its k and items sized to spread over all SMs */
int sparsep_batch_execute_per_matrix(sparsep_batch *b, void *stream);
/* one matrix alone with its committed items */
int sparsep_batch_execute_one(sparsep_batch *b, uint32_t m, void *stream);
/* the autotuner: every candidate variant of every matrix timed alone (median
 * of reps), the fastest kept and committed.  times_us: nmats x candidates,
 * 0 where a candidate does not apply. */
int sparsep_batch_candidates(sparsep_batch_variant *out, int max);
int sparsep_batch_autotune(sparsep_batch *b, int reps, double *times_us, int32_t *chosen);
/* median time of matrix m alone under variant v (ENOSYS: not applicable) */
int sparsep_batch_time_variant(sparsep_batch *b, uint32_t m, const sparsep_batch_variant *v, int reps,
                               double *us_out);
int sparsep_batch_get_info(const sparsep_batch *b, uint64_t *compulsory_bytes, uint64_t *items, uint64_t *nnz);
/* committed work items by kind: window items (a row range with its x tile
 * staged in shared memory) and chunk items (rows longer than 5120 nonzeros,
 * one item per 5120-nonzero chunk) */
int sparsep_batch_item_kinds(const sparsep_batch *b, uint64_t *window_items, uint64_t *chunk_items);

/* ------------------------------------------------------------------------ */
/* COO -> CSR on the device (no reference counterpart on the device; the     */
/* arrays equal coo2csr's, spmv/1D/CSR-row/support/matrix.h:113-152)         */
/* ------------------------------------------------------------------------ */
/* d_rows / d_cols / d_vals: nnz device entries in any order; d_rowptr:
 * nrows + 1, d_colind / d_vals_out: nnz.  Rows ascending, input order kept
 * inside a row (stable).  EINVAL if a row index is >= nrows.  Allocates its
 * own scratch (16 bytes per nonzero); synchronises the stream. */
#define SPARSEP_DECLARE_C2C(T, S)                                                                               \
  int sparsep_coo2csr_device_##S(const uint32_t *d_rows, const uint32_t *d_cols, const T *d_vals, uint32_t nnz, \
                                 uint32_t nrows, uint32_t *d_rowptr, uint32_t *d_colind, T *d_vals_out,         \
                                 void *stream);
SPARSEP_DECLARE_C2C(int8_t, i8)
SPARSEP_DECLARE_C2C(int16_t, i16)
SPARSEP_DECLARE_C2C(int32_t, i32)
SPARSEP_DECLARE_C2C(int64_t, i64)
SPARSEP_DECLARE_C2C(float, f32)
SPARSEP_DECLARE_C2C(double, f64)
/* A plan from a CSR matrix already on the device (e.g. the output above):
 * the row pointers are read back for the planner, the column indices checked
 * on the device, the arrays copied into the plan (the caller keeps its own). */
#define SPARSEP_DECLARE_PLAN_DEVICE(T, S)                                                         \
  int sparsep_plan_csr_device_##S(uint32_t nrows, uint32_t ncols, uint32_t nnz, const uint32_t *d_rowptr, \
                                  const uint32_t *d_colind, const T *d_values, const sparsep_opts *o,     \
                                  sparsep_plan **out);
SPARSEP_DECLARE_PLAN_DEVICE(int8_t, i8)
SPARSEP_DECLARE_PLAN_DEVICE(int16_t, i16)
SPARSEP_DECLARE_PLAN_DEVICE(int32_t, i32)
SPARSEP_DECLARE_PLAN_DEVICE(int64_t, i64)
SPARSEP_DECLARE_PLAN_DEVICE(float, f32)
SPARSEP_DECLARE_PLAN_DEVICE(double, f64)

/* ------------------------------------------------------------------------ */
/* CSR -> BCSR on the device (the arrays of sparsep_csr2bcsr_<t>:           */
/* spmv/1D/BCSR-nnz/support/matrix.h:202-485, csr2bcsr + sortBCSRMatrix +   */
/* countNNZperBlockBCSRMatrix)                                              */
/* ------------------------------------------------------------------------ */
/* Two steps.  sparsep_bcsr_layout_device sorts the nonzeros of a device CSR
 * (rowptr nrows + 1, colind nnz) into rb x cb blocks and returns the block
 * count; EINVAL for a malformed rowptr or a column >= ncols.  The fill then
 * writes caller-allocated device arrays: browptr[ceil(nrows/rb) + 1],
 * bcolind[nblocks], bval[nblocks * rb * cb] (row-major blocks, blocks of a
 * block row by ascending block column, a later duplicate entry overwrites an
 * earlier one) and nnz_per_block[nblocks] (entries != 0).  One layout serves
 * any number of fills (e.g. several value arrays of one pattern) while the
 * CSR's colind stays unchanged; both steps synchronise the stream. */
typedef struct sparsep_bcsr_layout sparsep_bcsr_layout;
int sparsep_bcsr_layout_device(const uint32_t *d_rowptr, const uint32_t *d_colind, uint32_t nrows, uint32_t ncols,
                               uint32_t nnz, uint32_t rb, uint32_t cb, sparsep_bcsr_layout **out, uint64_t *nblocks,
                               void *stream);
void sparsep_bcsr_layout_free(sparsep_bcsr_layout *layout);
#define SPARSEP_DECLARE_C2B(T, S)                                                                                \
  int sparsep_csr2bcsr_device_##S(const sparsep_bcsr_layout *layout, const T *d_values, uint32_t *d_browptr, \
                                  uint32_t *d_bcolind, T *d_bval, uint32_t *d_nnz_per_block, void *stream);
SPARSEP_DECLARE_C2B(int8_t, i8)
SPARSEP_DECLARE_C2B(int16_t, i16)
SPARSEP_DECLARE_C2B(int32_t, i32)
SPARSEP_DECLARE_C2B(int64_t, i64)
SPARSEP_DECLARE_C2B(float, f32)
SPARSEP_DECLARE_C2B(double, f64)
/* A 1D BCSR plan from device arrays (the output above): browptr (and, for
 * nnz-balanced parts, nnz_per_block, which may otherwise be NULL) read back
 * for the planner, block columns checked on the device, arrays copied. */
#define SPARSEP_DECLARE_PLAN_BCSR_DEVICE(T, S)                                                                   \
  int sparsep_plan_bcsr_device_##S(uint32_t nrows, uint32_t ncols, uint32_t rb, uint32_t cb, uint64_t nblocks, \
                                   uint64_t nnz, const uint32_t *d_browptr, const uint32_t *d_bcolind,         \
                                   const T *d_bval, const uint32_t *d_nnz_per_block, const sparsep_opts *o,    \
                                   sparsep_plan **out);
SPARSEP_DECLARE_PLAN_BCSR_DEVICE(int8_t, i8)
SPARSEP_DECLARE_PLAN_BCSR_DEVICE(int16_t, i16)
SPARSEP_DECLARE_PLAN_BCSR_DEVICE(int32_t, i32)
SPARSEP_DECLARE_PLAN_BCSR_DEVICE(int64_t, i64)
SPARSEP_DECLARE_PLAN_BCSR_DEVICE(float, f32)
SPARSEP_DECLARE_PLAN_BCSR_DEVICE(double, f64)

/* ------------------------------------------------------------------------ */
/* Gather floor (measurement support; no reference counterpart)              */
/* ------------------------------------------------------------------------ */
/* Reads x[d_idx[i]] for i < n (column indices all < length of x) and
 * nothing else, on `ctas` CTAs of 512 threads; d_out receives one float per
 * thread (ctas * 512).  Timing it on a matrix's column indices gives the
 * random-gather bound of that matrix's SpMV. */
int sparsep_probe_gather_f32(const uint32_t *d_idx, uint64_t n, const float *d_x, float *d_out, int ctas,
                             void *stream);

/* ------------------------------------------------------------------------ */
/* Conjugate gradient on a plan (no reference counterpart)                   */
/* ------------------------------------------------------------------------ */
/* The iterative-solver caller of the SpMV: CG for a symmetric positive
 * definite matrix planned in FP32 or FP64 (any format / scheme).  One
 * iteration (the plan's SpMV + four vector kernels, scalars kept on the
 * device) is captured once as a CUDA graph and replayed; the residual is read
 * every check_every iterations.  d_b, d_x: device vectors of n elements;
 * d_x holds the start on entry and the solution on return.  Stops at
 * ||b - A x|| / ||b|| <= rel_tol or after max_iters.  Deterministic.  The
 * plan must outlive the solver; a plan is used by one solve at a time. */
typedef struct sparsep_cg sparsep_cg;
int sparsep_cg_create(sparsep_plan *plan, sparsep_cg **out);
int sparsep_cg_solve(sparsep_cg *cg, const void *d_b, void *d_x, uint32_t max_iters, double rel_tol,
                     uint32_t check_every, uint32_t *iters, double *rel_residual, void *stream);
void sparsep_cg_free(sparsep_cg *cg);

/* Power iteration on a square FP32 / FP64 plan (ENOSYS for integer plans):
 * d_x (n device elements) holds the start vector and receives the unit-norm
 * estimate of the dominant eigenvector.  Each iteration -- SpMV, the Rayleigh
 * quotient lambda = p . Ap and ||Ap|| as fixed-order double sums, p = Ap/||Ap||
 * -- is one CUDA graph replayed on `stream`; lambda is read back every
 * check_every iterations and the run stops when two reads differ by at most
 * rel_tol * |lambda| (or A p = 0, or after max_iters).  Bit-identical from run
 * to run. */
typedef struct sparsep_power sparsep_power;
int sparsep_power_create(sparsep_plan *plan, sparsep_power **out);
int sparsep_power_run(sparsep_power *pw, void *d_x, uint32_t max_iters, double rel_tol, uint32_t check_every,
                      double *lambda, uint32_t *iters, void *stream);
void sparsep_power_free(sparsep_power *pw);

/* ------------------------------------------------------------------------ */
/* Learned variant selector (no reference counterpart)                       */
/* ------------------------------------------------------------------------ */
/* Sixteen cheap sparsity features of a CSR structure with k right-hand sides
 * (log sizes, row-length mean / spread / max, long- and short-row shares,
 * distance from the diagonal, 4x4 and 8x8 block fill, x footprint, column
 * step), an MLP 16-64-64-K over them (BF16 weights, FP32 accumulate; K =
 * SPARSEP_NVARIANTS = the batch variants of sparsep_batch_candidates, in that
 * order), and its hand-written CUDA training and inference kernels.  The
 * selector only chooses a batch variant; results are those of the variant. */
#define SPARSEP_NFEATURES 16
#define SPARSEP_NVARIANTS 36
int sparsep_features(uint32_t nrows, uint32_t ncols, const uint32_t *rowptr, const uint32_t *colind, uint32_t k,
                     float *out);
/* network primitives on device buffers: weights d_wb (BF16 bits, nparams),
 * standardised features d_x (n x 16), times d_t (n x K, 0 = variant does not
 * apply); loss_grad writes the mean loss and its gradient: per matrix,
 * (t_best * wscale)^alpha x (expected regret of a softmax pick + ce_weight x
 * cross-entropy to softmax(-regret / tau)) (d_scratch:
 * sparsep_mlp_scratch_floats(n) floats); adam updates the FP32 master
 * weights and their BF16 copy */
uint32_t sparsep_mlp_nparams(void);
size_t sparsep_mlp_scratch_floats(uint32_t n);
int sparsep_mlp_forward(const uint16_t *d_wb, const float *d_x, uint32_t n, float *d_logits, void *stream);
int sparsep_mlp_loss_grad(const uint16_t *d_wb, const float *d_x, const float *d_t, uint32_t n, float wscale,
                          float alpha, float ce_weight, float tau, float *d_grad, float *d_loss, float *d_scratch,
                          void *stream);
int sparsep_mlp_adam(float *d_w, uint16_t *d_wb, const float *d_grad, float *d_m, float *d_v, uint32_t step,
                     float lr, float beta1, float beta2, float eps, float weight_decay, void *stream);
int sparsep_mlp_to_bf16(const float *d_w, uint16_t *d_wb, void *stream);
/* a trained network (host BF16 weights, feature standardisation) on the GPU */
typedef struct sparsep_selector sparsep_selector;
int sparsep_selector_create(const uint16_t *wb, const float *feat_mean, const float *feat_std,
                            sparsep_selector **out);
void sparsep_selector_free(sparsep_selector *s);
int sparsep_selector_scores(sparsep_selector *s, const float *feats, uint32_t n, float *logits);
/* features of every matrix of a batch (nmats x 16, computed at creation) */
int sparsep_batch_features(const sparsep_batch *b, float *out);
/* learned variants for the whole batch: each matrix gets the applicable
 * variant the network scores highest; where that variant's softmax
 * probability is below min_confidence, the matrix is autotuned exhaustively
 * instead (reps timings per candidate).  Commits.  chosen / fallback (nmats,
 * may be NULL) receive the candidate index and 1 where the fallback ran. */
int sparsep_batch_select(sparsep_batch *b, sparsep_selector *s, float min_confidence, int reps, int32_t *chosen,
                         int32_t *fallback);

/* ------------------------------------------------------------------------ */
/* Allocation-free SpMV                                                      */
/* ------------------------------------------------------------------------ */
/* No counterpart in the reference.  For callers that cannot allocate device
 * memory when they multiply -- code inside a memory pool or arena that owns
 * the device heap, or work issued between someone else's stream operations,
 * where a cudaMalloc would synchronise the device or be refused.
 * y = A x for a row-sorted FP32 COO matrix already on the device (d_elems:
 * nnz reference elem_t entries, 16-byte aligned; d_x: ncols; d_y: nrows),
 * lock-free COO kernel, stream-ordered on `stream`.  It allocates nothing:
 * its scratch is a fixed array in the library's device image, sized for at
 * most 2^28 nonzeros (larger inputs return SPARSEP_ERANGE), that every GPU
 * loading the library holds until exit.  The first call on a device looks
 * the array up (cudaGetSymbolAddress) and should come before any stream
 * capture; after a device reset the next call looks it up again.  All calls
 * share the array: calls that overlap on the GPU race, so serialise them
 * (one stream, or events).  Unchecked preconditions (the call does no pass
 * over the input): entries sorted by row, rowind < nrows and colind < ncols.
 * A row index out of range writes nothing; a column index out of range reads
 * outside d_x (undefined). */
int sparsep_spmv_cooe_f32_noalloc(const sparsep_elem_f32 *d_elems, uint32_t nnz, uint32_t nrows, uint32_t ncols,
                                  const float *d_x, float *d_y, void *stream);

/* ------------------------------------------------------------------------ */
/* Plan variants of a CSR matrix (sparsep_opts.autotune; no reference        */
/* counterpart: there each choice is a separate program)                    */
/* ------------------------------------------------------------------------ */
/* A CSR input can run as any of SPARSEP_NPLANVARIANTS plans -- CSR auto items,
 * CSR 2048-nonzero items, the CSR TMA pipeline, the heavy-row stripes, COO
 * lock-free, COO atomic, BCSR 4x4, BCSR 8x8, BCOO 4x4, 2D equal-tile COO
 * 16x16 atomic -- all computing the same y (integers bit-exact, FP within the
 * per-row gamma bound).  sparsep_plan_csr_<t> with o->autotune = 2 times every
 * applicable one (block formats need a block fill >= 1/4; the stripes an x of
 * at least 1 MB) and keeps the fastest; autotune = 1 lets the learned selector
 * (the MLP of the batch selector, trained on these timings) pick, falling back
 * to timing when its confidence is below one half.  The plan's info.variant
 * names the choice.  autotune applies to 1D CSR inputs with one right-hand
 * side on host arrays (ENOSYS otherwise). */
#define SPARSEP_NPLANVARIANTS 10
const char *sparsep_plan_variant_name(int v);
/* every variant timed (median of reps after a warm-up, device x and y), us;
 * 0 where a variant does not apply; best receives the fastest's index */
/* sparsep_plan_variant_csr_<t>: the plan of variant v (0 .. SPARSEP_NPLANVARIANTS-1)
 * of A, the other options as in o */
#define SPARSEP_DECLARE_AUTOTUNE(T, S) \
  int sparsep_plan_autotune_csr_##S(const sparsep_csr_##S *A, int reps, double *times_us, int32_t *best); \
  int sparsep_plan_variant_csr_##S(const sparsep_csr_##S *A, int v, const sparsep_opts *o, sparsep_plan **out);
SPARSEP_DECLARE_AUTOTUNE(int8_t, i8)
SPARSEP_DECLARE_AUTOTUNE(int16_t, i16)
SPARSEP_DECLARE_AUTOTUNE(int32_t, i32)
SPARSEP_DECLARE_AUTOTUNE(int64_t, i64)
SPARSEP_DECLARE_AUTOTUNE(float, f32)
SPARSEP_DECLARE_AUTOTUNE(double, f64)

/* ------------------------------------------------------------------------ */
/* Test support: failures on purpose, without faulting a GPU                 */
/* ------------------------------------------------------------------------ */
/* No counterpart in the reference (its failures abort, DPU_ASSERT in
 * spmv/1D/CSR-row/host/app.c:91-93).  sparsep_test_fail_alloc(n): the n-th
 * device allocation the library makes from now on fails as a full device
 * would (the call returns SPARSEP_ENOMEM); 0 switches it off.
 * sparsep_test_live_allocations: device allocations the library holds now
 * (a call that failed must leave it unchanged).  sparsep_test_wait_fault(1):
 * kernels with a bounded staging wait (2D tiles staging their x segment, the
 * batched launch) add, after their own copies have landed, one wait that
 * nothing completes; it runs out after 1024 tries and the call reports
 * SPARSEP_ETIMEDOUT (the batch: sparsep_batch_status).  Nothing is left in
 * flight, so the next call with the switch off succeeds. */
int sparsep_test_fail_alloc(int nth);
long long sparsep_test_live_allocations(void);
int sparsep_test_wait_fault(int on);

/* ------------------------------------------------------------------------ */
/* Device information                                                        */
/* ------------------------------------------------------------------------ */
/* Number of SMs of the current device, or a negative status. */
int sparsep_device_sms(void);
/* Library version string. */
const char *sparsep_version(void);

#ifdef __cplusplus
}
#endif

#endif /* SPARSEP_H_ */
