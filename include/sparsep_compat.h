/*
 * sparsep_compat.h -- the reference's own names over the sparsep_b200 C-ABI.
 *
 * A SparseP host program (spmv/<1D|2D>/<kernel>/host/app.c) includes
 * support/utils.h and support/matrix.h and selects its element type with
 * -DINT8 / -DINT16 / -DINT32 / -DINT64 / -DFP32 / -DFP64 (default INT32,
 * spmv/1D/CSR-row/support/utils.h:12-34).  Including this header instead gives
 * the same names -- val_dt, byte_dt, struct CSRMatrix, struct BCSRMatrix, ... --
 * as typedefs of the byte-compatible sparsep structs for that element type,
 * and generic spellings of the entry points (sparsep_spmv_csr(A, x, y, o) ->
 * sparsep_spmv_csr_f32 under -DFP32).
 *
 * The two COO layouts of the reference share the name `struct COOMatrix`
 * (SoA in the CSR / BCSR families, spmv/1D/CSR-row/support/matrix.h:19-26;
 * AoS elem_t in the COO and 2D families, spmv/1D/COO-nnz/support/matrix.h:19-25).
 * Define SPARSEP_COO_ELEM to get the AoS one under that name.
 *
 * The reference's BDCSR struct of the BDBCSR/BDBCOO directories orders its
 * arrays differently from spmv/2D/BDCSR's (an intermediate only; the SpMV
 * runs on BDBCSRMatrix); this header follows spmv/2D/BDCSR.
 */
#ifndef SPARSEP_COMPAT_H_
#define SPARSEP_COMPAT_H_

#include "sparsep.h"

#if defined(INT8)
#define SPARSEP_SFX i8
typedef int8_t val_dt;
#define byte_dt 1
#elif defined(INT16)
#define SPARSEP_SFX i16
typedef int16_t val_dt;
#define byte_dt 2
#elif defined(INT64)
#define SPARSEP_SFX i64
typedef int64_t val_dt;
#define byte_dt 8
#elif defined(FP32)
#define SPARSEP_SFX f32
typedef float val_dt;
#define byte_dt 4
#elif defined(FP64)
#define SPARSEP_SFX f64
typedef double val_dt;
#define byte_dt 8
#else
#define SPARSEP_SFX i32
typedef int32_t val_dt;
#define byte_dt 4
#endif

#define SPARSEP_CAT_(a, b) a##_##b
#define SPARSEP_CAT(a, b) SPARSEP_CAT_(a, b)
#define SPARSEP_T(kind) SPARSEP_CAT(sparsep_##kind, SPARSEP_SFX)

/* struct tags of the reference, as aliases of the sparsep structs */
#define elem_t SPARSEP_T(elem)
#define bind_t sparsep_bind

#define CSRMatrix SPARSEP_T(csr)
#ifdef SPARSEP_COO_ELEM
#define COOMatrix SPARSEP_T(cooe)
#else
#define COOMatrix SPARSEP_T(coo)
#endif
#define BCSRMatrix SPARSEP_T(bcsr)
#define BCOOMatrix SPARSEP_T(bcoo)
#define DCSRMatrix SPARSEP_T(dcsr)
#define RBDCSRMatrix SPARSEP_T(rbdcsr)
#define BDCSRMatrix SPARSEP_T(bdcsr)
#define DCOOMatrix SPARSEP_T(dcoo)
#define RBDCOOMatrix SPARSEP_T(rbdcoo)
#define BDCOOMatrix SPARSEP_T(bdcoo)
#define DBCSRMatrix SPARSEP_T(dbcsr)
#define DBCOOMatrix SPARSEP_T(dbcoo)
#define RBDBCSRMatrix SPARSEP_T(rbdbcsr)
#define RBDBCOOMatrix SPARSEP_T(rbdbcoo)
#define BDBCSRMatrix SPARSEP_T(bdbcsr)
#define BDBCOOMatrix SPARSEP_T(bdbcoo)

/* generic entry points for the selected element type */
#define SPARSEP_FN(name) SPARSEP_CAT(sparsep_##name, SPARSEP_SFX)
#define sparsep_spmv_csr SPARSEP_FN(spmv_csr)
#define sparsep_spmv_coo SPARSEP_FN(spmv_coo)
#define sparsep_spmv_cooe SPARSEP_FN(spmv_cooe)
#define sparsep_spmv_bcsr SPARSEP_FN(spmv_bcsr)
#define sparsep_spmv_bcoo SPARSEP_FN(spmv_bcoo)
#define sparsep_spmv_dcsr SPARSEP_FN(spmv_dcsr)
#define sparsep_spmv_rbdcsr SPARSEP_FN(spmv_rbdcsr)
#define sparsep_spmv_bdcsr SPARSEP_FN(spmv_bdcsr)
#define sparsep_spmv_dcoo SPARSEP_FN(spmv_dcoo)
#define sparsep_spmv_rbdcoo SPARSEP_FN(spmv_rbdcoo)
#define sparsep_spmv_bdcoo SPARSEP_FN(spmv_bdcoo)
#define sparsep_spmv_dbcsr SPARSEP_FN(spmv_dbcsr)
#define sparsep_spmv_dbcoo SPARSEP_FN(spmv_dbcoo)
#define sparsep_spmv_rbdbcsr SPARSEP_FN(spmv_rbdbcsr)
#define sparsep_spmv_rbdbcoo SPARSEP_FN(spmv_rbdbcoo)
#define sparsep_spmv_bdbcsr SPARSEP_FN(spmv_bdbcsr)
#define sparsep_spmv_bdbcoo SPARSEP_FN(spmv_bdbcoo)
#define sparsep_plan_csr SPARSEP_FN(plan_csr)
#define sparsep_plan_cooe SPARSEP_FN(plan_cooe)
#define sparsep_plan_bcsr SPARSEP_FN(plan_bcsr)
#define sparsep_plan_bcoo SPARSEP_FN(plan_bcoo)
/* readers and converters under the reference's names (status-returning) */
#define sparsep_readCOOMatrix SPARSEP_FN(read_coo)
#define sparsep_coo2csr SPARSEP_FN(coo2csr)
#define sparsep_csr2bcsr SPARSEP_FN(csr2bcsr)
#define sparsep_bcsr2bcoo SPARSEP_FN(bcsr2bcoo)

/*
 * With -DSPARSEP_REFERENCE_NAMES, the reference's own reader, converter and
 * free functions with its own signatures, so an unmodified host/app.c keeps
 * its calls: pointer-returning as in spmv/1D/CSR-row/support/matrix.h:44
 * (readCOOMatrix), :113 (coo2csr), :102 / :158 (freeCOOMatrix /
 * freeCSRMatrix), spmv/1D/BCSR-nnz/support/matrix.h:202 (csr2bcsr), :515
 * (freeBCSRMatrix), spmv/1D/BCOO-nnz/support/matrix.h:549 (bcsr2bcoo), :607
 * (freeBCOOMatrix) and spmv/1D/COO-nnz/support/matrix.h:31 / :88
 * (readCOOMatrix, sortCOOMatrix of the AoS layout).  readCOOMatrix pads
 * nrows / ncols as the CSR-family reader does; -DSPARSEP_COO_NOPAD selects
 * the BCSR / BCOO families' reader, which does not.  Where the reference
 * aborts, these return NULL (the status is in sparsep_last_error /
 * the status-returning forms above).
 */
#ifdef SPARSEP_REFERENCE_NAMES
/* typed entry point of the selected element type, pasted directly (the
   generic names above are macros themselves) */
#define SPARSEP_TFN2(name, sfx) sparsep_##name##_##sfx
#define SPARSEP_TFN1(name, sfx) SPARSEP_TFN2(name, sfx)
#define SPARSEP_TFN(name) SPARSEP_TFN1(name, SPARSEP_SFX)
#ifdef SPARSEP_COO_ELEM
static inline struct COOMatrix *readCOOMatrix(const char *fileName) {
  struct COOMatrix *A = NULL;
  return SPARSEP_TFN(read_cooe)(fileName, &A) == SPARSEP_OK ? A : NULL;
}
static inline void sortCOOMatrix(struct COOMatrix *A) { (void)SPARSEP_TFN(sort_cooe)(A); }
static inline void freeCOOMatrix(struct COOMatrix *A) { SPARSEP_TFN(free_cooe)(A); }
#else
static inline struct COOMatrix *readCOOMatrix(const char *fileName) {
  struct COOMatrix *A = NULL;
#ifdef SPARSEP_COO_NOPAD
  return SPARSEP_TFN(read_coo_nopad)(fileName, &A) == SPARSEP_OK ? A : NULL;
#else
  return SPARSEP_TFN(read_coo)(fileName, &A) == SPARSEP_OK ? A : NULL;
#endif
}
static inline void freeCOOMatrix(struct COOMatrix *A) { SPARSEP_TFN(free_coo)(A); }
static inline struct CSRMatrix *coo2csr(struct COOMatrix *B) {
  struct CSRMatrix *A = NULL;
  return SPARSEP_TFN(coo2csr)(B, &A) == SPARSEP_OK ? A : NULL;
}
#endif
static inline void freeCSRMatrix(struct CSRMatrix *A) { SPARSEP_TFN(free_csr)(A); }
static inline struct BCSRMatrix *csr2bcsr(struct CSRMatrix *A, uint32_t row_block_size, uint32_t col_block_size) {
  struct BCSRMatrix *B = NULL;
  return SPARSEP_TFN(csr2bcsr)(A, row_block_size, col_block_size, &B) == SPARSEP_OK ? B : NULL;
}
static inline void freeBCSRMatrix(struct BCSRMatrix *B) { SPARSEP_TFN(free_bcsr)(B); }
static inline struct BCOOMatrix *bcsr2bcoo(struct BCSRMatrix *B) {
  struct BCOOMatrix *O = NULL;
  return SPARSEP_TFN(bcsr2bcoo)(B, &O) == SPARSEP_OK ? O : NULL;
}
static inline void freeBCOOMatrix(struct BCOOMatrix *O) { SPARSEP_TFN(free_bcoo)(O); }
#endif /* SPARSEP_REFERENCE_NAMES */

#endif /* SPARSEP_COMPAT_H_ */
