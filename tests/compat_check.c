/* a reference-style host program over the compat header (test fixture) */
#include "sparsep_compat.h"
#include <stdlib.h>
static void spmv_like_reference(struct CSRMatrix *A, val_dt *x, val_dt *y) {
  sparsep_opts o;
  sparsep_opts_default(&o);
  o.nr_parts = 2048; /* NR_DPUS */
  o.part_balance = SPARSEP_BAL_NNZ;
  (void)sparsep_spmv_csr(A, x, y, &o);
}
int main(void) {
  struct COOMatrix *B = NULL;
  struct CSRMatrix *A = NULL;
  struct elem_t e; struct bind_t b; (void)e; (void)b;
  if (sparsep_readCOOMatrix("m.mtx", &B) == 0 && sparsep_coo2csr(B, &A) == 0) {
    val_dt *x = calloc(A->ncols, sizeof(val_dt)), *y = calloc(A->nrows, sizeof(val_dt));
    spmv_like_reference(A, x, y);
  }
  return (int)sizeof(val_dt) + byte_dt;
}
