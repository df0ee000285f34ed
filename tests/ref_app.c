/* A reference-style host program (test fixture): the reference's own reader,
 * converter and free names (readCOOMatrix, coo2csr, csr2bcsr, bcsr2bcoo,
 * free*Matrix) and val_dt from sparsep_compat.h with -DSPARSEP_REFERENCE_NAMES
 * and -D<TYPE>, then the SpMV through the C-ABI in CSR (one-shot, 64 parts by
 * nonzeros, and a plan run twice on host buffers), BCSR 4x4, BCOO 4x4 and the
 * plan variant the learned selector picks (autotune = 1).
 * Usage: ref_app <file.mtx> <out-prefix>; writes <prefix>.{rowptr,colind,
 * values,x,y_csr,y_plan,y_bcsr,y_bcoo,y_auto} as raw arrays for the test to check. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "sparsep_compat.h"

static int dump(const char *prefix, const char *name, const void *p, size_t bytes) {
  char path[1024];
  snprintf(path, sizeof path, "%s.%s", prefix, name);
  FILE *f = fopen(path, "wb");
  if (!f) return 1;
  const size_t w = bytes ? fwrite(p, 1, bytes, f) : 0;
  fclose(f);
  return w != bytes;
}

int main(int argc, char **argv) {
  if (argc < 3) return 2;
  struct COOMatrix *B = readCOOMatrix(argv[1]);
  if (!B) return 3;
  struct CSRMatrix *A = coo2csr(B);
  struct BCSRMatrix *Bc = A ? csr2bcsr(A, 4, 4) : NULL;
  struct BCOOMatrix *Bo = Bc ? bcsr2bcoo(Bc) : NULL;
  if (!Bo) return 4;
  val_dt *x = calloc(A->ncols + 16, sizeof(val_dt));
  val_dt *y[5];
  for (int k = 0; k < 5; ++k) y[k] = calloc(A->nrows + 8, sizeof(val_dt));
  for (uint32_t i = 0; i < A->ncols; ++i) x[i] = (val_dt)((int)(i % 7) - 3);
  sparsep_opts o;
  sparsep_opts_default(&o);
  o.nr_parts = 64; /* NR_DPUS */
  o.part_balance = SPARSEP_BAL_NNZ;
  int st = sparsep_spmv_csr(A, x, y[0], &o);
  sparsep_plan *plan = NULL;
  if (!st) st = sparsep_plan_csr(A, NULL, &plan);
  for (int rep = 0; rep < 2 && !st; ++rep) st = sparsep_execute_host(plan, x, y[1]);
  double ms[5];
  if (!st) st = sparsep_timings(plan, ms);
  sparsep_plan_free(plan);
  if (!st) st = sparsep_spmv_bcsr(Bc, x, y[2], NULL);
  if (!st) st = sparsep_spmv_bcoo(Bo, x, y[3], NULL);
  /* the plan variant chosen by the learned selector (autotune = 1) */
  sparsep_opts ao;
  sparsep_opts_default(&ao);
  ao.autotune = 1;
  if (!st) st = sparsep_plan_csr(A, &ao, &plan);
  if (!st) st = sparsep_execute_host(plan, x, y[4]);
  sparsep_plan_info info;
  if (!st) st = sparsep_plan_get_info(plan, &info);
  if (!st) fprintf(stderr, "autotune=1 chose %s\n", info.variant);
  sparsep_plan_free(plan);
  if (st) {
    fprintf(stderr, "ref_app: %s %s\n", sparsep_strerror(st), sparsep_last_error());
    return 5;
  }
  const char *p = argv[2];
  int bad = dump(p, "rowptr", A->rowptr, ((size_t)A->nrows + 1) * 4) | dump(p, "colind", A->colind, (size_t)A->nnz * 4) |
            dump(p, "values", A->values, (size_t)A->nnz * sizeof(val_dt)) |
            dump(p, "x", x, (size_t)A->ncols * sizeof(val_dt)) |
            dump(p, "y_csr", y[0], (size_t)A->nrows * sizeof(val_dt)) |
            dump(p, "y_plan", y[1], (size_t)A->nrows * sizeof(val_dt)) |
            dump(p, "y_bcsr", y[2], (size_t)A->nrows * sizeof(val_dt)) |
            dump(p, "y_bcoo", y[3], (size_t)A->nrows * sizeof(val_dt)) |
            dump(p, "y_auto", y[4], (size_t)A->nrows * sizeof(val_dt));
  printf("%u %u %u\n", A->nrows, A->ncols, A->nnz);
  freeBCOOMatrix(Bo);
  freeBCSRMatrix(Bc);
  freeCSRMatrix(A);
  freeCOOMatrix(B);
  free(x);
  for (int k = 0; k < 5; ++k) free(y[k]);
  return bad ? 6 : 0;
}
