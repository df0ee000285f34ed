/* A C caller of the entry points with no reference counterpart: the batched
 * multi-RHS launch with learned variants, conjugate gradient on a plan, and
 * the value-keeping Matrix Market reader.  Compiled and linked by
 * tests/test_abi.py (not run: it needs a GPU and device buffers). */
#include <stdio.h>
#include <stdlib.h>

#include "sparsep.h"

int run_batch(uint32_t nmats, const sparsep_csr_f32 *const *mats, const uint32_t *nrhs, const float *const *x,
              float *const *y, const uint16_t *wb, const float *mean, const float *stdev) {
  sparsep_batch *b = NULL;
  sparsep_selector *sel = NULL;
  int st = sparsep_batch_create_f32(nmats, mats, nrhs, NULL, &b);
  for (uint32_t m = 0; !st && m < nmats; ++m) st = sparsep_batch_set_x(b, m, x[m]);
  if (!st) st = sparsep_selector_create(wb, mean, stdev, &sel);
  if (!st) st = sparsep_batch_select(b, sel, 0.3f, 3, NULL, NULL);
  if (!st) st = sparsep_batch_execute(b, NULL);
  for (uint32_t m = 0; !st && m < nmats; ++m) st = sparsep_batch_get_y(b, m, y[m]);
  if (st) fprintf(stderr, "batch: %s %s\n", sparsep_strerror(st), sparsep_last_error());
  sparsep_selector_free(sel);
  sparsep_batch_free(b);
  return st;
}

int run_cg(const char *mtx, const void *d_b, void *d_x) {
  sparsep_coo_f64 *coo = NULL;
  sparsep_csr_f64 *csr = NULL;
  sparsep_plan *plan = NULL;
  sparsep_cg *cg = NULL;
  uint32_t iters = 0;
  double res = 0.0;
  int st = sparsep_read_mtx_values_f64(mtx, &coo);
  if (!st) st = sparsep_coo2csr_f64(coo, &csr);
  if (!st) st = sparsep_plan_csr_f64(csr, NULL, &plan);
  if (!st) st = sparsep_cg_create(plan, &cg);
  if (!st) st = sparsep_cg_solve(cg, d_b, d_x, 1000, 1e-8, 25, &iters, &res, NULL);
  if (!st) printf("cg: %u iterations, relative residual %.3e\n", iters, res);
  else fprintf(stderr, "cg: %s\n", sparsep_strerror(st));
  sparsep_cg_free(cg);
  sparsep_plan_free(plan);
  sparsep_free_csr_f64(csr);
  sparsep_free_coo_f64(coo);
  return st;
}

int main(int argc, char **argv) {
  (void)argc;
  (void)argv;
  printf("%s\n", sparsep_version());
  return 0;
}
