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

/* Device CSR -> 4x4 BCSR -> plan -> SpMV without the matrix leaving the GPU;
 * dalloc is the caller's device allocator (the library's own buffers are
 * inside the layout and the plan). */
typedef void *(*dev_alloc_fn)(size_t bytes);
int run_device_bcsr(const uint32_t *d_rowptr, const uint32_t *d_colind, const float *d_vals, uint32_t nrows,
                    uint32_t ncols, uint32_t nnz, dev_alloc_fn dalloc, const float *d_x, float *d_y) {
  sparsep_bcsr_layout *layout = NULL;
  sparsep_plan *plan = NULL;
  uint64_t nb = 0;
  uint32_t *bp = NULL, *bc = NULL, *npb = NULL;
  float *bv = NULL;
  int st = sparsep_bcsr_layout_device(d_rowptr, d_colind, nrows, ncols, nnz, 4, 4, &layout, &nb, NULL);
  if (!st) {
    bp = dalloc(((size_t)(nrows + 3) / 4 + 1) * sizeof(uint32_t));
    bc = dalloc((size_t)nb * sizeof(uint32_t) + 4);
    bv = dalloc((size_t)nb * 16 * sizeof(float) + 4);
    npb = dalloc((size_t)nb * sizeof(uint32_t) + 4);
    if (!bp || !bc || !bv || !npb) st = SPARSEP_ENOMEM;
  }
  if (!st) st = sparsep_csr2bcsr_device_f32(layout, d_vals, bp, bc, bv, npb, NULL);
  sparsep_bcsr_layout_free(layout);
  if (!st) st = sparsep_plan_bcsr_device_f32(nrows, ncols, 4, 4, nb, nnz, bp, bc, bv, npb, NULL, &plan);
  if (!st) st = sparsep_execute_device(plan, d_x, d_y, NULL);
  sparsep_plan_free(plan);
  return st;
}

int main(int argc, char **argv) {
  (void)argc;
  (void)argv;
  printf("%s\n", sparsep_version());
  return 0;
}
