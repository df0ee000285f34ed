// autotune.cu -- the plan variants of a CSR matrix, timed (exhaustive) or
// chosen by the learned selector (sparsep_opts.autotune).
//
// No counterpart in the reference: there every format / scheme / balance /
// sync choice is a separate program fixed at compile time
// (spmv/1D/CSR-row/Makefile:4-8, spmv/1D/COO-nnz/Makefile:7-9,
// spmv/2D/BDCSR/support/params.h:8-75).  Here one CSR input can run as any of
// SPARSEP_NPLANVARIANTS plans; every one computes y = A x over the same rows
// and columns (integers bit-exact, FP within the per-row gamma bound), so the
// choice changes the schedule only.  Candidates are built through the public
// C-ABI one at a time (converted on the host, planned, timed with CUDA events
// on device-resident x and y, freed) so the peak memory is one candidate's.
// Block formats are skipped where their blocks would be mostly explicit zeros
// (fill below FILL_MIN), the heavy-row split where x fits L1 anyway.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include <cuda_runtime.h>

#include "internal.hpp"

namespace sparsep {
namespace {

constexpr double FILL_MIN = 0.25;  // block formats: at most 4x the nonzeros stored

struct Variant {
  const char *name;
  int kind;  // 0 csr, 1 cooe, 2 bcsr, 3 bcoo, 4 dcoo
  uint32_t b;
  void (*opts)(sparsep_opts &);
};

const Variant kVariants[SPARSEP_NPLANVARIANTS] = {
    {"csr/1d/auto", 0, 0, [](sparsep_opts &) {}},
    {"csr/1d/items-2048", 0, 0, [](sparsep_opts &o) { o.item_nnz = 2048; }},
    {"csr/1d/tma-pipeline", 0, 0, [](sparsep_opts &o) { o.pipeline = 1; }},
    {"csr/1d/heavy-row-stripes", 0, 0, [](sparsep_opts &) {}},  // threshold set per matrix
    {"coo/1d/lock-free", 1, 0, [](sparsep_opts &) {}},
    {"coo/1d/atomic", 1, 0, [](sparsep_opts &o) { o.sync = SPARSEP_SYNC_ATOMIC; }},
    {"bcsr/1d/4x4", 2, 4, [](sparsep_opts &) {}},
    {"bcsr/1d/8x8", 2, 8, [](sparsep_opts &) {}},
    {"bcoo/1d/4x4", 3, 4, [](sparsep_opts &) {}},
    {"coo/2d-equal/16x16/atomic", 4, 0, [](sparsep_opts &o) { o.sync = SPARSEP_SYNC_ATOMIC; }},
};

// The typed C-ABI entry points of one element type.
template <typename T> struct Api;
#define SPARSEP_API(T, S)                                                                                   \
  template <> struct Api<T> {                                                                               \
    static int plan_csr(const sparsep_csr_##S *A, const sparsep_opts *o, sparsep_plan **p) {                \
      return sparsep_plan_csr_##S(A, o, p);                                                                 \
    }                                                                                                       \
    static int plan_cooe(const sparsep_cooe_##S *A, const sparsep_opts *o, sparsep_plan **p) {              \
      return sparsep_plan_cooe_##S(A, o, p);                                                                \
    }                                                                                                       \
    static int plan_bcsr(const sparsep_bcsr_##S *A, const sparsep_opts *o, sparsep_plan **p) {              \
      return sparsep_plan_bcsr_##S(A, o, p);                                                                \
    }                                                                                                       \
    static int plan_bcoo(const sparsep_bcoo_##S *A, const sparsep_opts *o, sparsep_plan **p) {              \
      return sparsep_plan_bcoo_##S(A, o, p);                                                                \
    }                                                                                                       \
    static int plan_dcoo(const sparsep_dcoo_##S *A, const sparsep_opts *o, sparsep_plan **p) {              \
      return sparsep_plan_dcoo_##S(A, o, p);                                                                \
    }                                                                                                       \
    static int csr2bcsr(const sparsep_csr_##S *A, uint32_t b, sparsep_bcsr_##S **out) {                     \
      return sparsep_csr2bcsr_##S(A, b, b, out);                                                            \
    }                                                                                                       \
    static int bcsr2bcoo(const sparsep_bcsr_##S *A, sparsep_bcoo_##S **out) { return sparsep_bcsr2bcoo_##S(A, out); } \
    static int cooe2dcoo(const sparsep_cooe_##S *A, sparsep_dcoo_##S **out) {                               \
      return sparsep_cooe2dcoo_##S(A, 16, 16, out);                                                         \
    }                                                                                                       \
    static void free_bcsr(sparsep_bcsr_##S *A) { sparsep_free_bcsr_##S(A); }                                \
    static void free_bcoo(sparsep_bcoo_##S *A) { sparsep_free_bcoo_##S(A); }                                \
    static void free_dcoo(sparsep_dcoo_##S *A) { sparsep_free_dcoo_##S(A); }                                \
  };
SPARSEP_API(int8_t, i8)
SPARSEP_API(int16_t, i16)
SPARSEP_API(int32_t, i32)
SPARSEP_API(int64_t, i64)
SPARSEP_API(float, f32)
SPARSEP_API(double, f64)
#undef SPARSEP_API

// The AoS COO of a CSR matrix, sorted by (row, column) as the reference's
// sortCOOMatrix leaves it (spmv/1D/COO-nnz/support/matrix.h:88-125; the 2D
// converters expect that order), owning its arrays.  The sort within a row is
// stable, so duplicate entries keep their order.
template <typename T> struct CooeOf {
  typename Types<T>::cooe s{};
  std::vector<uint32_t> rows;
  std::vector<typename Types<T>::elem> elems;
  explicit CooeOf(const typename Types<T>::csr *A) {
    rows.resize((size_t)A->nrows + 1);
    elems.resize((size_t)A->nnz + 8);
    for (uint32_t r = 0; r < A->nrows; ++r) {
      rows[r] = A->rowptr[r + 1] - A->rowptr[r];
      for (uint32_t j = A->rowptr[r]; j < A->rowptr[r + 1]; ++j) {
        elems[j].rowind = r;
        elems[j].colind = A->colind[j];
        elems[j].val = A->values[j];
      }
      std::stable_sort(elems.begin() + A->rowptr[r], elems.begin() + A->rowptr[r + 1],
                       [](const auto &a, const auto &b) { return a.colind < b.colind; });
    }
    s.nrows = A->nrows;
    s.ncols = A->ncols;
    s.nnz = A->nnz;
    s.rows = rows.data();
    s.nnzs = elems.data();
  }
};

// Whether variant v applies to a matrix with these features (16 floats).
bool applies(int v, const float *f, uint32_t ncols, size_t esize) {
  const Variant &V = kVariants[v];
  if (V.kind == 2 || V.kind == 3) return f[V.b == 4 ? 12 : 13] >= FILL_MIN;
  if (v == 3) return (uint64_t)ncols * esize >= (1u << 20);  // x past L1: worth its stripes
  return true;
}

// Heavy-row threshold of the split variant: about two nonzeros per stripe row.
uint32_t split_rows(uint32_t ncols, size_t esize) {
  const uint64_t W = std::min<uint64_t>(65536, (128 * 1024) / esize);
  return (uint32_t)std::max<uint64_t>(8, 2 * ((ncols + W - 1) / W));
}

}  // namespace

// Build the plan of variant v for CSR matrix A (opts as given otherwise).
template <typename T>
int build_variant(const typename Types<T>::csr *A, int v, const sparsep_opts &base, sparsep_plan **out) {
  using I = Api<T>;
  sparsep_opts o = base;
  o.autotune = 0;
  kVariants[v].opts(o);
  if (v == 3) o.heavy_rows = (int32_t)split_rows(A->ncols, sizeof(T));
  try {
    switch (kVariants[v].kind) {
      case 0: return I::plan_csr(A, &o, out);
      case 1: {
        CooeOf<T> E(A);
        return I::plan_cooe(&E.s, &o, out);
      }
      case 2:
      case 3: {
        typename Types<T>::bcsr *B = nullptr;
        int st = I::csr2bcsr(A, kVariants[v].b, &B);
        if (!st && kVariants[v].kind == 2) st = I::plan_bcsr(B, &o, out);
        if (!st && kVariants[v].kind == 3) {
          typename Types<T>::bcoo *O = nullptr;
          st = I::bcsr2bcoo(B, &O);
          if (!st) st = I::plan_bcoo(O, &o, out);
          I::free_bcoo(O);
        }
        I::free_bcsr(B);
        return st;
      }
      default: {
        CooeOf<T> E(A);
        typename Types<T>::dcoo *D = nullptr;
        int st = I::cooe2dcoo(&E.s, &D);
        if (!st) st = I::plan_dcoo(D, &o, out);
        I::free_dcoo(D);
        return st;
      }
    }
  } catch (const std::bad_alloc &) {
    return SPARSEP_ENOMEM;
  }
}

// Median device time (us) of `reps` runs of a plan on its own x / y buffers,
// after one warm-up run.
static int time_plan(sparsep_plan *p, int reps, cudaStream_t s, double *us) {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    if (e0) cudaEventDestroy(e0);
    return SPARSEP_EIO;
  }
  int st = sparsep_execute_device(p, sparsep_plan_x(p), sparsep_plan_y(p), s);
  std::vector<double> t;
  for (int r = 0; r < reps && !st; ++r) {
    cudaEventRecord(e0, s);
    st = sparsep_execute_device(p, sparsep_plan_x(p), sparsep_plan_y(p), s);
    cudaEventRecord(e1, s);
    float ms = 0;
    if (!st && cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess)
      t.push_back(ms * 1e3);
    else if (!st)
      st = SPARSEP_EIO;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st) return st;
  std::nth_element(t.begin(), t.begin() + t.size() / 2, t.end());
  *us = t[t.size() / 2];
  return SPARSEP_OK;
}

// Time every applicable variant; times_us[v] = 0 where v does not apply.
template <typename T>
int autotune_times(const typename Types<T>::csr *A, const sparsep_opts &base, int reps, double *times_us,
                   int32_t *best) {
  float f[SPARSEP_NFEATURES];
  if (int st = sparsep_features(A->nrows, A->ncols, A->rowptr, A->colind, 1, f)) return st;
  cudaStream_t s = nullptr;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return SPARSEP_EIO;
  int st = SPARSEP_OK, b = -1;
  for (int v = 0; v < SPARSEP_NPLANVARIANTS && !st; ++v) {
    times_us[v] = 0;
    if (!applies(v, f, A->ncols, sizeof(T))) continue;
    sparsep_plan *p = nullptr;
    st = build_variant<T>(A, v, base, &p);
    if (st == SPARSEP_ENOSYS || st == SPARSEP_ERANGE) {  // not offered for this matrix
      st = SPARSEP_OK;
      continue;
    }
    if (!st) st = time_plan(p, std::max(1, reps), s, &times_us[v]);
    sparsep_plan_free(p);
    if (!st && (b < 0 || times_us[v] < times_us[b])) b = v;
  }
  cudaStreamDestroy(s);
  if (best) *best = b;
  return st;
}

// The plan-variant network (16 features -> 64 -> 64 -> SPARSEP_NVARIANTS
// logits, of which the first SPARSEP_NPLANVARIANTS are used), trained on
// autotune_times databases; plan_model.cpp holds its weights.
const uint16_t *plan_model_weights();
const float *plan_model_mean();
const float *plan_model_std();

// sparsep_opts.autotune: 2 = the fastest variant by timing; 1 = the variant
// the network scores highest among the applicable ones, unless its softmax
// probability is below LEARNED_MIN_CONFIDENCE, then as 2.
constexpr float LEARNED_MIN_CONFIDENCE = 0.5f;

template <typename T>
int plan_autotuned(const typename Types<T>::csr *A, const sparsep_opts &o, sparsep_plan **out) {
  double t[SPARSEP_NPLANVARIANTS];
  int32_t best = -1;
  int how = 2;  // how the variant was chosen: 1 by the network, 2 by timing
  if (o.autotune == 1 && plan_model_weights()) {
    float f[SPARSEP_NFEATURES], logits[SPARSEP_NVARIANTS];
    sparsep_selector *sel = nullptr;
    int st = sparsep_features(A->nrows, A->ncols, A->rowptr, A->colind, 1, f);
    if (!st) st = sparsep_selector_create(plan_model_weights(), plan_model_mean(), plan_model_std(), &sel);
    if (!st) st = sparsep_selector_scores(sel, f, 1, logits);
    sparsep_selector_free(sel);
    if (st) return st;
    float mx = -1e30f, z = 0;
    int arg = -1;
    for (int v = 0; v < SPARSEP_NPLANVARIANTS; ++v)
      if (applies(v, f, A->ncols, sizeof(T)) && logits[v] > mx) {
        mx = logits[v];
        arg = v;
      }
    for (int v = 0; v < SPARSEP_NPLANVARIANTS; ++v)
      if (applies(v, f, A->ncols, sizeof(T))) z += std::exp(logits[v] - mx);
    if (arg >= 0 && 1.0f / z >= LEARNED_MIN_CONFIDENCE) {
      best = arg;
      how = 1;
    }
  }
  if (best < 0) {
    if (int st = autotune_times<T>(A, o, 3, t, &best)) return st;
    if (best < 0) return SPARSEP_ENOSYS;
  }
  int st = build_variant<T>(A, best, o, out);
  if (!st) note_variant(*out, kVariants[best].name, how);
  return st;
}

}  // namespace sparsep

using namespace sparsep;

extern "C" {

const char *sparsep_plan_variant_name(int v) {
  return v >= 0 && v < SPARSEP_NPLANVARIANTS ? kVariants[v].name : nullptr;
}

#define SPARSEP_AUTOTUNE_ENTRY(T, S)                                                                         \
  int sparsep_plan_autotune_csr_##S(const sparsep_csr_##S *A, int reps, double *times_us, int32_t *best) {   \
    if (!A || !times_us || reps < 1) return SPARSEP_EINVAL;                                                  \
    sparsep_opts o;                                                                                          \
    sparsep_opts_default(&o);                                                                                \
    return autotune_times<T>(A, o, reps, times_us, best);                                                    \
  }                                                                                                          \
  int sparsep_plan_variant_csr_##S(const sparsep_csr_##S *A, int v, const sparsep_opts *o, sparsep_plan **out) { \
    if (!A || !out || v < 0 || v >= SPARSEP_NPLANVARIANTS) return SPARSEP_EINVAL;                            \
    sparsep_opts oo;                                                                                         \
    if (o) oo = *o; else sparsep_opts_default(&oo);                                                          \
    int st = build_variant<T>(A, v, oo, out);                                                                \
    if (!st) note_variant(*out, kVariants[v].name, 0);                                                       \
    return st;                                                                                               \
  }
SPARSEP_AUTOTUNE_ENTRY(int8_t, i8)
SPARSEP_AUTOTUNE_ENTRY(int16_t, i16)
SPARSEP_AUTOTUNE_ENTRY(int32_t, i32)
SPARSEP_AUTOTUNE_ENTRY(int64_t, i64)
SPARSEP_AUTOTUNE_ENTRY(float, f32)
SPARSEP_AUTOTUNE_ENTRY(double, f64)
#undef SPARSEP_AUTOTUNE_ENTRY

}  // extern "C"

namespace sparsep {
template int plan_autotuned<int8_t>(const Types<int8_t>::csr *, const sparsep_opts &, sparsep_plan **);
template int plan_autotuned<int16_t>(const Types<int16_t>::csr *, const sparsep_opts &, sparsep_plan **);
template int plan_autotuned<int32_t>(const Types<int32_t>::csr *, const sparsep_opts &, sparsep_plan **);
template int plan_autotuned<int64_t>(const Types<int64_t>::csr *, const sparsep_opts &, sparsep_plan **);
template int plan_autotuned<float>(const Types<float>::csr *, const sparsep_opts &, sparsep_plan **);
template int plan_autotuned<double>(const Types<double>::csr *, const sparsep_opts &, sparsep_plan **);
}  // namespace sparsep
