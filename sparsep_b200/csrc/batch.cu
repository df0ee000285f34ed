// batch.cu -- many CSR matrices with 1..32 right-hand sides in one persistent
// launch, fed by a device work queue and replayed as a CUDA graph.
//
// Each matrix m has its own device copy (rowptr, colind, values), its x
// (ncols x k, row-major) and y (nrows x k).  Work items are row ranges of one
// matrix sized for one warp; persistent warps pull items from a global counter
// (atomicAdd, no waiting) until the queue is empty, so matrices of very
// different sizes share the GPU without per-matrix launch gaps or tails.
//
// Two row routines, chosen per matrix (the autotuner picks `lanes`):
//   RHS mode (k >= 4): a group of G lanes per row, lane j holds right-hand
//     sides j, j+G, ...; each nonzero's x row x[c*k .. c*k+k) is one coalesced
//     load across the group.
//   NNZ mode: a group of G lanes per row splits the row's nonzeros, each lane
//     keeps k (<= 4) partial sums, then a shuffle reduction over the group.
// Same arithmetic as the single-vector path: integers accumulate in 32/64-bit
// unsigned and wrap exactly; FP in the element type.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <vector>

#include "device.cuh"
#include "internal.hpp"

namespace sparsep {
namespace batch {

template <typename T> struct Mat {
  const uint32_t *rowptr;
  const uint32_t *colind;
  const T *val;
  const T *x;
  T *y;
  uint32_t nrows, ncols, k, pad;
};

struct BItem {
  uint32_t mat;
  uint32_t r0, r1;
  uint16_t lanes;  // G
  uint16_t mode;   // 0 = lanes over right-hand sides, 1 = lanes over nonzeros
};

constexpr int KMAX_NNZ_MODE = 4;  // right-hand sides per lane in NNZ mode
constexpr int ACC_RHS = 8;        // accumulators per lane in RHS mode (k <= 8 * G)

template <typename T, int G>
__device__ __forceinline__ void rows_rhs(const Mat<T> &m, uint32_t r0, uint32_t r1, int lane) {
  using A = Acc<T>;
  constexpr int NG = 32 / G;
  const int g = lane / G, gl = lane % G;
  // shuffles stay inside the group: its lanes share a row, hence a trip count
  const unsigned gmask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << (g * G));
  for (uint32_t base = r0; base < r1; base += NG) {
    const uint32_t r = base + g;
    if (r >= r1) continue;
    A acc[ACC_RHS];
#pragma unroll
    for (int a = 0; a < ACC_RHS; ++a) acc[a] = A(0);
    const uint32_t s = __ldg(m.rowptr + r), e = __ldg(m.rowptr + r + 1);
    for (uint32_t p0 = s; p0 < e; p0 += G) {
      // the group loads G nonzeros at once, then every lane walks them with
      // all of their x loads independent of each other
      uint32_t cl = 0;
      T vl = T(0);
      if (p0 + gl < e) {
        cl = __ldcs(m.colind + p0 + gl);
        vl = __ldcs(m.val + p0 + gl);
      }
      const uint32_t cnt = e - p0 < (uint32_t)G ? e - p0 : (uint32_t)G;
#pragma unroll
      for (int q = 0; q < G; ++q) {
        if ((uint32_t)q < cnt) {
          const uint32_t c = __shfl_sync(gmask, cl, q, G);
          const T v = __shfl_sync(gmask, vl, q, G);
          const T *xr = m.x + (size_t)c * m.k;
#pragma unroll
          for (int a = 0; a < ACC_RHS; ++a) {
            const uint32_t j = gl + a * G;
            if (j < m.k) acc[a] += mul<T>(v, __ldg(xr + j));
          }
        }
      }
    }
    T *yr = m.y + (size_t)r * m.k;
#pragma unroll
    for (int a = 0; a < ACC_RHS; ++a) {
      const uint32_t j = gl + a * G;
      if (j < m.k) yr[j] = from_acc<T>(acc[a]);
    }
  }
}

template <typename T, int G>
__device__ __forceinline__ void rows_nnz(const Mat<T> &m, uint32_t r0, uint32_t r1, int lane) {
  using A = Acc<T>;
  constexpr int NG = 32 / G;
  const int g = lane / G, gl = lane % G;
  for (uint32_t base = r0; base < r1; base += NG) {
    const uint32_t r = base + g;
    const bool ok = r < r1;
    A acc[KMAX_NNZ_MODE];
#pragma unroll
    for (int a = 0; a < KMAX_NNZ_MODE; ++a) acc[a] = A(0);
    if (ok) {
      const uint32_t s = __ldg(m.rowptr + r), e = __ldg(m.rowptr + r + 1);
#pragma unroll 4
      for (uint32_t p = s + gl; p < e; p += G) {
        const uint32_t c = __ldcs(m.colind + p);
        const T v = __ldcs(m.val + p);
        const T *xr = m.x + (size_t)c * m.k;
#pragma unroll
        for (int a = 0; a < KMAX_NNZ_MODE; ++a)
          if (a < (int)m.k) acc[a] += mul<T>(v, __ldg(xr + a));
      }
    }
#pragma unroll
    for (int a = 0; a < KMAX_NNZ_MODE; ++a)
#pragma unroll
      for (int o = G / 2; o > 0; o >>= 1) acc[a] += __shfl_xor_sync(0xffffffffu, acc[a], o);
    if (ok && gl == 0) {
      T *yr = m.y + (size_t)r * m.k;
#pragma unroll
      for (int a = 0; a < KMAX_NNZ_MODE; ++a)
        if (a < (int)m.k) yr[a] = from_acc<T>(acc[a]);
    }
  }
}

template <typename T>
__device__ void run_item(const Mat<T> &m, const BItem &it, int lane) {
  if (it.mode == 0) {
    switch (it.lanes) {
      case 4: rows_rhs<T, 4>(m, it.r0, it.r1, lane); break;
      case 8: rows_rhs<T, 8>(m, it.r0, it.r1, lane); break;
      case 16: rows_rhs<T, 16>(m, it.r0, it.r1, lane); break;
      default: rows_rhs<T, 32>(m, it.r0, it.r1, lane); break;
    }
  } else {
    switch (it.lanes) {
      case 1: rows_nnz<T, 1>(m, it.r0, it.r1, lane); break;
      case 2: rows_nnz<T, 2>(m, it.r0, it.r1, lane); break;
      case 4: rows_nnz<T, 4>(m, it.r0, it.r1, lane); break;
      case 8: rows_nnz<T, 8>(m, it.r0, it.r1, lane); break;
      case 16: rows_nnz<T, 16>(m, it.r0, it.r1, lane); break;
      default: rows_nnz<T, 32>(m, it.r0, it.r1, lane); break;
    }
  }
}

// Persistent: every warp takes items from the queue until it is empty.
template <typename T>
__global__ void __launch_bounds__(256) persistent(const Mat<T> *mats, const BItem *items, uint32_t nitems,
                                                  unsigned int *head) {
  const int lane = threadIdx.x & 31;
  for (;;) {
    unsigned int i = 0;
    if (lane == 0) i = atomicAdd(head, 1u);
    i = __shfl_sync(0xffffffffu, i, 0);
    if (i >= nitems) break;
    const BItem it = items[i];
    const Mat<T> m = mats[it.mat];
    run_item<T>(m, it, lane);
  }
}

// One matrix, one warp per item, no queue (the per-matrix launches and the
// autotuner's timing runs).
template <typename T>
__global__ void __launch_bounds__(256) per_matrix(const Mat<T> *mats, const BItem *items, uint32_t i0, uint32_t n) {
  const uint32_t w = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  if (w >= n) return;
  const BItem it = items[i0 + w];
  const Mat<T> m = mats[it.mat];
  run_item<T>(m, it, threadIdx.x & 31);
}

}  // namespace batch
}  // namespace sparsep

using namespace sparsep;
using namespace sparsep::batch;

struct sparsep_batch {
  int dtype = 0;
  size_t esize = 4;
  uint32_t nmats = 0;
  int sms = 148;
  std::vector<void *> allocs;
  std::vector<Mat<float>> mats_h;  // pointers are type-agnostic; values reinterpreted per dtype
  std::vector<uint64_t> nnz;
  std::vector<sparsep_batch_variant> var;
  std::vector<BItem> items_h;
  std::vector<uint32_t> item0, nitem;  // per matrix: first item and count
  void *mats_d = nullptr;
  BItem *items_d = nullptr;
  unsigned int *head = nullptr;
  cudaStream_t stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint64_t bytes = 0;  // compulsory bytes of one batch execution
  int grid = 0;
};

static thread_local char g_batch_err[256] = "";
static int bmap(cudaError_t e) {
  if (e == cudaSuccess) return SPARSEP_OK;
  std::snprintf(g_batch_err, sizeof g_batch_err, "%s (%d)", cudaGetErrorString(e), (int)e);
  if (e == cudaErrorMemoryAllocation) return SPARSEP_ENOMEM;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver || e == cudaErrorNoKernelImageForDevice)
    return SPARSEP_ENODEV;
  return SPARSEP_EIO;
}
#define BCK(x)                                  \
  do {                                          \
    cudaError_t e_ = (x);                       \
    if (e_ != cudaSuccess) return bmap(e_);     \
  } while (0)

static int balloc(sparsep_batch *b, size_t bytes, void **out) {
  void *d = nullptr;
  BCK(cudaMalloc(&d, bytes ? bytes : 16));
  b->allocs.push_back(d);
  *out = d;
  return SPARSEP_OK;
}

// Items of one matrix for a variant: warp-sized row ranges holding about
// `target` nonzero x right-hand-side products.
static void make_items(sparsep_batch *b, uint32_t m, const uint32_t *rowptr) {
  const auto &M = b->mats_h[m];
  const sparsep_batch_variant &v = b->var[m];
  b->item0[m] = (uint32_t)b->items_h.size();
  const uint64_t target = v.item_work > 0 ? (uint64_t)v.item_work : 16384;
  const uint32_t rows_min = v.mode == 0 ? 32 / v.lanes : 32 / v.lanes;
  uint32_t r = 0;
  while (r < M.nrows) {
    uint32_t r1 = r;
    uint64_t work = 0;
    do {
      const uint32_t end = std::min(M.nrows, r1 + rows_min);
      work += ((uint64_t)rowptr[end] - rowptr[r1] + (end - r1)) * M.k;
      r1 = end;
    } while (r1 < M.nrows && work < target);
    BItem it;
    it.mat = m;
    it.r0 = r;
    it.r1 = r1;
    it.lanes = (uint16_t)v.lanes;
    it.mode = (uint16_t)v.mode;
    b->items_h.push_back(it);
    r = r1;
  }
  b->nitem[m] = (uint32_t)b->items_h.size() - b->item0[m];
}

static int check_variant(const sparsep_batch_variant &v, uint32_t k) {
  if (v.mode == 0) {
    if (v.lanes != 4 && v.lanes != 8 && v.lanes != 16 && v.lanes != 32) return SPARSEP_EINVAL;
    if (k > (uint32_t)ACC_RHS * v.lanes) return SPARSEP_ENOSYS;
  } else if (v.mode == 1) {
    if (v.lanes < 1 || v.lanes > 32 || (v.lanes & (v.lanes - 1))) return SPARSEP_EINVAL;
    if (k > (uint32_t)KMAX_NNZ_MODE) return SPARSEP_ENOSYS;
  } else {
    return SPARSEP_EINVAL;
  }
  return SPARSEP_OK;
}

extern "C" void sparsep_batch_variant_default(uint32_t k, sparsep_batch_variant *v) {
  if (!v) return;
  std::memset(v, 0, sizeof *v);
  if (k >= 4) {
    v->mode = 0;
    v->lanes = k >= 32 ? 32 : (k >= 16 ? 16 : (k >= 8 ? 8 : 4));
  } else {
    v->mode = 1;
    v->lanes = 8;
  }
  v->item_work = 16384;
}

template <typename T>
static int batch_create(uint32_t nmats, const typename Types<T>::csr *const *A, const uint32_t *nrhs,
                        const sparsep_batch_variant *var, sparsep_batch **out) {
  if (!out || !A || !nrhs || nmats == 0) return SPARSEP_EINVAL;
  *out = nullptr;
  auto *b = new (std::nothrow) sparsep_batch();
  if (!b) return SPARSEP_ENOMEM;
  std::unique_ptr<sparsep_batch, void (*)(sparsep_batch *)> guard(b, sparsep_batch_free);
  b->dtype = Types<T>::dtype;
  b->esize = sizeof(T);
  b->nmats = nmats;
  int dev = 0;
  BCK(cudaGetDevice(&dev));
  BCK(cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev));
  b->mats_h.resize(nmats);
  b->nnz.resize(nmats);
  b->var.resize(nmats);
  b->item0.resize(nmats);
  b->nitem.resize(nmats);
  std::vector<std::vector<uint32_t>> rowptrs(nmats);
  for (uint32_t m = 0; m < nmats; ++m) {
    const auto *M = A[m];
    if (!M || !M->rowptr || (M->nnz && (!M->colind || !M->values))) return SPARSEP_EINVAL;
    const uint32_t k = nrhs[m];
    if (k == 0 || k > 256) return SPARSEP_EINVAL;
    if (M->rowptr[M->nrows] != M->nnz) return SPARSEP_EINVAL;
    for (uint32_t q = 0; q < M->nnz; ++q)
      if (M->colind[q] >= M->ncols) return SPARSEP_EINVAL;
    if (var) b->var[m] = var[m];
    else sparsep_batch_variant_default(k, &b->var[m]);
    if (int st = check_variant(b->var[m], k)) return st;
    void *d[5];
    int st = balloc(b, ((size_t)M->nrows + 1) * 4, &d[0]);
    if (!st) st = balloc(b, ((size_t)M->nnz + 16) * 4, &d[1]);
    if (!st) st = balloc(b, ((size_t)M->nnz + 16) * sizeof(T), &d[2]);
    if (!st) st = balloc(b, ((size_t)M->ncols * k + 16) * sizeof(T), &d[3]);
    if (!st) st = balloc(b, ((size_t)M->nrows * k + 16) * sizeof(T), &d[4]);
    if (st) return st;
    BCK(cudaMemcpy(d[0], M->rowptr, ((size_t)M->nrows + 1) * 4, cudaMemcpyHostToDevice));
    if (M->nnz) {
      BCK(cudaMemcpy(d[1], M->colind, (size_t)M->nnz * 4, cudaMemcpyHostToDevice));
      BCK(cudaMemcpy(d[2], M->values, (size_t)M->nnz * sizeof(T), cudaMemcpyHostToDevice));
    }
    BCK(cudaMemset(d[3], 0, ((size_t)M->ncols * k + 16) * sizeof(T)));
    auto &h = b->mats_h[m];
    h.rowptr = (const uint32_t *)d[0];
    h.colind = (const uint32_t *)d[1];
    h.val = (const float *)d[2];
    h.x = (const float *)d[3];
    h.y = (float *)d[4];
    h.nrows = M->nrows;
    h.ncols = M->ncols;
    h.k = k;
    h.pad = 0;
    b->nnz[m] = M->nnz;
    rowptrs[m].assign(M->rowptr, M->rowptr + M->nrows + 1);
    b->bytes += (uint64_t)M->nnz * (4 + sizeof(T)) + ((uint64_t)M->nrows + 1) * 4 +
                ((uint64_t)M->ncols + M->nrows) * k * sizeof(T);
  }
  for (uint32_t m = 0; m < nmats; ++m) make_items(b, m, rowptrs[m].data());
  int st = balloc(b, sizeof(Mat<T>) * nmats, &b->mats_d);
  if (!st) st = balloc(b, sizeof(BItem) * b->items_h.size(), (void **)&b->items_d);
  if (!st) st = balloc(b, 64, (void **)&b->head);
  if (st) return st;
  BCK(cudaMemcpy(b->mats_d, b->mats_h.data(), sizeof(Mat<T>) * nmats, cudaMemcpyHostToDevice));
  BCK(cudaMemcpy(b->items_d, b->items_h.data(), sizeof(BItem) * b->items_h.size(), cudaMemcpyHostToDevice));
  BCK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
  int per_sm = 0;
  BCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, persistent<T>, 256, 0));
  b->grid = b->sms * std::max(per_sm, 1);
  *out = guard.release();
  return SPARSEP_OK;
}

template <typename T>
static int launch_persistent(sparsep_batch *b, cudaStream_t s) {
  BCK(cudaMemsetAsync(b->head, 0, 4, s));
  persistent<T><<<b->grid, 256, 0, s>>>((const Mat<T> *)b->mats_d, b->items_d, (uint32_t)b->items_h.size(),
                                         b->head);
  return bmap(cudaGetLastError());
}

template <typename T>
static int launch_one(sparsep_batch *b, uint32_t m, cudaStream_t s) {
  const uint32_t n = b->nitem[m];
  if (!n) return SPARSEP_OK;
  per_matrix<T><<<(n + 7) / 8, 256, 0, s>>>((const Mat<T> *)b->mats_d, b->items_d, b->item0[m], n);
  return bmap(cudaGetLastError());
}

static int dispatch_persistent(sparsep_batch *b, cudaStream_t s) {
  return b->dtype == SPARSEP_FP32 ? launch_persistent<float>(b, s) : launch_persistent<int32_t>(b, s);
}
static int dispatch_one(sparsep_batch *b, uint32_t m, cudaStream_t s) {
  return b->dtype == SPARSEP_FP32 ? launch_one<float>(b, m, s) : launch_one<int32_t>(b, m, s);
}

static void drop_graph(sparsep_batch *b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
}

extern "C" {

int sparsep_batch_create_f32(uint32_t nmats, const sparsep_csr_f32 *const *A, const uint32_t *nrhs,
                             const sparsep_batch_variant *var, sparsep_batch **out) {
  try {
    return batch_create<float>(nmats, A, nrhs, var, out);
  } catch (const std::bad_alloc &) {
    return SPARSEP_ENOMEM;
  }
}

int sparsep_batch_create_i32(uint32_t nmats, const sparsep_csr_i32 *const *A, const uint32_t *nrhs,
                             const sparsep_batch_variant *var, sparsep_batch **out) {
  try {
    return batch_create<int32_t>(nmats, A, nrhs, var, out);
  } catch (const std::bad_alloc &) {
    return SPARSEP_ENOMEM;
  }
}

void sparsep_batch_free(sparsep_batch *b) {
  if (!b) return;
  if (b->stream) cudaStreamSynchronize(b->stream);
  drop_graph(b);
  for (void *d : b->allocs) cudaFree(d);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

int sparsep_batch_set_variant(sparsep_batch *b, uint32_t m, const sparsep_batch_variant *v) {
  if (!b || !v || m >= b->nmats) return SPARSEP_EINVAL;
  if (int st = check_variant(*v, b->mats_h[m].k)) return st;
  b->var[m] = *v;
  return SPARSEP_OK;
}

// Rebuild the item queue after variants changed (needs each matrix's rowptr,
// read back from the device).
int sparsep_batch_commit(sparsep_batch *b) {
  if (!b) return SPARSEP_EINVAL;
  drop_graph(b);
  b->items_h.clear();
  for (uint32_t m = 0; m < b->nmats; ++m) {
    std::vector<uint32_t> rp((size_t)b->mats_h[m].nrows + 1);
    BCK(cudaMemcpy(rp.data(), b->mats_h[m].rowptr, rp.size() * 4, cudaMemcpyDeviceToHost));
    make_items(b, m, rp.data());
  }
  // replace the device item array
  for (auto i = b->allocs.begin(); i != b->allocs.end(); ++i)
    if (*i == (void *)b->items_d) {
      cudaFree(*i);
      b->allocs.erase(i);
      break;
    }
  void *d = nullptr;
  int st = balloc(b, sizeof(BItem) * b->items_h.size(), &d);
  if (st) return st;
  b->items_d = (BItem *)d;
  BCK(cudaMemcpy(b->items_d, b->items_h.data(), sizeof(BItem) * b->items_h.size(), cudaMemcpyHostToDevice));
  return SPARSEP_OK;
}

int sparsep_batch_x(sparsep_batch *b, uint32_t m, void **d_x, void **d_y) {
  if (!b || m >= b->nmats) return SPARSEP_EINVAL;
  if (d_x) *d_x = (void *)b->mats_h[m].x;
  if (d_y) *d_y = (void *)b->mats_h[m].y;
  return SPARSEP_OK;
}

int sparsep_batch_set_x(sparsep_batch *b, uint32_t m, const void *h_x) {
  if (!b || !h_x || m >= b->nmats) return SPARSEP_EINVAL;
  const auto &M = b->mats_h[m];
  BCK(cudaMemcpy((void *)M.x, h_x, (size_t)M.ncols * M.k * b->esize, cudaMemcpyHostToDevice));
  return SPARSEP_OK;
}

int sparsep_batch_get_y(sparsep_batch *b, uint32_t m, void *h_y) {
  if (!b || !h_y || m >= b->nmats) return SPARSEP_EINVAL;
  const auto &M = b->mats_h[m];
  BCK(cudaMemcpy(h_y, M.y, (size_t)M.nrows * M.k * b->esize, cudaMemcpyDeviceToHost));
  return SPARSEP_OK;
}

// The whole batch: one graph launch (queue reset + persistent kernel); the
// graph is captured on the first call after a (re)commit.
int sparsep_batch_execute(sparsep_batch *b, void *stream) {
  if (!b) return SPARSEP_EINVAL;
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : b->stream;
  if (!b->exec) {
    BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    int st = dispatch_persistent(b, b->stream);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (st) {
      if (g) cudaGraphDestroy(g);
      return st;
    }
    BCK(e);
    b->graph = g;
    BCK(cudaGraphInstantiate(&b->exec, b->graph, 0));
  }
  BCK(cudaGraphLaunch(b->exec, s));
  if (!stream) BCK(cudaStreamSynchronize(s));
  return SPARSEP_OK;
}

// The baseline: one kernel launch per matrix on `stream`, in matrix order.
int sparsep_batch_execute_per_matrix(sparsep_batch *b, void *stream) {
  if (!b) return SPARSEP_EINVAL;
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : b->stream;
  for (uint32_t m = 0; m < b->nmats; ++m)
    if (int st = dispatch_one(b, m, s)) return st;
  if (!stream) BCK(cudaStreamSynchronize(s));
  return SPARSEP_OK;
}

// One matrix alone (autotuner timing runs).
int sparsep_batch_execute_one(sparsep_batch *b, uint32_t m, void *stream) {
  if (!b || m >= b->nmats) return SPARSEP_EINVAL;
  return dispatch_one(b, m, static_cast<cudaStream_t>(stream));
}

// Exhaustive autotuner over the row-routine variants of every matrix: each
// candidate's items are built, uploaded to a scratch item array and timed
// alone with CUDA events (median of `reps`); the fastest is kept.  The chosen
// variants are committed (items rebuilt, graph recaptured on next execute).
// times_us (nmats x sparsep_batch_candidates()) receives the medians, 0 for
// candidates that do not apply to a matrix; chosen (nmats) the chosen index.
static const sparsep_batch_variant kCand[] = {
    {0, 4, 16384, 0},  {0, 8, 16384, 0},  {0, 16, 16384, 0},  {0, 32, 16384, 0}, {0, 4, 131072, 0},
    {0, 8, 131072, 0}, {0, 16, 131072, 0}, {0, 32, 131072, 0}, {1, 1, 16384, 0},  {1, 2, 16384, 0},
    {1, 4, 16384, 0},  {1, 8, 16384, 0},  {1, 16, 16384, 0},  {1, 32, 16384, 0}, {1, 1, 131072, 0},
    {1, 4, 131072, 0}, {1, 8, 131072, 0}, {1, 32, 131072, 0}};
constexpr int kNCand = sizeof(kCand) / sizeof(kCand[0]);

int sparsep_batch_candidates(sparsep_batch_variant *out, int max) {
  for (int i = 0; i < kNCand && out && i < max; ++i) out[i] = kCand[i];
  return kNCand;
}

int sparsep_batch_autotune(sparsep_batch *b, int reps, double *times_us, int32_t *chosen) {
  if (!b || reps < 1) return SPARSEP_EINVAL;
  cudaStream_t s = b->stream;
  cudaEvent_t e0, e1;
  BCK(cudaEventCreate(&e0));
  BCK(cudaEventCreate(&e1));
  int status = SPARSEP_OK;
  BItem *scratch = nullptr;
  size_t scratch_n = 0;
  std::vector<float> ms(reps);
  for (uint32_t m = 0; m < b->nmats && !status; ++m) {
    std::vector<uint32_t> rp((size_t)b->mats_h[m].nrows + 1);
    if ((status = bmap(cudaMemcpy(rp.data(), b->mats_h[m].rowptr, rp.size() * 4, cudaMemcpyDeviceToHost)))) break;
    double best = 1e300;
    int best_i = -1;
    const sparsep_batch_variant keep = b->var[m];
    for (int c = 0; c < kNCand && !status; ++c) {
      if (times_us) times_us[(size_t)m * kNCand + c] = 0.0;
      if (check_variant(kCand[c], b->mats_h[m].k)) continue;
      // candidate items of matrix m alone
      sparsep_batch tmp;
      tmp.mats_h = {b->mats_h[m]};
      tmp.var = {kCand[c]};
      tmp.item0.assign(1, 0);
      tmp.nitem.assign(1, 0);
      make_items(&tmp, 0, rp.data());
      for (auto &it : tmp.items_h) it.mat = m;
      tmp.mats_h.clear();
      const size_t n = tmp.items_h.size();
      if (n > scratch_n) {
        if (scratch) cudaFree(scratch);
        scratch = nullptr;
        if ((status = bmap(cudaMalloc(&scratch, n * sizeof(BItem))))) break;
        scratch_n = n;
      }
      if ((status = bmap(cudaMemcpy(scratch, tmp.items_h.data(), n * sizeof(BItem), cudaMemcpyHostToDevice)))) break;
      for (int r = -1; r < reps; ++r) {  // one untimed warm-up
        cudaEventRecord(e0, s);
        if (b->dtype == SPARSEP_FP32)
          per_matrix<float><<<(unsigned)((n + 7) / 8), 256, 0, s>>>((const Mat<float> *)b->mats_d, scratch, 0,
                                                                     (uint32_t)n);
        else
          per_matrix<int32_t><<<(unsigned)((n + 7) / 8), 256, 0, s>>>((const Mat<int32_t> *)b->mats_d, scratch, 0,
                                                                       (uint32_t)n);
        cudaEventRecord(e1, s);
        if ((status = bmap(cudaEventSynchronize(e1)))) break;
        if (r >= 0) cudaEventElapsedTime(&ms[r], e0, e1);
      }
      if (status) break;
      std::vector<float> sorted = ms;
      std::sort(sorted.begin(), sorted.end());
      const double us = 1e3 * sorted[sorted.size() / 2];
      if (times_us) times_us[(size_t)m * kNCand + c] = us;
      if (us < best) {
        best = us;
        best_i = c;
      }
    }
    b->var[m] = best_i >= 0 ? kCand[best_i] : keep;
    if (chosen) chosen[m] = best_i;
  }
  if (scratch) cudaFree(scratch);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (status) return status;
  return sparsep_batch_commit(b);
}

int sparsep_batch_get_info(const sparsep_batch *b, uint64_t *compulsory_bytes, uint64_t *items, uint64_t *nnz) {
  if (!b) return SPARSEP_EINVAL;
  if (compulsory_bytes) *compulsory_bytes = b->bytes;
  if (items) *items = b->items_h.size();
  if (nnz) {
    uint64_t t = 0;
    for (uint64_t v : b->nnz) t += v;
    *nnz = t;
  }
  return SPARSEP_OK;
}

}  // extern "C"
