// batch.cu -- host side of the batched multi-RHS SpMV: device copies of the
// matrices, work items and their queue order, the graph-captured batch
// launch, the per-matrix baseline and the exhaustive variant autotuner.  The
// kernels are in batch_kernels.cu.
#include <algorithm>
#include <cmath>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <thread>
#include <vector>

#include "fault.hpp"
#include "batch.hpp"
#include "internal.hpp"

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
  std::vector<std::vector<uint32_t>> rowptr;  // host copies: items are rebuilt without a read-back
  std::vector<std::vector<uint32_t>> clo, chi;  // per row: lowest and highest column (window items)
  std::vector<std::vector<uint32_t>> bbrp;      // host copies of the 4 x 4 BCSR block-row pointers (if any)
  std::vector<float> feat;                    // nmats x SPARSEP_NFEATURES selector features
  std::vector<sparsep_batch_variant> var;
  std::vector<BItem> items_h;          // committed items, matrix after matrix
  std::vector<uint32_t> item0, nitem;  // per matrix: first item and count
  std::vector<BItem> base_h;           // the per-matrix baseline's items
  std::vector<uint32_t> base0, nbase;
  int *err = nullptr;  // staging timeouts (SPARSEP_ETIMEDOUT), sticky until read
  bool ticket = true;  // batch launch: CTAs claim items by atomic ticket (else CTA b runs item b)
  BItem *items_d = nullptr;  // committed items (per-matrix launches of one matrix)
  BItem *queue_d = nullptr;  // the same items in queue order (long rows first)
  BItem *base_d = nullptr;
  unsigned int *head = nullptr;
  cudaStream_t stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint64_t bytes = 0;  // compulsory bytes of one batch execution
};

static int bmap(cudaError_t e) {
  if (e == cudaSuccess) return SPARSEP_OK;
  char msg[256];
  std::snprintf(msg, sizeof msg, "%s (%d)", cudaGetErrorString(e), (int)e);
  sparsep::record_error(msg);
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
  BCK(dev_malloc((void **)&d, bytes ? bytes : 16));
  b->allocs.push_back(d);
  *out = d;
  return SPARSEP_OK;
}

static void bfree(sparsep_batch *b, void *d) {
  if (!d) return;
  for (auto i = b->allocs.begin(); i != b->allocs.end(); ++i)
    if (*i == d) {
      dev_free(*i);
      b->allocs.erase(i);
      return;
    }
}

static uint32_t pow2ceil(uint32_t v) {
  uint32_t p = 1;
  while (p < v) p <<= 1;
  return p;
}

#ifndef SPARSEP_BATCH_ITEM_WORK
#define SPARSEP_BATCH_ITEM_WORK 163840
#endif
static constexpr uint32_t DEFAULT_ITEM_WORK = SPARSEP_BATCH_ITEM_WORK;  // nonzero x right-hand-side products per item

// Nonzeros per item for a variant: about item_work products, within [32, BCAP].
static uint32_t item_cap(const sparsep_batch_variant &v, uint32_t k) {
  const uint64_t w = v.item_work > 0 ? (uint64_t)v.item_work : DEFAULT_ITEM_WORK;
  return (uint32_t)std::min<uint64_t>(BCAP, std::max<uint64_t>(32, w / k));
}

// Items of one matrix: consecutive rows up to `cap` nonzeros and BRCAP rows;
// a row longer than BCAP becomes one item per BCAP-nonzero chunk, sharing the
// row's slot of chunk partials and its arrival counter.  Under a
// window variant (mode 2, 3) an item also stops growing when the x rows its
// columns span would no longer fit the staging arena beside its nonzeros, and
// it stages them (c0, cw) when they pay: at least two nonzeros per staged x
// row.  Rows whose own span does not fit start ordinary items.
static void make_block_items(const Mat<float> &M, const uint32_t *bbrp, const sparsep_batch_variant &v,
                             uint32_t cap, std::vector<BItem> &out);

static void make_items(const Mat<float> &M, const uint32_t *rowptr, const uint32_t *clo, const uint32_t *chi,
                       const uint32_t *bbrp, uint32_t es, const sparsep_batch_variant &v, uint32_t cap,
                       std::vector<BItem> &out) {
  if (v.mode == 4) return make_block_items(M, bbrp, v, cap, out);
  const uint32_t k = M.pitch;  // every routine computes the whole padded row
  const uint32_t V = (uint32_t)std::max(1, v.vec);
  const uint32_t acc = pow2ceil((k + v.lanes * V - 1) / (v.lanes * V));
  // chunks of long rows: the widest load the pitch allows, lanes for one pass
  const uint32_t v_long = k % 4 == 0 ? 4 : (k % 2 == 0 ? 2 : 1);
  const uint32_t g_long = std::min<uint32_t>(32, pow2ceil(k / v_long));
  const uint32_t acc_long = pow2ceil((k + g_long * v_long - 1) / (g_long * v_long));
  uint64_t part_off = 0;  // the long rows' partials and counters, in row order
  uint32_t slot = 0;
  const bool windows = (v.mode & 2) != 0;
  const uint32_t xrow = k * es;  // bytes of one staged x row
  BItem base{};
  base.rowptr = M.rowptr;
  base.colind = M.colind;
  base.val = M.val;
  base.x = M.x;
  base.y = M.y;
  base.k = (uint16_t)k;
  base.ncols = M.ncols;
  base.nrows = M.nrows;
  BItem cur{};
  bool open = false, win = false;
  uint32_t lo = 0, hi = 0;  // columns spanned by the open window item (hi exclusive; lo == hi: none yet)
  auto fits = [&](uint32_t nr, uint32_t n, uint32_t a, uint32_t b) {
    return carve(nr, n, es, (b - a) * xrow).end <= ARENA;
  };
  auto flush = [&]() {
    if (!open) return;
    open = false;
    if (win && hi > lo && 2ull * (hi - lo) <= cur.p1 - cur.p0) cur.c0 = lo, cur.cw = hi - lo;
    out.push_back(cur);
  };
  for (uint32_t r = 0; r < M.nrows; ++r) {
    const uint32_t len = rowptr[r + 1] - rowptr[r];
    if (len > BCAP) {
      flush();
      const uint32_t nch = (len + BCAP - 1) / BCAP;
      for (uint32_t c = 0; c < nch; ++c) {
        BItem it = base;
        it.r0 = r;
        it.nr = 1;
        it.p0 = rowptr[r] + c * BCAP;
        it.p1 = std::min(rowptr[r + 1], it.p0 + BCAP);
        it.mode = MODE_LONG;
        it.lanes = (uint8_t)g_long;
        it.vec = (uint8_t)v_long;
        it.acc = (uint8_t)acc_long;
        it.c0 = c;
        it.cw = nch;
        it.part = M.part + part_off;
        it.cnt = M.cnt + slot;
        out.push_back(it);
      }
      part_off += (uint64_t)nch * k;
      ++slot;
      continue;
    }
    // the span with this row added
    const uint32_t a = len ? (hi > lo ? std::min(lo, clo[r]) : clo[r]) : lo;
    const uint32_t b = len ? (hi > lo ? std::max(hi, chi[r] + 1) : chi[r] + 1) : hi;
    if (open && (cur.p1 - cur.p0 + len > cap || cur.nr == BRCAP ||
                 (win && !fits(cur.nr + 1, cur.p1 - cur.p0 + len, a, b))))
      flush();
    if (!open) {
      cur = base;
      cur.r0 = r;
      cur.nr = 0;
      cur.p0 = cur.p1 = rowptr[r];
      cur.mode = (v.mode & 1) ? MODE_MERGE : MODE_ROWS;
      cur.lanes = (uint8_t)v.lanes;
      cur.vec = (uint8_t)V;
      cur.acc = (uint8_t)acc;
      cur.c0 = cur.cw = 0;
      open = true;
      lo = hi = 0;
      win = windows && (!len || fits(1, len, clo[r], chi[r] + 1));
    }
    if (win && len) {
      lo = hi > lo ? std::min(lo, clo[r]) : clo[r];
      hi = std::max(hi, chi[r] + 1);
    }
    cur.nr = (uint16_t)(r + 1 - cur.r0);
    cur.p1 = rowptr[r + 1];
  }
  flush();
}

// Block items of one matrix (mode 4, its 4 x 4 BCSR copy): consecutive block
// rows up to `cap` nonzero slots (16 per block, at most BBCAP blocks) and
// BRCAP / 4 block rows.
static void make_block_items(const Mat<float> &M, const uint32_t *bbrp, const sparsep_batch_variant &v,
                             uint32_t cap, std::vector<BItem> &out) {
  const uint32_t nbr = (M.nrows + 3) / 4;
  const uint32_t bcap = std::max<uint32_t>(1, std::min<uint32_t>(BBCAP, cap / 16));
  BItem base{};
  base.rowptr = M.browptr;
  base.colind = M.bcol;
  base.val = M.bval;
  base.x = M.x;
  base.y = M.y;
  base.k = (uint16_t)M.pitch;
  base.ncols = M.ncols;
  base.nrows = M.nrows;
  base.mode = MODE_BCSR;
  base.lanes = (uint8_t)v.lanes;
  base.vec = 4;
  base.acc = 1;
  BItem cur{};
  bool open = false;
  for (uint32_t br = 0; br < nbr; ++br) {
    const uint32_t len = bbrp[br + 1] - bbrp[br];  // <= BBCAP (checked when the copy was built)
    if (open && (cur.p1 - cur.p0 + len > bcap || cur.nr == BRCAP / 4)) out.push_back(cur), open = false;
    if (!open) {
      cur = base;
      cur.r0 = br;
      cur.nr = 0;
      cur.p0 = cur.p1 = bbrp[br];
      open = true;
    }
    cur.nr = (uint16_t)(br + 1 - cur.r0);
    cur.p1 = bbrp[br + 1];
  }
  if (open) out.push_back(cur);
}

static int check_variant(const sparsep_batch_variant &v, uint32_t nrhs) {
  if (v.item_work < 0 || v.mode < 0 || v.mode > 4) return SPARSEP_EINVAL;
  const uint32_t k = row_pitch(nrhs);
  const int V = v.vec ? v.vec : 1;
  if (v.lanes < 1 || v.lanes > 32 || (v.lanes & (v.lanes - 1))) return SPARSEP_EINVAL;
  if (V != 1 && V != 2 && V != 4) return SPARSEP_EINVAL;
  if (k % V || ((v.mode & 2) && V != 4)) return SPARSEP_ENOSYS;  // windows: 4-wide variants
  if (v.mode == 4 && (V != 4 || (uint32_t)v.lanes * 4 < k)) return SPARSEP_ENOSYS;  // blocks: one pass of 4-wide
  if (pow2ceil((k + v.lanes * V - 1) / (v.lanes * V)) * V > (uint32_t)ACC_REGS) return SPARSEP_ENOSYS;
  return SPARSEP_OK;
}

static const uint32_t *bbrp_of(const sparsep_batch *b, uint32_t m) {
  return b->bbrp[m].empty() ? nullptr : b->bbrp[m].data();
}

// check_variant, and block variants only where the matrix has a BCSR copy.
static int variant_ok(const sparsep_batch *b, uint32_t m, const sparsep_batch_variant &v) {
  if (int st = check_variant(v, b->mats_h[m].k)) return st;
  return v.mode == 4 && !b->mats_h[m].browptr ? SPARSEP_ENOSYS : SPARSEP_OK;
}

// Merge mode, the widest vector load that divides the row pitch, and enough
// lanes for one pass over it (at most 32).
extern "C" void sparsep_batch_variant_default(uint32_t nrhs, sparsep_batch_variant *v) {
  if (!v) return;
  std::memset(v, 0, sizeof *v);
  const uint32_t k = row_pitch(nrhs);
  v->mode = 1;
  v->vec = k % 4 == 0 ? 4 : 1;
  v->lanes = (int)std::min<uint32_t>(32, pow2ceil((k + v->vec - 1) / v->vec));
  while (check_variant(*v, nrhs) && v->vec > 1) {
    v->vec >>= 1;
    v->lanes = (int)std::min<uint32_t>(32, pow2ceil((k + v->vec - 1) / v->vec));
  }
  v->item_work = 0;
}

// Queue order of the batch launch: long-row chunks first (rows with the most
// chunks first), then the rest matrix after matrix.
static void queue_order(const std::vector<BItem> &in, std::vector<BItem> &q) {
  q.clear();
  q.reserve(in.size());
  for (const BItem &it : in)
    if (it.mode == MODE_LONG) q.push_back(it);
  std::stable_sort(q.begin(), q.end(), [](const BItem &a, const BItem &b) { return a.cw > b.cw; });
  for (const BItem &it : in)
    if (it.mode != MODE_LONG) q.push_back(it);
}

// Committed variants -> items, queue, device copies; drops the captured graph.
static int rebuild(sparsep_batch *b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  b->items_h.clear();
  for (uint32_t m = 0; m < b->nmats; ++m) {
    b->item0[m] = (uint32_t)b->items_h.size();
    make_items(b->mats_h[m], b->rowptr[m].data(), b->clo[m].data(), b->chi[m].data(), bbrp_of(b, m), (uint32_t)b->esize, b->var[m],
               item_cap(b->var[m], b->mats_h[m].pitch), b->items_h);
    b->nitem[m] = (uint32_t)b->items_h.size() - b->item0[m];
  }
  std::vector<BItem> q;
  queue_order(b->items_h, q);
  bfree(b, b->items_d);
  bfree(b, b->queue_d);
  b->items_d = b->queue_d = nullptr;
  const size_t bytes = sizeof(BItem) * std::max<size_t>(1, b->items_h.size());
  int st = balloc(b, bytes, (void **)&b->items_d);
  if (!st) st = balloc(b, bytes, (void **)&b->queue_d);
  if (st) return st;
  if (!b->items_h.empty()) {
    BCK(cudaMemcpyAsync(b->items_d, b->items_h.data(), sizeof(BItem) * b->items_h.size(), cudaMemcpyHostToDevice,
                        b->stream));
    BCK(cudaMemcpyAsync(b->queue_d, q.data(), sizeof(BItem) * q.size(), cudaMemcpyHostToDevice, b->stream));
  }
  // landed before any launch on any stream reads them (q dies on return)
  BCK(cudaStreamSynchronize(b->stream));
  return SPARSEP_OK;
}

// The baseline's items: every matrix with the default variant for its k and
// items small enough that one launch per matrix spreads over all SMs.
static uint32_t grid_filling_cap(const sparsep_batch *b, uint32_t m, uint32_t cap) {
  const uint64_t want = (b->nnz[m] + 2ull * b->sms - 1) / (2ull * b->sms);
  return (uint32_t)std::min<uint64_t>(cap, std::max<uint64_t>(64, want));
}

// The 4 x 4 BCSR copy of matrix m for the block variants (mode 4), built on
// the device from its uploaded CSR, for matrices whose 4 x 4 blocks are at
// least a quarter full (selector feature 12) and whose pitch is a multiple of
// 4; dropped again when a block row holds more than BBCAP blocks.
template <typename T>
static int build_blocks(sparsep_batch *b, uint32_t m) {
  auto &h = b->mats_h[m];
  if (!b->nnz[m] || h.pitch % 4 || b->feat[(size_t)m * SPARSEP_NFEATURES + 12] < 0.25f) return SPARSEP_OK;
  sparsep_bcsr_layout *L = nullptr;
  uint64_t nb = 0;
  if (int st = sparsep_bcsr_layout_device(h.rowptr, h.colind, h.nrows, h.ncols, (uint32_t)b->nnz[m], 4, 4, &L, &nb,
                                          b->stream))
    return st;
  const uint32_t nbr = (h.nrows + 3) / 4;
  void *brp = nullptr, *bcol = nullptr, *bval = nullptr, *npb = nullptr;
  int st = balloc(b, ((size_t)nbr + 1 + 16) * 4, &brp);
  if (!st) st = balloc(b, (nb + 16) * 4, &bcol);
  if (!st) st = balloc(b, (nb * 16 + 16) * sizeof(T), &bval);
  if (!st) st = balloc(b, (nb + 16) * 4, &npb);
  if (!st) {
    if constexpr (std::is_same<T, float>::value)
      st = sparsep_csr2bcsr_device_f32(L, reinterpret_cast<const float *>(h.val), (uint32_t *)brp, (uint32_t *)bcol,
                                       (float *)bval, (uint32_t *)npb, b->stream);
    else
      st = sparsep_csr2bcsr_device_i32(L, reinterpret_cast<const int32_t *>(h.val), (uint32_t *)brp,
                                       (uint32_t *)bcol, (int32_t *)bval, (uint32_t *)npb, b->stream);
  }
  sparsep_bcsr_layout_free(L);
  bfree(b, npb);
  std::vector<uint32_t> hb;
  if (!st) {
    hb.resize((size_t)nbr + 1);
    st = bmap(cudaMemcpy(hb.data(), brp, hb.size() * 4, cudaMemcpyDeviceToHost));
  }
  uint32_t most = 0;
  for (uint32_t i = 0; !st && i < nbr; ++i) most = std::max(most, hb[i + 1] - hb[i]);
  if (st || most > BBCAP) {
    bfree(b, brp);
    bfree(b, bcol);
    bfree(b, bval);
    return st;
  }
  h.browptr = static_cast<const uint32_t *>(brp);
  h.bcol = static_cast<const uint32_t *>(bcol);
  h.bval = static_cast<const float *>(bval);
  b->bbrp[m] = std::move(hb);
  return SPARSEP_OK;
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
  // uploads and clears go on the batch's own stream, which rebuild() drains
  // before returning: a launch on any stream then sees them complete
  BCK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
  b->mats_h.resize(nmats);
  b->nnz.resize(nmats);
  b->var.resize(nmats);
  b->item0.resize(nmats);
  b->nitem.resize(nmats);
  b->base0.resize(nmats);
  b->nbase.resize(nmats);
  b->rowptr.resize(nmats);
  b->clo.resize(nmats);
  b->chi.resize(nmats);
  b->bbrp.resize(nmats);
  for (uint32_t m = 0; m < nmats; ++m) {
    const auto *M = A[m];
    if (!M || !M->rowptr || (M->nnz && (!M->colind || !M->values))) return SPARSEP_EINVAL;
    const uint32_t k = nrhs[m];
    if (k == 0 || k > 256) return SPARSEP_EINVAL;
    if (M->rowptr[0] != 0 || M->rowptr[M->nrows] != M->nnz) return SPARSEP_EINVAL;
    for (uint32_t r = 0; r < M->nrows; ++r)
      if (M->rowptr[r + 1] < M->rowptr[r]) return SPARSEP_EINVAL;
    for (uint32_t q = 0; q < M->nnz; ++q)
      if (M->colind[q] >= M->ncols) return SPARSEP_EINVAL;
    if (var) b->var[m] = var[m];
    else sparsep_batch_variant_default(k, &b->var[m]);
    if (int st = check_variant(b->var[m], k)) return st;
    const uint32_t kp = row_pitch(k);
    void *d[5];
    int st = balloc(b, ((size_t)M->nrows + 1 + 16) * 4, &d[0]);
    if (!st) st = balloc(b, ((size_t)M->nnz + 16) * 4, &d[1]);
    if (!st) st = balloc(b, ((size_t)M->nnz + 16) * sizeof(T), &d[2]);
    const size_t xrows = ((size_t)M->ncols + 3) / 4 * 4;  // whole 4-column blocks (block items read them)
    if (!st) st = balloc(b, (xrows * kp + 16) * sizeof(T), &d[3]);
    if (!st) st = balloc(b, ((size_t)M->nrows * kp + 16) * sizeof(T), &d[4]);
    if (st) return st;
    // rows longer than BCAP: a partial row per chunk and an arrival counter
    uint64_t chunks = 0, longrows = 0;
    for (uint32_t r = 0; r < M->nrows; ++r) {
      const uint32_t len = M->rowptr[r + 1] - M->rowptr[r];
      if (len > BCAP) chunks += (len + BCAP - 1) / BCAP, ++longrows;
    }
    void *part = nullptr, *cnt = nullptr;
    if (longrows) {
      if ((st = balloc(b, chunks * kp * sizeof(T), &part))) return st;
      if ((st = balloc(b, longrows * sizeof(unsigned), &cnt))) return st;
      BCK(cudaMemsetAsync(cnt, 0, longrows * sizeof(unsigned), b->stream));
    }
    BCK(cudaMemcpyAsync(d[0], M->rowptr, ((size_t)M->nrows + 1) * 4, cudaMemcpyHostToDevice, b->stream));
    if (M->nnz) {
      BCK(cudaMemcpyAsync(d[1], M->colind, (size_t)M->nnz * 4, cudaMemcpyHostToDevice, b->stream));
      BCK(cudaMemcpyAsync(d[2], M->values, (size_t)M->nnz * sizeof(T), cudaMemcpyHostToDevice, b->stream));
    }
    BCK(cudaMemsetAsync(d[3], 0, (xrows * kp + 16) * sizeof(T), b->stream));
    auto &h = b->mats_h[m];
    h.rowptr = (const uint32_t *)d[0];
    h.colind = (const uint32_t *)d[1];
    h.val = (const float *)d[2];
    h.x = (const float *)d[3];
    h.y = (float *)d[4];
    h.part = (float *)part;
    h.cnt = (unsigned *)cnt;
    h.nrows = M->nrows;
    h.ncols = M->ncols;
    h.k = k;
    h.pitch = kp;
    b->nnz[m] = M->nnz;
    b->rowptr[m].assign(M->rowptr, M->rowptr + M->nrows + 1);
    b->clo[m].assign(M->nrows, 0);
    b->chi[m].assign(M->nrows, 0);
    for (uint32_t r = 0; r < M->nrows; ++r)
      for (uint32_t q = M->rowptr[r]; q < M->rowptr[r + 1]; ++q) {
        const uint32_t c = M->colind[q];
        if (q == M->rowptr[r] || c < b->clo[m][r]) b->clo[m][r] = c;
        if (q == M->rowptr[r] || c > b->chi[m][r]) b->chi[m][r] = c;
      }
    b->bytes += (uint64_t)M->nnz * (4 + sizeof(T)) + ((uint64_t)M->nrows + 1) * 4 +
                ((uint64_t)M->ncols + M->nrows) * k * sizeof(T);
  }
  // selector features, matrices spread over the host's threads
  b->feat.assign((size_t)nmats * SPARSEP_NFEATURES, 0.f);
  {
    const unsigned nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < nt; ++t)
      pool.emplace_back([&, t]() {
        for (uint32_t m = t; m < nmats; m += nt)
          sparsep_features(A[m]->nrows, A[m]->ncols, A[m]->rowptr, A[m]->colind, nrhs[m],
                           &b->feat[(size_t)m * SPARSEP_NFEATURES]);
      });
    for (auto &th : pool) th.join();
  }
  for (uint32_t m = 0; m < nmats; ++m)
    if (int st = build_blocks<T>(b, m)) return st;
  for (uint32_t m = 0; m < nmats; ++m)
    if (int st = variant_ok(b, m, b->var[m])) return st;
  for (uint32_t m = 0; m < nmats; ++m) {
    sparsep_batch_variant dv;
    sparsep_batch_variant_default(b->mats_h[m].k, &dv);
    b->base0[m] = (uint32_t)b->base_h.size();
    make_items(b->mats_h[m], b->rowptr[m].data(), b->clo[m].data(), b->chi[m].data(), bbrp_of(b, m), (uint32_t)b->esize, dv,
               grid_filling_cap(b, m, item_cap(dv, b->mats_h[m].pitch)), b->base_h);
    b->nbase[m] = (uint32_t)b->base_h.size() - b->base0[m];
  }
  int st = balloc(b, 64, (void **)&b->err);
  if (!st) st = balloc(b, sizeof(BItem) * std::max<size_t>(1, b->base_h.size()), (void **)&b->base_d);
  if (!st) st = balloc(b, 64, (void **)&b->head);
  if (st) return st;
  BCK(cudaMemsetAsync(b->err, 0, 64, b->stream));
  if (!b->base_h.empty())
    BCK(cudaMemcpyAsync(b->base_d, b->base_h.data(), sizeof(BItem) * b->base_h.size(), cudaMemcpyHostToDevice,
                        b->stream));
  if ((st = rebuild(b))) return st;  // also waits for every upload above
  *out = guard.release();
  return SPARSEP_OK;
}

// err[1] carries the test-support wait fault to the kernel (read on the device,
// so a captured graph sees the switch as it is at launch)
static int set_fault_word(sparsep_batch *b, cudaStream_t s) {
  BCK(cudaMemsetAsync(b->err + 1, wait_fault() ? 1 : 0, sizeof(int), s));
  return SPARSEP_OK;
}

template <typename T>
static int launch_queue(sparsep_batch *b, cudaStream_t s) {
  if (b->ticket) BCK(cudaMemsetAsync(b->head, 0, 4, s));
  return bmap(batch_launch<T>(b->queue_d, 0, (uint32_t)b->items_h.size(), b->ticket ? b->head : nullptr, b->err, s));
}

template <typename T>
static int launch_items(sparsep_batch *b, const BItem *items, uint32_t i0, uint32_t n, cudaStream_t s) {
  return bmap(batch_launch<T>(items, i0, n, nullptr, b->err, s));
}

static int dispatch_queue(sparsep_batch *b, cudaStream_t s) {
  return b->dtype == SPARSEP_FP32 ? launch_queue<float>(b, s) : launch_queue<int32_t>(b, s);
}
static int dispatch_items(sparsep_batch *b, const BItem *items, uint32_t i0, uint32_t n, cudaStream_t s) {
  return b->dtype == SPARSEP_FP32 ? launch_items<float>(b, items, i0, n, s) : launch_items<int32_t>(b, items, i0, n, s);
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
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (void *d : b->allocs) dev_free(d);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

int sparsep_batch_set_variant(sparsep_batch *b, uint32_t m, const sparsep_batch_variant *v) {
  if (!b || !v || m >= b->nmats) return SPARSEP_EINVAL;
  if (int st = variant_ok(b, m, *v)) return st;
  b->var[m] = *v;
  return SPARSEP_OK;
}

int sparsep_batch_get_variant(const sparsep_batch *b, uint32_t m, sparsep_batch_variant *v) {
  if (!b || !v || m >= b->nmats) return SPARSEP_EINVAL;
  *v = b->var[m];
  return SPARSEP_OK;
}

// Rebuild the items and the queue after variants changed.
int sparsep_batch_commit(sparsep_batch *b) {
  if (!b) return SPARSEP_EINVAL;
  try {
    return rebuild(b);
  } catch (const std::bad_alloc &) {
    return SPARSEP_ENOMEM;
  }
}

int sparsep_batch_x(sparsep_batch *b, uint32_t m, void **d_x, void **d_y) {
  if (!b || m >= b->nmats) return SPARSEP_EINVAL;
  if (d_x) *d_x = (void *)b->mats_h[m].x;
  if (d_y) *d_y = (void *)b->mats_h[m].y;
  return SPARSEP_OK;
}

int sparsep_batch_pitch(const sparsep_batch *b, uint32_t m, uint32_t *pitch) {
  if (!b || !pitch || m >= b->nmats) return SPARSEP_EINVAL;
  *pitch = b->mats_h[m].pitch;
  return SPARSEP_OK;
}

// Host x (ncols x k, dense rows) into the device rows of `pitch` elements.
int sparsep_batch_set_x(sparsep_batch *b, uint32_t m, const void *h_x) {
  if (!b || !h_x || m >= b->nmats) return SPARSEP_EINVAL;
  const auto &M = b->mats_h[m];
  const size_t w = (size_t)M.k * b->esize;
  BCK(cudaMemcpy2DAsync((void *)M.x, (size_t)M.pitch * b->esize, h_x, w, w, M.ncols, cudaMemcpyHostToDevice,
                        b->stream));
  BCK(cudaStreamSynchronize(b->stream));  // in place before any later launch, on any stream
  return SPARSEP_OK;
}

int sparsep_batch_get_y(sparsep_batch *b, uint32_t m, void *h_y) {
  if (!b || !h_y || m >= b->nmats) return SPARSEP_EINVAL;
  const auto &M = b->mats_h[m];
  BCK(cudaStreamSynchronize(b->stream));
  const size_t w = (size_t)M.k * b->esize;
  BCK(cudaMemcpy2DAsync(h_y, w, M.y, (size_t)M.pitch * b->esize, w, M.nrows, cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  return SPARSEP_OK;
}

// The whole batch: one graph launch (queue reset + queue kernel); the
// graph is captured on the first call after a (re)commit.
int sparsep_batch_execute(sparsep_batch *b, void *stream) {
  if (!b) return SPARSEP_EINVAL;
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : b->stream;
  if (int st = set_fault_word(b, s)) return st;
  if (!b->exec) {
    BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    int st = dispatch_queue(b, b->stream);
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
  if (stream) return SPARSEP_OK;
  BCK(cudaStreamSynchronize(s));
  return sparsep_batch_status(b);
}

// The baseline: one plain launch per matrix, in matrix order, each matrix with
// the default (untuned) variant for its k and items sized to fill the GPU.
int sparsep_batch_execute_per_matrix(sparsep_batch *b, void *stream) {
  if (!b) return SPARSEP_EINVAL;
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : b->stream;
  if (int st = set_fault_word(b, s)) return st;
  for (uint32_t m = 0; m < b->nmats; ++m)
    if (int st = dispatch_items(b, b->base_d, b->base0[m], b->nbase[m], s)) return st;
  if (stream) return SPARSEP_OK;
  BCK(cudaStreamSynchronize(s));
  return sparsep_batch_status(b);
}

// One matrix alone with its committed items.
int sparsep_batch_execute_one(sparsep_batch *b, uint32_t m, void *stream) {
  if (!b || m >= b->nmats) return SPARSEP_EINVAL;
  return dispatch_items(b, b->items_d, b->item0[m], b->nitem[m], static_cast<cudaStream_t>(stream));
}

// Exhaustive autotuner over the row-routine variants of every matrix: each
// candidate's items (sized to fill the GPU) are uploaded to a scratch array
// and timed alone with CUDA events (median of `reps`, after one warm-up); the
// fastest is kept.  The chosen variants are committed (items rebuilt, graph
// recaptured on the next execute).  times_us (nmats x candidates) receives
// the medians, 0 where a candidate does not apply; chosen (nmats) the index.
static const sparsep_batch_variant kCand[] = {
    {0, 1, 0, 1},  {0, 1, 0, 4},  {0, 2, 0, 1},  {0, 2, 0, 4},  {0, 4, 0, 1},  {0, 4, 0, 4},
    {0, 8, 0, 1},  {0, 8, 0, 4},  {0, 16, 0, 1}, {0, 16, 0, 4}, {1, 1, 0, 1},  {1, 1, 0, 4},
    {1, 2, 0, 1},  {1, 2, 0, 4},  {1, 4, 0, 1},  {1, 4, 0, 4},  {1, 8, 0, 1},  {1, 8, 0, 4},
    {1, 16, 0, 1}, {1, 16, 0, 4}, {1, 32, 0, 4}, {2, 1, 0, 4},  {2, 2, 0, 4},  {2, 4, 0, 4},
    {2, 8, 0, 4},  {2, 16, 0, 4}, {3, 2, 0, 4},  {3, 4, 0, 4},  {3, 8, 0, 4},  {3, 16, 0, 4},
    {4, 1, 0, 4},  {4, 2, 0, 4},  {4, 4, 0, 4},  {4, 8, 0, 4},  {4, 16, 0, 4}, {4, 32, 0, 4}};
constexpr int kNCand = sizeof(kCand) / sizeof(kCand[0]);
static_assert(kNCand == SPARSEP_NVARIANTS, "the selector scores every candidate");

// SPARSEP_OK if variant v can run matrix m (its k, and for block variants a
// BCSR copy), else ENOSYS / EINVAL.
int sparsep_batch_variant_applies(const sparsep_batch *b, uint32_t m, const sparsep_batch_variant *v) {
  if (!b || !v || m >= b->nmats) return SPARSEP_EINVAL;
  return variant_ok(b, m, *v);
}

int sparsep_batch_candidates(sparsep_batch_variant *out, int max) {
  for (int i = 0; i < kNCand && out && i < max; ++i) out[i] = kCand[i];
  return kNCand;
}

int sparsep_batch_time_variant(sparsep_batch *b, uint32_t m, const sparsep_batch_variant *v, int reps,
                               double *us_out);

int sparsep_batch_autotune(sparsep_batch *b, int reps, double *times_us, int32_t *chosen) {
  if (!b || reps < 1) return SPARSEP_EINVAL;
  for (uint32_t m = 0; m < b->nmats; ++m) {
    double best = 1e300;
    int best_i = -1;
    for (int c = 0; c < kNCand; ++c) {
      double us = 0.0;
      const int st = sparsep_batch_time_variant(b, m, &kCand[c], reps, &us);
      if (st == SPARSEP_ENOSYS) us = 0.0;
      else if (st) return st;
      if (times_us) times_us[(size_t)m * kNCand + c] = us;
      if (us > 0.0 && us < best) {
        best = us;
        best_i = c;
      }
    }
    if (best_i >= 0) b->var[m] = kCand[best_i];
    if (chosen) chosen[m] = best_i;
  }
  return sparsep_batch_commit(b);
}

// Median time (us) of matrix m alone under variant v, items sized to fill the
// GPU; ENOSYS when v does not apply to m's right-hand-side count.
int sparsep_batch_time_variant(sparsep_batch *b, uint32_t m, const sparsep_batch_variant *v, int reps,
                               double *us_out) {
  if (!b || !v || !us_out || m >= b->nmats || reps < 1) return SPARSEP_EINVAL;
  if (int st = variant_ok(b, m, *v)) return st;
  std::vector<BItem> items;
  try {
    make_items(b->mats_h[m], b->rowptr[m].data(), b->clo[m].data(), b->chi[m].data(), bbrp_of(b, m), (uint32_t)b->esize, *v,
               grid_filling_cap(b, m, item_cap(*v, b->mats_h[m].pitch)), items);
  } catch (const std::bad_alloc &) {
    return SPARSEP_ENOMEM;
  }
  *us_out = 0.0;
  if (items.empty()) return SPARSEP_OK;
  BItem *d = nullptr;
  BCK(dev_malloc((void **)&d, items.size() * sizeof(BItem)));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  // same stream as the timed launches: the items are in place before the first
  int st = bmap(cudaMemcpyAsync(d, items.data(), items.size() * sizeof(BItem), cudaMemcpyHostToDevice, b->stream));
  if (!st) st = bmap(cudaEventCreate(&e0));
  if (!st) st = bmap(cudaEventCreate(&e1));
  std::vector<float> ms(reps);
  for (int r = -1; r < reps && !st; ++r) {
    cudaEventRecord(e0, b->stream);
    st = dispatch_items(b, d, 0, (uint32_t)items.size(), b->stream);
    cudaEventRecord(e1, b->stream);
    if (!st) st = bmap(cudaEventSynchronize(e1));
    if (!st && r >= 0) st = bmap(cudaEventElapsedTime(&ms[r], e0, e1));
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  dev_free(d);
  if (st) return st;
  std::sort(ms.begin(), ms.end());
  *us_out = 1e3 * ms[ms.size() / 2];
  return SPARSEP_OK;
}

// Staging timeouts since the last call (the failed items were skipped):
// SPARSEP_ETIMEDOUT, else OK.  Synchronises the batch's work.
int sparsep_batch_status(sparsep_batch *b) {
  if (!b) return SPARSEP_EINVAL;
  int h = 0;
  BCK(cudaStreamSynchronize(b->stream));
  BCK(cudaMemcpyAsync(&h, b->err, sizeof h, cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  if (!h) return SPARSEP_OK;
  BCK(cudaMemsetAsync(b->err, 0, sizeof h, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  if (h == SPARSEP_ETIMEDOUT) return h;
  char msg[96];
  std::snprintf(msg, sizeof msg, "batch kernel check failed at site %d", h);  // checked build only
  sparsep::record_error(msg);
  return SPARSEP_EIO;
}

// 1: CTAs of the batch launch claim items by atomic ticket (queue order
// guaranteed); 0: CTA b runs queue item b (order as the hardware schedules).
int sparsep_batch_set_ticket(sparsep_batch *b, int on) {
  if (!b) return SPARSEP_EINVAL;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  b->ticket = on != 0;
  return SPARSEP_OK;
}

int sparsep_batch_features(const sparsep_batch *b, float *out) {
  if (!b || !out) return SPARSEP_EINVAL;
  std::memcpy(out, b->feat.data(), sizeof(float) * b->feat.size());
  return SPARSEP_OK;
}

// Learned variants: the network's highest-scoring applicable candidate per
// matrix; below min_confidence (softmax probability over the applicable
// candidates) the matrix is autotuned exhaustively instead.
int sparsep_batch_select(sparsep_batch *b, sparsep_selector *sel, float min_confidence, int reps, int32_t *chosen,
                         int32_t *fallback) {
  if (!b || !sel || reps < 1) return SPARSEP_EINVAL;
  std::vector<float> z;
  try {
    z.resize((size_t)b->nmats * kNCand);
  } catch (const std::bad_alloc &) {
    return SPARSEP_ENOMEM;
  }
  if (int st = sparsep_selector_scores(sel, b->feat.data(), b->nmats, z.data())) return st;
  for (uint32_t m = 0; m < b->nmats; ++m) {
    const float *zm = &z[(size_t)m * kNCand];
    int best = -1;
    float zmax = -3.0e38f;
    for (int c = 0; c < kNCand; ++c)
      if (!variant_ok(b, m, kCand[c]) && zm[c] > zmax) zmax = zm[c], best = c;
    double sum = 0.0;
    for (int c = 0; c < kNCand; ++c)
      if (!variant_ok(b, m, kCand[c])) sum += std::exp((double)zm[c] - zmax);
    const double conf = best >= 0 ? 1.0 / sum : 0.0;
    int fb = 0;
    if (best < 0 || conf < min_confidence) {
      fb = 1;
      double tbest = 1e300;
      for (int c = 0; c < kNCand; ++c) {
        double us = 0.0;
        const int st = sparsep_batch_time_variant(b, m, &kCand[c], reps, &us);
        if (st == SPARSEP_ENOSYS) continue;
        if (st) return st;
        if (us > 0.0 && us < tbest) tbest = us, best = c;
      }
    }
    if (best >= 0) b->var[m] = kCand[best];
    if (chosen) chosen[m] = best;
    if (fallback) fallback[m] = fb;
  }
  return sparsep_batch_commit(b);
}

// Committed work items by kind: window items (x tile staged) and chunks of
// rows longer than one item.
int sparsep_batch_item_kinds(const sparsep_batch *b, uint64_t *window_items, uint64_t *chunk_items) {
  if (!b) return SPARSEP_EINVAL;
  uint64_t w = 0, c = 0;
  for (const BItem &it : b->items_h) {
    if (it.mode == MODE_LONG) ++c;
    else if (it.cw) ++w;
  }
  if (window_items) *window_items = w;
  if (chunk_items) *chunk_items = c;
  return SPARSEP_OK;
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
