// plan.cu -- plans (device-resident matrix + work items), execution and the
// per-dtype C-ABI entry points of sparsep_b200.
//
// A plan is the reference's "Load Matrix" phase done once: the reference
// partitions rows / nnz / blocks over NR_DPUS DPUs and NR_TASKLETS tasklets
// (support/partition.h) and scatters the pieces with dpu_push_xfer
// (spmv/1D/CSR-row/host/app.c:221-252).  Here the same partitions become CTA
// work items over one device copy of the matrix; nr_parts > 0 reproduces the
// reference split exactly (one part = one CTA, one tasklet = one warp) and
// nr_parts = 0 lets the planner size items for the GPU.
#include <algorithm>
#include <climits>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include <cuda.h>

#include "fault.hpp"
#include "internal.hpp"
#include "kernels.hpp"

using namespace sparsep;

// ---------------------------------------------------------------------------
// plan object
// ---------------------------------------------------------------------------
// Row bands of y for the host-buffer path (each >= BAND_MIN_BYTES of y).  Each
// band's wait and copy cost ~8 us on a B200 (32 bands of 4 MB: 249 us exposed),
// so few large bands win: 4 bands leave 37 us of a 4 MB copy after the kernel,
// 8 bands 62 us, one copy 84 us.
static constexpr uint32_t MAX_BANDS = 4;
static constexpr size_t BAND_MIN_BYTES = 512 * 1024;

struct sparsep_plan {
  int dtype = 0, format = 0, scheme = 0, nrhs = 1;
  size_t esize = 4;
  uint32_t nrows = 0, ncols = 0, V = 1;
  uint64_t nnz = 0, nblocks = 0;
  uint32_t rb = 1, cb = 1;
  int sms = 148, threads = 256;
  size_t smem = 0;
  int out_mode = OUT_DIRECT;
  uint32_t carry_w = 0;
  std::vector<void *> allocs;
  const uint32_t *rowptr = nullptr, *colind = nullptr, *bcolind = nullptr;
  const void *val = nullptr, *elems = nullptr, *bval = nullptr;
  const sparsep_bind *bind = nullptr;
  Item *items = nullptr;
  uint32_t nitems = 0;
  void *xpad = nullptr, *y = nullptr, *part = nullptr;
  unsigned long long *carry_val = nullptr, *carry_idx = nullptr;
  unsigned int *done = nullptr;
  int *err = nullptr;
  int *h_err = nullptr;  // pinned host copy of the error word (host-buffer path)
  // Host-buffer path: y goes back in row bands, each copied as soon as the
  // kernel has finished the items writing it (nbands = 0: one copy at the end).
  uint32_t nbands = 0;
  uint32_t band_row[MAX_BANDS + 1] = {};  // band b = rows [band_row[b], band_row[b+1])
  uint32_t band_items[MAX_BANDS] = {};    // items of band b: the count its copy waits for
  unsigned int *band_cnt = nullptr;       // device counters: items finished, over all host calls
  uint32_t band_calls = 0;                // host calls whose kernel was launched (mod 2^32)
  cudaStream_t copy_stream = nullptr;
  unsigned int *row_cnt = nullptr;  // long-row arrival counters (pipelined CSR)
  uint64_t n_rowptr = 0, n_idx = 0, n_val = 0, n_elems = 0;  // allocated extents
  bool stage = false;
  bool pipe = false;  // 1D CSR auto items run on the pipelined persistent kernel
  int pipe_grid = 0;
  uint32_t max_item_nnz = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[5] = {};
  double t[5] = {0, 0, 0, 0, 0};
  sparsep_plan_info info{};
  // Split 1D CSR plan (csr_stripes.cu): rows with >= `threshold` nonzeros (the
  // heavy rows) run stripe-major in column stripes of W columns; rowptr,
  // colind and val above hold the other rows (the heavy ones empty).  One
  // persistent kernel runs both, then a merge kernel sums the heavy rows'
  // stripe partials into y.
  struct Split {
    bool on = false;
    uint32_t threshold = 0, nH = 0, nS = 0, W = 0, ctas = 0, nchunks = 0;
    uint64_t nnz = 0;  // heavy nonzeros
    const uint32_t *hrow = nullptr, *vptr = nullptr, *cta_first = nullptr;
    const uint16_t *hcol = nullptr, *wsplit = nullptr;
    const void *hval = nullptr;
    const StripeChunk *chunks = nullptr;
    void *part = nullptr;
    uint64_t n_vptr = 0, n_h = 0, n_lptr = 0, n_l = 0, n_part = 0;
  } split;
  // nrhs > 1 (1D CSR, FP32 / INT32): the plan wraps a one-matrix batch, whose
  // row routines read each nonzero's k right-hand sides together
  sparsep_batch *batch = nullptr;
};

static thread_local char g_last_error[256] = "";

namespace sparsep {
void note_variant(sparsep_plan *p, const char *name, int mode) {
  if (!p || !name) return;
  if (mode == 0) std::snprintf(p->info.variant, sizeof p->info.variant, "%s", name);
  else std::snprintf(p->info.variant, sizeof p->info.variant, "%s (%s)", name, mode == 1 ? "learned" : "autotuned");
}
}  // namespace sparsep

namespace sparsep {
void record_error(const char *msg) { std::snprintf(g_last_error, sizeof g_last_error, "%s", msg); }
}  // namespace sparsep

static int map_cuda(cudaError_t e) {
  if (e != cudaSuccess) std::snprintf(g_last_error, sizeof g_last_error, "%s (%d)", cudaGetErrorString(e), (int)e);
  switch (e) {
    case cudaSuccess: return SPARSEP_OK;
    case cudaErrorMemoryAllocation: return SPARSEP_ENOMEM;
    case cudaErrorNoDevice:
    case cudaErrorInsufficientDriver:
    case cudaErrorNoKernelImageForDevice:
    case cudaErrorInvalidDevice: return SPARSEP_ENODEV;
    default: return SPARSEP_EIO;
  }
}
#define CK(x)                                   \
  do {                                          \
    cudaError_t e_ = (x);                       \
    if (e_ != cudaSuccess) return map_cuda(e_); \
  } while (0)

static size_t dtype_size(int d) {
  static const size_t s[6] = {1, 2, 4, 8, 4, 8};
  return (d >= 0 && d < 6) ? s[d] : 0;
}

static int dalloc(sparsep_plan *p, size_t bytes, void **out) {
  void *d = nullptr;
  if (bytes == 0) bytes = 16;
  CK(dev_malloc((void **)&d, bytes));
  p->allocs.push_back(d);
  // on the plan's stream: finish_plan waits for it, so every later launch,
  // on any stream, sees the buffer complete
  cudaError_t e = cudaMemsetAsync(d, 0, bytes, p->stream);
  if (e != cudaSuccess) return map_cuda(e);
  *out = d;
  return SPARSEP_OK;
}

// Copy n elements of size es to a fresh device buffer with `pad` zero elements after.
static int upload(sparsep_plan *p, const void *h, size_t n, size_t es, size_t pad, const void **out) {
  void *d = nullptr;
  int st = dalloc(p, (n + pad) * es, &d);
  if (st) return st;
  if (n && h) CK(cudaMemcpyAsync(d, h, n * es, cudaMemcpyDefault, p->stream));  // host or device source
  p->info.device_bytes += (n + pad) * es;
  *out = d;
  return SPARSEP_OK;
}

static uint32_t pow2ceil(uint64_t v) {
  uint32_t p = 1;
  while (p < v && p < 32) p <<= 1;
  return p;
}

// Auto-planner sizes: one CTA of 256 threads takes ~4k nonzeros.  Row items
// hold at most 4096 - 16 nonzeros so that, after the 16-byte alignment of the
// staged copy, they fit the pipelined kernel's 4096 slots.
static constexpr uint64_t AUTO_ITEM_NNZ = 4080;
static constexpr uint64_t AUTO_ITEM_ROWS = 1024;
static constexpr uint64_t AUTO_LONG_CHUNK = 4096;
static constexpr uint64_t AUTO_ITEM_ELEMS = 4096;
static constexpr uint64_t AUTO_ITEM_ENTRIES = 8192;  // stored block entries per item
static constexpr size_t STAGE_AUTO_MAX = 96 * 1024;
static constexpr size_t STAGE_MAX = 200 * 1024;

struct Opts {
  sparsep_opts o;
  int lanes() const { return o.lanes; }
};

static int check_opts(const sparsep_opts *o) {
  if (!o) return SPARSEP_OK;
  if (o->nr_parts < 0 || o->nr_workers < 0 || o->nr_workers > 16) return SPARSEP_EINVAL;
  if (o->lanes != 0 && (o->lanes < 1 || o->lanes > 32 || (o->lanes & (o->lanes - 1)))) return SPARSEP_EINVAL;
  if (o->part_balance < 0 || o->part_balance > SPARSEP_BAL_NNZ_ELEM) return SPARSEP_EINVAL;
  if (o->worker_balance < 0 || o->worker_balance > SPARSEP_BAL_INTERLEAVE) return SPARSEP_EINVAL;
  if (o->sync < 0 || o->sync > SPARSEP_SYNC_CG) return SPARSEP_EINVAL;
  if (o->autotune < 0 || o->autotune > 2 || o->heavy_rows < -1) return SPARSEP_EINVAL;
  if (o->nrhs < 0) return SPARSEP_EINVAL;
  if (o->nrhs > 256) return SPARSEP_ENOSYS;
  return SPARSEP_OK;
}

// ---------------------------------------------------------------------------
// Item builders
// ---------------------------------------------------------------------------
struct Tile {
  uint64_t ptr_base = 0, nnz_base = 0;
  uint32_t row_off = 0, row_end = 0, col_off = 0, xw = 0, slot = 0;
};

static Item make_item(const Tile &t, uint16_t kind) {
  Item it;
  std::memset(&it, 0, sizeof it);
  it.ptr_base = t.ptr_base;
  it.nnz_base = t.nnz_base;
  it.row_off = t.row_off;
  it.row_end = t.row_end;
  it.col_off = t.col_off;
  it.xlo = t.col_off;
  it.xw = t.xw;
  it.slot = t.slot;
  it.kind = kind;
  it.worker_bal = SPARSEP_BAL_INTERLEAVE;
  return it;
}


// CSR rows [r0, r1) of a tile (local rowptr rp) -> items.  faithful: exactly one
// item; otherwise split by nnz, with rows longer than AUTO_ITEM_NNZ chunked
// into LONG items when allow_long.
static void csr_tile_items(std::vector<Item> &items, const Tile &t, const uint32_t *rp, uint64_t r0, uint64_t r1,
                           const sparsep_opts &o, bool faithful, bool allow_long) {
  // item size: <= AUTO_ITEM_NNZ nonzeros, or the option's target rounded to a
  // stage size (2048 or 4096) less the 16 slots of copy alignment
  const uint64_t ITEM_NNZ = (o.item_nnz > 0 && o.item_nnz <= 2048) ? 2032 : AUTO_ITEM_NNZ;
  const uint64_t ROWS_CAP = ITEM_NNZ <= 2032 ? 512 : AUTO_ITEM_ROWS;
  const uint64_t LONG_CHUNK = ITEM_NNZ <= 2032 ? 2048 : AUTO_LONG_CHUNK;
  auto emit = [&](uint64_t a, uint64_t b) {
    if (a >= b) return;
    Item it = make_item(t, ITEM_ROWS);
    it.a0 = a;
    it.a1 = b;
    it.n0 = t.nnz_base + rp[a];
    it.n1 = t.nnz_base + rp[b];
    // lanes = 0 selects the staged (stream) row kernel, a fixed L the vector kernel
    it.lanes = (uint16_t)o.lanes;
    it.worker_bal = o.worker_balance == SPARSEP_BAL_NNZ_ELEM || o.worker_balance == SPARSEP_BAL_BLOCK
                        ? SPARSEP_BAL_NNZ
                        : (uint32_t)o.worker_balance;
    items.push_back(it);
  };
  if (faithful) {
    emit(r0, r1);
    return;
  }
  uint64_t a = r0, acc = 0;
  for (uint64_t r = r0; r < r1; ++r) {
    uint64_t len = (uint64_t)rp[r + 1] - rp[r];
    if (allow_long && len > ITEM_NNZ) {
      emit(a, r);
      uint64_t nch = (len + LONG_CHUNK - 1) / LONG_CHUNK;
      const uint32_t first = (uint32_t)items.size();
      for (uint64_t c = 0; c < nch; ++c) {
        Item it = make_item(t, ITEM_LONG);
        it.a0 = t.nnz_base + rp[r] + c * LONG_CHUNK;
        it.a1 = std::min<uint64_t>(t.nnz_base + rp[r + 1], it.a0 + LONG_CHUNK);
        it.crow = (uint32_t)(t.row_off + r);
        it.chunk = (uint32_t)c;
        it.n0 = it.a0;
        it.n1 = it.a1;
        it.nchunk = (uint32_t)nch;
        it.first = first;  // cslot is numbered by number_long_rows()
        it.lanes = 32;
        items.push_back(it);
      }
      a = r + 1;
      acc = 0;
      continue;
    }
    if (r > a && (acc + len > ITEM_NNZ || r - a >= ROWS_CAP)) {
      emit(a, r);
      a = r;
      acc = 0;
    }
    acc += len;
  }
  emit(a, r1);
}

// Long-row arrival counters: one per long row, numbered in item order.
static void number_long_rows(std::vector<Item> &items) {
  uint32_t n = 0;
  for (Item &it : items)
    if (it.kind == ITEM_LONG) {
      if (it.chunk == 0) ++n;
      it.cslot = n - 1;
    }
}

// Element (COO) / block (BCOO) range [e0, e1) of a tile whose keys (rows or
// block rows) run over [k_lo, k_hi): split into items, each owning the keys
// from its first unit's key to the next item's first key.
template <typename KeyFn>
static void elem_tile_items(std::vector<Item> &items, const Tile &t, uint64_t e0, uint64_t e1, uint32_t k_lo,
                            uint32_t k_hi, const std::vector<uint64_t> &cuts_in, KeyFn key) {
  std::vector<uint64_t> cuts = cuts_in;  // boundaries inside (e0, e1), sorted
  std::vector<uint64_t> b;
  b.push_back(e0);
  for (uint64_t c : cuts)
    if (c > e0 && c < e1) b.push_back(c);
  b.push_back(e1);
  for (size_t i = 0; i + 1 < b.size(); ++i) {
    Item it = make_item(t, ITEM_ELEMS);
    it.a0 = b[i];
    it.a1 = b[i + 1];
    it.own0 = (i == 0) ? k_lo : (b[i] < e1 ? key(b[i]) : k_hi);
    it.own1 = (i + 2 == b.size()) ? k_hi : (b[i + 1] < e1 ? key(b[i + 1]) : k_hi);
    if (it.own1 < it.own0) it.own1 = it.own0;
    items.push_back(it);
  }
}

static std::vector<uint64_t> even_cuts(uint64_t e0, uint64_t e1, uint64_t per) {
  std::vector<uint64_t> c;
  if (per == 0) per = 1;
  for (uint64_t e = e0 + per; e < e1; e += per) c.push_back(e);
  return c;
}

// ---------------------------------------------------------------------------
// Row bands of the host-buffer path
// ---------------------------------------------------------------------------
// cuStreamWaitValue32 from the driver, looked up through the runtime (the
// library does not link libcuda); null when the driver does not offer it.
using WaitValue32 = CUresult (*)(CUstream, CUdeviceptr, cuuint32_t, unsigned int);
static WaitValue32 wait_value32() {
  static const WaitValue32 fn = [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuStreamWaitValue32", &f, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<WaitValue32>(f);
  }();
  return fn;
}

// Splits a 1D CSR item list into up to MAX_BANDS row bands of y: contiguous
// item ranges whose written rows (row items [a0, a1), long-row chunks their
// row) are disjoint and ordered.  A cut before item i is valid when no earlier
// item writes a row at or past the first row written by item i or any later
// item.  Sets each item's band and the plan's band rows / item counts.
static void set_bands(sparsep_plan *p, std::vector<Item> &items) {
  p->nbands = 0;
  const size_t ybytes = (size_t)p->nrows * p->esize, n = items.size();
  if (p->format != SPARSEP_FMT_CSR || p->scheme != SPARSEP_1D || p->out_mode != OUT_DIRECT || p->pipe || n < 2 ||
      ybytes < 2 * BAND_MIN_BYTES || !wait_value32())
    return;
  std::vector<uint64_t> pm(n), sm(n);  // prefix max of row ends, suffix min of row starts
  for (size_t i = 0; i < n; ++i) {
    const Item &it = items[i];
    uint64_t hi;
    if (it.kind == ITEM_ROWS) {
      sm[i] = (uint64_t)it.row_off + it.a0;
      hi = (uint64_t)it.row_off + it.a1;
    } else if (it.kind == ITEM_LONG) {
      sm[i] = it.crow;
      hi = (uint64_t)it.crow + 1;
    } else {
      return;
    }
    pm[i] = std::max(hi, i ? pm[i - 1] : 0);
  }
  for (size_t i = n - 1; i-- > 0;) sm[i] = std::min(sm[i], sm[i + 1]);
  const uint32_t want = (uint32_t)std::min<size_t>(MAX_BANDS, ybytes / BAND_MIN_BYTES);
  std::vector<size_t> cut{0};
  for (uint32_t k = 1; k < want; ++k) {
    size_t i = std::max(cut.back() + 1, (size_t)k * n / want);
    while (i < n && pm[i - 1] > sm[i]) ++i;
    if (i >= n) break;
    cut.push_back(i);
  }
  if (cut.size() < 2) return;
  cut.push_back(n);
  p->nbands = (uint32_t)cut.size() - 1;
  p->band_row[0] = 0;
  for (uint32_t b = 0; b < p->nbands; ++b) {
    p->band_items[b] = (uint32_t)(cut[b + 1] - cut[b]);
    for (size_t i = cut[b]; i < cut[b + 1]; ++i) items[i].band = b;
    p->band_row[b + 1] = b + 1 < p->nbands ? (uint32_t)sm[cut[b + 1]] : p->nrows;
  }
}

// ---------------------------------------------------------------------------
// Plan finalisation
// ---------------------------------------------------------------------------
static int finish_plan(sparsep_plan *p, std::vector<Item> &items, const sparsep_opts &o) {
  p->nitems = (uint32_t)items.size();
  set_bands(p, items);
  int st = upload(p, items.data(), items.size(), sizeof(Item), 0, (const void **)&p->items);
  if (st) return st;
  // x with >= 16 bytes of zero slack (bulk-copy alignment), y, partial slices
  size_t xpad_elems = (size_t)p->ncols + 64;
  st = dalloc(p, xpad_elems * p->esize, &p->xpad);
  if (st) return st;
  st = dalloc(p, ((size_t)p->nrows + 64) * p->esize, &p->y);
  if (st) return st;
  p->info.device_bytes += (xpad_elems + p->nrows + 64) * p->esize;
  if (p->out_mode == OUT_PARTIAL) {
    size_t b = (size_t)p->V * p->nrows * p->esize + 64;
    st = dalloc(p, b, &p->part);
    if (st) return st;
    p->info.scratch_bytes += b;
  }
  if (p->carry_w) {
    size_t n = (size_t)p->nitems * p->carry_w + 1;
    st = dalloc(p, n * 8, (void **)&p->carry_val);
    if (!st) st = dalloc(p, n * 8, (void **)&p->carry_idx);
    if (!st) st = dalloc(p, 16, (void **)&p->done);
    if (st) return st;
    p->info.scratch_bytes += n * 16 + 16;
  }
  st = dalloc(p, 16, (void **)&p->err);
  if (st) return st;
  CK(cudaHostAlloc((void **)&p->h_err, sizeof(int), cudaHostAllocDefault));
  if (p->nbands) {
    st = dalloc(p, MAX_BANDS * sizeof(unsigned int), (void **)&p->band_cnt);
    if (st) return st;
    CK(cudaStreamCreateWithFlags(&p->copy_stream, cudaStreamNonBlocking));
  }
  uint32_t nlong = 0;
  for (const Item &it : items) nlong += it.kind == ITEM_LONG && it.chunk == 0;
  if (nlong) {
    st = dalloc(p, (size_t)nlong * 4, (void **)&p->row_cnt);
    if (st) return st;
    p->info.scratch_bytes += (size_t)nlong * 4;
  }
  size_t smem = 0;
  for (const Item &it : items) {
    if (it.xw) {
      size_t b = (size_t)it.xw * p->esize + 32;
      smem = std::max(smem, (b + 15) & ~(size_t)15);
      p->stage = true;
    }
  }
  p->smem = smem;
  int workers = o.nr_workers > 0 ? o.nr_workers : 8;
  p->threads = 32 * workers;
  for (auto &e : p->ev) CK(cudaEventCreate(&e));
  p->info.dtype = p->dtype;
  p->info.format = p->format;
  p->info.scheme = p->scheme;
  p->info.nrhs = p->nrhs;
  p->info.nrows = p->nrows;
  p->info.ncols = p->ncols;
  p->info.nnz = p->nnz;
  p->info.nblocks = p->nblocks;
  p->info.items = p->nitems;
  p->info.device_bytes += p->info.scratch_bytes;
  p->info.kernel_launches = p->split.on ? 2 : 1 + (p->out_mode == OUT_PARTIAL ? 1 : 0);
  p->info.workers = workers;
  p->info.stage_x = p->stage ? 1 : 0;
  p->info.y_bands = (int32_t)p->nbands;
  int lanes_min = 64, lanes_max = -1;  // over row items; 0 = staged stream kernel
  for (const Item &it : items)
    if (it.kind == ITEM_ROWS) {
      lanes_min = std::min<int>(lanes_min, it.lanes);
      lanes_max = std::max<int>(lanes_max, it.lanes);
    }
  p->info.lanes = lanes_max < 0 ? 0 : (lanes_min == lanes_max ? lanes_min : -1);
  static const char *fm[] = {"csr", "coo", "bcsr", "bcoo"};
  static const char *sc[] = {"1d", "2d-d", "2d-rbd", "2d-bd"};
  static const char *sy[] = {"lf", "atomic", "atomic(cg)"};
  const std::string split =
      p->split.on ? "/heavy>=" + std::to_string(p->split.threshold) + "x" + std::to_string(p->split.nS) + "stripes"
                  : std::string();
  std::snprintf(p->info.variant, sizeof p->info.variant, "%s/%s/%s/parts=%d/lanes=%s/V=%u%s%s%s", fm[p->format],
                sc[p->scheme], sy[o.sync], o.nr_parts, o.lanes ? std::to_string(o.lanes).c_str() : "auto", p->V,
                p->stage ? "/smem-x" : "", p->pipe ? "/tma-pipe" : "", split.c_str());
  // the uploads and clears above ran on the plan's stream: done before any
  // launch, on any stream, can read them
  CK(cudaStreamSynchronize(p->stream));
  return SPARSEP_OK;
}

static int begin_plan(sparsep_plan **out, int dtype, int format, int scheme, const sparsep_opts *o,
                      sparsep_plan **pp, sparsep_opts &oo) {
  if (!out) return SPARSEP_EINVAL;
  *out = nullptr;
  int st = check_opts(o);
  if (st) return st;
  if (o) oo = *o;
  else sparsep_opts_default(&oo);
  if (oo.autotune) return SPARSEP_ENOSYS;  // plan variants start from a host CSR (plan_csr)
  // several right-hand sides: 1D CSR in FP32 / INT32 with automatic items
  if (oo.nrhs > 1 && !(format == SPARSEP_FMT_CSR && scheme == SPARSEP_1D &&
                       (dtype == SPARSEP_FP32 || dtype == SPARSEP_INT32) && oo.nr_parts == 0))
    return SPARSEP_ENOSYS;
  int dev = 0;
  CK(cudaGetDevice(&dev));
  auto *p = new (std::nothrow) sparsep_plan();
  if (!p) return SPARSEP_ENOMEM;
  if (cudaError_t e = cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking)) {
    delete p;
    return map_cuda(e);
  }
  CK(cudaDeviceGetAttribute(&p->sms, cudaDevAttrMultiProcessorCount, dev));
  p->dtype = dtype;
  p->format = format;
  p->scheme = scheme;
  p->esize = dtype_size(dtype);
  p->nrhs = 1;
  p->out_mode = OUT_DIRECT;
  *pp = p;
  return SPARSEP_OK;
}

static int stage_width(const sparsep_plan *p, const sparsep_opts &o, uint32_t w) {
  size_t bytes = (size_t)w * p->esize + 32;
  if (o.stage_x == 0 || w == 0) return 0;
  if (o.stage_x > 0) return bytes <= STAGE_MAX ? (int)w : 0;
  return bytes <= STAGE_AUTO_MAX ? (int)w : 0;
}

static uint64_t compulsory_csr(uint64_t nnz, uint64_t nrows, uint64_t ncols, size_t s) {
  return nnz * (4 + s) + (nrows + 1) * 4 + ncols * s + nrows * s;
}

// Output mode of a V-stripe scheme.
static void set_out_mode(sparsep_plan *p, const sparsep_opts &o, uint32_t V, bool has_carries, uint32_t carry_w) {
  p->V = V;
  if (o.sync == SPARSEP_SYNC_ATOMIC || o.sync == SPARSEP_SYNC_CG) {
    p->out_mode = OUT_ATOMIC;
    p->carry_w = 0;
  } else {
    p->out_mode = V > 1 ? OUT_PARTIAL : OUT_DIRECT;
    p->carry_w = has_carries ? carry_w : 0;
  }
}

// ---------------------------------------------------------------------------
// Split CSR plans: heavy rows in column stripes (csr_stripes.cu)
// ---------------------------------------------------------------------------
// Cost model of the planner's choice, in bytes of HBM streaming: a random x
// gather through L2 costs about GATHER_BYTES (on a B200, 16.7 M gathers of a
// 4 MB x take as long as streaming ~25 bytes each); a heavy nonzero costs its
// 2-byte stripe column and value (its x is read from shared memory); each
// stripe row costs its offset, its partial's store and the merge's read.
static constexpr uint64_t GATHER_BYTES = 24;
static constexpr uint64_t SPLIT_MIN_X_BYTES = 1 << 20;  // smaller x: gathers mostly hit L1
// The planner chooses a split on its own only once the split path is measured
// faster than the row kernel alone; until then heavy_rows > 0 requests it.
static constexpr bool SPLIT_AUTO = false;

static bool split_eligible(const sparsep_opts &o, uint64_t nnz) {
  return o.heavy_rows >= 0 && o.lanes == 0 && o.pipeline != 1 && o.sync == SPARSEP_SYNC_LF && o.nrhs <= 1 &&
         nnz < (1ull << 31);
}

// Heavy-row threshold for a split plan, 0 for none.
static uint32_t split_threshold(const sparsep_opts &o, const uint32_t *rp, uint32_t nrows, uint32_t ncols, size_t s,
                                uint32_t W) {
  if (o.heavy_rows > 0) return (uint32_t)o.heavy_rows;
  if (!SPLIT_AUTO || (uint64_t)ncols * s < SPLIT_MIN_X_BYTES || nrows == 0) return 0;
  const uint64_t nS = (ncols + (uint64_t)W - 1) / W, nnz = rp[nrows];
  // candidates: about 1, 2, 4, 8 nonzeros per stripe row on average
  uint64_t cand[4], nH[4] = {0, 0, 0, 0}, nnzH[4] = {0, 0, 0, 0};
  for (int i = 0; i < 4; ++i) cand[i] = std::max<uint64_t>(8, nS << i);
  for (uint32_t r = 0; r < nrows; ++r) {
    const uint64_t len = rp[r + 1] - rp[r];
    for (int i = 0; i < 4; ++i)
      if (len >= cand[i]) {
        ++nH[i];
        nnzH[i] += len;
      }
  }
  const uint64_t per_light = 4 + s + GATHER_BYTES;
  const uint64_t none = per_light * nnz;
  uint64_t best = none;
  uint32_t thr = 0;
  for (int i = 0; i < 4; ++i) {
    if (nH[i] == 0) continue;
    const uint64_t c = (2 + s) * nnzH[i] + (4 + 2 * s) * nS * nH[i] + per_light * (nnz - nnzH[i]);
    if (c < best) {
      best = c;
      thr = (uint32_t)cand[i];
    }
  }
  return best * 5 < none * 4 ? thr : 0;  // at least 20% less modelled traffic
}

// Chunks of one CSR-like array set: rows [0, nrows) of offsets `ptr`, cut at
// `cap` nonzeros or `rcap` rows (and at stripe boundaries: rows v with
// v / stripe_rows different); a row longer than `cap` becomes a run of pieces.
static void cut_chunks(std::vector<StripeChunk> &ch, const std::vector<uint32_t> &ptr, uint64_t nrows, uint32_t cap,
                       uint32_t rcap, uint64_t stripe_rows, bool light) {
  StripeChunk c{};
  bool open = false;
  auto close = [&]() {
    if (open) ch.push_back(c);
    open = false;
  };
  for (uint64_t v = 0; v < nrows; ++v) {
    const uint32_t s = light ? STRIPE_LIGHT : (uint32_t)(v / stripe_rows), a = ptr[v], b = ptr[v + 1];
    if (b - a > cap) {
      close();
      for (uint32_t o = a; o < b; o += cap) {
        StripeChunk q{};
        q.n0 = o;
        q.n1 = std::min<uint32_t>(b, o + cap);
        q.v0 = (uint32_t)v;
        q.v1 = (uint32_t)v + 1;
        q.stripe = s;
        q.piece = 4u | (o == a ? 1u : 0u) | (q.n1 == b ? 2u : 0u);
        ch.push_back(q);
      }
      continue;
    }
    if (open && (c.stripe != s || c.n1 - c.n0 + (b - a) > cap || c.v1 - c.v0 >= rcap)) close();
    if (!open) {
      c = StripeChunk{};
      c.n0 = c.n1 = a;
      c.v0 = c.v1 = (uint32_t)v;
      c.stripe = s;
      open = true;
    }
    c.n1 = b;
    c.v1 = (uint32_t)v + 1;
  }
  close();
}

// Cuts a chunk list into C contiguous ranges of about equal cost (nonzeros
// times `per_nnz`, plus rows and a fixed cost per chunk); pieces of one row
// stay in one range.  Returns C + 1 boundaries.
static std::vector<uint32_t> cost_ranges(const std::vector<StripeChunk> &ch, uint32_t C, uint64_t per_nnz) {
  const uint32_t n = (uint32_t)ch.size();
  std::vector<uint64_t> pre(n + 1, 0);
  for (uint32_t i = 0; i < n; ++i)
    pre[i + 1] = pre[i] + per_nnz * (ch[i].n1 - ch[i].n0) + 2ull * (ch[i].v1 - ch[i].v0) + 256;
  std::vector<uint32_t> first(C + 1, 0);
  for (uint32_t b = 1; b < C; ++b) {
    uint32_t i = (uint32_t)(std::lower_bound(pre.begin(), pre.end(), pre[n] * b / C) - pre.begin());
    i = std::max(i, first[b - 1]);
    while (i < n && ch[i].piece && !(ch[i].piece & 1u)) ++i;
    first[b] = std::min(i, n);
  }
  first[C] = n;
  return first;
}

// Builds a split plan's device arrays: the heavy rows (length >= thr) laid out
// stripe-major, the light rows as a CSR (heavy rows empty), and per CTA one
// chunk list interleaving its share of both.  Leaves p->split.on false when no
// row is heavy or the stripe rows would outnumber the nonzeros.
template <typename T>
static int build_split(sparsep_plan *p, const typename Types<T>::csr *A, uint32_t thr) {
  uint32_t W = 0, cap = 0, cap_l = 0, rcap = 0;
  stripe_geometry<T>(&W, nullptr, &cap, &cap_l, &rcap);
  const uint32_t n = A->nrows;
  const uint32_t *rp = A->rowptr;
  std::vector<uint32_t> heavy;
  for (uint32_t r = 0; r < n; ++r)
    if (rp[r + 1] - rp[r] >= thr) heavy.push_back(r);
  const uint64_t nH = heavy.size(), nS = ((uint64_t)A->ncols + W - 1) / W, V = nS * nH;
  if (nH == 0 || V >= (1ull << 31) || V > 2 * (uint64_t)A->nnz + (1u << 20)) return SPARSEP_OK;
  std::vector<uint32_t> vptr, cur, lptr, lcol;
  std::vector<uint16_t> hcol;
  std::vector<T> hval, lval;
  std::vector<StripeChunk> hch, lch, ch;
  try {
    // heavy rows, stripe-major (counting sort of each row's nonzeros by stripe)
    vptr.assign(V + 1 + 8, 0);
    for (uint64_t k = 0; k < nH; ++k) {
      const uint32_t r = heavy[k];
      for (uint32_t j = rp[r]; j < rp[r + 1]; ++j) ++vptr[(uint64_t)(A->colind[j] / W) * nH + k + 1];
    }
    for (uint64_t v = 0; v < V; ++v) vptr[v + 1] += vptr[v];
    const uint64_t nnzH = vptr[V];
    for (uint64_t v = V + 1; v < vptr.size(); ++v) vptr[v] = (uint32_t)nnzH;
    hcol.assign(nnzH + 32, 0);
    hval.assign(nnzH + 32, T(0));
    cur.assign(vptr.begin(), vptr.begin() + V);
    for (uint64_t k = 0; k < nH; ++k) {
      const uint32_t r = heavy[k];
      for (uint32_t j = rp[r]; j < rp[r + 1]; ++j) {
        const uint32_t c = A->colind[j], s = c / W;
        const uint32_t pos = cur[(uint64_t)s * nH + k]++;
        hcol[pos] = (uint16_t)(c - s * W);
        hval[pos] = A->values[j];
      }
    }
    // light rows, a CSR over all rows with the heavy ones empty
    const uint64_t nnzL = (uint64_t)A->nnz - nnzH;
    lptr.assign((size_t)n + 1 + 8, 0);
    lcol.reserve(nnzL + 32);
    lval.reserve(nnzL + 32);
    for (uint32_t r = 0; r < n; ++r) {
      if (rp[r + 1] - rp[r] < thr)
        for (uint32_t j = rp[r]; j < rp[r + 1]; ++j) {
          lcol.push_back(A->colind[j]);
          lval.push_back(A->values[j]);
        }
      lptr[r + 1] = (uint32_t)lcol.size();
    }
    for (size_t i = (size_t)n + 1; i < lptr.size(); ++i) lptr[i] = (uint32_t)nnzL;
    lcol.resize(nnzL + 32, 0);
    lval.resize(nnzL + 32, T(0));
    cut_chunks(hch, vptr, V, cap, rcap, nH, false);
    cut_chunks(lch, lptr, n, cap_l, rcap, 1, true);
  } catch (const std::bad_alloc &) {
    return SPARSEP_ENOMEM;
  }
  // per CTA (one per SM): a contiguous share of the heavy chunks and one of the
  // light chunks, interleaved by progress through each share, so that light
  // gathers and heavy streaming overlap on every SM
  const uint32_t C = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)p->sms, hch.size() + lch.size()));
  const std::vector<uint32_t> fh = cost_ranges(hch, C, 1), fl = cost_ranges(lch, C, 3);
  std::vector<uint32_t> first(C + 1, 0);
  try {
    ch.reserve(hch.size() + lch.size());
    for (uint32_t b = 0; b < C; ++b) {
      first[b] = (uint32_t)ch.size();
      const uint64_t th = fh[b + 1] - fh[b], tl = fl[b + 1] - fl[b];
      uint32_t i = fh[b], j = fl[b];
      while (i < fh[b + 1] || j < fl[b + 1]) {
        const bool h = j >= fl[b + 1] || (i < fh[b + 1] && (uint64_t)(i - fh[b]) * tl <= (uint64_t)(j - fl[b]) * th);
        ch.push_back(h ? hch[i++] : lch[j++]);
      }
    }
    first[C] = (uint32_t)ch.size();
  } catch (const std::bad_alloc &) {
    return SPARSEP_ENOMEM;
  }
  // each chunk's rows split over the consumer warps: warp w takes the rows
  // whose first nonzero lies in [n*w/NW, n*(w+1)/NW) of the chunk's n nonzeros
  constexpr uint32_t NW = SPLIT_WARPS;
  std::vector<uint16_t> wsplit;
  try {
    wsplit.assign(ch.size() * (NW + 1), 0);
  } catch (const std::bad_alloc &) {
    return SPARSEP_ENOMEM;
  }
  for (size_t i = 0; i < ch.size(); ++i) {
    const StripeChunk &c = ch[i];
    uint16_t *w = wsplit.data() + i * (NW + 1);
    const uint32_t nr = c.v1 - c.v0, nn = c.n1 - c.n0;
    w[NW] = (uint16_t)nr;
    if (c.piece) continue;
    const uint32_t *pt = (c.stripe == STRIPE_LIGHT ? lptr.data() : vptr.data()) + c.v0;
    uint32_t r = 0;
    for (uint32_t q = 1; q < NW; ++q) {
      const uint32_t t = (uint32_t)((uint64_t)nn * q / NW);
      while (r < nr && pt[r] - c.n0 < t) ++r;
      w[q] = (uint16_t)r;
    }
  }
  auto &S = p->split;
  int st;
  if ((st = upload(p, wsplit.data(), wsplit.size(), 2, 0, (const void **)&S.wsplit))) return st;
  if ((st = upload(p, heavy.data(), nH, 4, 0, (const void **)&S.hrow))) return st;
  if ((st = upload(p, vptr.data(), vptr.size(), 4, 0, (const void **)&S.vptr))) return st;
  if ((st = upload(p, hcol.data(), hcol.size(), 2, 0, (const void **)&S.hcol))) return st;
  if ((st = upload(p, hval.data(), hval.size(), sizeof(T), 0, &S.hval))) return st;
  if ((st = upload(p, lptr.data(), lptr.size(), 4, 0, (const void **)&p->rowptr))) return st;
  if ((st = upload(p, lcol.data(), lcol.size(), 4, 0, (const void **)&p->colind))) return st;
  if ((st = upload(p, lval.data(), lval.size(), sizeof(T), 0, &p->val))) return st;
  if ((st = upload(p, ch.data(), ch.size(), sizeof(StripeChunk), 0, (const void **)&S.chunks))) return st;
  if ((st = upload(p, first.data(), first.size(), 4, 0, (const void **)&S.cta_first))) return st;
  if ((st = dalloc(p, (V + 8) * sizeof(T), &S.part))) return st;
  p->info.scratch_bytes += (V + 8) * sizeof(T);
  S.on = true;
  S.threshold = thr;
  S.nH = (uint32_t)nH;
  S.nS = (uint32_t)nS;
  S.W = W;
  S.ctas = C;
  S.nchunks = (uint32_t)ch.size();
  S.nnz = vptr[V];
  S.n_vptr = vptr.size();
  S.n_h = hcol.size();
  S.n_lptr = lptr.size();
  S.n_l = lcol.size();
  S.n_part = V;
  return SPARSEP_OK;
}

// ---------------------------------------------------------------------------
// Several right-hand sides on one plan: x is ncols x k and y nrows x k, both
// row-major (one nonzero's k right-hand sides contiguous).  The plan wraps a
// batch of this one matrix, whose work items read the k values of x a nonzero
// needs with one load per lane group (the batch's row routines, default
// variant for k).
// ---------------------------------------------------------------------------
template <typename T>
static int plan_multi_rhs(sparsep_plan *p, const typename Types<T>::csr *A, uint32_t k) {
  const typename Types<T>::csr *mats[1] = {A};
  int st;
  if constexpr (std::is_same<T, float>::value) st = sparsep_batch_create_f32(1, mats, &k, nullptr, &p->batch);
  else st = sparsep_batch_create_i32(1, mats, &k, nullptr, &p->batch);
  if (st) return st;
  if ((st = sparsep_batch_x(p->batch, 0, &p->xpad, &p->y))) return st;  // the batch owns them
  uint64_t cb = 0, items = 0, nnz = 0;
  sparsep_batch_get_info(p->batch, &cb, &items, &nnz);
  p->nrhs = (int)k;
  p->info.dtype = p->dtype;
  p->info.format = SPARSEP_FMT_CSR;
  p->info.scheme = SPARSEP_1D;
  p->info.nrhs = (int32_t)k;
  p->info.nrows = p->nrows;
  p->info.ncols = p->ncols;
  p->info.nnz = p->nnz;
  p->info.items = items;
  p->info.compulsory_bytes = cb;
  p->info.kernel_launches = 1;
  sparsep_batch_variant v{};
  sparsep_batch_get_variant(p->batch, 0, &v);
  std::snprintf(p->info.variant, sizeof p->info.variant, "csr/1d/rows x %u rhs/%s/lanes=%d/vec=%d", k,
                v.mode ? "merge" : "rows", v.lanes, v.vec);
  for (auto &e : p->ev) CK(cudaEventCreate(&e));
  return SPARSEP_OK;
}

// ---------------------------------------------------------------------------
// CSR
// ---------------------------------------------------------------------------
template <typename T>
static int plan_csr(const typename Types<T>::csr *A, const sparsep_opts *o, sparsep_plan **out,
                    bool device_arrays = false) {
  if (o && o->autotune) {  // one of the plan variants, timed or learned (autotune.cu)
    if (!out) return SPARSEP_EINVAL;
    *out = nullptr;
    if (int st = check_opts(o)) return st;
    if (device_arrays || o->nrhs > 1) return SPARSEP_ENOSYS;
    if (!A || (A->nrows && !A->rowptr) || (A->nnz && (!A->colind || !A->values))) return SPARSEP_EINVAL;
    if (A->rowptr[0] != 0 || A->rowptr[A->nrows] != A->nnz) return SPARSEP_EINVAL;
    return plan_autotuned<T>(A, *o, out);
  }
  sparsep_plan *p = nullptr;
  sparsep_opts oo;
  int st = begin_plan(out, Types<T>::dtype, SPARSEP_FMT_CSR, SPARSEP_1D, o, &p, oo);
  if (st) return st;
  auto t0 = std::chrono::steady_clock::now();
  std::unique_ptr<sparsep_plan, void (*)(sparsep_plan *)> guard(p, sparsep_plan_free);
  if (!A || (A->nrows && !A->rowptr) || (A->nnz && (!A->colind || !A->values))) return SPARSEP_EINVAL;
  if (A->rowptr[0] != 0 || A->rowptr[A->nrows] != A->nnz) return SPARSEP_EINVAL;
  for (uint32_t r = 0; r < A->nrows; ++r)
    if (A->rowptr[r + 1] < A->rowptr[r]) return SPARSEP_EINVAL;
  if (!device_arrays)  // device column indices are checked on the device by the caller
    for (uint32_t k = 0; k < A->nnz; ++k)
      if (A->colind[k] >= A->ncols) return SPARSEP_EINVAL;
  p->nrows = A->nrows;
  p->ncols = A->ncols;
  p->nnz = A->nnz;
  if (oo.nrhs > 1) {
    if (device_arrays) return SPARSEP_ENOSYS;  // the batch reads the host arrays
    if constexpr (std::is_same<T, float>::value || std::is_same<T, int32_t>::value) {
      if ((st = plan_multi_rhs<T>(p, A, (uint32_t)oo.nrhs))) return st;
      p->t[0] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
      *out = guard.release();
      return SPARSEP_OK;
    }
    return SPARSEP_ENOSYS;
  }
  std::vector<Item> items;
  Tile t;
  t.row_end = A->nrows;
  const bool faithful = oo.nr_parts > 0;
  bool has_long = false;
  if (faithful) {
    std::vector<uint32_t> split(oo.nr_parts + 2);
    if (oo.part_balance == SPARSEP_BAL_ROW) sparsep_partition_by_row(A->nrows, oo.nr_parts, split.data());
    else sparsep_partition_by_nnz(A->rowptr, A->nrows, oo.nr_parts, split.data());
    for (int i = 0; i < oo.nr_parts; ++i) csr_tile_items(items, t, A->rowptr, split[i], split[i + 1], oo, true, false);
  } else {
    // a split plan when the heavy rows' x gathers are worth moving into
    // shared-memory stripes (host arrays only: the re-layout reads columns)
    if (!device_arrays && split_eligible(oo, A->nnz)) {
      uint32_t W = 0;
      stripe_geometry<T>(&W, nullptr, nullptr, nullptr, nullptr);
      const uint32_t thr = split_threshold(oo, A->rowptr, A->nrows, A->ncols, sizeof(T), W);
      if (thr && (st = build_split<T>(p, A, thr))) return st;
      if (p->split.on) {  // no row items: one persistent kernel runs both parts
        set_out_mode(p, oo, 1, false, 1);
        p->info.compulsory_bytes = compulsory_csr(A->nnz, A->nrows, A->ncols, sizeof(T));
        if ((st = finish_plan(p, items, oo))) return st;
        p->t[0] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        *out = guard.release();
        return SPARSEP_OK;
      }
    }
    csr_tile_items(items, t, A->rowptr, 0, A->nrows, oo, false, true);
    number_long_rows(items);
    for (auto &it : items) has_long |= it.kind == ITEM_LONG;
  }
  set_out_mode(p, oo, 1, has_long, 1);
  p->pipe = !faithful && oo.lanes == 0 && p->out_mode == OUT_DIRECT && oo.pipeline == 1;
  for (const Item &it : items) p->max_item_nnz = std::max<uint32_t>(p->max_item_nnz, (uint32_t)(it.n1 - it.n0));
  if ((st = upload(p, A->rowptr, (size_t)A->nrows + 1, 4, 16, (const void **)&p->rowptr))) return st;
  if ((st = upload(p, A->colind, A->nnz, 4, 16, (const void **)&p->colind))) return st;
  if ((st = upload(p, A->values, A->nnz, sizeof(T), 16, &p->val))) return st;
  p->n_rowptr = (uint64_t)A->nrows + 17;
  p->n_idx = p->n_val = (uint64_t)A->nnz + 16;
  p->info.compulsory_bytes = compulsory_csr(A->nnz, A->nrows, A->ncols, sizeof(T));
  if ((st = finish_plan(p, items, oo))) return st;
  p->t[0] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  *out = guard.release();
  return SPARSEP_OK;
}

// 2D CSR tiles.  D: tile (h, c) has a local rowptr of tile_height+1 entries at
// p*(tile_height+1) (spmv/2D/DCSR/support/matrix.h:190-205).  RBD/BD: stripe c
// has a full-height rowptr at c*(nrows+1) split into H nnz-balanced row ranges
// (partition_by_nnz, spmv/2D/BDCSR/support/partition.h:47-91).
template <typename T>
static int plan_csr_tiles(int scheme, uint32_t nrows, uint32_t ncols, uint64_t nnz, uint32_t H, uint32_t V,
                          const uint32_t *drowptr, size_t rowptr_len, const uint32_t *dcolind, const T *dval,
                          const std::vector<Tile> &tiles_in, const std::vector<std::pair<uint64_t, uint64_t>> &ranges,
                          const sparsep_opts *o, sparsep_plan **out) {
  sparsep_plan *p = nullptr;
  sparsep_opts oo;
  int st = begin_plan(out, Types<T>::dtype, SPARSEP_FMT_CSR, scheme, o, &p, oo);
  if (st) return st;
  auto t0 = std::chrono::steady_clock::now();
  std::unique_ptr<sparsep_plan, void (*)(sparsep_plan *)> guard(p, sparsep_plan_free);
  p->nrows = nrows;
  p->ncols = ncols;
  p->nnz = nnz;
  std::vector<Item> items;
  const bool faithful = oo.nr_parts > 0;
  for (size_t i = 0; i < tiles_in.size(); ++i) {
    Tile t = tiles_in[i];
    t.xw = stage_width(p, oo, t.xw);
    csr_tile_items(items, t, drowptr + t.ptr_base, ranges[i].first, ranges[i].second, oo, faithful, false);
  }
  (void)H;
  set_out_mode(p, oo, V, false, 1);
  if ((st = upload(p, drowptr, rowptr_len, 4, 16, (const void **)&p->rowptr))) return st;
  if ((st = upload(p, dcolind, nnz, 4, 16, (const void **)&p->colind))) return st;
  if ((st = upload(p, dval, nnz, sizeof(T), 16, &p->val))) return st;
  p->n_rowptr = rowptr_len + 16;
  p->n_idx = p->n_val = nnz + 16;
  p->info.compulsory_bytes = compulsory_csr(nnz, nrows, ncols, sizeof(T));
  if ((st = finish_plan(p, items, oo))) return st;
  p->t[0] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  *out = guard.release();
  return SPARSEP_OK;
}

// per-stripe H row ranges of a full-height stripe CSR (RBD / BD)
static std::vector<uint32_t> stripe_row_split(const uint32_t *rp, uint32_t nrows, uint32_t H) {
  std::vector<uint32_t> s(H + 2);
  std::vector<uint64_t> pre(rp, rp + nrows + 1);
  greedy_split(pre.data(), nrows, H, s.data());
  return s;
}

template <typename T>
static int plan_dcsr(const typename Types<T>::dcsr *A, const sparsep_opts *o, sparsep_plan **out) {
  if (!A || !A->horz_partitions || !A->vert_partitions || !A->tile_height || !A->tile_width) return SPARSEP_EINVAL;
  const uint32_t H = A->horz_partitions, V = A->vert_partitions, th = A->tile_height, tw = A->tile_width;
  std::vector<Tile> tiles;
  std::vector<std::pair<uint64_t, uint64_t>> ranges;
  uint64_t base = 0;
  for (uint32_t h = 0; h < H; ++h)
    for (uint32_t c = 0; c < V; ++c) {
      uint64_t pidx = (uint64_t)h * V + c;
      Tile t;
      t.ptr_base = pidx * (th + 1);
      t.nnz_base = base;
      t.row_off = h * th;
      uint32_t rows = t.row_off >= A->nrows ? 0 : std::min(th, A->nrows - t.row_off);
      t.row_end = t.row_off + rows;
      t.col_off = c * tw;
      t.xw = t.col_off >= A->ncols ? 0 : std::min(tw, A->ncols - t.col_off);
      t.slot = c;
      base += A->nnzs_per_partition[pidx];
      if (A->drowptr[t.ptr_base + th] != A->nnzs_per_partition[pidx]) return SPARSEP_EINVAL;
      tiles.push_back(t);
      ranges.push_back({0, rows});
    }
  if (base != A->nnz) return SPARSEP_EINVAL;
  for (uint64_t k = 0; k < A->nnz; ++k)
    if (A->dcolind[k] >= tw) return SPARSEP_EINVAL;
  return plan_csr_tiles<T>(SPARSEP_2D_EQUAL, A->nrows, A->ncols, A->nnz, H, V, A->drowptr,
                           (size_t)H * V * (th + 1) + 1, A->dcolind, A->dval, tiles, ranges, o, out);
}

template <typename T, typename S>
static int plan_stripes_csr(int scheme, const S *A, const uint32_t *widths, const sparsep_opts *o,
                            sparsep_plan **out) {
  const uint32_t H = A->horz_partitions, V = A->vert_partitions, nr = A->nrows;
  if (!H || !V) return SPARSEP_EINVAL;
  std::vector<Tile> tiles;
  std::vector<std::pair<uint64_t, uint64_t>> ranges;
  uint64_t base = 0;
  for (uint32_t c = 0; c < V; ++c) {
    const uint32_t *rp = A->drowptr + (size_t)c * (nr + 1);
    if (rp[nr] != A->nnzs_per_vert_partition[c]) return SPARSEP_EINVAL;
    auto split = stripe_row_split(rp, nr, H);
    for (uint32_t h = 0; h < H; ++h) {
      Tile t;
      t.ptr_base = (uint64_t)c * (nr + 1);
      t.nnz_base = base;
      t.row_off = 0;
      t.row_end = nr;
      t.col_off = widths[c];
      t.xw = widths[c + 1] > widths[c] ? widths[c + 1] - widths[c] : 0;
      t.slot = c;
      tiles.push_back(t);
      ranges.push_back({split[h], split[h + 1]});
    }
    for (uint64_t k = base; k < base + A->nnzs_per_vert_partition[c]; ++k)
      if (A->dcolind[k] >= std::max<uint32_t>(1, widths[c + 1] - widths[c])) return SPARSEP_EINVAL;
    base += A->nnzs_per_vert_partition[c];
  }
  if (base != A->nnz) return SPARSEP_EINVAL;
  return plan_csr_tiles<T>(scheme, A->nrows, A->ncols, A->nnz, H, V, A->drowptr, (size_t)V * (nr + 1) + 1,
                           A->dcolind, A->dval, tiles, ranges, o, out);
}

static std::vector<uint32_t> eq_widths(uint32_t ncols, uint32_t V, uint32_t tw) {
  std::vector<uint32_t> w(V + 1);
  for (uint32_t c = 0; c <= V; ++c) w[c] = (uint32_t)std::min<uint64_t>((uint64_t)c * tw, ncols);
  return w;
}

template <typename T>
static int plan_rbdcsr(const typename Types<T>::rbdcsr *A, const sparsep_opts *o, sparsep_plan **out) {
  if (!A || !A->vert_partitions || !A->tile_width) return SPARSEP_EINVAL;
  auto w = eq_widths(A->ncols, A->vert_partitions, A->tile_width);
  return plan_stripes_csr<T>(SPARSEP_2D_EQUAL_W, A, w.data(), o, out);
}

template <typename T>
static int plan_bdcsr(const typename Types<T>::bdcsr *A, const sparsep_opts *o, sparsep_plan **out) {
  if (!A || !A->vert_partitions || !A->vert_tile_widths) return SPARSEP_EINVAL;
  return plan_stripes_csr<T>(SPARSEP_2D_VAR, A, A->vert_tile_widths, o, out);
}

// ---------------------------------------------------------------------------
// COO (AoS elem_t, sorted by row)
// ---------------------------------------------------------------------------
struct ElemTile {
  Tile t;
  uint64_t e0, e1;
  uint32_t k_lo, k_hi;
  std::vector<uint64_t> cuts;  // faithful part boundaries inside [e0, e1)
};

template <typename T>
static int plan_elems(int fmt, int scheme, uint32_t nrows, uint32_t ncols, uint64_t nnz, uint64_t nunits,
                      uint32_t V, const void *elems, size_t elem_size, const std::vector<ElemTile> &tiles,
                      std::function<uint32_t(uint64_t)> key, uint64_t per_item, const sparsep_opts *o,
                      sparsep_plan **out, const typename Types<T>::bcoo *B = nullptr, uint32_t rb = 1,
                      uint32_t cb = 1) {
  sparsep_plan *p = nullptr;
  sparsep_opts oo;
  int st = begin_plan(out, Types<T>::dtype, fmt, scheme, o, &p, oo);
  if (st) return st;
  auto t0 = std::chrono::steady_clock::now();
  std::unique_ptr<sparsep_plan, void (*)(sparsep_plan *)> guard(p, sparsep_plan_free);
  p->nrows = nrows;
  p->ncols = ncols;
  p->nnz = nnz;
  p->rb = rb;
  p->cb = cb;
  std::vector<Item> items;
  const bool faithful = oo.nr_parts > 0;
  for (const ElemTile &et : tiles) {
    Tile t = et.t;
    t.xw = stage_width(p, oo, t.xw);
    std::vector<uint64_t> cuts = et.cuts;
    if (!faithful) cuts = even_cuts(et.e0, et.e1, per_item);
    elem_tile_items(items, t, et.e0, et.e1, et.k_lo, et.k_hi, cuts, key);
  }
  const uint32_t W = fmt == SPARSEP_FMT_BCOO ? rb : 1;
  set_out_mode(p, oo, V, true, W);
  if (fmt == SPARSEP_FMT_COO) {
    if ((st = upload(p, elems, nunits, elem_size, 8, &p->elems))) return st;
    p->n_elems = nunits + 8;
    p->info.compulsory_bytes = nnz * (8 + sizeof(T)) + (uint64_t)ncols * sizeof(T) + (uint64_t)nrows * sizeof(T);
  } else {
    p->nblocks = nunits;
    if ((st = upload(p, B->bind, nunits, sizeof(sparsep_bind), 4, (const void **)&p->bind))) return st;
    if ((st = upload(p, B->bval, nunits * rb * cb, sizeof(T), 16 * rb * cb, &p->bval))) return st;
    p->n_elems = nunits + 4;
    p->n_val = (nunits + 16) * rb * cb;
    p->info.compulsory_bytes = nunits * (8 + (uint64_t)rb * cb * sizeof(T)) + (uint64_t)ncols * sizeof(T) +
                               (uint64_t)nrows * sizeof(T);
  }
  if ((st = finish_plan(p, items, oo))) return st;
  p->t[0] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  *out = guard.release();
  return SPARSEP_OK;
}

// Part boundaries for element-wise formats with the reference's balance options.
// units [0, n) with keys key(u) (sorted); per-key unit counts via prefix.
static std::vector<uint64_t> faithful_elem_cuts(const sparsep_opts &o, uint64_t n, uint32_t nkeys,
                                                const std::vector<uint64_t> &key_prefix,
                                                const std::vector<uint64_t> &weight_prefix) {
  std::vector<uint64_t> cuts;
  uint32_t P = (uint32_t)o.nr_parts;
  if (o.part_balance == SPARSEP_BAL_NNZ_ELEM) {
    // equal units (COO-nnz, spmv/1D/COO-nnz/host/app.c:118-156) or, with weights,
    // the greedy nnz split at unit granularity (BCOO-nnz, spmv/1D/BCOO-nnz/support/partition.h:37-97)
    if (weight_prefix.empty()) {
      std::vector<uint64_t> s(P + 1);
      sparsep_partition_by_elem(n, P, s.data());
      for (uint32_t i = 1; i < P; ++i) cuts.push_back(s[i]);
    } else {
      std::vector<uint32_t> s(P + 2);
      greedy_split_bcsr(weight_prefix.data(), (uint32_t)n, P, s.data());
      for (uint32_t i = 1; i < P; ++i) cuts.push_back(s[i]);
    }
  } else {
    // row / block-row granularity (COO-row, COO-nnz-rgrn, BCOO-block)
    std::vector<uint32_t> s(P + 2);
    if (o.part_balance == SPARSEP_BAL_ROW) {
      sparsep_partition_by_row(nkeys, P, s.data());
    } else {
      greedy_split(key_prefix.data(), nkeys, P, s.data());
    }
    for (uint32_t i = 1; i < P; ++i) cuts.push_back(key_prefix[s[i]]);
  }
  return cuts;
}

template <typename T>
static int plan_cooe(const typename Types<T>::cooe *A, const sparsep_opts *o, sparsep_plan **out) {
  if (!A || (A->nnz && !A->nnzs)) return SPARSEP_EINVAL;
  using E = typename Types<T>::elem;
  for (uint32_t n = 0; n < A->nnz; ++n) {
    if (A->nnzs[n].rowind >= A->nrows || A->nnzs[n].colind >= A->ncols) return SPARSEP_EINVAL;
    if (n && A->nnzs[n].rowind < A->nnzs[n - 1].rowind) return SPARSEP_EINVAL;  // must be row-sorted
  }
  sparsep_opts oo;
  if (o) oo = *o; else sparsep_opts_default(&oo);
  ElemTile et;
  et.t.row_end = A->nrows;
  et.t.xw = 0;
  et.e0 = 0;
  et.e1 = A->nnz;
  et.k_lo = 0;
  et.k_hi = A->nrows;
  const E *el = A->nnzs;
  if (oo.nr_parts > 0) {
    std::vector<uint64_t> kp(A->nrows + 1, 0);
    for (uint32_t n = 0; n < A->nnz; ++n) kp[el[n].rowind + 1]++;
    for (uint32_t r = 0; r < A->nrows; ++r) kp[r + 1] += kp[r];
    et.cuts = faithful_elem_cuts(oo, A->nnz, A->nrows, kp, {});
  }
  std::vector<ElemTile> tiles{et};
  return plan_elems<T>(SPARSEP_FMT_COO, SPARSEP_1D, A->nrows, A->ncols, A->nnz, A->nnz, 1, A->nnzs, sizeof(E), tiles,
                       [el](uint64_t u) { return el[u].rowind; }, AUTO_ITEM_ELEMS, o, out);
}

// SoA COO (the CSR-family reader's output, in file order): sorted into the
// AoS layout, then planned as above.
template <typename T>
static int plan_coo(const typename Types<T>::coo *A, const sparsep_opts *o, sparsep_plan **out) {
  if (!A || (A->nnz && (!A->rowindx || !A->colind || !A->values))) return SPARSEP_EINVAL;
  using E = typename Types<T>::elem;
  std::vector<E> e(A->nnz);
  for (uint32_t n = 0; n < A->nnz; ++n) {
    if (A->rowindx[n] >= A->nrows || A->colind[n] >= A->ncols) return SPARSEP_EINVAL;
    e[n].rowind = A->rowindx[n];
    e[n].colind = A->colind[n];
    e[n].val = A->values[n];
  }
  std::stable_sort(e.begin(), e.end(), [](const E &a, const E &b) {
    return a.rowind != b.rowind ? a.rowind < b.rowind : a.colind < b.colind;
  });
  typename Types<T>::cooe C;
  C.nrows = A->nrows;
  C.ncols = A->ncols;
  C.nnz = A->nnz;
  C.rows = nullptr;
  C.nnzs = e.data();
  return plan_cooe<T>(&C, o, out);
}

// 2D COO.  D: tile p holds nnzs_per_partition[p] elements with tile-local
// row / col (spmv/2D/DCOO/support/matrix.h:158-217).  RBD/BD: stripe c holds its
// elements with global rows and stripe-local columns, split into H parts at
// element granularity (spmv/2D/BDCOO/support/partition.h:47-100).
template <typename T>
static int plan_dcoo(const typename Types<T>::dcoo *A, const sparsep_opts *o, sparsep_plan **out) {
  if (!A || !A->horz_partitions || !A->vert_partitions || !A->tile_height || !A->tile_width) return SPARSEP_EINVAL;
  using E = typename Types<T>::elem;
  const uint32_t H = A->horz_partitions, V = A->vert_partitions, th = A->tile_height, tw = A->tile_width;
  sparsep_opts oo;
  if (o) oo = *o; else sparsep_opts_default(&oo);
  std::vector<ElemTile> tiles;
  uint64_t base = 0;
  for (uint32_t h = 0; h < H; ++h)
    for (uint32_t c = 0; c < V; ++c) {
      uint64_t pidx = (uint64_t)h * V + c;
      ElemTile et;
      et.t.row_off = h * th;
      uint32_t rows = et.t.row_off >= A->nrows ? 0 : std::min(th, A->nrows - et.t.row_off);
      et.t.row_end = et.t.row_off + rows;
      et.t.col_off = c * tw;
      et.t.xw = et.t.col_off >= A->ncols ? 0 : std::min(tw, A->ncols - et.t.col_off);
      et.t.slot = c;
      et.e0 = base;
      et.e1 = base + A->nnzs_per_partition[pidx];
      et.k_lo = et.t.row_off;
      et.k_hi = et.t.row_end;
      for (uint64_t n = et.e0; n < et.e1; ++n) {
        if (A->nnzs[n].rowind >= rows || A->nnzs[n].colind >= tw) return SPARSEP_EINVAL;
        if (n > et.e0 && A->nnzs[n].rowind < A->nnzs[n - 1].rowind) return SPARSEP_EINVAL;
      }
      base = et.e1;
      tiles.push_back(et);
    }
  if (base != A->nnz) return SPARSEP_EINVAL;
  const E *el = A->nnzs;
  // keys are output rows: tile-local row + tile row offset (tile found from the unit)
  std::vector<uint32_t> tile_of_unit_off;  // row offset per unit, computed lazily
  std::vector<uint32_t> roff(A->nnz);
  for (auto &et : tiles)
    for (uint64_t n = et.e0; n < et.e1; ++n) roff[n] = et.t.row_off;
  auto key = [el, r = std::move(roff)](uint64_t u) { return el[u].rowind + r[u]; };
  return plan_elems<T>(SPARSEP_FMT_COO, SPARSEP_2D_EQUAL, A->nrows, A->ncols, A->nnz, A->nnz, V, A->nnzs, sizeof(E),
                       tiles, key, AUTO_ITEM_ELEMS, &oo, out);
}

template <typename T, typename S>
static int plan_stripes_coo(int scheme, const S *A, const uint32_t *widths, const sparsep_opts *o,
                            sparsep_plan **out) {
  using E = typename Types<T>::elem;
  const uint32_t H = A->horz_partitions, V = A->vert_partitions;
  if (!H || !V) return SPARSEP_EINVAL;
  sparsep_opts oo;
  if (o) oo = *o; else sparsep_opts_default(&oo);
  std::vector<ElemTile> tiles;
  uint64_t base = 0;
  for (uint32_t c = 0; c < V; ++c) {
    ElemTile et;
    et.t.row_off = 0;
    et.t.row_end = A->nrows;
    et.t.col_off = widths[c];
    et.t.xw = widths[c + 1] > widths[c] ? widths[c + 1] - widths[c] : 0;
    et.t.slot = c;
    et.e0 = base;
    et.e1 = base + A->nnzs_per_vert_partition[c];
    et.k_lo = 0;
    et.k_hi = A->nrows;
    for (uint64_t n = et.e0; n < et.e1; ++n) {
      if (A->nnzs[n].rowind >= A->nrows || A->nnzs[n].colind >= std::max<uint32_t>(1, et.t.xw))
        return SPARSEP_EINVAL;
      if (n > et.e0 && A->nnzs[n].rowind < A->nnzs[n - 1].rowind) return SPARSEP_EINVAL;
    }
    // H parts at element granularity per stripe (the reference's 2D COO split)
    std::vector<uint64_t> s(H + 1);
    sparsep_partition_by_elem(et.e1 - et.e0, H, s.data());
    for (uint32_t h = 1; h < H; ++h) et.cuts.push_back(et.e0 + s[h]);
    base = et.e1;
    tiles.push_back(et);
  }
  if (base != A->nnz) return SPARSEP_EINVAL;
  if (oo.nr_parts <= 0) oo.nr_parts = 0;
  const E *el = A->nnzs;
  sparsep_opts o2 = oo;
  if (o2.nr_parts == 0) {
    // GPU sizing, but never coarser than the reference's H parts per stripe
    for (auto &et : tiles) {
      auto extra = even_cuts(et.e0, et.e1, AUTO_ITEM_ELEMS);
      et.cuts.insert(et.cuts.end(), extra.begin(), extra.end());
      std::sort(et.cuts.begin(), et.cuts.end());
      et.cuts.erase(std::unique(et.cuts.begin(), et.cuts.end()), et.cuts.end());
    }
    o2.nr_parts = 1;  // cuts are final
  }
  return plan_elems<T>(SPARSEP_FMT_COO, scheme, A->nrows, A->ncols, A->nnz, A->nnz, V, A->nnzs, sizeof(E), tiles,
                       [el](uint64_t u) { return el[u].rowind; }, AUTO_ITEM_ELEMS, &o2, out);
}

template <typename T>
static int plan_rbdcoo(const typename Types<T>::rbdcoo *A, const sparsep_opts *o, sparsep_plan **out) {
  if (!A || !A->vert_partitions || !A->tile_width) return SPARSEP_EINVAL;
  auto w = eq_widths(A->ncols, A->vert_partitions, A->tile_width);
  return plan_stripes_coo<T>(SPARSEP_2D_EQUAL_W, A, w.data(), o, out);
}

template <typename T>
static int plan_bdcoo(const typename Types<T>::bdcoo *A, const sparsep_opts *o, sparsep_plan **out) {
  if (!A || !A->vert_partitions || !A->vert_tile_widths) return SPARSEP_EINVAL;
  return plan_stripes_coo<T>(SPARSEP_2D_VAR, A, A->vert_tile_widths, o, out);
}

// ---------------------------------------------------------------------------
// BCSR
// ---------------------------------------------------------------------------
template <typename T>
static int plan_bcsr_tiles(int scheme, uint32_t nrows, uint32_t ncols, uint64_t nnz, uint64_t nblocks, uint32_t rb,
                           uint32_t cb, uint32_t V, const uint32_t *browptr, size_t browptr_len,
                           const uint32_t *bcolind, const T *bval, const std::vector<Tile> &tiles,
                           const std::vector<std::vector<uint32_t>> &splits, const sparsep_opts &oo,
                           sparsep_plan **out) {
  sparsep_plan *p = nullptr;
  sparsep_opts o2 = oo;
  int st = begin_plan(out, Types<T>::dtype, SPARSEP_FMT_BCSR, scheme, &oo, &p, o2);
  if (st) return st;
  auto t0 = std::chrono::steady_clock::now();
  std::unique_ptr<sparsep_plan, void (*)(sparsep_plan *)> guard(p, sparsep_plan_free);
  if (rb == 0 || cb == 0 || rb > 16) return SPARSEP_ENOSYS;
  p->nrows = nrows;
  p->ncols = ncols;
  p->nnz = nnz;
  p->nblocks = nblocks;
  p->rb = rb;
  p->cb = cb;
  std::vector<Item> items;
  const bool faithful = oo.nr_parts > 0;
  const uint64_t per = std::max<uint64_t>(1, AUTO_ITEM_ENTRIES / ((uint64_t)rb * cb));
  for (size_t i = 0; i < tiles.size(); ++i) {
    Tile t = tiles[i];
    t.xw = stage_width(p, oo, t.xw);
    const uint32_t *bp = browptr + t.ptr_base;
    const auto &sp = splits[i];
    for (size_t k = 0; k + 1 < sp.size(); ++k) {
      uint64_t a = sp[k], b = sp[k + 1];
      auto emit = [&](uint64_t x0, uint64_t x1) {
        if (x0 >= x1) return;
        Item it = make_item(t, ITEM_ROWS);
        it.a0 = x0;
        it.a1 = x1;
        uint64_t m = ((uint64_t)bp[x1] - bp[x0] + (x1 - x0) - 1) / (x1 - x0);
        it.lanes = oo.lanes ? (uint16_t)oo.lanes : (uint16_t)pow2ceil((m + 1) / 2);
        items.push_back(it);
      };
      if (faithful) {
        emit(a, b);
        continue;
      }
      uint64_t s0 = a, acc = 0;
      for (uint64_t r = a; r < b; ++r) {
        uint64_t n = (uint64_t)bp[r + 1] - bp[r];
        if (r > s0 && acc + n > per) {
          emit(s0, r);
          s0 = r;
          acc = 0;
        }
        acc += n;
      }
      emit(s0, b);
    }
  }
  set_out_mode(p, oo, V, false, 1);
  if ((st = upload(p, browptr, browptr_len, 4, 16, (const void **)&p->rowptr))) return st;
  if ((st = upload(p, bcolind, nblocks, 4, 16, (const void **)&p->bcolind))) return st;
  if ((st = upload(p, bval, nblocks * rb * cb, sizeof(T), 16 * rb * cb, &p->bval))) return st;
  p->n_rowptr = browptr_len + 16;
  p->n_idx = nblocks + 16;
  p->n_val = (nblocks + 16) * rb * cb;
  uint64_t nbr = (nrows + rb - 1) / rb;
  p->info.compulsory_bytes = nblocks * (4 + (uint64_t)rb * cb * sizeof(T)) + (nbr + 1) * 4 +
                             (uint64_t)ncols * sizeof(T) + (uint64_t)nrows * sizeof(T);
  if ((st = finish_plan(p, items, o2))) return st;
  p->t[0] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  *out = guard.release();
  return SPARSEP_OK;
}

// block-row split of [0, nbr) with the reference's BCSR balance options
static std::vector<uint32_t> bcsr_split(const sparsep_opts &o, const uint32_t *browptr, uint32_t nbr,
                                        const uint32_t *nnz_per_block, uint32_t parts) {
  std::vector<uint32_t> s(parts + 2);
  if (o.part_balance == SPARSEP_BAL_ROW) sparsep_partition_by_row(nbr, parts, s.data());
  else if (o.part_balance == SPARSEP_BAL_BLOCK) sparsep_partition_block_rows(browptr, nbr, nullptr, parts, s.data());
  else sparsep_partition_block_rows(browptr, nbr, nnz_per_block, parts, s.data());
  s.resize(parts + 1);
  return s;
}

template <typename T>
static int plan_bcsr(const typename Types<T>::bcsr *A, const sparsep_opts *o, sparsep_plan **out) {
  if (!out) return SPARSEP_EINVAL;
  if (!A || !A->row_block_size || !A->col_block_size || (A->num_blocks && (!A->bcolind || !A->bval)) ||
      !A->browptr)
    return SPARSEP_EINVAL;
  sparsep_opts oo;
  if (o) oo = *o; else sparsep_opts_default(&oo);
  if (int st = check_opts(&oo)) return st;
  const uint32_t nbr = A->num_block_rows;
  if (A->browptr[nbr] != A->num_blocks) return SPARSEP_EINVAL;
  for (uint64_t b = 0; b < A->num_blocks; ++b)
    if (A->bcolind[b] >= A->num_block_cols) return SPARSEP_EINVAL;
  Tile t;
  t.row_end = A->nrows;
  std::vector<uint32_t> sp;
  if (oo.nr_parts > 0) sp = bcsr_split(oo, A->browptr, nbr, A->nnz_per_block, oo.nr_parts);
  else sp = {0, nbr};
  return plan_bcsr_tiles<T>(SPARSEP_1D, A->nrows, A->ncols, A->nnz, A->num_blocks, (uint32_t)A->row_block_size,
                            (uint32_t)A->col_block_size, 1, A->browptr, (size_t)nbr + 1, A->bcolind, A->bval, {t},
                            {sp}, oo, out);
}

// 2D BCSR: D tiles have local browptr of num_block_rows+1 at p*(nbr+1)
// (spmv/2D/DBCSR/support/matrix.h:311-330); stripes (RBD/BD) have a
// full-height browptr at c*(nbr+1) split into H parts
// (spmv/2D/BDBCSR-nnz/support/partition.h:52).
template <typename T>
static int plan_dbcsr(const typename Types<T>::dbcsr *A, const sparsep_opts *o, sparsep_plan **out) {
  if (!out) return SPARSEP_EINVAL;
  if (!A || !A->horz_partitions || !A->vert_partitions || !A->row_block_size || !A->col_block_size)
    return SPARSEP_EINVAL;
  sparsep_opts oo;
  if (o) oo = *o; else sparsep_opts_default(&oo);
  if (int st = check_opts(&oo)) return st;
  const uint32_t H = A->horz_partitions, V = A->vert_partitions, nbr = A->num_block_rows;
  const uint32_t cb = (uint32_t)A->col_block_size;
  std::vector<Tile> tiles;
  std::vector<std::vector<uint32_t>> splits;
  uint64_t base = 0;
  for (uint32_t h = 0; h < H; ++h)
    for (uint32_t c = 0; c < V; ++c) {
      uint64_t pidx = (uint64_t)h * V + c;
      Tile t;
      t.ptr_base = pidx * (nbr + 1);
      t.nnz_base = base;
      t.row_off = (uint32_t)(h * A->tile_height);
      t.row_end = (uint32_t)std::min<uint64_t>((uint64_t)t.row_off + A->tile_height, A->nrows);
      if (t.row_end < t.row_off) t.row_end = t.row_off;
      t.col_off = (uint32_t)(c * A->tile_width);
      uint64_t span = (uint64_t)A->num_block_cols * cb;
      t.xw = t.col_off >= A->ncols ? 0 : (uint32_t)std::min<uint64_t>(span, A->ncols - t.col_off);
      t.slot = c;
      const uint32_t *bp = A->browptr + t.ptr_base;
      if (bp[nbr] != A->blocks_per_partition[pidx]) return SPARSEP_EINVAL;
      for (uint64_t b = base; b < base + A->blocks_per_partition[pidx]; ++b)
        if (A->bcolind[b] >= A->num_block_cols) return SPARSEP_EINVAL;
      base += A->blocks_per_partition[pidx];
      tiles.push_back(t);
      splits.push_back({0, nbr});
    }
  if (base != A->nblocks) return SPARSEP_EINVAL;
  return plan_bcsr_tiles<T>(SPARSEP_2D_EQUAL, A->nrows, A->ncols, A->nnz, A->nblocks, (uint32_t)A->row_block_size,
                            cb, V, A->browptr, (size_t)H * V * (nbr + 1) + 1, A->bcolind, A->bval, tiles, splits, oo,
                            out);
}

template <typename T, typename S>
static int plan_stripes_bcsr(int scheme, const S *A, const uint32_t *widths, const sparsep_opts *o,
                             sparsep_plan **out) {
  if (!out) return SPARSEP_EINVAL;
  if (!A->horz_partitions || !A->vert_partitions || !A->row_block_size || !A->col_block_size) return SPARSEP_EINVAL;
  sparsep_opts oo;
  if (o) oo = *o; else sparsep_opts_default(&oo);
  if (int st = check_opts(&oo)) return st;
  const uint32_t H = A->horz_partitions, V = A->vert_partitions, nbr = A->num_block_rows;
  const uint32_t cb = (uint32_t)A->col_block_size;
  std::vector<Tile> tiles;
  std::vector<std::vector<uint32_t>> splits;
  uint64_t base = 0;
  for (uint32_t c = 0; c < V; ++c) {
    Tile t;
    t.ptr_base = (uint64_t)c * (nbr + 1);
    t.nnz_base = base;
    t.row_off = 0;
    t.row_end = A->nrows;
    t.col_off = widths[c];
    uint64_t span = (uint64_t)A->num_block_cols * cb;
    t.xw = t.col_off >= A->ncols ? 0 : (uint32_t)std::min<uint64_t>(span, A->ncols - t.col_off);
    t.slot = c;
    const uint32_t *bp = A->browptr + t.ptr_base;
    if (bp[nbr] != A->blocks_per_vert_partition[c]) return SPARSEP_EINVAL;
    for (uint64_t b = base; b < base + A->blocks_per_vert_partition[c]; ++b)
      if (A->bcolind[b] >= A->num_block_cols) return SPARSEP_EINVAL;
    // H parts of the stripe's block rows, by nnz (the -nnz variants) or blocks
    std::vector<uint32_t> npb(A->nnz_per_block + base, A->nnz_per_block + base + A->blocks_per_vert_partition[c]);
    sparsep_opts ob = oo;
    if (ob.part_balance != SPARSEP_BAL_BLOCK && ob.part_balance != SPARSEP_BAL_ROW) ob.part_balance = SPARSEP_BAL_NNZ;
    splits.push_back(bcsr_split(ob, bp, nbr, npb.data(), H));
    tiles.push_back(t);
    base += A->blocks_per_vert_partition[c];
  }
  if (base != A->nblocks) return SPARSEP_EINVAL;
  return plan_bcsr_tiles<T>(scheme, A->nrows, A->ncols, A->nnz, A->nblocks, (uint32_t)A->row_block_size, cb, V,
                            A->browptr, (size_t)V * (nbr + 1) + 1, A->bcolind, A->bval, tiles, splits, oo, out);
}

template <typename T>
static int plan_rbdbcsr(const typename Types<T>::rbdbcsr *A, const sparsep_opts *o, sparsep_plan **out) {
  if (!A || !A->vert_partitions || !A->tile_width) return SPARSEP_EINVAL;
  auto w = eq_widths(A->ncols, A->vert_partitions, A->tile_width);
  return plan_stripes_bcsr<T>(SPARSEP_2D_EQUAL_W, A, w.data(), o, out);
}

template <typename T>
static int plan_bdbcsr(const typename Types<T>::bdbcsr *A, const sparsep_opts *o, sparsep_plan **out) {
  if (!A || !A->vert_partitions || !A->vert_tile_widths) return SPARSEP_EINVAL;
  return plan_stripes_bcsr<T>(SPARSEP_2D_VAR, A, A->vert_tile_widths, o, out);
}

// ---------------------------------------------------------------------------
// BCOO
// ---------------------------------------------------------------------------
template <typename T>
static int plan_bcoo(const typename Types<T>::bcoo *A, const sparsep_opts *o, sparsep_plan **out) {
  if (!out) return SPARSEP_EINVAL;
  if (!A || !A->row_block_size || !A->col_block_size || (A->num_blocks && (!A->bind || !A->bval)))
    return SPARSEP_EINVAL;
  if (A->row_block_size > 16) return SPARSEP_ENOSYS;
  sparsep_opts oo;
  if (o) oo = *o; else sparsep_opts_default(&oo);
  for (uint64_t b = 0; b < A->num_blocks; ++b) {
    if (A->bind[b].rowind >= A->num_block_rows || A->bind[b].colind >= A->num_block_cols) return SPARSEP_EINVAL;
    if (b && A->bind[b].rowind < A->bind[b - 1].rowind) return SPARSEP_EINVAL;
  }
  ElemTile et;
  et.t.row_end = A->nrows;
  et.e0 = 0;
  et.e1 = A->num_blocks;
  et.k_lo = 0;
  et.k_hi = A->num_block_rows;
  const sparsep_bind *bi = A->bind;
  if (oo.nr_parts > 0) {
    std::vector<uint64_t> kp(A->num_block_rows + 1, 0), wp(A->num_blocks + 1, 0);
    for (uint64_t b = 0; b < A->num_blocks; ++b) kp[bi[b].rowind + 1]++;
    for (uint32_t r = 0; r < A->num_block_rows; ++r) kp[r + 1] += kp[r];
    for (uint64_t b = 0; b < A->num_blocks; ++b) wp[b + 1] = wp[b] + (A->nnz_per_block ? A->nnz_per_block[b] : 1);
    sparsep_opts ob = oo;
    if (ob.part_balance == SPARSEP_BAL_NNZ) ob.part_balance = SPARSEP_BAL_NNZ_ELEM;
    et.cuts = faithful_elem_cuts(ob, A->num_blocks, A->num_block_rows, kp,
                                 ob.part_balance == SPARSEP_BAL_NNZ_ELEM ? wp : std::vector<uint64_t>{});
  }
  const uint32_t rb = (uint32_t)A->row_block_size, cb = (uint32_t)A->col_block_size;
  uint64_t per = std::max<uint64_t>(1, AUTO_ITEM_ENTRIES / ((uint64_t)rb * cb));
  return plan_elems<T>(SPARSEP_FMT_BCOO, SPARSEP_1D, A->nrows, A->ncols, A->nnz, A->num_blocks, 1, nullptr, 0, {et},
                       [bi](uint64_t u) { return bi[u].rowind; }, per, &oo, out, A, rb, cb);
}

// 2D BCOO: blocks of tile p (D) or stripe c (RBD/BD), keys = tile-local block rows.
template <typename T, typename S>
static int plan_tiles_bcoo(int scheme, const S *A, uint32_t ntiles, const uint32_t *blocks_per,
                           std::function<Tile(uint32_t)> tile_of, uint32_t H, bool stripes, const sparsep_opts *o,
                           sparsep_plan **out) {
  if (!out) return SPARSEP_EINVAL;
  if (!A->row_block_size || !A->col_block_size) return SPARSEP_EINVAL;
  if (A->row_block_size > 16) return SPARSEP_ENOSYS;
  sparsep_opts oo;
  if (o) oo = *o; else sparsep_opts_default(&oo);
  const uint32_t rb = (uint32_t)A->row_block_size, cb = (uint32_t)A->col_block_size, nbr = A->num_block_rows;
  std::vector<ElemTile> tiles;
  uint64_t base = 0;
  for (uint32_t p = 0; p < ntiles; ++p) {
    ElemTile et;
    et.t = tile_of(p);
    et.e0 = base;
    et.e1 = base + blocks_per[p];
    et.k_lo = 0;
    et.k_hi = stripes ? nbr : (uint32_t)std::min<uint64_t>(nbr, (et.t.row_end - et.t.row_off + rb - 1) / rb);
    for (uint64_t b = et.e0; b < et.e1; ++b) {
      if (A->bind[b].rowind >= nbr || A->bind[b].colind >= A->num_block_cols) return SPARSEP_EINVAL;
      if (b > et.e0 && A->bind[b].rowind < A->bind[b - 1].rowind) return SPARSEP_EINVAL;
    }
    if (stripes) {
      // H parts per stripe by nnz at block granularity (spmv/2D/BDBCOO-nnz/support/partition.h:52-100)
      std::vector<uint64_t> wp(blocks_per[p] + 1, 0);
      for (uint64_t b = 0; b < blocks_per[p]; ++b) wp[b + 1] = wp[b] + A->nnz_per_block[base + b];
      std::vector<uint32_t> s(H + 2);
      greedy_split_bcsr(wp.data(), blocks_per[p], H, s.data());
      for (uint32_t h = 1; h < H; ++h) et.cuts.push_back(et.e0 + s[h]);
    }
    base = et.e1;
    tiles.push_back(et);
  }
  if (base != A->nblocks) return SPARSEP_EINVAL;
  typename Types<T>::bcoo B;
  std::memset(&B, 0, sizeof B);
  B.bind = A->bind;
  B.bval = A->bval;
  sparsep_opts o2 = oo;
  uint64_t per = std::max<uint64_t>(1, AUTO_ITEM_ENTRIES / ((uint64_t)rb * cb));
  if (o2.nr_parts == 0) {
    for (auto &et : tiles) {
      auto extra = even_cuts(et.e0, et.e1, per);
      et.cuts.insert(et.cuts.end(), extra.begin(), extra.end());
      std::sort(et.cuts.begin(), et.cuts.end());
      et.cuts.erase(std::unique(et.cuts.begin(), et.cuts.end()), et.cuts.end());
    }
    o2.nr_parts = 1;
  }
  const sparsep_bind *bi = A->bind;
  uint32_t V = A->vert_partitions;
  return plan_elems<T>(SPARSEP_FMT_BCOO, scheme, A->nrows, A->ncols, A->nnz, A->nblocks, V, nullptr, 0, tiles,
                       [bi](uint64_t u) { return bi[u].rowind; }, per, &o2, out, &B, rb, cb);
}

template <typename T>
static int plan_dbcoo(const typename Types<T>::dbcoo *A, const sparsep_opts *o, sparsep_plan **out) {
  if (!A || !A->horz_partitions || !A->vert_partitions) return SPARSEP_EINVAL;
  const uint32_t V = A->vert_partitions;
  const uint64_t span = (uint64_t)A->num_block_cols * A->col_block_size;
  auto tile_of = [A, V, span](uint32_t p) {
    Tile t;
    uint32_t h = p / V, c = p % V;
    t.row_off = (uint32_t)(h * A->tile_height);
    t.row_end = (uint32_t)std::min<uint64_t>((uint64_t)t.row_off + A->tile_height, A->nrows);
    if (t.row_end < t.row_off) t.row_end = t.row_off;
    t.col_off = (uint32_t)(c * A->tile_width);
    t.xw = t.col_off >= A->ncols ? 0 : (uint32_t)std::min<uint64_t>(span, A->ncols - t.col_off);
    t.slot = c;
    return t;
  };
  return plan_tiles_bcoo<T>(SPARSEP_2D_EQUAL, A, A->horz_partitions * V, A->blocks_per_partition, tile_of,
                            A->horz_partitions, false, o, out);
}

template <typename T, typename S>
static int plan_stripes_bcoo(int scheme, const S *A, std::vector<uint32_t> widths, const sparsep_opts *o,
                             sparsep_plan **out) {
  const uint64_t span = (uint64_t)A->num_block_cols * A->col_block_size;
  auto tile_of = [A, widths, span](uint32_t c) {
    Tile t;
    t.row_off = 0;
    t.row_end = A->nrows;
    t.col_off = widths[c];
    t.xw = t.col_off >= A->ncols ? 0 : (uint32_t)std::min<uint64_t>(span, A->ncols - t.col_off);
    t.slot = c;
    return t;
  };
  return plan_tiles_bcoo<T>(scheme, A, A->vert_partitions, A->blocks_per_vert_partition, tile_of,
                            A->horz_partitions, true, o, out);
}

template <typename T>
static int plan_rbdbcoo(const typename Types<T>::rbdbcoo *A, const sparsep_opts *o, sparsep_plan **out) {
  if (!A || !A->vert_partitions || !A->tile_width || !A->horz_partitions) return SPARSEP_EINVAL;
  return plan_stripes_bcoo<T>(SPARSEP_2D_EQUAL_W, A, eq_widths(A->ncols, A->vert_partitions, A->tile_width), o, out);
}

template <typename T>
static int plan_bdbcoo(const typename Types<T>::bdbcoo *A, const sparsep_opts *o, sparsep_plan **out) {
  if (!A || !A->vert_partitions || !A->vert_tile_widths || !A->horz_partitions) return SPARSEP_EINVAL;
  std::vector<uint32_t> w(A->vert_tile_widths, A->vert_tile_widths + A->vert_partitions + 1);
  return plan_stripes_bcoo<T>(SPARSEP_2D_VAR, A, w, o, out);
}

// ---------------------------------------------------------------------------
// Execution
// ---------------------------------------------------------------------------
template <typename T>
static int run_t(sparsep_plan *p, const void *d_x, void *d_y, cudaStream_t s, unsigned int *band_cnt) {
  const T *x = static_cast<const T *>(d_x);
  if (p->stage && d_x != p->xpad) {
    CK(cudaMemcpyAsync(p->xpad, d_x, (size_t)p->ncols * sizeof(T), cudaMemcpyDeviceToDevice, s));
    x = static_cast<const T *>(p->xpad);
  }
  if (p->out_mode == OUT_ATOMIC) CK(cudaMemsetAsync(d_y, 0, (size_t)p->nrows * sizeof(T), s));
  Params<T> P;
  std::memset(&P, 0, sizeof P);
  P.items = p->items;
  P.nitems = p->nitems;
  P.nrows = p->nrows;
  P.ncols = p->ncols;
  P.rowptr = p->rowptr;
  P.colind = p->colind;
  P.val = static_cast<const T *>(p->val);
  P.elems = p->elems;
  P.bcolind = p->bcolind;
  P.bind = p->bind;
  P.bval = static_cast<const T *>(p->bval);
  P.rb = p->rb;
  P.cb = p->cb;
  P.x = x;
  P.y = static_cast<T *>(d_y);
  P.part = static_cast<T *>(p->part);
  P.out_mode = p->out_mode;
  P.carry_val = p->carry_w ? p->carry_val : nullptr;
  // CSR long rows complete through per-row counters; the carry list and the
  // last-CTA fix-up serve the element-wise (COO / BCOO) formats
  P.carry_idx = (p->carry_w && p->format != SPARSEP_FMT_CSR) ? p->carry_idx : nullptr;
  P.done = p->done;
  P.row_cnt = p->row_cnt;
  P.band_cnt = band_cnt;
  P.err = p->err;
  P.n_rowptr = p->n_rowptr;
  P.n_idx = p->n_idx;
  P.n_val = p->n_val;
  P.n_elems = p->n_elems;
  P.n_x = p->ncols;
  P.n_xalloc = x == p->xpad ? (uint64_t)p->ncols + 64 : p->ncols;  // staging reads into the slack
  P.n_carry = p->carry_w ? (uint64_t)p->nitems * p->carry_w + 1 : 0;
  P.nslots = p->out_mode == OUT_PARTIAL ? p->V : 1;
  P.smem_bytes = (uint32_t)p->smem;
  P.fault_wait = wait_fault();
  if (p->split.on) {
    // one persistent kernel over the heavy stripes and the light rows, then
    // the heavy rows' stripe partials summed into y
    const auto &S = p->split;
    StripeParams<T> Q;
    std::memset(&Q, 0, sizeof Q);
    Q.chunks = S.chunks;
    Q.cta_first = S.cta_first;
    Q.wsplit = S.wsplit;
    Q.vptr = S.vptr;
    Q.hcol = S.hcol;
    Q.hval = static_cast<const T *>(S.hval);
    Q.lptr = p->rowptr;
    Q.lcol = p->colind;
    Q.lval = static_cast<const T *>(p->val);
    Q.x = static_cast<const T *>(d_x);
    Q.y = static_cast<T *>(d_y);
    Q.part = static_cast<T *>(S.part);
    Q.ncols = p->ncols;
    Q.nrows = p->nrows;
    Q.W = S.W;
    Q.err = p->err;
    Q.n_vptr = S.n_vptr;
    Q.n_h = S.n_h;
    Q.n_lptr = S.n_lptr;
    Q.n_l = S.n_l;
    Q.n_part = S.n_part;
    CK(launch_stripes<T>(Q, S.ctas, s));
    CK(launch_heavy_merge<T>(static_cast<const T *>(S.part), S.hrow, S.nH, S.nS, static_cast<T *>(d_y), p->sms, s));
    return SPARSEP_OK;
  }
  if (p->pipe) CK(launch_csr_pipe<T>(P, p->sms, s, &p->pipe_grid, p->max_item_nnz));
  else CK(launch_items<T>(P, p->format, p->carry_w, p->threads, p->smem, s));
  if (p->out_mode == OUT_PARTIAL) {
    CK(cudaEventRecord(p->ev[2], s));
    CK(launch_merge<T>(static_cast<const T *>(p->part), static_cast<T *>(d_y), p->nrows, p->V, p->sms, s));
  }
  return SPARSEP_OK;
}

// A multi-RHS plan on device buffers: x into the batch, one launch, y out
// (stream-ordered on s; on the legacy stream, synchronous around the batch's
// own stream).
// The batch's rows are `pitch` elements apart, the caller's k: 2D copies.
static int run_multi(sparsep_plan *p, const void *d_x, void *d_y, cudaStream_t s) {
  uint32_t pitch = 0;
  if (int st = sparsep_batch_pitch(p->batch, 0, &pitch)) return st;
  const size_t w = (size_t)p->nrhs * p->esize, pw = (size_t)pitch * p->esize;
  if (!s) {
    if (d_x != p->xpad) CK(cudaMemcpy2D(p->xpad, pw, d_x, w, w, p->ncols, cudaMemcpyDeviceToDevice));
    if (int st = sparsep_batch_execute(p->batch, nullptr)) return st;
    if (d_y != p->y) CK(cudaMemcpy2D(d_y, w, p->y, pw, w, p->nrows, cudaMemcpyDeviceToDevice));
    return SPARSEP_OK;
  }
  if (d_x != p->xpad) CK(cudaMemcpy2DAsync(p->xpad, pw, d_x, w, w, p->ncols, cudaMemcpyDeviceToDevice, s));
  if (int st = sparsep_batch_execute(p->batch, s)) return st;
  if (d_y != p->y) CK(cudaMemcpy2DAsync(d_y, w, p->y, pw, w, p->nrows, cudaMemcpyDeviceToDevice, s));
  return SPARSEP_OK;
}

static int run_any(sparsep_plan *p, const void *d_x, void *d_y, cudaStream_t s,
                   unsigned int *band_cnt = nullptr) {
  if (p->batch) return run_multi(p, d_x, d_y, s);
  switch (p->dtype) {
    case SPARSEP_INT8: return run_t<int8_t>(p, d_x, d_y, s, band_cnt);
    case SPARSEP_INT16: return run_t<int16_t>(p, d_x, d_y, s, band_cnt);
    case SPARSEP_INT32: return run_t<int32_t>(p, d_x, d_y, s, band_cnt);
    case SPARSEP_INT64: return run_t<int64_t>(p, d_x, d_y, s, band_cnt);
    case SPARSEP_FP32: return run_t<float>(p, d_x, d_y, s, band_cnt);
    case SPARSEP_FP64: return run_t<double>(p, d_x, d_y, s, band_cnt);
  }
  return SPARSEP_EINVAL;
}

// Columns of a device CSR inside [0, ncols): one flag for the whole array.
__global__ void cols_in_range(const uint32_t *__restrict__ c, uint64_t n, uint32_t ncols, int *__restrict__ bad) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    if (c[i] >= ncols) *bad = 1;
}

// A plan from a CSR matrix already on the device: the row pointers are read
// back for the planner (4 bytes per row), the column indices are checked on
// the device, and the arrays are copied device to device into the plan.
template <typename T>
static int plan_csr_device(uint32_t nrows, uint32_t ncols, uint32_t nnz, const uint32_t *d_rowptr,
                           const uint32_t *d_colind, const T *d_values, const sparsep_opts *o, sparsep_plan **out) {
  if (!out || !d_rowptr || (nnz && (!d_colind || !d_values))) return SPARSEP_EINVAL;
  *out = nullptr;
  std::vector<uint32_t> rp;
  try {
    rp.resize((size_t)nrows + 1);
  } catch (const std::bad_alloc &) {
    return SPARSEP_ENOMEM;
  }
  CK(cudaMemcpy(rp.data(), d_rowptr, rp.size() * 4, cudaMemcpyDeviceToHost));
  if (nnz) {
    int *bad = nullptr, h = 0;
    CK(dev_malloc((void **)&bad, sizeof(int)));
    cudaError_t e = cudaMemset(bad, 0, sizeof(int));
    if (e == cudaSuccess) {
      cols_in_range<<<std::min<uint64_t>(4096, (nnz + 255) / 256), 256>>>(d_colind, nnz, ncols, bad);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(&h, bad, sizeof(int), cudaMemcpyDeviceToHost);
    dev_free(bad);
    CK(e);
    if (h) return SPARSEP_EINVAL;
  }
  typename Types<T>::csr A;
  A.nrows = nrows;
  A.ncols = ncols;
  A.nnz = nnz;
  A.rowptr = rp.data();
  A.colind = const_cast<uint32_t *>(d_colind);
  A.values = const_cast<T *>(d_values);
  return plan_csr<T>(&A, o, out, true);
}

// A plan from a BCSR matrix already on the device (the device converter's
// output, or any BCSR of the reference layout): the block row pointers -- and,
// for nnz-balanced parts, the nonzeros per block -- are read back for the
// planner, the block columns checked on the device, the arrays copied into the
// plan (the caller keeps its own).
template <typename T>
static int plan_bcsr_device(uint32_t nrows, uint32_t ncols, uint32_t rb, uint32_t cb, uint64_t nblocks, uint64_t nnz,
                            const uint32_t *d_browptr, const uint32_t *d_bcolind, const T *d_bval,
                            const uint32_t *d_nnz_per_block, const sparsep_opts *o, sparsep_plan **out) {
  if (!out) return SPARSEP_EINVAL;
  *out = nullptr;
  if (!d_browptr || rb == 0 || cb == 0 || nblocks > UINT32_MAX || (nblocks && (!d_bcolind || !d_bval)))
    return SPARSEP_EINVAL;
  sparsep_opts oo;
  if (o) oo = *o; else sparsep_opts_default(&oo);
  if (int st = check_opts(&oo)) return st;
  const uint32_t nbr = (uint32_t)(((uint64_t)nrows + rb - 1) / rb);
  const uint32_t nbc = (uint32_t)(((uint64_t)ncols + cb - 1) / cb);
  std::vector<uint32_t> bp((size_t)nbr + 1);
  CK(cudaMemcpy(bp.data(), d_browptr, bp.size() * 4, cudaMemcpyDeviceToHost));
  if (bp[0] != 0 || bp[nbr] != nblocks) return SPARSEP_EINVAL;
  for (uint32_t i = 0; i < nbr; ++i)
    if (bp[i] > bp[i + 1]) return SPARSEP_EINVAL;
  if (nblocks) {
    int *bad = nullptr, h = 0;
    CK(dev_malloc((void **)&bad, sizeof(int)));
    cudaError_t e = cudaMemset(bad, 0, sizeof(int));
    if (e == cudaSuccess) {
      cols_in_range<<<std::min<uint64_t>(4096, (nblocks + 255) / 256), 256>>>(d_bcolind, nblocks, nbc, bad);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(&h, bad, sizeof(int), cudaMemcpyDeviceToHost);
    dev_free(bad);
    CK(e);
    if (h) return SPARSEP_EINVAL;
  }
  std::vector<uint32_t> npb;
  const bool need_npb = oo.nr_parts > 0 && oo.part_balance != SPARSEP_BAL_ROW && oo.part_balance != SPARSEP_BAL_BLOCK;
  if (need_npb) {
    if (!d_nnz_per_block) return SPARSEP_EINVAL;
    npb.resize(nblocks);
    if (nblocks) CK(cudaMemcpy(npb.data(), d_nnz_per_block, nblocks * 4, cudaMemcpyDeviceToHost));
  }
  Tile t;
  t.row_end = nrows;
  std::vector<uint32_t> sp;
  if (oo.nr_parts > 0) sp = bcsr_split(oo, bp.data(), nbr, need_npb ? npb.data() : nullptr, oo.nr_parts);
  else sp = {0, nbr};
  return plan_bcsr_tiles<T>(SPARSEP_1D, nrows, ncols, nnz, nblocks, rb, cb, 1, bp.data(), (size_t)nbr + 1, d_bcolind,
                            d_bval, {t}, {sp}, oo, out);
}

// ---------------------------------------------------------------------------
// C-ABI
// ---------------------------------------------------------------------------
extern "C" {

const char *sparsep_version(void) {
#ifdef SPARSEP_CHECK
  return "sparsep_b200 0.1 (sm_100a, bounds-checked)";
#else
  return "sparsep_b200 0.1 (sm_100a)";
#endif
}

const char *sparsep_last_error(void) { return g_last_error; }

const char *sparsep_strerror(int s) {
  switch (s) {
    case SPARSEP_OK: return "ok";
    case SPARSEP_EIO: return "CUDA runtime error";
    case SPARSEP_ENOMEM: return "out of memory";
    case SPARSEP_ENODEV: return "no usable CUDA device";
    case SPARSEP_EINVAL: return "invalid argument";
    case SPARSEP_ENOSYS: return "option combination not provided";
    case SPARSEP_ERANGE: return "size beyond the supported maximum";
    case SPARSEP_ETIMEDOUT: return "bounded device wait timed out";
    case SPARSEP_EBADF: return "matrix file missing or malformed";
  }
  return "unknown status";
}

void sparsep_opts_default(sparsep_opts *o) {
  if (!o) return;
  std::memset(o, 0, sizeof *o);
  o->format = SPARSEP_FMT_CSR;
  o->scheme = SPARSEP_1D;
  o->part_balance = SPARSEP_BAL_NNZ;
  o->worker_balance = SPARSEP_BAL_INTERLEAVE;
  o->sync = SPARSEP_SYNC_LF;
  o->nr_parts = 0;
  o->nr_workers = 0;
  o->vert_partitions = 1;
  o->row_block_size = 4;
  o->col_block_size = 4;
  o->lanes = 0;
  o->nrhs = 1;
  o->stage_x = -1;
}

int sparsep_device_sms(void) {
  int dev = 0, n = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
  return n;
}

void sparsep_plan_free(sparsep_plan *p) {
  if (!p) return;
  if (p->batch) sparsep_batch_free(p->batch);
  if (p->stream) cudaStreamSynchronize(p->stream);
  if (p->copy_stream) {
    cudaStreamSynchronize(p->copy_stream);
    cudaStreamDestroy(p->copy_stream);
  }
  for (void *d : p->allocs) dev_free(d);
  if (p->h_err) cudaFreeHost(p->h_err);
  for (auto &e : p->ev)
    if (e) cudaEventDestroy(e);
  if (p->stream) cudaStreamDestroy(p->stream);
  delete p;
}

int sparsep_plan_get_info(const sparsep_plan *p, sparsep_plan_info *info) {
  if (!p || !info) return SPARSEP_EINVAL;
  *info = p->info;
  return SPARSEP_OK;
}

int sparsep_timings(const sparsep_plan *p, double ms[5]) {
  if (!p || !ms) return SPARSEP_EINVAL;
  for (int i = 0; i < 5; ++i) ms[i] = p->t[i];
  return SPARSEP_OK;
}

void *sparsep_plan_x(sparsep_plan *p) { return p ? p->xpad : nullptr; }
void *sparsep_plan_y(sparsep_plan *p) { return p ? p->y : nullptr; }

int sparsep_execute_device(sparsep_plan *p, const void *d_x, void *d_y, void *stream) {
  if (!p || !d_x || !d_y) return SPARSEP_EINVAL;
  return run_any(p, d_x, d_y, static_cast<cudaStream_t>(stream));
}

// y in row bands: each band's copy, on the plan's copy stream, waits
// (cuStreamWaitValue32) until the kernel has counted all items of the band, so
// the copies of the early bands overlap the kernel's later items.  The
// counters are never cleared: after the n-th launch counter b holds
// n * band_items[b] (mod 2^32, which the wait's wrap-around comparison
// handles), so a wait for call n cannot be met by an earlier call's counts.
static int copy_y_banded(sparsep_plan *p, void *h_y) {
  cudaStream_t c = p->copy_stream;
  const size_t es = p->esize;
  char *hy = static_cast<char *>(h_y);
  const char *dy = static_cast<const char *>(p->y);
  uint32_t b = 0;
  for (; b < p->nbands; ++b) {
    const cuuint32_t target = p->band_calls * p->band_items[b];
    if (wait_value32()(c, (CUdeviceptr)(uintptr_t)(p->band_cnt + b), target, CU_STREAM_WAIT_VALUE_GEQ) != CUDA_SUCCESS)
      break;
    const size_t r0 = p->band_row[b], r1 = p->band_row[b + 1];
    if (r1 > r0) CK(cudaMemcpyAsync(hy + r0 * es, dy + r0 * es, (r1 - r0) * es, cudaMemcpyDeviceToHost, c));
  }
  if (b < p->nbands) {  // the driver refused a wait: the remaining rows after the whole kernel
    CK(cudaStreamWaitEvent(c, p->ev[2], 0));
    const size_t r0 = p->band_row[b];
    CK(cudaMemcpyAsync(hy + r0 * es, dy + r0 * es, (p->nrows - r0) * es, cudaMemcpyDeviceToHost, c));
  }
  return SPARSEP_OK;
}

int sparsep_execute_host(sparsep_plan *p, const void *h_x, void *h_y) {
  if (!p || !h_x || !h_y) return SPARSEP_EINVAL;
  if (p->batch) {  // several right-hand sides: the batch's host copies around one launch
    using clk = std::chrono::steady_clock;
    const auto t0 = clk::now();
    int st = sparsep_batch_set_x(p->batch, 0, h_x);
    const auto t1 = clk::now();
    if (!st) st = sparsep_batch_execute(p->batch, nullptr);
    const auto t2 = clk::now();
    if (!st) st = sparsep_batch_get_y(p->batch, 0, h_y);
    const auto t3 = clk::now();
    p->t[1] = std::chrono::duration<double, std::milli>(t1 - t0).count();
    p->t[2] = std::chrono::duration<double, std::milli>(t2 - t1).count();
    p->t[3] = std::chrono::duration<double, std::milli>(t3 - t2).count();
    p->t[4] = 0;
    return st;
  }
  cudaStream_t s = p->stream;
  CK(cudaEventRecord(p->ev[0], s));
  CK(cudaMemcpyAsync(p->xpad, h_x, (size_t)p->ncols * p->esize, cudaMemcpyHostToDevice, s));
  CK(cudaEventRecord(p->ev[1], s));
  if (p->nbands) {
    if (int st = run_any(p, p->xpad, p->y, s, p->band_cnt)) return st;
    ++p->band_calls;  // the launch adds band_items[b] to counter b
    CK(cudaEventRecord(p->ev[2], s));
    CK(cudaEventRecord(p->ev[3], s));
    const int cst = copy_y_banded(p, h_y);
    // the copy stream is drained before the call returns, also when a copy
    // failed: no band wait may outlive this call and read the next call's counters
    CK(cudaEventRecord(p->ev[4], p->copy_stream));
    CK(cudaStreamWaitEvent(s, p->ev[4], 0));
    if (cst) {
      cudaStreamSynchronize(s);
      return cst;
    }
  } else {
    if (int st = run_any(p, p->xpad, p->y, s)) return st;
    if (p->out_mode != OUT_PARTIAL) CK(cudaEventRecord(p->ev[2], s));
    CK(cudaEventRecord(p->ev[3], s));
    CK(cudaMemcpyAsync(h_y, p->y, (size_t)p->nrows * p->esize, cudaMemcpyDeviceToHost, s));
    CK(cudaEventRecord(p->ev[4], s));
  }
  // the error word rides behind y: one synchronisation for the whole call
  CK(cudaMemcpyAsync(p->h_err, p->err, sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  float a = 0, b = 0, c = 0, d = 0;
  CK(cudaEventElapsedTime(&a, p->ev[0], p->ev[1]));
  CK(cudaEventElapsedTime(&b, p->ev[1], p->ev[2]));
  CK(cudaEventElapsedTime(&c, p->ev[2], p->ev[3]));
  CK(cudaEventElapsedTime(&d, p->ev[3], p->ev[4]));
  p->t[1] = a;
  p->t[2] = b;
  p->t[4] = c;
  p->t[3] = std::max(d, 0.f);  // banded: the part of the y copy left after the kernel
  if (const int e = *p->h_err) {
    CK(cudaMemsetAsync(p->err, 0, sizeof(int), s));
    CK(cudaStreamSynchronize(s));
    return e;
  }
  return SPARSEP_OK;
}

#define SPARSEP_KIND_ENTRIES(T, S, K)                                                                 \
  int sparsep_plan_##K##_##S(const sparsep_##K##_##S *A, const sparsep_opts *o, sparsep_plan **out) { \
    try {                                                                                             \
      return plan_##K<T>(A, o, out);                                                                  \
    } catch (const std::bad_alloc &) {                                                                \
      return SPARSEP_ENOMEM;                                                                          \
    }                                                                                                 \
  }                                                                                                   \
  int sparsep_spmv_##K##_##S(const sparsep_##K##_##S *A, const T *x, T *y, const sparsep_opts *o) {   \
    if (!x || !y) return SPARSEP_EINVAL;                                                              \
    sparsep_plan *p = nullptr;                                                                        \
    int st = sparsep_plan_##K##_##S(A, o, &p);                                                        \
    if (st) return st;                                                                                \
    st = sparsep_execute_host(p, x, y);                                                               \
    sparsep_plan_free(p);                                                                             \
    return st;                                                                                        \
  }                                                                                                   \
  void sparsep_free_##K##_##S(sparsep_##K##_##S *A) { free_any(A); }

#define SPARSEP_DTYPE_ENTRIES(T, S)      \
  SPARSEP_KIND_ENTRIES(T, S, csr)        \
  SPARSEP_KIND_ENTRIES(T, S, coo)        \
  SPARSEP_KIND_ENTRIES(T, S, cooe)       \
  SPARSEP_KIND_ENTRIES(T, S, bcsr)       \
  SPARSEP_KIND_ENTRIES(T, S, bcoo)       \
  SPARSEP_KIND_ENTRIES(T, S, dcsr)       \
  SPARSEP_KIND_ENTRIES(T, S, rbdcsr)     \
  SPARSEP_KIND_ENTRIES(T, S, bdcsr)      \
  SPARSEP_KIND_ENTRIES(T, S, dcoo)       \
  SPARSEP_KIND_ENTRIES(T, S, rbdcoo)     \
  SPARSEP_KIND_ENTRIES(T, S, bdcoo)      \
  SPARSEP_KIND_ENTRIES(T, S, dbcsr)      \
  SPARSEP_KIND_ENTRIES(T, S, dbcoo)      \
  SPARSEP_KIND_ENTRIES(T, S, rbdbcsr)    \
  SPARSEP_KIND_ENTRIES(T, S, rbdbcoo)    \
  SPARSEP_KIND_ENTRIES(T, S, bdbcsr)     \
  SPARSEP_KIND_ENTRIES(T, S, bdbcoo)

SPARSEP_DTYPE_ENTRIES(int8_t, i8)
SPARSEP_DTYPE_ENTRIES(int16_t, i16)
SPARSEP_DTYPE_ENTRIES(int32_t, i32)
SPARSEP_DTYPE_ENTRIES(int64_t, i64)
SPARSEP_DTYPE_ENTRIES(float, f32)
SPARSEP_DTYPE_ENTRIES(double, f64)

}  // extern "C"

#define SPARSEP_PLAN_DEVICE_ENTRY(T, S)                                                                   \
  extern "C" int sparsep_plan_csr_device_##S(uint32_t nrows, uint32_t ncols, uint32_t nnz,                 \
                                             const uint32_t *d_rowptr, const uint32_t *d_colind,          \
                                             const T *d_values, const sparsep_opts *o, sparsep_plan **out) { \
    try {                                                                                                 \
      return plan_csr_device<T>(nrows, ncols, nnz, d_rowptr, d_colind, d_values, o, out);                 \
    } catch (const std::bad_alloc &) {                                                                    \
      return SPARSEP_ENOMEM;                                                                              \
    }                                                                                                     \
  }
SPARSEP_PLAN_DEVICE_ENTRY(int8_t, i8)
SPARSEP_PLAN_DEVICE_ENTRY(int16_t, i16)
SPARSEP_PLAN_DEVICE_ENTRY(int32_t, i32)
SPARSEP_PLAN_DEVICE_ENTRY(int64_t, i64)
SPARSEP_PLAN_DEVICE_ENTRY(float, f32)
SPARSEP_PLAN_DEVICE_ENTRY(double, f64)

#define SPARSEP_PLAN_BCSR_DEVICE_ENTRY(T, S)                                                                       \
  extern "C" int sparsep_plan_bcsr_device_##S(uint32_t nrows, uint32_t ncols, uint32_t rb, uint32_t cb,           \
                                              uint64_t nblocks, uint64_t nnz, const uint32_t *d_browptr,          \
                                              const uint32_t *d_bcolind, const T *d_bval,                         \
                                              const uint32_t *d_nnz_per_block, const sparsep_opts *o,             \
                                              sparsep_plan **out) {                                               \
    try {                                                                                                          \
      return plan_bcsr_device<T>(nrows, ncols, rb, cb, nblocks, nnz, d_browptr, d_bcolind, d_bval, d_nnz_per_block, \
                                 o, out);                                                                          \
    } catch (const std::bad_alloc &) {                                                                             \
      return SPARSEP_ENOMEM;                                                                                       \
    }                                                                                                              \
  }
SPARSEP_PLAN_BCSR_DEVICE_ENTRY(int8_t, i8)
SPARSEP_PLAN_BCSR_DEVICE_ENTRY(int16_t, i16)
SPARSEP_PLAN_BCSR_DEVICE_ENTRY(int32_t, i32)
SPARSEP_PLAN_BCSR_DEVICE_ENTRY(int64_t, i64)
SPARSEP_PLAN_BCSR_DEVICE_ENTRY(float, f32)
SPARSEP_PLAN_BCSR_DEVICE_ENTRY(double, f64)
