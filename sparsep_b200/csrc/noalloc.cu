// noalloc.cu -- an SpMV entry point that allocates nothing.
//
// Some callers cannot allocate device memory at the time they need an SpMV:
// code running inside a memory pool or arena that owns the whole device heap,
// a host process whose allocator is locked down after start-up, or a routine
// that runs between another component's stream operations, where a
// cudaMalloc would synchronise the device or be refused.  For them,
// sparsep_spmv_cooe_f32_noalloc multiplies a sorted FP32 COO matrix that is
// already on the device with the lock-free COO kernel, using a fixed scratch
// area that lives in this library's own device image instead of memory
// allocated per call.
//
// The scratch is a file-scope __device__ array of MAX_ITEMS carry slots
// (16 bytes each, about 1 MB); every GPU that loads the library holds it until
// the process exits.  Calls share it, so calls that overlap on the GPU race.
// Each call derives its work items from blockIdx (4096 nonzeros each), so no
// plan or item table is needed either.
#include <cstring>
#include <mutex>

#include <cuda.h>

#include "kernels_impl.cuh"

namespace sparsep {
namespace noalloc {

constexpr uint32_t ELEMS_PER_ITEM = 4096;
constexpr uint32_t MAX_ITEMS = 1u << 16;  // nonzeros <= 2^28 (one carry slot per item)

// [0, MAX_ITEMS): carry values, [MAX_ITEMS, 2*MAX_ITEMS): carry targets,
// [2*MAX_ITEMS]: completion counter
static __device__ __align__(256) unsigned long long g_scratch[2 * MAX_ITEMS + 2];

__global__ void __launch_bounds__(256) coo_f32(Params<float> P, uint64_t nnz) {
  __shared__ uint32_t is_last;
  const uint32_t k = blockIdx.x;
  const auto *el = reinterpret_cast<const sparsep_elem_f32 *>(P.elems);
  Item it;
  it.a0 = (uint64_t)k * ELEMS_PER_ITEM;
  it.a1 = it.a0 + ELEMS_PER_ITEM < nnz ? it.a0 + ELEMS_PER_ITEM : nnz;
  it.ptr_base = it.nnz_base = 0;
  it.row_off = it.col_off = 0;
  // item k owns the rows from its first nonzero's row to the next item's first
  // row (clamped to nrows: a row index out of range, which is the caller's
  // error, then writes nothing instead of walking past y)
  const uint32_t f0 = k == 0 ? 0u : el[it.a0].rowind, f1 = k + 1 == P.nitems ? P.nrows : el[it.a1].rowind;
  it.own0 = f0 < P.nrows ? f0 : P.nrows;
  it.own1 = f1 < P.nrows ? f1 : P.nrows;
  if (it.own1 < it.own0) it.own1 = it.own0;
  it.xlo = it.xw = 0;
  it.slot = 0;
  it.kind = ITEM_ELEMS;
  it.lanes = 0;
  it.row_end = P.nrows;
  elems_lf<float, 1, 0, 0>(P, it, P.x, k, 1);
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    is_last = atomicAdd(P.done, 1u) == P.nitems - 1;
  }
  __syncthreads();
  if (is_last) {
    __threadfence();
    carry_fixup<float>(P, P.nitems, 1);
    if (threadIdx.x == 0) *P.done = 0;
  }
}

// Device address of g_scratch, looked up once per device and context: a
// device reset gives the device a new primary context (and the library's
// device image a new address), so the lookup is redone when the current
// context is not the one the address was found in.
using CtxGetCurrent = CUresult (*)(CUcontext *);
static CtxGetCurrent ctx_get_current() {
  static const CtxGetCurrent fn = [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<CtxGetCurrent>(f);
  }();
  return fn;
}
struct Slot {
  CUcontext ctx = nullptr;
  unsigned long long *addr = nullptr;
};
static Slot g_slot[64];
static std::mutex g_mu;

}  // namespace noalloc
}  // namespace sparsep

using namespace sparsep;

static int noalloc_status(cudaError_t e) {
  if (e == cudaSuccess) return SPARSEP_OK;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver || e == cudaErrorNoKernelImageForDevice)
    return SPARSEP_ENODEV;
  return SPARSEP_EIO;
}

extern "C" int sparsep_spmv_cooe_f32_noalloc(const sparsep_elem_f32 *d_elems, uint32_t nnz, uint32_t nrows,
                                             uint32_t ncols, const float *d_x, float *d_y, void *stream) {
  if (!d_x || !d_y || (nnz && !d_elems)) return SPARSEP_EINVAL;
  if ((reinterpret_cast<uintptr_t>(d_elems) & 15) != 0) return SPARSEP_EINVAL;  // 16-byte vector loads
  const uint64_t nitems = ((uint64_t)nnz + noalloc::ELEMS_PER_ITEM - 1) / noalloc::ELEMS_PER_ITEM;
  if (nitems > noalloc::MAX_ITEMS) return SPARSEP_ERANGE;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return noalloc_status(e);
  if (dev < 0 || dev >= 64) return SPARSEP_ENODEV;
  // set-up, once per device (and again after a device reset): the array's
  // device address; the first call on a device should come before any
  // stream capture
  CUcontext ctx = nullptr;
  if (noalloc::ctx_get_current() && noalloc::ctx_get_current()(&ctx) != CUDA_SUCCESS) ctx = nullptr;
  unsigned long long *scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(noalloc::g_mu);
    noalloc::Slot &sl = noalloc::g_slot[dev];
    if (!sl.addr || sl.ctx != ctx) {
      void *p = nullptr;
      e = cudaGetSymbolAddress(&p, noalloc::g_scratch);
      if (e != cudaSuccess) return noalloc_status(e);
      sl.addr = static_cast<unsigned long long *>(p);
      sl.ctx = ctx;
    }
    scratch = sl.addr;
  }
  if (nnz == 0) return noalloc_status(cudaMemsetAsync(d_y, 0, (size_t)nrows * sizeof(float), st));
  // the completion counter must start at zero
  e = cudaMemsetAsync(scratch + 2 * noalloc::MAX_ITEMS, 0, sizeof(unsigned long long), st);
  if (e != cudaSuccess) return noalloc_status(e);
  Params<float> P;
  std::memset(&P, 0, sizeof P);
  P.nitems = (uint32_t)nitems;
  P.nrows = nrows;
  P.ncols = ncols;
  P.elems = d_elems;
  P.x = d_x;
  P.y = d_y;
  P.out_mode = OUT_DIRECT;
  P.carry_val = scratch;
  P.carry_idx = scratch + noalloc::MAX_ITEMS;
  P.done = reinterpret_cast<unsigned int *>(scratch + 2 * noalloc::MAX_ITEMS);
  P.n_elems = nnz;  // no padding past the caller's last nonzero
  P.n_x = ncols;
  P.n_xalloc = ncols;
  P.n_carry = nitems;
  P.nslots = 1;
  noalloc::coo_f32<<<(unsigned)nitems, 256, 0, st>>>(P, nnz);
  return noalloc_status(cudaGetLastError());
}
