// fault.cpp -- device allocations and failure injection for tests.
//
// No counterpart in the reference, whose failures abort (DPU_ASSERT,
// spmv/1D/CSR-row/host/app.c:91-93).  Here every failure is a status, and
// these switches let tests make the two kinds of failure happen on purpose
// without faulting a GPU: a device allocation that fails (SPARSEP_ENOMEM) and
// a bounded device wait that runs out (SPARSEP_ETIMEDOUT).
#include <atomic>

#include "fault.hpp"
#include "sparsep.h"

namespace sparsep {

static std::atomic<long long> g_live{0};  // live device allocations
static std::atomic<int> g_fail_in{0};     // the g_fail_in-th allocation from now fails (0: none)
static std::atomic<int> g_wait_fault{0};

cudaError_t dev_malloc(void **p, size_t bytes) {
  int n = g_fail_in.load();
  while (n > 0 && !g_fail_in.compare_exchange_weak(n, n - 1)) {
  }
  if (n == 1) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  const cudaError_t e = cudaMalloc(p, bytes);
  if (e == cudaSuccess) ++g_live;
  return e;
}

void dev_free(void *p) {
  if (!p) return;
  cudaFree(p);
  --g_live;
}

int wait_fault() { return g_wait_fault.load(); }

}  // namespace sparsep

extern "C" {

int sparsep_test_fail_alloc(int nth) {
  if (nth < 0) return SPARSEP_EINVAL;
  sparsep::g_fail_in.store(nth);
  return SPARSEP_OK;
}

long long sparsep_test_live_allocations(void) { return sparsep::g_live.load(); }

int sparsep_test_wait_fault(int on) {
  sparsep::g_wait_fault.store(on ? 1 : 0);
  return SPARSEP_OK;
}

}  // extern "C"
