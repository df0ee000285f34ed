// fault.hpp -- device allocations of the library and the test-support fault
// switches (fault.cpp).
#pragma once
#include <cstddef>
#include <cuda_runtime.h>

namespace sparsep {

// Every device allocation of the library goes through dev_malloc / dev_free:
// test support can make the n-th allocation fail (as cudaMalloc does when the
// device is full), and the count of live allocations shows leaks.
cudaError_t dev_malloc(void **p, size_t bytes);
void dev_free(void *p);

// Nonzero while test support asks the kernels with bounded staging waits to
// add one wait that nothing completes (after their own copies have landed).
int wait_fault();

}  // namespace sparsep
