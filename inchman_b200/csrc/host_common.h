// Error reporting shared by the host translation units of the C ABI.
#pragma once
#include <cstdarg>
#include <cstdio>
#include <string>
#include <cuda_runtime.h>

namespace gpgmp {
// Records a message for gpgmp_last_error() on the calling thread and returns code.
int set_error(int code, const char* fmt, ...);

// Stream-ordered allocation from a pool per device that keeps freed memory mapped
// (devpool.cpp); for entry points that allocate device copies of host buffers on
// every call.
cudaError_t pool_alloc(void** p, size_t bytes, cudaStream_t st);
cudaError_t pool_free(void* p, cudaStream_t st);
}  // namespace gpgmp
