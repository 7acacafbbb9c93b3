// Host stand-in for <hip/hip_runtime.h>: the memory calls the reference's
// BiCGSTAB makes, on host memory (see ../rocm_shim_blas.h).
#pragma once

#include <cstddef>
#include <cstdlib>
#include <cstring>

typedef int hipError_t;
enum { hipSuccess = 0 };
typedef enum { hipMemcpyHostToHost = 0, hipMemcpyHostToDevice = 1, hipMemcpyDeviceToHost = 2,
               hipMemcpyDeviceToDevice = 3, hipMemcpyDefault = 4 } hipMemcpyKind;

template <typename T>
inline hipError_t hipMalloc(T** p, size_t bytes) {
  *p = (T*)std::calloc(bytes ? bytes : 1, 1);
  return *p ? hipSuccess : 2;
}
inline hipError_t hipFree(void* p) {
  std::free(p);
  return hipSuccess;
}
inline hipError_t hipMemcpy(void* dst, const void* src, size_t bytes, hipMemcpyKind) {
  std::memmove(dst, src, bytes);
  return hipSuccess;
}
