// Host (CPU) stand-ins for the handful of HIP runtime, hipBLAS and hipSPARSE
// calls that the reference's BiCGSTAB (include/bicgstab/bicgstab_solver.h)
// makes, so that file compiles unmodified as plain C++ into the oracle's
// reference harness.  TEST INFRASTRUCTURE ONLY.
//
// "Device" memory is host memory.  The library arithmetic is restated from
// the routines' published definitions (ROCm is not present here, and the
// reference does not pin its version): dot and nrm2 sum in fixed chunks of
// 8192 elements, then the chunk sums in order (the oracle's own reduction);
// axpy y = alpha x + y, scal x = alpha x, copy; SpMV y = alpha A x + beta y
// with each CSR row summed in stored order.  What this pins is the order of
// the reference's own recurrence steps, not the libraries' rounding.
#pragma once

#include <cmath>
#include <cstddef>
#include <cstdlib>
#include <cstring>

namespace rocm_shim {
constexpr long kChunk = 8192;
inline double chunked_dot(long n, const double* a, long inca, const double* b, long incb) {
  double t = 0.0;
  for (long s = 0; s < n; s += kChunk) {
    long e = s + kChunk < n ? s + kChunk : n;
    double acc = 0.0;
    for (long i = s; i < e; ++i) acc += a[i * inca] * b[i * incb];
    t += acc;
  }
  return t;
}
}  // namespace rocm_shim
