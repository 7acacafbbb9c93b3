// Host stand-in for <hipblas.h>: the level-1 routines of the reference's
// BiCGSTAB (see rocm_shim_blas.h for the arithmetic).
#pragma once

#include <cmath>

#include "rocm_shim_blas.h"

typedef struct hipblas_shim_handle* hipblasHandle_t;
typedef enum { HIPBLAS_STATUS_SUCCESS = 0 } hipblasStatus_t;

inline hipblasStatus_t hipblasCreate(hipblasHandle_t* h) {
  *h = nullptr;
  return HIPBLAS_STATUS_SUCCESS;
}
inline hipblasStatus_t hipblasDestroy(hipblasHandle_t) { return HIPBLAS_STATUS_SUCCESS; }
inline hipblasStatus_t hipblasDdot(hipblasHandle_t, int n, const double* x, int incx, const double* y, int incy,
                                   double* result) {
  *result = rocm_shim::chunked_dot(n, x, incx, y, incy);
  return HIPBLAS_STATUS_SUCCESS;
}
inline hipblasStatus_t hipblasDnrm2(hipblasHandle_t, int n, const double* x, int incx, double* result) {
  *result = std::sqrt(rocm_shim::chunked_dot(n, x, incx, x, incx));
  return HIPBLAS_STATUS_SUCCESS;
}
inline hipblasStatus_t hipblasDaxpy(hipblasHandle_t, int n, const double* alpha, const double* x, int incx,
                                    double* y, int incy) {
  const double a = *alpha;
  for (long i = 0; i < n; ++i) y[i * incy] = a * x[i * incx] + y[i * incy];
  return HIPBLAS_STATUS_SUCCESS;
}
inline hipblasStatus_t hipblasDscal(hipblasHandle_t, int n, const double* alpha, double* x, int incx) {
  const double a = *alpha;
  for (long i = 0; i < n; ++i) x[i * incx] = a * x[i * incx];
  return HIPBLAS_STATUS_SUCCESS;
}
inline hipblasStatus_t hipblasDcopy(hipblasHandle_t, int n, const double* x, int incx, double* y, int incy) {
  for (long i = 0; i < n; ++i) y[i * incy] = x[i * incx];
  return HIPBLAS_STATUS_SUCCESS;
}
