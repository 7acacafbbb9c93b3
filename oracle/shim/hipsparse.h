// Host stand-in for <hipsparse.h>: the generic CSR SpMV of the reference's
// BiCGSTAB (see rocm_shim_blas.h for the arithmetic).
#pragma once

#include <cstddef>

typedef enum { HIPSPARSE_STATUS_SUCCESS = 0 } hipsparseStatus_t;
typedef struct hipsparse_shim_handle* hipsparseHandle_t;
typedef enum { HIPSPARSE_INDEX_32I = 0 } hipsparseIndexType_t;
typedef enum { HIPSPARSE_INDEX_BASE_ZERO = 0 } hipsparseIndexBase_t;
typedef enum { HIP_R_64F = 0 } hipDataType;
typedef enum { HIPSPARSE_OPERATION_NON_TRANSPOSE = 0 } hipsparseOperation_t;
typedef enum { HIPSPARSE_MV_ALG_DEFAULT = 0 } hipsparseSpMVAlg_t;

struct hipsparse_shim_csr {
  long rows, cols, nnz;
  const int* rp;
  const int* ci;
  const double* v;
};
struct hipsparse_shim_vec {
  long n;
  double* p;
};
typedef hipsparse_shim_csr* hipsparseSpMatDescr_t;
typedef hipsparse_shim_vec* hipsparseDnVecDescr_t;

inline hipsparseStatus_t hipsparseCreate(hipsparseHandle_t* h) {
  *h = nullptr;
  return HIPSPARSE_STATUS_SUCCESS;
}
inline hipsparseStatus_t hipsparseDestroy(hipsparseHandle_t) { return HIPSPARSE_STATUS_SUCCESS; }
inline hipsparseStatus_t hipsparseCreateCsr(hipsparseSpMatDescr_t* m, long rows, long cols, long nnz, void* rp,
                                            void* ci, void* v, hipsparseIndexType_t, hipsparseIndexType_t,
                                            hipsparseIndexBase_t, hipDataType) {
  *m = new hipsparse_shim_csr{rows, cols, nnz, (const int*)rp, (const int*)ci, (const double*)v};
  return HIPSPARSE_STATUS_SUCCESS;
}
inline hipsparseStatus_t hipsparseDestroySpMat(hipsparseSpMatDescr_t m) {
  delete m;
  return HIPSPARSE_STATUS_SUCCESS;
}
inline hipsparseStatus_t hipsparseCreateDnVec(hipsparseDnVecDescr_t* d, long n, void* p, hipDataType) {
  *d = new hipsparse_shim_vec{n, (double*)p};
  return HIPSPARSE_STATUS_SUCCESS;
}
inline hipsparseStatus_t hipsparseDestroyDnVec(hipsparseDnVecDescr_t d) {
  delete d;
  return HIPSPARSE_STATUS_SUCCESS;
}
inline hipsparseStatus_t hipsparseSpMV_bufferSize(hipsparseHandle_t, hipsparseOperation_t, const void*,
                                                  hipsparseSpMatDescr_t, hipsparseDnVecDescr_t, const void*,
                                                  hipsparseDnVecDescr_t, hipDataType, hipsparseSpMVAlg_t,
                                                  size_t* bytes) {
  *bytes = 0;
  return HIPSPARSE_STATUS_SUCCESS;
}
// y = alpha A x + beta y (beta == 0 ignores y's old contents)
inline hipsparseStatus_t hipsparseSpMV(hipsparseHandle_t, hipsparseOperation_t, const void* alpha,
                                       hipsparseSpMatDescr_t A, hipsparseDnVecDescr_t x, const void* beta,
                                       hipsparseDnVecDescr_t y, hipDataType, hipsparseSpMVAlg_t, void*) {
  const double a = *(const double*)alpha, b = *(const double*)beta;
  for (long r = 0; r < A->rows; ++r) {
    double acc = 0.0;
    for (int e = A->rp[r]; e < A->rp[r + 1]; ++e) acc += A->v[e] * x->p[A->ci[e]];
    y->p[r] = (a == 1.0 ? acc : a * acc) + (b == 0.0 ? 0.0 : b * y->p[r]);
  }
  return HIPSPARSE_STATUS_SUCCESS;
}
