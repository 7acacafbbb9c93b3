// C++ drop-in entry points of include/common/spai_multi_dcu_api.h, built with
// g++ on top of the C ABI (dcu_spai.h).  Reference behaviour is cited per
// function; the differences are listed in the header.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <new>
#include <string>

#include "common/spai_multi_dcu_api.h"
#include "dcu_spai.h"

struct MultiDCU_Context {
  int numDCUs = 1;          // one B200 stands in for every DCU unit
  dcu_spai_ctx* spai = nullptr;
  CSC_Matrix devA{};        // device copy of A (the reference's devCSC_A[0])
  size_t devA_cap_n = 0, devA_cap_nnz = 0;
  std::string err;
};

namespace {

void free_dev_csc(CSC_Matrix* m) {
  if (m->mPtr) cudaFree(m->mPtr);
  if (m->mIndex) cudaFree(m->mIndex);
  if (m->mData) cudaFree(m->mData);
  m->mPtr = nullptr;
  m->mIndex = nullptr;
  m->mData = nullptr;
}

bool cuda_ok(MultiDCU_Context* ctx, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return true;
  ctx->err = std::string(what) + ": " + cudaGetErrorString(e);
  return false;
}

// Upload host A into ctx->devA (grown on demand).
bool upload_a(MultiDCU_Context* ctx, const CSC_Matrix* A) {
  const size_t n = (size_t)A->n, nnz = (size_t)(A->nonzeroes > 0 ? A->nonzeroes : 0);
  if (ctx->devA_cap_n < n || ctx->devA_cap_nnz < nnz || !ctx->devA.mPtr) {
    free_dev_csc(&ctx->devA);
    if (!cuda_ok(ctx, cudaMalloc((void**)&ctx->devA.mPtr, sizeof(int) * (n + 1)), "cudaMalloc") ||
        !cuda_ok(ctx, cudaMalloc((void**)&ctx->devA.mIndex, sizeof(int) * (nnz ? nnz : 1)), "cudaMalloc") ||
        !cuda_ok(ctx, cudaMalloc((void**)&ctx->devA.mData, sizeof(double) * (nnz ? nnz : 1)), "cudaMalloc"))
      return false;
    ctx->devA_cap_n = n;
    ctx->devA_cap_nnz = nnz;
  }
  ctx->devA.n = ctx->devA.nRow = ctx->devA.nCol = A->n;
  ctx->devA.nonzeroes = (int)nnz;
  if (!cuda_ok(ctx, cudaMemcpy(ctx->devA.mPtr, A->mPtr, sizeof(int) * (n + 1), cudaMemcpyHostToDevice), "H2D"))
    return false;
  if (nnz) {
    if (!cuda_ok(ctx, cudaMemcpy(ctx->devA.mIndex, A->mIndex, sizeof(int) * nnz, cudaMemcpyHostToDevice), "H2D") ||
        !cuda_ok(ctx, cudaMemcpy(ctx->devA.mData, A->mData, sizeof(double) * nnz, cudaMemcpyHostToDevice), "H2D"))
      return false;
  }
  return true;
}

bool valid_host_csc(MultiDCU_Context* ctx, const CSC_Matrix* A) {
  // validateMatrix, src/spai_multi_dcu.cpp:1455-1480
  if (!A) { ctx->err = "matrix is null"; return false; }
  if (A->n <= 0 || A->nCol <= 0 || A->nRow <= 0) { ctx->err = "matrix dimensions are invalid"; return false; }
  if (A->nonzeroes < 0) { ctx->err = "negative nonzero count"; return false; }
  if (!A->mPtr || (A->nonzeroes > 0 && (!A->mIndex || !A->mData))) { ctx->err = "matrix arrays are null"; return false; }
  if (A->nRow != A->nCol || A->n != A->nCol) { ctx->err = "matrix must be square"; return false; }
  return true;
}

float run_spai(MultiDCU_Context* ctx, const CSC_Matrix* A, CSC_Matrix* devM, int colStart, int colEnd,
               int schedule) {
  if (!ctx || !ctx->spai) return -1.0f;
  if (!valid_host_csc(ctx, A) || !devM) {
    if (!devM) ctx->err = "output matrix is null";
    return -1.0f;
  }
  // the reference returns 0.0f for an invalid range (:1560-1561)
  if (colStart < 0 || colEnd > A->nCol || colStart >= colEnd) {
    ctx->err = "invalid column range";
    return -1.0f;
  }
  if (!upload_a(ctx, A)) return -1.0f;
  const int n = A->n, nnz = A->nonzeroes;
  CSC_Matrix M{};
  M.n = M.nRow = M.nCol = n;
  M.nonzeroes = nnz;
  if (!cuda_ok(ctx, cudaMalloc((void**)&M.mPtr, sizeof(int) * (size_t)(n + 1)), "cudaMalloc") ||
      !cuda_ok(ctx, cudaMalloc((void**)&M.mIndex, sizeof(int) * (size_t)(nnz > 0 ? nnz : 1)), "cudaMalloc") ||
      !cuda_ok(ctx, cudaMalloc((void**)&M.mData, sizeof(double) * (size_t)(nnz > 0 ? nnz : 1)), "cudaMalloc")) {
    free_dev_csc(&M);
    return -1.0f;
  }
  bool ok = cuda_ok(ctx, cudaMemcpy(M.mPtr, ctx->devA.mPtr, sizeof(int) * (size_t)(n + 1), cudaMemcpyDeviceToDevice),
                    "D2D");
  if (ok && nnz > 0)
    ok = cuda_ok(ctx, cudaMemcpy(M.mIndex, ctx->devA.mIndex, sizeof(int) * (size_t)nnz, cudaMemcpyDeviceToDevice),
                 "D2D");
  dcu_options opt;
  dcu_options_default(&opt);
  opt.schedule = schedule;
  opt.col_start = colStart;
  opt.col_end = colEnd;
  dcu_build_info info{};
  if (ok) {
    int rc = dcu_spai_build_d(ctx->spai, n, nnz, ctx->devA.mPtr, ctx->devA.mIndex, ctx->devA.mData, &opt, M.mData,
                              nullptr, &info);
    if (rc != DCU_OK) {
      ctx->err = dcu_spai_last_error(ctx->spai);
      ok = false;
    }
  }
  if (!ok) {
    free_dev_csc(&M);
    return -1.0f;
  }
  *devM = M;
  return info.ms;
}

}  // namespace

MultiDCU_Context* initMultiDCU(int requestedDCUs) {
  (void)requestedDCUs;  // capped to the devices used, like :1306-1312; one B200 here
  MultiDCU_Context* ctx = new (std::nothrow) MultiDCU_Context();
  if (!ctx) return nullptr;
  int rc = dcu_spai_create(&ctx->spai, 0, 0);
  if (rc != DCU_OK) {
    fprintf(stderr, "initMultiDCU: no usable CUDA device (status %d)\n", rc);
    delete ctx;
    return nullptr;
  }
  return ctx;
}

void cleanupMultiDCU(MultiDCU_Context* ctx) {
  if (!ctx) return;
  free_dev_csc(&ctx->devA);
  dcu_spai_destroy(ctx->spai);
  delete ctx;
}

float RunStaticSPAI_MultiDCU_MPI(MultiDCU_Context* ctx, const CSC_Matrix* CSC_A, CSC_Matrix* devCSC_M_global,
                                 int globalColStart, int globalColEnd) {
  return run_spai(ctx, CSC_A, devCSC_M_global, globalColStart, globalColEnd, DCU_SCHED_BALANCED_COLUMNS);
}

float RunDynamicSPAI_MultiDCU_MPI(MultiDCU_Context* ctx, const CSC_Matrix* CSC_A, CSC_Matrix* devCSC_M_global,
                                  int globalColStart, int globalColEnd) {
  return run_spai(ctx, CSC_A, devCSC_M_global, globalColStart, globalColEnd, DCU_SCHED_BALANCED_NNZ);
}

void replicateMatrixA(MultiDCU_Context* ctx, CSC_Matrix* CSC_A) {
  if (ctx && valid_host_csc(ctx, CSC_A)) upload_a(ctx, CSC_A);
}

CSC_Matrix* deviceMatrixA(MultiDCU_Context* ctx) { return (ctx && ctx->devA.mPtr) ? &ctx->devA : nullptr; }

int numDCUUnits(MultiDCU_Context* ctx) { return ctx ? ctx->numDCUs : 0; }

const char* lastErrorMultiDCU(MultiDCU_Context* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int runBiCGSTABOnRank0(CSC_Matrix* devA, CSC_Matrix* devM) {
  return runBiCGSTABOnRank0Info(devA, devM, nullptr, nullptr, nullptr, nullptr);
}

int runBiCGSTABOnRank0Info(CSC_Matrix* devA, CSC_Matrix* devM, double* solverMs, int* converged, double* tol,
                           int* maxIters) {
  if (solverMs) *solverMs = 0.0;
  if (converged) *converged = 0;
  if (tol) *tol = 1e-7;
  if (maxIters) *maxIters = 10000;
  if (!devA || !devM || devA->n <= 0 || devM->n != devA->n || devM->nonzeroes != devA->nonzeroes) return 0;
  const int n = devA->n;
  dcu_spai_ctx* s = nullptr;
  int dev = 0;
  cudaGetDevice(&dev);
  if (dcu_spai_create(&s, dev, 0) != DCU_OK) return 0;
  double *b = nullptr, *x = nullptr;
  int iters = 0;
  if (cudaMalloc((void**)&b, sizeof(double) * (size_t)n) == cudaSuccess &&
      cudaMalloc((void**)&x, sizeof(double) * (size_t)n) == cudaSuccess) {
    // b = 1, x0 = 1 (:1922-1927)
    double* h = new (std::nothrow) double[n];
    if (h) {
      for (int i = 0; i < n; ++i) h[i] = 1.0;
      cudaMemcpy(b, h, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice);
      cudaMemcpy(x, h, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice);
      delete[] h;
      dcu_options opt;
      dcu_options_default(&opt);
      opt.tol = 1e-7;
      opt.tol_mode = DCU_TOL_ABS;
      opt.maxiter = 10000;
      opt.verify = 0;
      dcu_solve_info info{};
      if (dcu_bicgstab_d(s, n, devA->nonzeroes, devA->mPtr, devA->mIndex, devA->mData, devM->mData, b, x, &opt,
                         &info) == DCU_OK) {
        // a breakdown leaves NaN in the reference, whose loop then runs to MAX_ITER
        iters = (info.status == DCU_SOLVE_BREAKDOWN) ? opt.maxiter : info.iters;
        if (solverMs) *solverMs = info.ms;
        if (converged) *converged = info.status == DCU_SOLVE_CONVERGED;
      }
    }
  }
  if (b) cudaFree(b);
  if (x) cudaFree(x);
  dcu_spai_destroy(s);
  return iters;
}

void printAlgoReport(const char* mode, int dcuUnits, const char* partition, float preconditionerMs,
                     int iterationCount) {
  printf("[ALGO_REPORT] mode=%s, dcu_units=%d, partition=%s, preconditioner_ms=%.4f, iteration_count=%d\n", mode,
         dcuUnits, partition, preconditionerMs, iterationCount);
  fflush(stdout);
}
