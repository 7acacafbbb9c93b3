// Command-line driver with the flags of the reference's spai_multi_dcu
// (printUsage / main, src/spai_multi_dcu.cpp:2386-2440):
//   spai_multi_dcu [dcu_count] [--algo static|dynamic]
//                  [--partition balanced_columns|balanced_nnz]
//                  [--matrix <path>] [--precondition-only] [--help]
// It reads the matrix, builds M on one B200 (RunStatic/RunDynamic...), runs
// BiCGSTAB with the reference's settings (runBiCGSTABOnRank0) unless
// --precondition-only, and prints the [ALGO_REPORT] line.  MPI launchers
// with one rank behave the same; more ranks are not used.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "common/spai_multi_dcu_api.h"
#include "dcu_spai.h"

static void usage(const char* prog) {
  printf("usage: %s [dcu_count] [--algo static|dynamic] [--partition balanced_columns|balanced_nnz]\n", prog);
  printf("          [--matrix <path>] [--precondition-only] [--help]\n");
}

int main(int argc, char** argv) {
  std::string filename = "matrices/circuit_2.mtx";
  bool useNnz = false, partitionGiven = false, precondOnly = false;
  int requested = -1;
  std::string algo = "static";
  for (int i = 1; i < argc; ++i) {
    if (!strcmp(argv[i], "--help") || !strcmp(argv[i], "-h")) {
      usage(argv[0]);
      return 0;
    } else if (!strcmp(argv[i], "--matrix") && i + 1 < argc) {
      filename = argv[++i];
    } else if (!strcmp(argv[i], "--algo") && i + 1 < argc) {
      algo = argv[++i];
    } else if (!strcmp(argv[i], "--partition") && i + 1 < argc) {
      partitionGiven = true;
      useNnz = !strcmp(argv[++i], "balanced_nnz");
    } else if (!strcmp(argv[i], "--precondition-only")) {
      precondOnly = true;
    } else if (argv[i][0] != '-') {
      requested = atoi(argv[i]);
    }
  }
  if (!partitionGiven) useNnz = (algo == "dynamic");

  CSC_Matrix A{};
  if (dcu_mtx_read(filename.c_str(), &A.n, &A.nonzeroes, &A.mPtr, &A.mIndex, &A.mData) != 0 || A.n <= 0) {
    fprintf(stderr, "cannot read matrix %s\n", filename.c_str());
    return EXIT_FAILURE;
  }
  A.nRow = A.nCol = A.n;
  printf("matrix %s: n = %d, nnz = %d\n", filename.c_str(), A.n, A.nonzeroes);

  MultiDCU_Context* ctx = initMultiDCU(requested);
  if (!ctx) return EXIT_FAILURE;
  CSC_Matrix M{};
  float ms = (algo == "dynamic") ? RunDynamicSPAI_MultiDCU_MPI(ctx, &A, &M, 0, A.nCol)
                                 : RunStaticSPAI_MultiDCU_MPI(ctx, &A, &M, 0, A.nCol);
  if (ms < 0.0f) {
    fprintf(stderr, "SPAI build failed: %s\n", lastErrorMultiDCU(ctx));
    cleanupMultiDCU(ctx);
    return EXIT_FAILURE;
  }
  int iters = 0, converged = 0, maxIters = 0;
  double solverMs = 0.0, tol = 0.0;
  if (!precondOnly) iters = runBiCGSTABOnRank0Info(deviceMatrixA(ctx), &M, &solverMs, &converged, &tol, &maxIters);
  printAlgoReport(algo.c_str(), numDCUUnits(ctx), useNnz ? "balanced_nnz" : "balanced_columns", ms, iters);
  // Not printed by the reference: the solver's own numbers, for the results
  // database (dcu_b200/results_db.py), on a line of its own so that scripts
  // reading [ALGO_REPORT] are unaffected.
  if (!precondOnly)
    printf("[SOLVER_REPORT] gpupbicgstab_ms=%.4f, converged=%d, solver_tol=%.3e, max_iters=%d\n", solverMs, converged,
           tol, maxIters);
  cudaFree(M.mPtr);
  cudaFree(M.mIndex);
  cudaFree(M.mData);
  cleanupMultiDCU(ctx);
  dcu_mtx_free(A.mPtr);
  dcu_mtx_free(A.mIndex);
  dcu_mtx_free(A.mData);
  return EXIT_SUCCESS;
}
