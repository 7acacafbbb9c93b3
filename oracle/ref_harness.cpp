// Harness that compiles the reference's own CPU helpers, unmodified, from
// where they lie in the reference tree (include path given by the Makefile),
// into oracle/_ref/libref_harness.so.  TEST INFRASTRUCTURE ONLY: it pins the
// oracle's MatrixMarket reader, CSC->CSR and |I_k| sizing against the
// reference's code (tests/test_oracle_pinned.py).  Nothing here ships.
//
// Wrapped reference functions:
//   readMatrixToCSC   include/common/read.h:1296-1320
//   computeN1MAX      include/common/init.h:43-75 (whole matrix: max |I_k|;
//                     one-column M per call: |I_k| of every column)
//   computeN2MAX      include/common/init.h:80-92
//   CSC2CSR           include/common/assemble.h:34-67
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <unistd.h>
#include <fcntl.h>

#include "dataType.h"
#include "read.h"
#include "init.h"
#include "assemble.h"

namespace {
// The reference helpers print progress to stdout; silence it around calls.
struct Quiet {
  int saved;
  Quiet() {
    fflush(stdout);
    saved = dup(1);
    int devnull = open("/dev/null", O_WRONLY);
    dup2(devnull, 1);
    close(devnull);
  }
  ~Quiet() {
    fflush(stdout);
    dup2(saved, 1);
    close(saved);
  }
};
}  // namespace

extern "C" {

void ref_free(void* p) { free(p); }

int ref_read(const char* path, int* n, int* nnz, int** ptr, int** idx, double** val) {
  CSC_Matrix A;
  memset(&A, 0, sizeof A);
  {
    Quiet q;
    readMatrixToCSC(const_cast<char*>(path), &A);
  }
  *n = A.n;
  *nnz = A.nonzeroes;
  *ptr = A.mPtr;
  *idx = A.mIndex;
  *val = A.mData;
  return 0;
}

int ref_n1max(int n, int* ptr, int* idx, double* val) {
  CSC_Matrix A;
  A.n = A.nRow = A.nCol = n;
  A.nonzeroes = ptr[n];
  A.mPtr = ptr;
  A.mIndex = idx;
  A.mData = val;
  return computeN1MAX(&A, &A);
}

// |I_k| of every column k in [c0, c1), each from computeN1MAX called on a
// one-column M whose only column holds J_k = the rows of A(:, k)
// (mPtr = {0, |J_k|}, mIndex = A's indices of column k).  The reference
// function keeps its own vector per call, so columns run in parallel.
void ref_n1_per_column(int n, int* ptr, int* idx, double* val, int c0, int c1, int* out) {
  CSC_Matrix A;
  A.n = A.nRow = A.nCol = n;
  A.nonzeroes = ptr[n];
  A.mPtr = ptr;
  A.mIndex = idx;
  A.mData = val;
#pragma omp parallel for schedule(dynamic, 256)
  for (int k = c0; k < c1; ++k) {
    int mp[2] = {0, ptr[k + 1] - ptr[k]};
    CSC_Matrix M;
    M.n = M.nCol = 1;
    M.nRow = n;
    M.nonzeroes = mp[1];
    M.mPtr = mp;
    M.mIndex = idx + ptr[k];
    M.mData = val + ptr[k];
    out[k - c0] = computeN1MAX(&A, &M);
  }
}

int ref_n2max(int n, int* ptr, int* idx, double* val) {
  CSC_Matrix A;
  A.n = A.nRow = A.nCol = n;
  A.nonzeroes = ptr[n];
  A.mPtr = ptr;
  A.mIndex = idx;
  A.mData = val;
  return computeN2MAX(&A);
}

void ref_csc2csr(int n, int* ptr, int* idx, double* val, int* rptr, int* ridx, double* rval) {
  CSC_Matrix A;
  A.n = A.nRow = A.nCol = n;
  A.nonzeroes = ptr[n];
  A.mPtr = ptr;
  A.mIndex = idx;
  A.mData = val;
  CSR_Matrix R;
  memset(&R, 0, sizeof R);
  {
    Quiet q;
    CSC2CSR(&A, &R, (unsigned)n);
  }
  memcpy(rptr, R.mPtr, sizeof(int) * (n + 1));
  memcpy(ridx, R.mIndex, sizeof(int) * R.nonzeroes);
  memcpy(rval, R.mData, sizeof(double) * R.nonzeroes);
  free(R.mPtr);
  free(R.mIndex);
  free(R.mData);
}

}  // extern "C"
