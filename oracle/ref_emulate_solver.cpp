// The reference's BiCGSTAB (cublas2_pbicgstabv2, include/bicgstab/
// bicgstab_solver.h:33-275) compiled unmodified against the host stand-ins
// of oracle/shim/ (HIP runtime, hipBLAS, hipSPARSE), with A and M converted
// by the reference's CSC2CSR (include/common/assemble.h:34-67).  TEST
// INFRASTRUCTURE ONLY; part of oracle/_ref/libref_emu.so (see
// ref_emulate.cpp).  Compiled without floating-point contraction: the
// stand-ins restate the libraries' arithmetic as the oracle does, so that
// what differs between the two is the recurrence code alone.
#include <fcntl.h>
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "dataType.h"
#include "assemble.h"
#include "bicgstab/bicgstab_solver.h"

extern "C" {

// x (in: x0, out: the solution); b is not modified (the reference overwrites
// its b with A x on exit, so it runs on a copy).  TOL is the reference's
// absolute threshold on ||r||_2, MAX_ITER its cap.  Returns the reference's
// iter_times; *final_err = its final ||r||_2 (read from the line it prints).
int refemu_bicgstab(int n, int* ptr, int* idx, double* val, double* mval, const double* b, double* x, double tol,
                    int maxiter, double* final_err) {
  CSC_Matrix A{}, M{};
  A.n = A.nRow = A.nCol = M.n = M.nRow = M.nCol = n;
  A.nonzeroes = M.nonzeroes = ptr[n];
  A.mPtr = M.mPtr = ptr;
  A.mIndex = M.mIndex = idx;
  A.mData = val;
  M.mData = mval;
  CSR_Matrix Ar{}, Mr{};
  std::vector<double> bb(b, b + n);
  char path[] = "/tmp/refemu_bicgstabXXXXXX";
  int fd = mkstemp(path);
  if (fd < 0) return -1;
  fflush(stdout);
  int saved = dup(1);
  dup2(fd, 1);
  CSC2CSR(&A, &Ar, (unsigned)n);
  CSC2CSR(&M, &Mr, (unsigned)n);
  int it = cublas2_pbicgstabv2(&Ar, &Mr, bb.data(), x, tol, maxiter);
  fflush(stdout);
  dup2(saved, 1);
  close(saved);
  // the last "iter_times = %d, err/err0=%18.14f" line carries the final ||r||
  std::string text;
  lseek(fd, 0, SEEK_SET);
  char buf[4096];
  ssize_t k;
  while ((k = read(fd, buf, sizeof buf)) > 0) text.append(buf, (size_t)k);
  close(fd);
  unlink(path);
  if (final_err) {
    *final_err = -1.0;
    size_t pos = text.rfind("err/err0=");
    if (pos != std::string::npos) *final_err = strtod(text.c_str() + pos + 9, nullptr);
  }
  free(Ar.mPtr);
  free(Ar.mIndex);
  free(Ar.mData);
  free(Mr.mPtr);
  free(Mr.mIndex);
  free(Mr.mData);
  return it;
}

}  // extern "C"
