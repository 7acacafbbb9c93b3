// Command-line driver with the flags and timing lines of the reference's
// single-device program (main, src/spai_single_dcu.cpp:2692-2916):
//   spai_single_dcu [--matrix <path>] [--strategy <label>] [--device <id>]
// It reads the matrix (readMatrixToCSC semantics), uploads A and builds M on
// the device (preconditioningTime = the upload + the build, as the reference
// adds its H2D time to StaticSPAIv20's), then solves A x = b with the
// reference's settings -- b = 1, x0 = 1, ||r||_2 < 1e-7 absolute, MAX_ITER
// 10000 -- (solvingTime = the x/b upload + the solve, which here includes the
// CSC->CSR/SELL layout of A and M), and prints
//   iter_times = <iters>, err/err0=<final ||r||>
//   preconditioningTime = : <ms> ms
//   solvingTime = : <ms> ms
//   totalTime = : <ms> ms
// in the reference's formats.  The device description lines are printed in
// English.  Exit status 0 on success (also when the solver stops at
// MAX_ITER, as the reference's does), 1 on a read or library error.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "dcu_spai.h"

namespace {

struct Timer {
  cudaEvent_t a{}, b{};
  Timer() {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
  }
  ~Timer() {
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  }
  void start() { cudaEventRecord(a, 0); }
  float stop() {
    float ms = 0.f;
    cudaEventRecord(b, 0);
    cudaEventSynchronize(b);
    cudaEventElapsedTime(&ms, a, b);
    return ms;
  }
};

int fail(const char* what, dcu_spai_ctx* ctx) {
  fprintf(stderr, "error: %s%s%s\n", what, ctx ? ": " : "", ctx ? dcu_spai_last_error(ctx) : "");
  return 1;
}

}  // namespace

int main(int argc, char** argv) {
  std::string filename = "matrices/circuit_2.mtx";
  std::string strategy = "static";
  int deviceId = 0;
  for (int i = 1; i < argc; ++i) {
    if (!strcmp(argv[i], "--matrix") && i + 1 < argc) {
      filename = argv[++i];
    } else if (!strcmp(argv[i], "--strategy") && i + 1 < argc) {
      strategy = argv[++i];
    } else if (!strcmp(argv[i], "--device") && i + 1 < argc) {
      deviceId = atoi(argv[++i]);
    } else if (!strcmp(argv[i], "--help") || !strcmp(argv[i], "-h")) {
      printf("usage: %s [--matrix <path>] [--strategy <label>] [--device <id>]\n", argv[0]);
      return 0;
    }
  }
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count < 1) {
    printf("error: no CUDA device found\n");
    return 1;
  }
  if (deviceId < 0 || deviceId >= count) deviceId = 0;  // as the reference (:2711)
  printf("detected %d device(s), running on device %d\n", count, deviceId);
  cudaSetDevice(deviceId);
  cudaDeviceProp prop{};
  cudaGetDeviceProperties(&prop, deviceId);
  printf("device: %s\n", prop.name);
  printf("compute capability: %d.%d\n", prop.major, prop.minor);
  printf("warp size: %d\n", prop.warpSize);
  printf("strategy label: %s\n", strategy.c_str());
  printf("matrix file: %s\n", filename.c_str());

  int n = 0, nnz = 0;
  int *hp = nullptr, *hi = nullptr;
  double* hv = nullptr;
  if (dcu_mtx_read(filename.c_str(), &n, &nnz, &hp, &hi, &hv) != 0 || n <= 0 || !hp || !hi || !hv) {
    printf("error: cannot read the matrix or it is invalid: %s\n", filename.c_str());
    return 1;
  }
  dcu_spai_ctx* ctx = nullptr;
  if (dcu_spai_create(&ctx, deviceId, 0) != DCU_OK) return fail("cannot create a context", nullptr);
  // Each timed library call returns after its work has finished on the
  // device, so the events on the legacy stream bracket it as a whole.

  Timer t;
  float preconditioningTime = 0.f, solvingTime = 0.f;
  printf("--------Transfer A values to GPU\n");
  t.start();
  int *dp = nullptr, *di = nullptr;
  double *dv = nullptr, *dm = nullptr;
  cudaMalloc(&dp, sizeof(int) * (size_t)(n + 1));
  cudaMalloc(&di, sizeof(int) * (size_t)(nnz > 0 ? nnz : 1));
  cudaMalloc(&dv, sizeof(double) * (size_t)(nnz > 0 ? nnz : 1));
  cudaMalloc(&dm, sizeof(double) * (size_t)(nnz > 0 ? nnz : 1));
  cudaMemcpyAsync(dv, hv, sizeof(double) * (size_t)nnz, cudaMemcpyHostToDevice, 0);
  cudaMemcpyAsync(di, hi, sizeof(int) * (size_t)nnz, cudaMemcpyHostToDevice, 0);
  cudaMemcpyAsync(dp, hp, sizeof(int) * (size_t)(n + 1), cudaMemcpyHostToDevice, 0);
  float ms = t.stop();
  if (cudaGetLastError() != cudaSuccess) return fail("device allocation or copy failed", nullptr);
  printf("elapsedTime = : %8.4f ms \n ", ms);
  preconditioningTime += ms;

  dcu_options o;
  dcu_options_default(&o);
  dcu_build_info bi{};
  t.start();
  if (dcu_spai_build_d(ctx, n, nnz, dp, di, dv, &o, dm, nullptr, &bi) != DCU_OK)
    return fail("SPAI build failed", ctx);
  ms = t.stop();
  printf("SPAI build: n = %d, nnz = %d, max |J| = %d, max |I| = %d, singular columns = %d\n", n, nnz, bi.max_nj,
         bi.max_ni, bi.cols_singular);
  printf("elapsedTime = : %8.4f ms \n ", ms);
  preconditioningTime += ms;

  std::vector<double> ones((size_t)n, 1.0);
  double *db = nullptr, *dx = nullptr;
  t.start();
  cudaMalloc(&db, sizeof(double) * (size_t)n);
  cudaMalloc(&dx, sizeof(double) * (size_t)n);
  cudaMemcpyAsync(dx, ones.data(), sizeof(double) * (size_t)n, cudaMemcpyHostToDevice, 0);
  cudaMemcpyAsync(db, ones.data(), sizeof(double) * (size_t)n, cudaMemcpyHostToDevice, 0);
  dcu_options so;
  dcu_options_default(&so);
  so.tol_mode = DCU_TOL_ABS;
  so.tol = 1e-7;
  so.maxiter = 10000;
  so.verify = 0;  // stop on the recurrence residual, as the reference
  dcu_solve_info si{};
  if (dcu_bicgstab_d(ctx, n, nnz, dp, di, dv, dm, db, dx, &so, &si) != DCU_OK) return fail("solve failed", ctx);
  ms = t.stop();
  printf("iter_times = %d, err/err0=%18.14f \n", si.iters, si.res);
  printf("elapsedTime = : %8.4f ms \n ", ms);
  solvingTime += ms;

  printf("-----------------++++++++++++++++++++++++++++++++++++++++\n");
  printf("preconditioningTime = : %12.4f ms \n ", preconditioningTime);
  printf("solvingTime = : %12.4f ms \n ", solvingTime);
  printf("\n");
  printf("totalTime = : %12.4f ms \n ", preconditioningTime + solvingTime);

  cudaFree(dp);
  cudaFree(di);
  cudaFree(dv);
  cudaFree(dm);
  cudaFree(db);
  cudaFree(dx);
  dcu_spai_destroy(ctx);
  dcu_mtx_free(hp);
  dcu_mtx_free(hi);
  dcu_mtx_free(hv);
  return 0;
}
