// The reference's own SPAI kernels and BiCGSTAB, executed on the host.
// TEST INFRASTRUCTURE ONLY (the oracle's reference harness): built by
// `make emu` into oracle/_ref/libref_emu.so, used by tests and by
// tests/golden/make_golden.py to pin the oracle's restatement against code
// the reference ships.  Nothing in the product links or loads it.
//
// * SPAI: the kernels of src/spai_single_dcu.cpp (computeJ*, computeI*,
//   ComputeTildeACSR, QR_RShared, ComputeTildeE*, Sol, modifyData*) are
//   compiled unmodified from oracle/_ref/ref_spai_kernels.inc (extracted from
//   the reference tree by oracle/extract_ref_kernels.py) and run on the SIMT
//   emulator of oracle/simt_emu.h with the reference's launch shapes: 256
//   threads per block, the logical warp width and shared-memory sizes chosen
//   from n2max / n1max as StaticSPAIv20 chooses them
//   (src/spai_single_dcu.cpp:1224-2687), the single-pass path when
//   nCol * n1max * n2max fits its compareSize, else the column tiles.
//   refemu_spai() below restates that host sequence (the file itself cannot
//   be compiled here: triple-chevron launches, HIP runtime).  One deliberate
//   difference: in the tiled path the tile may hold fewer columns than the
//   reference's, to bound host memory (the padded A(I,J) of one circuit_2
//   column is 46 MB); every column's result depends only on that column.
//   n2max and n1max come from the reference's CPU computeN2MAX/computeN1MAX
//   (include/common/init.h), equal to what its GPU sizing kernels find.
//   ComputeTildeE* run with a one-lane logical warp (see run_width): the
//   only kernel here whose lanes exchange data without a barrier in a way
//   that depends on lockstep execution.  (computeI*'s lanes read the
//   column's shared counter while others append to it; any order of those
//   appends gives the same set, which the kernel then sorts.)
//   Arrays the reference leaves uninitialised after hipMalloc are zeroed.
// * BiCGSTAB: cublas2_pbicgstabv2 (include/bicgstab/bicgstab_solver.h) is
//   compiled unmodified against the host stand-ins in oracle/shim/ for the HIP
//   runtime, hipBLAS and hipSPARSE; A and M reach it in CSR from the
//   reference's CSC2CSR (include/common/assemble.h).
//
// Compiled with -ffp-contract=fast and FMA (as HIP device code is compiled by
// default) for the kernels' arithmetic; the BiCGSTAB stand-ins are compiled
// in a separate unit without contraction (ref_emulate_solver.cpp).
#include <fcntl.h>
#include <unistd.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "simt_emu.h"

#include "dataType.h"
#include "init.h"

using std::sqrt;

#include "ref_spai_kernels.inc"

namespace {

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

constexpr int kThreads = 256;                       // threadsPerBlock (:1238)
constexpr long kCompareSize = 1024L * 1024 * 100 * 4 * 3;  // compareSize (:1495)

// Logical warp width of the J / I / A(I,J) / QR / E / Sol kernels: the n2max
// bucket (:1549-1571, :2153-2178, ...).
int width_of(int n2max) {
  if (n2max <= 2) return 2;
  if (n2max <= 4) return 4;
  if (n2max <= 8) return 8;
  if (n2max <= 16) return 16;
  if (n2max <= 32) return 32;
  if (n2max <= 64) return 64;
  if (n2max <= 128) return 128;
  return 256;
}

// Width of modifyData*: the bucket capped at 32 (:2060-2071, :2629-2640).
int store_width_of(int n2max) { return width_of(n2max) < 32 ? width_of(n2max) : 32; }

// Shared I-list size of computeIShared*_Symbol_SpMMv1, 0 for the global
// kernel.  The tables at :1590-1790 and :2196-2365 give every logical warp a
// segment of next_pow2(n1max) rows, at least max(8, W) (512 when n2max > 256),
// and fall back to the global kernel beyond 8192 per block.
int ishared_size_of(int W, int n1max, int n2max) {
  int seg = W > 8 ? W : 8;
  if (n2max > 256) seg = 512;
  while (seg < n1max) seg <<= 1;
  long size = (long)(kThreads / W) * seg;
  return size <= 8192 ? (int)size : 0;
}

// R's shared size of QR_RShared_SSPAIv10 (:2446-2480); 0 = the reference
// exits (n2max > 2048).
int rshared_size_of(int n2max) {
  if (n2max <= 256) return 256;
  if (n2max <= 512) return 512;
  if (n2max <= 1024) return 1024;
  if (n2max <= 2048) return 2048;
  return 0;
}

struct Arrays {
  std::vector<int> J, jPTR, I, iPTR, E, atomic;
  std::vector<double> tildeA, R, X;
  Arrays(long cols, int n1max, int n2max)
      : J(cols * n2max), jPTR(cols), I(cols * n1max), iPTR(cols), E(cols), atomic(cols),
        tildeA(cols * n1max * n2max), R(cols * n2max * n2max), X(cols * n2max) {}
  void clear_counts() {
    std::fill(jPTR.begin(), jPTR.end(), 0);
    std::fill(iPTR.begin(), iPTR.end(), 0);
    std::fill(E.begin(), E.end(), 0);
  }
};

#define LAUNCH(grid, KERNEL, ...) simt::launch((unsigned)(grid), kThreads, [&] { KERNEL(__VA_ARGS__); })

template <int W>
int run_width(bool tiled, int nCol, int n1max, int n2max, int* ptr, int* idx, double* val, int sK, int eGrid,
              Arrays& a, double* out) {
  const int blocks = (eGrid - 1) / (kThreads / 32) + 1;  // :1540, :1564
  int* J = a.J.data();
  int* jPTR = a.jPTR.data();
  int* I = a.I.data();
  int* iPTR = a.iPTR.data();
  int* E = a.E.data();
  int* at = a.atomic.data();
  double* tA = a.tildeA.data();
  double* R = a.R.data();
  double* X = a.X.data();
  if (tiled)
    LAUNCH(blocks, computeJ2_SSPAIv10<W>, ptr, idx, eGrid, J, jPTR, n2max, sK);
  else
    LAUNCH(blocks, computeJ_SSPAIv10<W>, ptr, idx, nCol, J, jPTR, n2max);
  const int isz = ishared_size_of(W, n1max, n2max);
#define ISHARED(S)                                                                                     \
  case S:                                                                                              \
    if (tiled)                                                                                         \
      LAUNCH(blocks, (computeIShared_iter_Symbol_SpMMv1<W, S>), ptr, idx, eGrid, I, iPTR, n1max, J, jPTR, \
             n2max, at);                                                                               \
    else                                                                                               \
      LAUNCH(blocks, (computeIShared_Symbol_SpMMv1<W, S>), ptr, idx, eGrid, I, iPTR, n1max, J, jPTR, n2max, \
             at);                                                                                      \
    break;
  switch (isz) {
    ISHARED(256)
    ISHARED(512)
    ISHARED(1024)
    ISHARED(2048)
    ISHARED(4096)
    ISHARED(8192)
    default:
      if (tiled)
        LAUNCH(blocks, computeI_iter_Symbol_SpMMv1<W>, ptr, idx, eGrid, I, iPTR, n1max, J, jPTR, n2max, at);
      else if (W == 128)  // the single-pass table's fallback for this bucket is the width-32 kernel (:2352)
        LAUNCH(blocks, computeI_Symbol_SpMMv1<32>, ptr, idx, eGrid, I, iPTR, n1max, J, jPTR, n2max, at);
      else
        LAUNCH(blocks, computeI_Symbol_SpMMv1<W>, ptr, idx, eGrid, I, iPTR, n1max, J, jPTR, n2max, at);
  }
#undef ISHARED
  LAUNCH(blocks, ComputeTildeACSR_SSPAIv10<W>, tA, val, ptr, idx, eGrid, I, iPTR, J, jPTR, n1max, n2max);
  switch (rshared_size_of(n2max)) {
    case 256: LAUNCH(blocks, (QR_RShared_SSPAIv10<W, 256>), tA, R, iPTR, jPTR, n1max, n2max, eGrid); break;
    case 512: LAUNCH(blocks, (QR_RShared_SSPAIv10<W, 512>), tA, R, iPTR, jPTR, n1max, n2max, eGrid); break;
    case 1024: LAUNCH(blocks, (QR_RShared_SSPAIv10<W, 1024>), tA, R, iPTR, jPTR, n1max, n2max, eGrid); break;
    case 2048: LAUNCH(blocks, (QR_RShared_SSPAIv10<W, 2048>), tA, R, iPTR, jPTR, n1max, n2max, eGrid); break;
    default: return -2;
  }
  // ComputeTildeE*: every lane first stores E = -1, then the lanes search
  // I_k for the diagonal.  Lockstep execution orders all those stores before
  // any lane's match; the emulator's fibers run one lane's whole loop before
  // the next lane's store.  With one lane per logical warp the same code
  // finds the same E without relying on that order (I_k's rows are distinct,
  // so at most one position matches).
  const int eblocks = (eGrid - 1) / kThreads + 1;
  if (tiled)
    LAUNCH(eblocks, ComputeTildeE2_SSPAIv10<1>, E, I, iPTR, n1max, eGrid, sK);
  else
    LAUNCH(eblocks, ComputeTildeE_SSPAIv10<1>, E, I, iPTR, n1max, eGrid);
  LAUNCH(blocks, Sol_SSPAIv10<W>, tA, R, X, E, jPTR, n1max, n2max, eGrid);
  const int W1 = store_width_of(n2max);
  const int b1 = (eGrid - 1) / (kThreads / W1) + 1;
#define STORE(S)                                                                          \
  case S:                                                                                 \
    if (tiled)                                                                            \
      LAUNCH(b1, modifyData24_SSPAIv10<S>, out, ptr, X, jPTR, n2max, eGrid, sK);          \
    else                                                                                  \
      LAUNCH(b1, modifyData4_SSPAIv10<S>, out, ptr, X, jPTR, n2max, eGrid);               \
    break;
  switch (W1) {
    STORE(2)
    STORE(4)
    STORE(8)
    STORE(16)
    STORE(32)
  }
#undef STORE
  return 0;
}

int run(bool tiled, int nCol, int n1max, int n2max, int* ptr, int* idx, double* val, int sK, int eGrid, Arrays& a,
        double* out) {
  switch (width_of(n2max)) {
    case 2: return run_width<2>(tiled, nCol, n1max, n2max, ptr, idx, val, sK, eGrid, a, out);
    case 4: return run_width<4>(tiled, nCol, n1max, n2max, ptr, idx, val, sK, eGrid, a, out);
    case 8: return run_width<8>(tiled, nCol, n1max, n2max, ptr, idx, val, sK, eGrid, a, out);
    case 16: return run_width<16>(tiled, nCol, n1max, n2max, ptr, idx, val, sK, eGrid, a, out);
    case 32: return run_width<32>(tiled, nCol, n1max, n2max, ptr, idx, val, sK, eGrid, a, out);
    case 64: return run_width<64>(tiled, nCol, n1max, n2max, ptr, idx, val, sK, eGrid, a, out);
    case 128: return run_width<128>(tiled, nCol, n1max, n2max, ptr, idx, val, sK, eGrid, a, out);
    default: return run_width<256>(tiled, nCol, n1max, n2max, ptr, idx, val, sK, eGrid, a, out);
  }
}

}  // namespace

extern "C" {

// M's values on A's pattern (mval[nnz], A's CSC order) from the reference's
// kernels.  tile_budget_bytes bounds the padded A(I,J) of one tile in the
// tiled path (0: the reference's own tile).  Returns 0, -1 on bad input, -2
// where the reference exits (n2max > 2048).  info[0..3] = n1max, n2max,
// tiles used, 1 when the single-pass path ran.
int refemu_spai(int n, int* ptr, int* idx, double* val, double* mval, long long tile_budget_bytes, int* info) {
  if (n <= 0 || !ptr || !idx || !val || !mval) return -1;
  CSC_Matrix A;
  A.n = A.nRow = A.nCol = n;
  A.nonzeroes = ptr[n];
  A.mPtr = ptr;
  A.mIndex = idx;
  A.mData = val;
  const int n2max = computeN2MAX(&A);
  const int n1max = computeN1MAX(&A, &A);
  const long real = (long)n * n1max * n2max;
  const int iterations = (int)((real - 1) / kCompareSize + 1);
  std::memset(mval, 0, sizeof(double) * (size_t)A.nonzeroes);
  int rc = 0;
  if (iterations == 1) {
    Arrays a(n, n1max, n2max);
    rc = run(false, n, n1max, n2max, ptr, idx, val, 0, n, a, mval);
    if (info) info[2] = 1, info[3] = 1;
  } else {
    long cols = (n - 1) / iterations + 1;  // nCols (:1501)
    const long per_col = (long)n1max * n2max * (long)sizeof(double);
    if (tile_budget_bytes > 0 && cols * per_col > tile_budget_bytes)
      cols = tile_budget_bytes / per_col > 0 ? tile_budget_bytes / per_col : 1;
    Arrays a(cols, n1max, n2max);
    int tiles = 0;
    for (long sK = 0; sK < n && rc == 0; sK += cols, ++tiles) {
      const int eGrid = (int)(sK + cols <= n ? cols : n - sK);
      a.clear_counts();
      rc = run(true, n, n1max, n2max, ptr, idx, val, (int)sK, eGrid, a, mval);
    }
    if (info) info[2] = tiles, info[3] = 0;
  }
  if (info) info[0] = n1max, info[1] = n2max;
  return rc;
}

}  // extern "C"
