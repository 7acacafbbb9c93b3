// Right-preconditioned BiCGSTAB (the recurrences of cublas2_pbicgstabv2,
// include/bicgstab/bicgstab_solver.h:33-275) as five fused kernels per
// iteration, all scalars resident on the device, one CUDA graph per chunk of
// iterations:
//
//   K1 k_bi_py     p = r + beta (p - omega ay) (computed on the fly at every
//                  gathered column, own row stored), y = M p
//   K2 k_bi_ay     ay = A y, (r*, ay)                 -> alpha = rho / (r*, ay)
//   K3 k_bi_sz     s = r - alpha ay (on the fly, own row stored), z = M s
//   K4 k_bi_az     az = A z, (az, s), (az, az)         -> omega
//   K5 k_bi_xr     x += alpha y + omega z, r = s - omega az, (r*, r), (r, r)
//                                                     -> rho, beta, ||r||, stop test
//
// The reference issues 4 SpMV + 12 BLAS-1 calls and 5 blocking host reads per
// iteration (bicgstab_solver.h:138-232).  Reductions end in the last block to
// arrive (per-block partials summed in block order), so every dot product is
// deterministic for a given grid.
//
// Precision forms (template VT / MT / IT):
//   FP64   p, y, z, r* double; M double; int32 column indices
//   mixed  p, y, z, r* float; M float or bf16; int16 column deltas when
//          every |col - row| < 32768.  A, x, r, s, ay, az, every dot product and
//          the rho/alpha/omega/beta recurrences stay FP64.  x and r are updated
//          with exactly the y, z, A y, A z that were stored, so the recurrence
//          residual tracks b - A x to FP64 rounding.
#include <array>
#include <cmath>
#include <algorithm>
#include <cstddef>
#include <type_traits>

#include "internal.cuh"

namespace dcu {
namespace {

constexpr int BI_BLOCK = 256;
constexpr int BI_WARPS = BI_BLOCK / 32;
// Iterations per graph launch.  The host launches each chunk one ahead of
// the stop flag it reads back, so after convergence up to a chunk and a half
// of early-exit launches run; each chunk boundary costs a flag copy.  Long
// iterations (large operators) favour short chunks, short iterations long
// ones: 4 iterations from kChunkShortNnz stored entries on (128^3: 10.80 ->
// 10.71 ms against 8), 8 below.
constexpr int kChunkShort = 4, kChunkLong = 8;
constexpr long long kChunkShortNnz = 1ll << 22;

enum { ST_RUN = -1 };

struct Scal {
  double rho, alpha, omega, beta, res, thr, bnorm, true_res;
  int it, done, status, pidx;
  int verify, verify_pending, maxiter, replacements;
  int a32;  // the A products read the FP32 copy of A's values (every value exact in FP32)
  unsigned counter[8];
};

// ---- loads -----------------------------------------------------------------
__device__ __forceinline__ double ldm(const double* p) { return __ldcs(p); }
__device__ __forceinline__ double ldm(const float* p) { return (double)__ldcs(p); }
__device__ __forceinline__ double ldm(const __nv_bfloat16* p) {
  const unsigned short u = __ldcs(reinterpret_cast<const unsigned short*>(p));
  return (double)__uint_as_float((unsigned)u << 16);
}
__device__ __forceinline__ int ldcol(const int* ix, long long q, int) { return __ldcs(ix + q); }
__device__ __forceinline__ int ldcol(const int16_t* ix, long long q, int r) { return r + (int)__ldcs(ix + q); }

template <typename T>
__device__ __forceinline__ double ldv(const T* p) { return (double)__ldg(p); }

// kNarrow values of one row of a narrow slice, read row-major from the
// narrow array (an FP32 / BF16 M): one 16-byte load for BF16, two for FP32.
template <typename MT>
struct Row8;
template <>
struct Row8<__nv_bfloat16> {
  uint4 u;
  __device__ __forceinline__ void load(const __nv_bfloat16* p) { u = __ldcs(reinterpret_cast<const uint4*>(p)); }
  __device__ __forceinline__ double at(int t) const {
    const unsigned w = (t < 2) ? u.x : (t < 4) ? u.y : (t < 6) ? u.z : u.w;
    return (double)__uint_as_float((t & 1) ? (w & 0xffff0000u) : (w << 16));
  }
};
template <>
struct Row8<float> {
  float4 a, b;
  __device__ __forceinline__ void load(const float* p) {
    a = __ldcs(reinterpret_cast<const float4*>(p));
    b = __ldcs(reinterpret_cast<const float4*>(p) + 1);
  }
  __device__ __forceinline__ double at(int t) const {
    const float4& q = (t < 4) ? a : b;
    const int u = t & 3;
    return (double)((u == 0) ? q.x : (u == 1) ? q.y : (u == 2) ? q.z : q.w);
  }
};
template <>
struct Row8<double> {  // never loaded: an FP64 M has no narrow array
  __device__ __forceinline__ void load(const double*) {}
  __device__ __forceinline__ double at(int) const { return 0.0; }
};

// One SELL-32 row: sum_k val[q] * xf(col[q]).  A warp covers one slice, so
// each k step reads 32 consecutive slots.  Slots are taken 8 at a time with
// every value and index load issued before the dependent gathers, so a thread
// keeps up to 16 independent loads in flight.  A slice whose every k has one
// column offset for all its rows (su[s]; SellPlan::kd) reads no index at all:
// the column is the row plus the slice's offset, one broadcast load per k
// from a table 1/32 the size of the index array.  For a narrow slice (at most
// kNarrow wide, SellPlan::kd8) those offsets come from a table indexed by the
// slice, so they load together with the slice's flags and slot offset rather
// than after them; with M8 (an FP32 / BF16 M) its values come row-major from
// val8 as well, so a row needs one round trip for its values and offsets and
// one for its gathers.  Every path sums the row's products in entry order.
// The rows of a slice that the plan flagged wide (su bit 2) were summed by
// the wide pre-pass (k_bi_wide) into wv.
// A narrow slice's kNarrow offsets: int16 (one 16-byte load) with 16-bit
// column deltas, else int32 (two).
template <typename IT>
struct Kd8 {
  int4 a, b;
  __device__ __forceinline__ void load(const int* kd8, const int16_t*, int s) {
    const int4* q = reinterpret_cast<const int4*>(kd8 + (long long)s * kNarrow);
    a = __ldg(q);
    b = __ldg(q + 1);
  }
  __device__ __forceinline__ void unpack(int (&d)[kNarrow]) const {
    d[0] = a.x; d[1] = a.y; d[2] = a.z; d[3] = a.w; d[4] = b.x; d[5] = b.y; d[6] = b.z; d[7] = b.w;
  }
};
template <>
struct Kd8<int16_t> {
  int4 a;
  __device__ __forceinline__ void load(const int*, const int16_t* kd8h, int s) {
    a = __ldg(reinterpret_cast<const int4*>(kd8h + (long long)s * kNarrow));
  }
  __device__ __forceinline__ void unpack(int (&d)[kNarrow]) const {
    const int w[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      d[2 * k] = (int)(short)(w[k] & 0xffff);
      d[2 * k + 1] = w[k] >> 16;
    }
  }
};

template <bool M8, typename MT, typename IT, typename F>
__device__ __forceinline__ double sell_row(const long long* __restrict__ off, const int* __restrict__ kd,
                                           const int* __restrict__ kd8, const int16_t* __restrict__ kd8h,
                                           const int* __restrict__ su, const double* __restrict__ wv,
                                           const MT* __restrict__ val, const MT* __restrict__ val8,
                                           const IT* __restrict__ ix, int r, F xf) {
  const int s = r >> 5;
  const int f = __ldg(su + s);
  Kd8<IT> kq;
  kq.load(kd8, kd8h, s);
  Row8<MT> m8;
  long long o0 = 0, o1 = 0;
  if (M8) {
    m8.load(val8 + (long long)r * kNarrow);
  } else {
    o0 = __ldg(off + s);
    o1 = __ldg(off + s + 1);
  }
  if (f & 4) return __ldg(wv + ((long long)(f >> 3) << 5) + (r & 31));
  if (f & 2) {
    const int w = (f >> 3) & 15;
    int d[kNarrow];
    kq.unpack(d);
    double av[kNarrow];
    const long long base = o0 + (r & 31);
#pragma unroll
    for (int t = 0; t < kNarrow; ++t) av[t] = (t < w) ? (M8 ? m8.at(t) : ldm(val + base + 32ll * t)) : 0.0;
    double acc = 0.0;
#pragma unroll
    for (int t = 0; t < kNarrow; ++t)
      if (t < w) acc += av[t] * xf(r + d[t]);
    return acc;
  }
  if (M8) {
    o0 = __ldg(off + s);
    o1 = __ldg(off + s + 1);
  }
  const long long base = o0 + (r & 31);
  const int w = (int)((o1 - o0) >> 5);
  double acc = 0.0;
  if (f & 1) {
    const int* __restrict__ kp = kd + (o0 >> 5);
    for (int k0 = 0; k0 < w; k0 += 8) {
      double av[8];
      int cv[8];
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        if (k0 + t < w) {
          av[t] = ldm(val + base + 32ll * (k0 + t));
          cv[t] = r + (__ldg(kp + k0 + t) >> 1);
        } else {
          av[t] = 0.0;
          cv[t] = r;
        }
      }
#pragma unroll
      for (int t = 0; t < 8; ++t)
        if (k0 + t < w) acc += av[t] * xf(cv[t]);
    }
    return acc;
  }
  for (int k0 = 0; k0 < w; k0 += 8) {
    double av[8];
    int cv[8];
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      if (k0 + t < w) {
        const long long q = base + 32ll * (k0 + t);
        av[t] = ldm(val + q);
        cv[t] = ldcol(ix, q, r);
      } else {
        av[t] = 0.0;
        cv[t] = r;
      }
    }
#pragma unroll
    for (int t = 0; t < 8; ++t)
      if (k0 + t < w) acc += av[t] * xf(cv[t]);
  }
  return acc;
}

// Block partial -> per-block slot; the last block to finish sums the slots in
// block order and returns true (with the totals in tot[] for every thread).
template <int ND>
__device__ __forceinline__ bool grid_reduce(double (&v)[ND], double* __restrict__ part, unsigned* counter,
                                            double (&tot)[ND]) {
  __shared__ double red[ND][BI_WARPS];
  __shared__ int amlast;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int d = 0; d < ND; ++d) {
    double x = v[d];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) red[d][wid] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int d = 0; d < ND; ++d) {
      double s = 0.0;
#pragma unroll
      for (int w = 0; w < BI_WARPS; ++w) s += red[d][w];
      part[d * gridDim.x + blockIdx.x] = s;
    }
    __threadfence();
    const unsigned t = atomicAdd(counter, 1u);
    amlast = (t == gridDim.x - 1) ? 1 : 0;
  }
  __syncthreads();
  if (!amlast) return false;
  __threadfence();
#pragma unroll
  for (int d = 0; d < ND; ++d) {
    double s = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += BI_BLOCK) s += __ldcg(part + d * gridDim.x + i);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __syncthreads();
    if (lane == 0) red[d][wid] = s;
    __syncthreads();
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < BI_WARPS; ++w) t += red[d][w];
    tot[d] = t;
  }
  if (threadIdx.x == 0) *counter = 0u;
  return true;
}

template <typename MT, typename IT, typename VT>
struct BiArgs {
  int n;
  const long long* off;
  const int* kd;        // per (slice, k) offset descriptors (SellPlan::kd)
  const int* kd8;       // per narrow slice, its offsets (SellPlan::kd8)
  const int16_t* kd8h;  // the same as int16 (with 16-bit column deltas)
  const int* su;        // per slice flags (SellPlan::su)
  const IT* ix;         // shared by A and M (same pattern)
  const double* aval;
  const float* aval32;   // FP32 copy of aval, or null
  const int* a_inexact;  // nonzero when some A value is not exact in FP32
  const MT* mval;
  const MT* mval8;      // narrow slices' M values, row-major (FP32 / BF16 M), or null
  const double* b;
  double* x;
  double* r;
  VT* rs;
  VT* p0;
  VT* p1;
  VT* y;
  double* ay;
  double* s;
  VT* z;
  double* az;
  double* part;
  Scal* S;
  const int* rptr;       // CSR row pointers (row lengths of the wide slices)
  const int* wide_list;  // slices wider than kWideSlice (SellPlan::wide)
  double* wide_val;      // their row values for the next SpMV, 32 per listed slice
  int nwide;
};

// A's row (FP64 values in SELL order).
template <typename MT, typename IT, typename VT, typename F>
__device__ __forceinline__ double a_row(const BiArgs<MT, IT, VT>& a, int r, F xf) {
  return sell_row<false, double, IT>(a.off, a.kd, a.kd8, a.kd8h, a.su, a.wide_val, a.aval, nullptr, a.ix, r, xf);
}
// The plain FP64 form (FP64 M) never reads A's FP32 copy.
template <typename MT>
constexpr bool kA32 = !std::is_same<MT, double>::value;

// A's row from the FP32 copy of its values: the same numbers when every
// value of A is exact in FP32 (Scal::a32), widened to FP64 before the
// multiply, so the row's sum is bit-identical to a_row's.
template <typename MT, typename IT, typename VT, typename F>
__device__ __forceinline__ double a_row32(const BiArgs<MT, IT, VT>& a, int r, F xf) {
  return sell_row<false, float, IT>(a.off, a.kd, a.kd8, a.kd8h, a.su, a.wide_val, a.aval32, nullptr, a.ix, r, xf);
}
// M's row: narrow slices from the row-major narrow array where the form has one.
template <typename MT, typename IT, typename VT, typename F>
__device__ __forceinline__ double m_row(const BiArgs<MT, IT, VT>& a, int r, F xf) {
  constexpr bool narrow = !std::is_same<MT, double>::value;
  if (narrow && a.mval8)
    return sell_row<narrow, MT, IT>(a.off, a.kd, a.kd8, a.kd8h, a.su, a.wide_val, a.mval, a.mval8, a.ix, r, xf);
  return sell_row<false, MT, IT>(a.off, a.kd, a.kd8, a.kd8h, a.su, a.wide_val, a.mval, nullptr, a.ix, r, xf);
}

// Kernels K1..K5 are launched with programmatic dependent launch: their blocks
// may start while the previous kernel drains, and wait here for its results.
// Every kernel of the iteration starts here.  It first lets the next kernel
// in the stream (launched with programmatic dependent launch) be scheduled:
// that launch happens once every block of this grid has passed this point,
// so its blocks only take slots this grid no longer needs, and they become
// resident while this grid finishes instead of after it.  Then it waits for
// the previous kernel to complete with its memory visible (the wait covers
// completion, not the trigger), and reads the stop flag.
__device__ __forceinline__ bool finished(const Scal* S) {
  cudaTriggerProgrammaticLaunchCompletion();
  cudaGridDependencySynchronize();
  return *(volatile const int*)&S->done != 0;
}

__device__ __forceinline__ bool bad(double v) { return !isfinite(v); }

// ---- wide pre-pass ---------------------------------------------------------
// A full slice made wider than kWideSlice by a few long rows; in sell_row its
// warp would walk every slot of the slice, with one gather latency per 8 slots.
// Here a warp takes one such slice: each lane sums its own row up to its own
// length (rptr), 8 slots at a time as in sell_row; then the rows longer than
// kWideSlice are summed one at a time by the whole warp, each lane loading one
// entry in 32 and its gather (two chunks of 32 prefetched), and one chain of
// multiply-adds consuming them in k order through shuffles.  Every row's sum
// is formed in sell_row's order with its operations, stopping at the row's
// length instead of running over the zero padding, so the iterates do not
// change.  Launched just before the kernel whose SpMV it serves.
enum { WIDE_AX = 0, WIDE_PY, WIDE_Y, WIDE_AY, WIDE_SZ, WIDE_AZ };

template <typename MT, typename IT, typename F>
__device__ __forceinline__ double wide_row(long long o0, const int* __restrict__ rptr, const MT* __restrict__ val,
                                           const IT* __restrict__ ix, int r, F xf) {
  const int lane = r & 31;
  const int len = __ldg(rptr + r + 1) - __ldg(rptr + r);
  const long long base = o0 + lane;
  double acc = 0.0;
  if (len <= kWideSlice) {
    for (int k0 = 0; k0 < len; k0 += 8) {
      double av[8];
      int cv[8];
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        if (k0 + t < len) {
          const long long q = base + 32ll * (k0 + t);
          av[t] = ldm(val + q);
          cv[t] = ldcol(ix, q, r);
        } else {
          av[t] = 0.0;
          cv[t] = r;
        }
      }
#pragma unroll
      for (int t = 0; t < 8; ++t)
        if (k0 + t < len) acc += av[t] * xf(cv[t]);
    }
  }
  unsigned longs = __ballot_sync(0xffffffffu, len > kWideSlice);
  while (longs) {
    const int j = __ffs(longs) - 1;
    longs &= longs - 1;
    const int lj = __shfl_sync(0xffffffffu, len, j);
    const int rj = (r & ~31) + j;
    const long long bj = o0 + j;
    auto load = [&](int k, double& av, double& xv) {
      if (k < lj) {
        const long long q = bj + 32ll * k;
        av = ldm(val + q);
        xv = xf(ldcol(ix, q, rj));
      } else {
        av = 0.0;
        xv = 0.0;
      }
    };
    // two chunks in flight ahead of the one being consumed
    double chain = 0.0, av0, xv0, av1, xv1;
    load(lane, av0, xv0);
    load(32 + lane, av1, xv1);
    for (int c0 = 0; c0 < lj; c0 += 32) {
      double av2, xv2;
      load(c0 + 64 + lane, av2, xv2);
      const int cnt = min(32, lj - c0);
      for (int t = 0; t < cnt; ++t) {
        const double at = __shfl_sync(0xffffffffu, av0, t);
        const double xt = __shfl_sync(0xffffffffu, xv0, t);
        chain += at * xt;
      }
      av0 = av1;
      xv0 = xv1;
      av1 = av2;
      xv1 = xv2;
    }
    if (lane == j) acc = chain;
  }
  return acc;
}

template <typename MT, typename IT, typename VT, int WHICH>
__global__ void __launch_bounds__(BI_BLOCK) k_bi_wide(BiArgs<MT, IT, VT> a) {
  if (WHICH != WIDE_AX && finished(a.S)) return;  // WIDE_AX serves k_bi_init / k_bi_true (plain launches)
  const int wv = (int)(((long long)blockIdx.x * BI_BLOCK + threadIdx.x) >> 5);
  if (wv >= a.nwide) return;  // whole warps
  const int s = a.wide_list[wv];
  const int r = (s << 5) + (threadIdx.x & 31);
  const long long o0 = a.off[s];
  double v;
  if constexpr (WHICH == WIDE_AX) {
    v = wide_row(o0, a.rptr, a.aval, a.ix, r, [&](int c) { return ldv(a.x + c); });
  } else if constexpr (WHICH == WIDE_PY) {
    const double beta = a.S->beta, omega = a.S->omega;
    const VT* __restrict__ pold = a.S->pidx ? a.p1 : a.p0;
    const double* __restrict__ rr = a.r;
    const double* __restrict__ ay = a.ay;
    v = wide_row(o0, a.rptr, a.mval, a.ix, r,
                 [&](int c) { return ldv(rr + c) + beta * (ldv(pold + c) - omega * ldv(ay + c)); });
  } else if constexpr (WHICH == WIDE_Y) {
    const VT* __restrict__ p = a.p0;
    v = wide_row(o0, a.rptr, a.mval, a.ix, r, [&](int c) { return ldv(p + c); });
  } else if constexpr (WHICH == WIDE_AY) {
    const VT* __restrict__ y = a.y;
    v = wide_row(o0, a.rptr, a.aval, a.ix, r, [&](int c) { return ldv(y + c); });
  } else if constexpr (WHICH == WIDE_SZ) {
    const double nalpha = -1.0 * a.S->alpha;
    const double* __restrict__ rr = a.r;
    const double* __restrict__ ay = a.ay;
    v = wide_row(o0, a.rptr, a.mval, a.ix, r, [&](int c) { return ldv(rr + c) + nalpha * ldv(ay + c); });
  } else {
    const VT* __restrict__ z = a.z;
    v = wide_row(o0, a.rptr, a.aval, a.ix, r, [&](int c) { return ldv(z + c); });
  }
  a.wide_val[((long long)wv << 5) + (threadIdx.x & 31)] = v;
}

// K0: r = b - A x, r* = r, p = ay = 0, rho = (r*, r), ||r||, ||b||
template <typename MT, typename IT, typename VT>
__global__ void __launch_bounds__(BI_BLOCK) k_bi_init(BiArgs<MT, IT, VT> a, double tol, int tol_mode, int maxiter,
                                                      int verify) {
  double v[3] = {0.0, 0.0, 0.0};
  // with every value of A exact in FP32 its FP64 SELL copy may be absent
  const bool a32 = kA32<MT> && a.aval32 && *a.a_inexact == 0;
  auto xf = [&](int c) { return ldv(a.x + c); };
  const int stride = gridDim.x * BI_BLOCK;
  for (int r = blockIdx.x * BI_BLOCK + threadIdx.x; r < a.n; r += stride) {
    const double ax = a32 ? a_row32(a, r, xf) : a_row(a, r, xf);
    const double br = a.b[r];
    const double rr = br + (-1.0) * ax;
    a.r[r] = rr;
    const VT rsv = (VT)rr;
    a.rs[r] = rsv;
    a.p0[r] = (VT)0.0;
    a.p1[r] = (VT)0.0;
    a.ay[r] = 0.0;
    v[0] += (double)rsv * rr;
    v[1] += rr * rr;
    v[2] += br * br;
  }
  double tot[3];
  if (grid_reduce<3>(v, a.part, &a.S->counter[0], tot) && threadIdx.x == 0) {
    Scal* S = a.S;
    S->rho = tot[0];
    S->res = sqrt(tot[1]);
    S->bnorm = sqrt(tot[2]);
    S->thr = (tol_mode == DCU_TOL_REL) ? tol * S->bnorm : tol;
    S->alpha = 0.0;
    S->omega = 1.0;
    S->beta = 0.0;
    S->pidx = 0;
    S->it = 1;
    S->maxiter = maxiter;
    S->verify = verify;
    S->verify_pending = 0;
    S->replacements = 0;
    S->true_res = -1.0;
    S->a32 = (a.aval32 && *a.a_inexact == 0) ? 1 : 0;
    S->status = ST_RUN;
    S->done = 0;
    if (S->res == 0.0) {  // x0 already solves the system
      S->status = DCU_SOLVE_CONVERGED;
      S->done = 1;
    } else if (maxiter <= 1) {
      S->status = DCU_SOLVE_MAXITER;
      S->done = 1;
    }
  }
}

// K1: p = r + beta (p - omega ay); y = M p
template <typename MT, typename IT, typename VT>
__global__ void __launch_bounds__(BI_BLOCK) k_bi_py(BiArgs<MT, IT, VT> a) {
  if (finished(a.S)) return;
  const double beta = a.S->beta, omega = a.S->omega;
  const int pidx = a.S->pidx;
  const VT* __restrict__ pold = pidx ? a.p1 : a.p0;
  VT* __restrict__ pnew = pidx ? a.p0 : a.p1;
  const double* __restrict__ rr = a.r;
  const double* __restrict__ ay = a.ay;
  auto pf = [&](int c) { return ldv(rr + c) + beta * (ldv(pold + c) - omega * ldv(ay + c)); };
  const int stride = gridDim.x * BI_BLOCK;
  for (int r = blockIdx.x * BI_BLOCK + threadIdx.x; r < a.n; r += stride) {
    const double yv = m_row(a, r, pf);
    pnew[r] = (VT)pf(r);
    a.y[r] = (VT)yv;
  }
}

// Split form of K1, used with a narrow (FP32 / BF16) preconditioner: p is
// formed once per row by a streaming kernel and then read by a one-vector
// SpMV, instead of at every gathered column (three gathered vectors per
// entry).  Same arithmetic as the fused kernel.  This is the untuned default:
// split with a narrow M, fused with an FP64 M (whose SpMV moves 8 bytes of
// value per entry, so the gathers the split saves weigh less).  The autotuner
// compares both in whole solves where they compute the same values (FP64
// vectors); at 128^3 it finds the split faster with an FP64 M too.  K3
// gathers two vectors and stays fused always.
template <typename MT>
constexpr bool split_k1() {
  return !std::is_same<MT, double>::value;
}

__device__ __forceinline__ double2 ld2(const double* p) { return *reinterpret_cast<const double2*>(p); }
__device__ __forceinline__ double2 ld2(const float* p) {
  const float2 f = *reinterpret_cast<const float2*>(p);
  return make_double2((double)f.x, (double)f.y);
}
__device__ __forceinline__ void st2(double* p, double u, double v) {
  *reinterpret_cast<double2*>(p) = make_double2(u, v);
}
__device__ __forceinline__ void st2(float* p, double u, double v) {
  *reinterpret_cast<float2*>(p) = make_float2((float)u, (float)v);
}

// K1a: p = r + beta (p - omega ay), in place (p0)
template <typename MT, typename IT, typename VT>
__global__ void __launch_bounds__(BI_BLOCK) k_bi_p(BiArgs<MT, IT, VT> a) {
  if (finished(a.S)) return;
  const double beta = a.S->beta, omega = a.S->omega;
  auto pf = [&](double rv, double pv, double ayv) { return rv + beta * (pv - omega * ayv); };
  const int npair = a.n >> 1;
  const int stride = gridDim.x * BI_BLOCK;
  for (int q = blockIdx.x * BI_BLOCK + threadIdx.x; q < npair; q += stride) {
    const int r = 2 * q;
    const double2 r2 = ld2(a.r + r), p2 = ld2(a.p0 + r), y2 = ld2(a.ay + r);
    st2(a.p0 + r, pf(r2.x, p2.x, y2.x), pf(r2.y, p2.y, y2.y));
  }
  if ((a.n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
    const int r = a.n - 1;
    a.p0[r] = (VT)pf(a.r[r], (double)a.p0[r], a.ay[r]);
  }
}

// K1b: y = M p (held to 32 registers: 8 blocks per SM; at 34 it ran 6)
template <typename MT, typename IT, typename VT>
__global__ void __launch_bounds__(BI_BLOCK, 8) k_bi_y(BiArgs<MT, IT, VT> a) {
  if (finished(a.S)) return;
  const VT* __restrict__ p = a.p0;
  const int stride = gridDim.x * BI_BLOCK;
  for (int r = blockIdx.x * BI_BLOCK + threadIdx.x; r < a.n; r += stride)
    a.y[r] = (VT)m_row(a, r, [&](int c) { return ldv(p + c); });
}

// K2: ay = A y; alpha = rho / (r*, ay)
// 32 registers (8 blocks per SM) with 16-bit columns and a narrow M; with
// int32 columns or an FP64 M up to 48 without spilling (5 blocks).  (An
// explicit minimum of one block lets the compiler take 64 for the former.)
template <typename MT, typename IT, typename VT>
__global__ void __launch_bounds__(BI_BLOCK, (std::is_same<MT, double>::value || std::is_same<IT, int>::value) ? 5 : 8)
    k_bi_ay(BiArgs<MT, IT, VT> a) {
  if (finished(a.S)) return;
  double v[1] = {0.0};
  const VT* __restrict__ y = a.y;
  auto yf = [&](int c) { return ldv(y + c); };
  const int stride = gridDim.x * BI_BLOCK;
  // r*[r] is loaded with the row's values, not after the store of Ay[r]
  // (which the load could alias): one round trip per row instead of two
  auto row = [&](int r, double rsv, double ayv) {
    a.ay[r] = ayv;
    v[0] += rsv * ayv;
  };
  const VT* __restrict__ rs = a.rs;
  if (kA32<MT> && a.S->a32) {
    for (int r = blockIdx.x * BI_BLOCK + threadIdx.x; r < a.n; r += stride) {
      const double rsv = ldv(rs + r);
      row(r, rsv, a_row32(a, r, yf));
    }
  } else {
    for (int r = blockIdx.x * BI_BLOCK + threadIdx.x; r < a.n; r += stride) {
      const double rsv = ldv(rs + r);
      row(r, rsv, a_row(a, r, yf));
    }
  }
  double tot[1];
  if (grid_reduce<1>(v, a.part, &a.S->counter[1], tot) && threadIdx.x == 0) {
    Scal* S = a.S;
    const double alpha = S->rho / tot[0];
    S->alpha = alpha;
    if (tot[0] == 0.0 || bad(alpha)) {
      S->status = DCU_SOLVE_BREAKDOWN;
      S->done = 1;
    }
  }
}

// K3: s = r - alpha ay; z = M s
template <typename MT, typename IT, typename VT>
__global__ void __launch_bounds__(BI_BLOCK) k_bi_sz(BiArgs<MT, IT, VT> a) {
  if (finished(a.S)) return;
  const double nalpha = -1.0 * a.S->alpha;
  const double* __restrict__ rr = a.r;
  const double* __restrict__ ay = a.ay;
  auto sf = [&](int c) { return ldv(rr + c) + nalpha * ldv(ay + c); };
  const int stride = gridDim.x * BI_BLOCK;
  for (int r = blockIdx.x * BI_BLOCK + threadIdx.x; r < a.n; r += stride) {
    // the row's own r and Ay load with its values, not after the SpMV
    const double rv = ldv(rr + r), ayv = ldv(ay + r);
    const double zv = m_row(a, r, sf);
    a.s[r] = rv + nalpha * ayv;
    a.z[r] = (VT)zv;
  }
}

// K4: az = A z; omega = (az, s) / (az, az)
template <typename MT, typename IT, typename VT>
__global__ void __launch_bounds__(BI_BLOCK) k_bi_az(BiArgs<MT, IT, VT> a) {
  if (finished(a.S)) return;
  double v[2] = {0.0, 0.0};
  const VT* __restrict__ z = a.z;
  auto zf = [&](int c) { return ldv(z + c); };
  const int stride = gridDim.x * BI_BLOCK;
  // s[r] is loaded with the row's values, not after the store of Az[r]
  // (which the load could alias): one round trip per row instead of two
  auto row = [&](int r, double sv, double azv) {
    a.az[r] = azv;
    v[0] += azv * sv;
    v[1] += azv * azv;
  };
  const double* __restrict__ s = a.s;
  if (kA32<MT> && a.S->a32) {
    for (int r = blockIdx.x * BI_BLOCK + threadIdx.x; r < a.n; r += stride) {
      const double sv = ldv(s + r);
      row(r, sv, a_row32(a, r, zf));
    }
  } else {
    for (int r = blockIdx.x * BI_BLOCK + threadIdx.x; r < a.n; r += stride) {
      const double sv = ldv(s + r);
      row(r, sv, a_row(a, r, zf));
    }
  }
  double tot[2];
  if (grid_reduce<2>(v, a.part, &a.S->counter[2], tot) && threadIdx.x == 0) {
    Scal* S = a.S;
    // Az = 0 (s = 0 when the half step solved the system): omega = 0, and K5
    // finds r = s; the reference's 0 / 0 would make x NaN
    const double omega = (tot[1] == 0.0) ? 0.0 : tot[0] / tot[1];
    S->omega = omega;
    if (bad(omega)) {
      S->status = DCU_SOLVE_BREAKDOWN;
      S->done = 1;
    }
  }
}

// K5: x += alpha y + omega z; r = s - omega az; rho, beta, ||r||, stop test.
// Rows are taken in pairs with every load issued before the first store
// (16-byte loads of the FP64 vectors), so one DRAM round trip covers a pair.
template <typename MT, typename IT, typename VT>
__global__ void __launch_bounds__(BI_BLOCK, 6) k_bi_xr(BiArgs<MT, IT, VT> a) {
  if (finished(a.S)) return;
  const double alpha = a.S->alpha, omega = a.S->omega, nomega = -1.0 * omega;
  double v[2] = {0.0, 0.0};
  auto row = [&](double& xv, double yv, double zv, double sv, double azv, double rsv) {
    xv = xv + alpha * yv;
    xv = xv + omega * zv;
    const double rn = sv + nomega * azv;
    v[0] += rsv * rn;
    v[1] += rn * rn;
    return rn;
  };
  const int npair = a.n >> 1;
  const int stride = gridDim.x * BI_BLOCK;
  for (int q = blockIdx.x * BI_BLOCK + threadIdx.x; q < npair; q += stride) {
    const int r = 2 * q;
    double2 x2 = *reinterpret_cast<const double2*>(a.x + r);
    const double2 s2 = *reinterpret_cast<const double2*>(a.s + r);
    const double2 az2 = *reinterpret_cast<const double2*>(a.az + r);
    const double y0 = (double)a.y[r], y1 = (double)a.y[r + 1];
    const double z0 = (double)a.z[r], z1 = (double)a.z[r + 1];
    const double rs0 = (double)a.rs[r], rs1 = (double)a.rs[r + 1];
    const double r0 = row(x2.x, y0, z0, s2.x, az2.x, rs0);
    const double r1 = row(x2.y, y1, z1, s2.y, az2.y, rs1);
    *reinterpret_cast<double2*>(a.x + r) = x2;
    *reinterpret_cast<double2*>(a.r + r) = make_double2(r0, r1);
  }
  if ((a.n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
    const int r = a.n - 1;
    double xv = a.x[r];
    const double rn = row(xv, (double)a.y[r], (double)a.z[r], a.s[r], a.az[r], (double)a.rs[r]);
    a.x[r] = xv;
    a.r[r] = rn;
  }
  double tot[2];
  if (grid_reduce<2>(v, a.part, &a.S->counter[3], tot) && threadIdx.x == 0) {
    Scal* S = a.S;
    const double rho_new = tot[0];
    const double beta = (rho_new / S->rho) * (alpha / omega);
    S->beta = beta;
    S->rho = rho_new;
    S->res = sqrt(tot[1]);
    S->pidx ^= 1;
    // the stop test first, as in the reference (it never examines beta)
    if (bad(S->res)) {
      S->status = DCU_SOLVE_BREAKDOWN;
      S->done = 1;
    } else if (S->res < S->thr) {
      if (S->verify) S->verify_pending = 1;
      else S->status = DCU_SOLVE_CONVERGED;
      S->done = 1;
    } else if (bad(beta) || rho_new == 0.0) {
      S->status = DCU_SOLVE_BREAKDOWN;
      S->done = 1;
    } else {
      S->it += 1;
      if (S->it >= S->maxiter) {
        S->status = DCU_SOLVE_MAXITER;
        S->done = 1;
      }
    }
  }
}

// K6: true residual b - A x.  replace = 1: residual replacement after the
// recurrence met the threshold (continue unless the true residual meets it
// too); replace = 0: report only.
template <typename MT, typename IT, typename VT>
__global__ void __launch_bounds__(BI_BLOCK) k_bi_true(BiArgs<MT, IT, VT> a, int replace) {
  double v[2] = {0.0, 0.0};
  const bool a32 = kA32<MT> && a.S->a32;  // (k_bi_init decided it)
  auto xf = [&](int c) { return ldv(a.x + c); };
  const int stride = gridDim.x * BI_BLOCK;
  for (int r = blockIdx.x * BI_BLOCK + threadIdx.x; r < a.n; r += stride) {
    const double ax = a32 ? a_row32(a, r, xf) : a_row(a, r, xf);
    const double rt = a.b[r] - ax;
    if (replace) a.r[r] = rt;
    v[0] += (double)a.rs[r] * rt;
    v[1] += rt * rt;
  }
  double tot[2];
  if (grid_reduce<2>(v, a.part, &a.S->counter[4], tot) && threadIdx.x == 0) {
    Scal* S = a.S;
    S->true_res = sqrt(tot[1]);
    if (replace) {
      S->verify_pending = 0;
      if (S->true_res < S->thr) {
        S->status = DCU_SOLVE_CONVERGED;
        S->done = 1;
      } else {
        S->rho = tot[0];
        S->res = S->true_res;
        S->replacements += 1;
        S->it += 1;
        if (S->it >= S->maxiter) {
          S->status = DCU_SOLVE_MAXITER;
          S->done = 1;
        } else {
          S->done = 0;
        }
      }
    }
  }
}

template <typename K, typename A>
cudaError_t launch_pdl(K kernel, int grid, cudaStream_t st, const A& args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(BI_BLOCK);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, args);
}

// Grid of a grid-stride kernel over `items` rows (or row pairs) for a tuning
// selector: 0 one wave of `per_sm` resident blocks per SM, -1 one block per
// BI_BLOCK items (no loop), k > 0 k blocks per SM (at most `per_sm`).
int grid_for(const Ctx* c, long long items, int per_sm, int sel) {
  if (sel < 0) return (int)std::max(1LL, (items + BI_BLOCK - 1) / BI_BLOCK);
  return waves_grid(c, items, BI_BLOCK, sel > 0 ? std::min(sel, per_sm) : per_sm);
}

template <typename MT, typename IT, typename VT>
int run_solver(Ctx* c, const SellPlan& plan, const SellA& aval, const MT* mval, const IT* ix, const double* b,
               double* x, const dcu_options* opt, const dcu_tuning* tu, dcu_solve_info* info,
               const MT* mval8 = nullptr) {
  const int n = plan.n;
  // blocks of each kernel resident on one SM at once
  auto resident = [&](const void* fn) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, BI_BLOCK, 0) != cudaSuccess || per_sm < 1) {
      cudaGetLastError();
      per_sm = 1;
    }
    return per_sm;
  };
  std::array<int, IK_COUNT> rs;
  rs[IK_P] = resident((const void*)k_bi_p<MT, IT, VT>);
  rs[IK_Y] = resident((const void*)k_bi_y<MT, IT, VT>);
  rs[IK_PY] = resident((const void*)k_bi_py<MT, IT, VT>);
  rs[IK_AY] = resident((const void*)k_bi_ay<MT, IT, VT>);
  rs[IK_SZ] = resident((const void*)k_bi_sz<MT, IT, VT>);
  rs[IK_AZ] = resident((const void*)k_bi_az<MT, IT, VT>);
  rs[IK_XR] = resident((const void*)k_bi_xr<MT, IT, VT>);
  // rows each kernel's threads stride over (the p pass takes row pairs); the
  // kernels that end in a reduction keep one full wave over n, whatever the
  // tuning: their grid fixes the summation order of the partial sums
  std::array<long long, IK_COUNT> items = {std::max(1, n >> 1), n, n, n, n, n, n};
  std::array<int, IK_COUNT> sel = {0, 0, 0, 0, 0, 0, 0};
  if (tu) {
    sel[IK_P] = tu->grid_p;
    sel[IK_Y] = tu->grid_y;
    sel[IK_PY] = tu->grid_py;
    sel[IK_SZ] = tu->grid_sz;
  }
  auto grid_of = [c, rs, items](int kind, int s) {
    const bool tunable = kind == IK_P || kind == IK_Y || kind == IK_PY || kind == IK_SZ;
    return grid_for(c, items[kind], rs[kind], tunable ? s : 0);
  };
  const int g_init = waves_grid(c, n, BI_BLOCK, resident((const void*)k_bi_init<MT, IT, VT>));
  const int g_tr = waves_grid(c, n, BI_BLOCK, resident((const void*)k_bi_true<MT, IT, VT>));
  const int g_p = grid_of(IK_P, sel[IK_P]);
  const int g_y = grid_of(IK_Y, sel[IK_Y]);
  const int g_py = grid_of(IK_PY, sel[IK_PY]);
  const int g_ay = grid_of(IK_AY, 0);
  const int g_sz = grid_of(IK_SZ, sel[IK_SZ]);
  const int g_az = grid_of(IK_AZ, 0);
  const int g_xr = grid_of(IK_XR, 0);
  const int grid = std::max({g_init, g_ay, g_az, g_xr, g_tr});  // partial-sum slots
  // The fused and the split first step compute bit-identical p and y when the
  // vectors are FP64 (the fused step's p is exact in VT); with FP32 vectors
  // the fused step multiplies by the unrounded p, so the form keeps its split.
  constexpr bool k1_free = std::is_same<VT, double>::value;
  const bool split = (k1_free && tu && tu->k1_split >= 0) ? tu->k1_split == 1 : split_k1<MT>();
  // vectors: r, ay, s, az (double) + rs, p0, p1, y, z (VT), 256-byte aligned
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t nd = al(sizeof(double) * (size_t)n), nv = al(sizeof(VT) * (size_t)n);
  DCU_TRY(ensure(c, B_VEC, 4 * nd + 5 * nv));
  DCU_TRY(ensure(c, B_PART, sizeof(double) * 3 * (size_t)grid + 256));
  DCU_TRY(ensure(c, B_SCAL, sizeof(Scal)));
  char* base = bp<char>(c, B_VEC);
  BiArgs<MT, IT, VT> a;
  std::memset(&a, 0, sizeof(a));  // padding included: the struct keys the graph cache
  a.n = n;
  a.off = plan.off;
  a.kd = plan.kd;
  a.kd8 = plan.kd8;
  a.kd8h = plan.kd8h;
  a.su = plan.su;
  a.ix = ix;
  a.aval = aval.v64;
  a.aval32 = aval.v32;
  a.a_inexact = aval.inexact;
  a.mval = mval;
  a.mval8 = mval8;
  a.b = b;
  a.x = x;
  a.r = (double*)(base);
  a.ay = (double*)(base + nd);
  a.s = (double*)(base + 2 * nd);
  a.az = (double*)(base + 3 * nd);
  a.rs = (VT*)(base + 4 * nd);
  a.p0 = (VT*)(base + 4 * nd + nv);
  a.p1 = (VT*)(base + 4 * nd + 2 * nv);
  a.y = (VT*)(base + 4 * nd + 3 * nv);
  a.z = (VT*)(base + 4 * nd + 4 * nv);
  a.part = bp<double>(c, B_PART);
  a.S = bp<Scal>(c, B_SCAL);
  // slices wider than kWideSlice: their rows come from the wide pre-pass
  a.rptr = plan.rptr;
  a.wide_list = plan.wide;
  a.nwide = plan.nwide;
  if (plan.nwide > 0) {
    DCU_TRY(ensure(c, B_WIDEVAL, sizeof(double) * 32 * (size_t)plan.nwide));
    a.wide_val = bp<double>(c, B_WIDEVAL);
  }
  const int g_wide = (int)(((long long)plan.nwide * 32 + BI_BLOCK - 1) / BI_BLOCK);
  const bool wide = plan.nwide > 0;
  if (reinterpret_cast<uintptr_t>(x) % 16 != 0)
    return fail(c, DCU_ERR_ARG, "x must be 16-byte aligned (cudaMalloc pointers are)");
  DCU_CUDA(c, cudaMemsetAsync(a.S, 0, sizeof(Scal), c->stream));
  int maxiter = opt->maxiter > 0 ? opt->maxiter : n;  // bicgstab_solver.h:134
  DCU_CUDA(c, cudaEventRecord(c->ev[0], c->stream));
  if (wide) {
    k_bi_wide<MT, IT, VT, WIDE_AX><<<g_wide, BI_BLOCK, 0, c->stream>>>(a);
    DCU_LAUNCHED(c, "k_bi_wide");
  }
  k_bi_init<MT, IT, VT><<<g_init, BI_BLOCK, 0, c->stream>>>(a, opt->tol, opt->tol_mode, maxiter, opt->verify);
  DCU_LAUNCHED(c, "k_bi_init");

  // graph of `chunk` iterations
  const int chunk = (long long)plan.nnz >= kChunkShortNnz ? kChunkShort : kChunkLong;
  // the key names the kernel instantiation too: the same buffers are reused
  // by every precision form
  std::vector<const void*> key = {(const void*)&k_bi_py<MT, IT, VT>, (const void*)(intptr_t)grid,
                                  (const void*)(intptr_t)split,
                                  (const void*)(intptr_t)g_py, (const void*)(intptr_t)g_ay, (const void*)(intptr_t)g_sz,
                                  (const void*)(intptr_t)g_az, (const void*)(intptr_t)g_xr, (const void*)(intptr_t)g_p,
                                  (const void*)(intptr_t)g_y, (const void*)(intptr_t)chunk};
  key_append(key, a);
  GraphSlot* ge = nullptr;
  for (auto& e : c->graphs)
    if (e.key == key) ge = &e;
  if (!ge) {
    cudaGraph_t g = nullptr;
    DCU_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t le = cudaSuccess;
    // a wide pre-pass node ahead of each SpMV kernel when the layout has wide slices
    auto pre = [&](auto kernel) {
      if (wide && le == cudaSuccess) le = launch_pdl(kernel, g_wide, c->stream, a);
    };
    for (int i = 0; i < chunk && le == cudaSuccess; ++i) {
      if (split) {
        le = launch_pdl(k_bi_p<MT, IT, VT>, g_p, c->stream, a);
        pre(k_bi_wide<MT, IT, VT, WIDE_Y>);
        if (le == cudaSuccess) le = launch_pdl(k_bi_y<MT, IT, VT>, g_y, c->stream, a);
      } else {
        pre(k_bi_wide<MT, IT, VT, WIDE_PY>);
        if (le == cudaSuccess) le = launch_pdl(k_bi_py<MT, IT, VT>, g_py, c->stream, a);
      }
      pre(k_bi_wide<MT, IT, VT, WIDE_AY>);
      if (le == cudaSuccess) le = launch_pdl(k_bi_ay<MT, IT, VT>, g_ay, c->stream, a);
      pre(k_bi_wide<MT, IT, VT, WIDE_SZ>);
      if (le == cudaSuccess) le = launch_pdl(k_bi_sz<MT, IT, VT>, g_sz, c->stream, a);
      pre(k_bi_wide<MT, IT, VT, WIDE_AZ>);
      if (le == cudaSuccess) le = launch_pdl(k_bi_az<MT, IT, VT>, g_az, c->stream, a);
      if (le == cudaSuccess) le = launch_pdl(k_bi_xr<MT, IT, VT>, g_xr, c->stream, a);
    }
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    if (le != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return cuda_fail(c, le, "cudaLaunchKernelEx (capture)", __FILE__, __LINE__);
    }
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaStreamEndCapture", __FILE__, __LINE__);
    GraphSlot ne;
    ne.key = key;
    ne.nodes = ((split ? 6 : 5) + (wide ? 4 : 0)) * chunk;
    e = cudaGraphInstantiate(&ne.exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaGraphInstantiate", __FILE__, __LINE__);
    if (c->graphs.size() >= 8) {  // bounded cache: drop the oldest
      cudaGraphExecDestroy(c->graphs.front().exec);
      c->graphs.erase(c->graphs.begin());
    }
    c->graphs.push_back(ne);
    ge = &c->graphs.back();
  }

  // Chunks are launched one ahead of the flag that is read back, so the GPU
  // never idles on the host; after convergence at most one chunk of
  // early-exit kernels runs.
  if (split) {
    c->profile_order = {IK_P, IK_Y, IK_AY, IK_SZ, IK_AZ, IK_XR};
    c->profile_sel = {sel[IK_P], sel[IK_Y], 0, sel[IK_SZ], 0, 0};
  } else {
    c->profile_order = {IK_PY, IK_AY, IK_SZ, IK_AZ, IK_XR};
    c->profile_sel = {sel[IK_PY], 0, sel[IK_SZ], 0, 0};
  }
  c->profile_k1_free = k1_free;
  c->profile_default_split = split_k1<MT>() ? 1 : 0;
  c->profile_launch = [c, a, grid_of](int kind, int s) -> int {
    const int g = grid_of(kind, s);
    DCU_CUDA(c, cudaMemsetAsync(&a.S->done, 0, sizeof(int), c->stream));
    switch (kind) {
      case IK_P: k_bi_p<MT, IT, VT><<<g, BI_BLOCK, 0, c->stream>>>(a); break;
      case IK_Y: k_bi_y<MT, IT, VT><<<g, BI_BLOCK, 0, c->stream>>>(a); break;
      case IK_PY: k_bi_py<MT, IT, VT><<<g, BI_BLOCK, 0, c->stream>>>(a); break;
      case IK_AY: k_bi_ay<MT, IT, VT><<<g, BI_BLOCK, 0, c->stream>>>(a); break;
      case IK_SZ: k_bi_sz<MT, IT, VT><<<g, BI_BLOCK, 0, c->stream>>>(a); break;
      case IK_AZ: k_bi_az<MT, IT, VT><<<g, BI_BLOCK, 0, c->stream>>>(a); break;
      default: k_bi_xr<MT, IT, VT><<<g, BI_BLOCK, 0, c->stream>>>(a); break;
    }
    DCU_LAUNCHED(c, "profile kernel");
    return DCU_OK;
  };
  c->profile_grid = grid_of;

  Scal hs;
  Scal* pin = reinterpret_cast<Scal*>(c->pinned);
  int* flag = reinterpret_cast<int*>(reinterpret_cast<char*>(c->pinned) + 1024);
  // Every chunk either finishes or advances the counter by `chunk`, and
  // each replacement advances it by one, so these bounds are never reached
  // by a working solver; they turn a logic error into a failure, not a hang.
  const long long max_chunks = (long long)maxiter / chunk + 4;
  for (int restarts = 0;; ++restarts) {
    if (restarts > maxiter + 1) return fail(c, DCU_ERR_CUDA, "solver did not terminate (restarts)");
    for (long long i = 0;; ++i) {
      if (i > max_chunks) return fail(c, DCU_ERR_CUDA, "solver did not terminate (chunks)");
      DCU_CUDA(c, cudaGraphLaunch(ge->exec, c->stream));
      c->launches += ge->nodes;
      DCU_CUDA(c, cudaMemcpyAsync(flag + (i & 1), &a.S->done, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
      DCU_CUDA(c, cudaEventRecord(c->ev[2 + (i & 1)], c->stream));
      if (i > 0) {
        DCU_CUDA(c, cudaEventSynchronize(c->ev[2 + ((i - 1) & 1)]));
        if (flag[(i - 1) & 1]) break;
      }
    }
    DCU_CUDA(c, cudaMemcpyAsync(pin, a.S, sizeof(Scal), cudaMemcpyDeviceToHost, c->stream));
    DCU_CUDA(c, cudaStreamSynchronize(c->stream));
    hs = *pin;
    if (hs.verify_pending) {
      if (wide) {
        k_bi_wide<MT, IT, VT, WIDE_AX><<<g_wide, BI_BLOCK, 0, c->stream>>>(a);
        DCU_LAUNCHED(c, "k_bi_wide");
      }
      k_bi_true<MT, IT, VT><<<g_tr, BI_BLOCK, 0, c->stream>>>(a, 1);
      DCU_LAUNCHED(c, "k_bi_true");
      DCU_CUDA(c, cudaMemcpyAsync(pin, a.S, sizeof(Scal), cudaMemcpyDeviceToHost, c->stream));
      DCU_CUDA(c, cudaStreamSynchronize(c->stream));
      hs = *pin;
      if (!hs.done) continue;
    }
    break;
  }
  if (hs.true_res < 0.0) {
    if (wide) {
      k_bi_wide<MT, IT, VT, WIDE_AX><<<g_wide, BI_BLOCK, 0, c->stream>>>(a);
      DCU_LAUNCHED(c, "k_bi_wide");
    }
    k_bi_true<MT, IT, VT><<<g_tr, BI_BLOCK, 0, c->stream>>>(a, 0);
    DCU_LAUNCHED(c, "k_bi_true");
  }
  DCU_CUDA(c, cudaEventRecord(c->ev[1], c->stream));
  DCU_CUDA(c, cudaMemcpyAsync(pin, a.S, sizeof(Scal), cudaMemcpyDeviceToHost, c->stream));
  DCU_CUDA(c, cudaStreamSynchronize(c->stream));
  hs = *pin;
  if (info) {
    info->iters = hs.it;
    info->status = hs.status;
    info->replacements = hs.replacements;
    info->res = hs.res;
    info->true_res = hs.true_res;
    info->bnorm = hs.bnorm;
    info->a_fp32 = hs.a32;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
    info->ms = ms;
  }
  return DCU_OK;
}

}  // namespace

int bicgstab_solve(Ctx* c, const SellPlan& plan, const SellA& aval_sell, const void* mval_sell, const double* b,
                   double* x, const dcu_options* opt, dcu_solve_info* info, const void* mval8_sell) {
  const int p = opt->precision;
  const dcu_tuning* tu = (p >= 0 && p < 5 && c->tune_set[p]) ? &c->tune[p] : nullptr;
  if (p == DCU_PREC_FP64)
    return run_solver<double, int, double>(c, plan, aval_sell, (const double*)mval_sell, plan.idx, b, x, opt, tu, info);
  const bool m32 = (p == DCU_PREC_MIXED_FP32 || p == DCU_PREC_M_FP32);
  const bool v32 = (p == DCU_PREC_MIXED_FP32 || p == DCU_PREC_MIXED_BF16);
  const float* mf = (const float*)mval_sell;
  const __nv_bfloat16* mb = (const __nv_bfloat16*)mval_sell;
  const float* mf8 = (const float*)mval8_sell;
  const __nv_bfloat16* mb8 = (const __nv_bfloat16*)mval8_sell;
  if (plan.delta16) {
    if (m32) return v32 ? run_solver<float, int16_t, float>(c, plan, aval_sell, mf, plan.del, b, x, opt, tu, info, mf8)
                        : run_solver<float, int16_t, double>(c, plan, aval_sell, mf, plan.del, b, x, opt, tu, info, mf8);
    return v32 ? run_solver<__nv_bfloat16, int16_t, float>(c, plan, aval_sell, mb, plan.del, b, x, opt, tu, info, mb8)
               : run_solver<__nv_bfloat16, int16_t, double>(c, plan, aval_sell, mb, plan.del, b, x, opt, tu, info, mb8);
  }
  if (m32) return v32 ? run_solver<float, int, float>(c, plan, aval_sell, mf, plan.idx, b, x, opt, tu, info, mf8)
                      : run_solver<float, int, double>(c, plan, aval_sell, mf, plan.idx, b, x, opt, tu, info, mf8);
  return v32 ? run_solver<__nv_bfloat16, int, float>(c, plan, aval_sell, mb, plan.idx, b, x, opt, tu, info, mb8)
             : run_solver<__nv_bfloat16, int, double>(c, plan, aval_sell, mb, plan.idx, b, x, opt, tu, info, mb8);
}

namespace {

// Mean device time (ms) of the stop-flag reset that precedes every profiled launch.
int reset_ms(Ctx* c, int reps, float* out) {
  int* done = reinterpret_cast<int*>(c->buf[B_SCAL].p) + offsetof(Scal, done) / sizeof(int);
  DCU_CUDA(c, cudaEventRecord(c->ev[0], c->stream));
  for (int r = 0; r < reps; ++r) DCU_CUDA(c, cudaMemsetAsync(done, 0, sizeof(int), c->stream));
  DCU_CUDA(c, cudaEventRecord(c->ev[1], c->stream));
  DCU_CUDA(c, cudaEventSynchronize(c->ev[1]));
  float t = 0.f;
  cudaEventElapsedTime(&t, c->ev[0], c->ev[1]);
  *out = t / reps;
  return DCU_OK;
}

// Mean device time (ms) of `kind` at selector `sel`.  Each timed launch
// follows an untimed launch of the kernel that precedes it in the iteration
// (`pred` at `pred_sel`), so L2 holds what it holds in a solve (A alone is
// larger than L2; back-to-back launches of one kernel would find part of
// their own data there).
int time_kernel(Ctx* c, int kind, int sel, int pred, int pred_sel, int reps, float reset, float* out) {
  DCU_TRY(c->profile_launch(kind, sel));  // warm-up
  float total = 0.f;
  for (int r = 0; r < reps; ++r) {
    DCU_TRY(c->profile_launch(pred, pred_sel));
    DCU_CUDA(c, cudaEventRecord(c->ev[0], c->stream));
    DCU_TRY(c->profile_launch(kind, sel));
    DCU_CUDA(c, cudaEventRecord(c->ev[1], c->stream));
    DCU_CUDA(c, cudaEventSynchronize(c->ev[1]));
    float t = 0.f;
    cudaEventElapsedTime(&t, c->ev[0], c->ev[1]);
    total += t;
  }
  *out = total / reps - reset;
  return DCU_OK;
}

}  // namespace

int profile_iteration(Ctx* c, int reps, float* ms, int cap, int* count) {
  if (!c->profile_launch) return fail(c, DCU_ERR_ARG, "no solve has run on this context");
  const int nk = (int)c->profile_order.size();
  if (count) *count = nk;
  if (cap < nk) return fail(c, DCU_ERR_ARG, "ms_out holds fewer entries than kernels");
  if (reps < 1) reps = 1;
  float reset = 0.f;
  DCU_TRY(reset_ms(c, reps, &reset));
  for (int j = 0; j < nk; ++j) {
    const int pj = (j + nk - 1) % nk;
    DCU_TRY(time_kernel(c, c->profile_order[j], c->profile_sel[j], c->profile_order[pj], c->profile_sel[pj], reps,
                        reset, &ms[j]));
  }
  return DCU_OK;
}

int tune_iteration(Ctx* c, int reps, dcu_tuning* t, int* timed) {
  if (!c->profile_launch) return fail(c, DCU_ERR_ARG, "no solve has run on this context");
  if (reps < 1) reps = 10;
  float reset = 0.f;
  DCU_TRY(reset_ms(c, reps, &reset));
  // the kernels without a reduction, each after its predecessor in the iteration
  std::vector<std::pair<int, int>> kinds = {{IK_P, IK_XR}, {IK_Y, IK_P}, {IK_SZ, IK_AY}};
  if (c->profile_k1_free) kinds.push_back({IK_PY, IK_XR});
  float def[IK_COUNT] = {}, best[IK_COUNT] = {};
  int best_sel[IK_COUNT] = {};
  int n_timed = 0;
  for (auto [kind, pred] : kinds) {
    // candidates: one wave (the default), one block per 256 rows, half the
    // resident blocks per SM; a candidate with the same grid as an earlier one
    // is not timed again
    std::vector<int> cands = {0, -1};
    const int full = c->profile_grid(kind, 0);
    for (int k = 1; k <= 32; ++k) {
      if (c->profile_grid(kind, k) == full) {  // k reaches the resident count
        if (k / 2 >= 1) cands.push_back(k / 2);
        break;
      }
    }
    std::vector<int> grids;
    for (int s : cands) {
      const int g = c->profile_grid(kind, s);
      bool seen = false;
      for (int h : grids) seen = seen || h == g;
      if (seen) continue;
      grids.push_back(g);
      float ms = 0.f;
      DCU_TRY(time_kernel(c, kind, s, pred, 0, reps, reset, &ms));
      ++n_timed;
      if (s == 0) {
        def[kind] = best[kind] = ms;
        best_sel[kind] = 0;
      } else if (ms < 0.99f * best[kind]) {  // a change must win by more than 1%
        best[kind] = ms;
        best_sel[kind] = s;
      }
    }
  }
  const bool dsplit = c->profile_default_split != 0;
  bool split = dsplit;
  if (c->profile_k1_free) {
    const float fused = best[IK_PY], sp = best[IK_P] + best[IK_Y];
    if (dsplit ? fused < 0.99f * sp : sp < 0.99f * fused) split = !dsplit;
    t->k1_split = split ? 1 : 0;
  } else {
    t->k1_split = -1;
  }
  t->grid_p = best_sel[IK_P];
  t->grid_y = best_sel[IK_Y];
  t->grid_py = c->profile_k1_free ? best_sel[IK_PY] : 0;
  t->grid_sz = best_sel[IK_SZ];
  t->iter_us_default = 1000.f * ((dsplit ? def[IK_P] + def[IK_Y] : def[IK_PY]) + def[IK_SZ]);
  t->iter_us_tuned = 1000.f * ((split ? best[IK_P] + best[IK_Y] : best[IK_PY]) + best[IK_SZ]);
  if (timed) *timed = n_timed;
  return DCU_OK;
}

void release_graphs(Ctx* c) {
  for (auto& g : c->graphs) cudaGraphExecDestroy(g.exec);
  c->graphs.clear();
}

}  // namespace dcu
