// SPAI build: for every column k of M (pattern of M = pattern of A)
//   J_k = rows of A(:,k) in stored order            (computeJ_SSPAIv10,
//                                                     src/spai_multi_dcu.cpp:275-295)
//   I_k = sorted, duplicate-free union of the rows of A(:,j), j in J_k
//                                                    (computeI*_Symbol_SpMMv1 :321-834)
//   At  = A(I_k, J_k), dense                        (ComputeTildeACSR_SSPAIv10 :945-983)
//   E   = position of k in I_k, -1 if absent        (ComputeTildeE_SSPAIv10 :985-1004)
//   m_k = argmin || At m - e_E ||_2                  (QR_RShared_SSPAIv10 :1069-1133 and
//                                                     Sol_SSPAIv10 :1028-1067 do this by
//                                                     modified Gram-Schmidt; here by
//                                                     Householder QR of [At | e_E])
//   M(J_k, k) = m_k                                  (modifyData4_SSPAIv10 :1135-1152)
//
// Two kernels share the column range through a device work queue:
//   k_spai_small  one 16-lane group per column (two per warp), |J_k| <= 7,
//                 <= 64 candidate rows, |I_k| <= 32 (or the tuned
//                 group_max_ni below it): candidates sorted in registers
//                 (bitonic network across the group), At staged in shared
//                 memory, two lanes per column of [At | e_E], each holding
//                 half its rows in registers.
//   k_spai_large  one CTA per column for everything else: I_k by a bitmap
//                 over the candidate row range, At in shared memory or a
//                 global slab, Householder with warp-per-trailing-column
//                 updates, column-oriented back substitution.
// Columns that do not fit the small kernel are appended to a list the large
// kernel drains with an atomic counter.  Each column's arithmetic is fixed by
// its own data (fixed reduction trees, no float atomics), so M is identical
// for every schedule and grid size.
#include <algorithm>
#include <climits>
#include <type_traits>
#include <vector>

#include "internal.cuh"

namespace dcu {
namespace {

enum { MODE_COUNT = 0, MODE_LIST = 1, MODE_BUILD = 2 };

// stats[] layout (int32 unless noted)
enum {
  ST_BIG_COUNT = 0,   // columns queued for the CTA kernel
  ST_BIG_MAXNJ = 1,   // max |J_k| over queued columns
  ST_SINGULAR = 2,    // columns with a zero / non-finite pivot
  ST_MAXNI = 3,       // max |I_k|
  ST_SMALL_COLS = 4,  // columns finished by the small kernel
  ST_LIMIT = 5,       // a column exceeded a CTA-kernel limit
  ST_MAXNJ = 6,       // max |J_k|
  ST_BIG_HEAD = 7,    // queue head of the CTA kernel
  ST_DYN_HEAD = 8,    // queue head of the dynamic schedule
  ST_BIG_DONE = 9,    // columns finished by the CTA kernel
  ST_FB_COUNT = 10,   // columns the thread kernel hands to the group kernel
  ST_FB_HEAD = 11,    // queue head of that hand-off list
  ST_NE_COLS = 12,    // columns finished by the thread kernel
  ST_STAGE_FAIL = 13, // a bulk copy into shared memory did not complete in time
  ST_STAGED = 16,     // CTA-kernel columns whose J columns were staged by bulk copies
  ST_HUB_COUNT = 17,  // columns handed to the hub kernels
  ST_INTS = 24,
  ST_AREA64 = 7,      // long long index (ints 14-15): max candidates * (|J|+1) over queued columns
  ST_AREASUM64 = 9,   // long long index (ints 18-19): sum of (candidates + 2) * (|J|+1) over queued columns
  ST_HUBHEAD64 = 10   // long long index (ints 20-21): elements of the hub pool handed out
};

constexpr int GL = 16;          // lanes per least-squares problem: 2 per column of [At | e_E]
constexpr int SG_GPW = 2;       // problems (groups) per warp
constexpr int SG_BLOCK = 64;    // 2 warps, 4 groups
constexpr int SG_WARPS = SG_BLOCK / 32;
constexpr int SG_MMAX = 32;     // max |I_k| on the group path
constexpr int SG_CMAX = 64;     // max candidate rows on the group path
constexpr int SG_NJMAX = 7;     // max |J_k| ([At | e_E] has <= 8 columns)
constexpr int SG_COLS = 8;
constexpr unsigned kPad = 0xFFFFFFFFu;

struct SmallArgs {
  int n;
  const int* ptr;
  const int* idx;
  const double* val;
  int col_start, col_end;
  int schedule;
  const int* chunks;  // dynamic schedule: nnz-balanced chunk bounds
  int nchunks;
  double* mval;
  double* colres;
  int* icount;
  const long long* iptr;
  int* ilist;
  int* big_list;
  int* stats;
  const int* list;    // when set: process these columns (count in stats[ST_FB_COUNT])
  int max_ni;         // largest |I_k| this kernel takes (<= SG_MMAX); larger go to the CTA kernel
};

// Shared state of the two groups of a warp.  Row strides are padded so the
// groups' broadcasts of v fall in different banks.
template <typename T>
struct WarpSmem {
  T At[SG_GPW][SG_COLS][SG_MMAX + 1];  // column j of [A(I,J) | e_E]; later R
  T v[SG_GPW][SG_MMAX + 2];            // Householder vector; then y; then x
  T dinv[SG_GPW][SG_COLS];             // 1 / R_jj
  T beta[SG_GPW][2];
  unsigned key[SG_GPW][SG_CMAX];       // candidate keys (row << 6 | candidate)
  int src[SG_GPW][SG_CMAX];            // candidate -> position in A's arrays
  signed char jj[SG_GPW][SG_CMAX];
};

__device__ __forceinline__ void queue_big(const SmallArgs& a, int k, int nj, long long area) {
  int q = atomicAdd(&a.stats[ST_BIG_COUNT], 1);
  a.big_list[q] = k;
  atomicMax(&a.stats[ST_BIG_MAXNJ], nj);
  atomicMax(reinterpret_cast<unsigned long long*>(a.stats) + ST_AREA64, (unsigned long long)area);
  // bound of the column's hub slab: |I| (<= candidates) x (|J| + 1), plus two scalars per step
  atomicAdd(reinterpret_cast<unsigned long long*>(a.stats) + ST_AREASUM64, (unsigned long long)(area + 2LL * (nj + 1)));
}

// Bitonic sort of GL*PER keys held PER per lane (element e = lane*PER + s),
// ascending, across the GL lanes of a group.
template <int PER>
__device__ __forceinline__ void group_sort(unsigned (&key)[PER], int lane, unsigned gmask) {
  constexpr int N = GL * PER;
#pragma unroll
  for (int kk = 2; kk <= N; kk <<= 1) {
#pragma unroll
    for (int jj = kk >> 1; jj > 0; jj >>= 1) {
      if (jj >= PER) {
        const int lx = jj / PER;
#pragma unroll
        for (int s = 0; s < PER; ++s) {
          const unsigned other = __shfl_xor_sync(gmask, key[s], lx, GL);
          const int e = lane * PER + s;
          const bool up = (e & kk) == 0;
          const bool lower = (e & jj) == 0;
          const unsigned mn = min(key[s], other), mx = max(key[s], other);
          key[s] = (lower == up) ? mn : mx;
        }
      } else {
#pragma unroll
        for (int s = 0; s < PER; ++s) {
          const int p = s ^ jj;
          if (p > s) {
            const int e = lane * PER + s;
            const bool up = (e & kk) == 0;
            const unsigned x = key[s], y = key[p];
            const unsigned lo = min(x, y), hi = max(x, y);
            key[s] = up ? lo : hi;
            key[p] = up ? hi : lo;
          }
        }
      }
    }
  }
}

// Householder QR of [At | e_E] and back substitution.  Lane = 2 * column +
// half: each lane holds RPL = MMAX / 2 consecutive rows of one column in
// registers.  The step loop is fully unrolled (steps < 8 <= RPL, so the
// diagonal entry of every step lives in the first half).  Rows above the step
// are excluded from the reflector by zeros in v.  Returns true for a zero /
// non-finite pivot.
template <int MMAX, typename T>
__device__ __forceinline__ bool group_qr_solve(const SmallArgs& a, WarpSmem<T>& ws, int g, int lane,
                                               unsigned gmask, int k, int cs, int nj, int m) {
  constexpr int RPL = MMAX / 2;
  const int j = lane >> 1, h = lane & 1, row0 = h * RPL;
  T r[RPL];
#pragma unroll
  for (int t = 0; t < RPL; ++t) r[t] = ws.At[g][j][row0 + t];
  T* v = ws.v[g];
  bool sing = false;
  const int steps = min(nj, m);
#pragma unroll
  for (int c = 0; c < SG_NJMAX; ++c) {
    if (c >= steps) break;
    // both lanes of column c: norm of rows >= c (two independent partial
    // sums: a shorter dependent chain), reflector, R_cc
    T pp[2] = {T(0), T(0)};
#pragma unroll
    for (int t = 0; t < RPL; ++t) pp[t & 1] += (row0 + t >= c) ? r[t] * r[t] : T(0);
    T part = pp[0] + pp[1];
    part += __shfl_xor_sync(gmask, part, 1, GL);
    const T nrm2 = __shfl_sync(gmask, part, 2 * c, GL);
    const T x0 = __shfl_sync(gmask, r[c], 2 * c, GL);  // row c < RPL: first half
    const T nrm = sqrt(nrm2);
    T alpha = T(0), beta = T(0);
    if (nrm > T(0)) {
      alpha = (x0 > T(0)) ? -nrm : nrm;
      beta = T(1) / (nrm * (nrm + fabs(x0)));  // 2 / (v^T v)
    } else {
      sing = true;
    }
    if (j == c) {
#pragma unroll
      for (int t = 0; t < RPL; ++t) {
        const int i = row0 + t;
        v[i] = (i < c) ? T(0) : ((i == c) ? x0 - alpha : r[t]);
        if (i == c) r[t] = alpha;
        else if (i > c) r[t] = T(0);
      }
    }
    __syncwarp(gmask);
    const bool trailing = (j > c) && (j <= nj);
    // v is re-read from shared memory in both loops (volatile) rather than
    // held in RPL more registers: fewer registers, more resident problems
    const volatile T* vv = v + row0;
    T wp[2] = {T(0), T(0)};
    if (trailing) {
#pragma unroll
      for (int t = 0; t < RPL; ++t) wp[t & 1] += vv[t] * r[t];
    }
    T w = wp[0] + wp[1];
    w += __shfl_xor_sync(gmask, w, 1, GL);
    if (trailing) {
      w *= beta;
#pragma unroll
      for (int t = 0; t < RPL; ++t) r[t] -= w * vv[t];
    }
    __syncwarp(gmask);
  }
  // R -> At (rows <= column), y -> v, 1/R_jj -> dinv, ||(Q^T e_E)[nj:]||^2
  T res2 = T(0);
  if (j < nj && h == 0) {
    T d = T(0);
#pragma unroll
    for (int t = 0; t < SG_COLS; ++t) {
      if (t <= j) ws.At[g][j][t] = r[t];
      if (t == j) d = r[t];
    }
    if (!(d != T(0)) || !isfinite((double)d)) sing = true;
    ws.dinv[g][j] = T(1) / d;
  } else if (j == nj) {
#pragma unroll
    for (int t = 0; t < RPL; ++t) {
      const int i = row0 + t;
      if (i < nj) v[i] = r[t];
      else res2 += r[t] * r[t];
    }
  }
  res2 += __shfl_xor_sync(gmask, res2, 1, GL);
  __syncwarp(gmask);
  // R x = y, column by column: lane i holds y_i; at step jc lane jc's x_jc
  // is final, goes to every lane, and the lanes above it subtract its column
  // (one shuffle per step instead of one lane walking the whole triangle)
  T yi = (lane < nj) ? v[lane] : T(0);
  const T di = (lane < nj) ? ws.dinv[g][lane] : T(0);
  for (int jc = nj - 1; jc >= 0; --jc) {
    const T xj = __shfl_sync(gmask, yi * di, jc, GL);
    if (lane < jc) yi -= ws.At[g][jc][lane] * xj;
    else if (lane == jc) yi = xj;
  }
  if (lane < nj) a.mval[cs + lane] = (double)yi;
  if (j == nj && h == 0 && a.colres) a.colres[k - a.col_start] = sqrt((double)res2);
  const unsigned any_sing = __ballot_sync(gmask, sing) & gmask;
  __syncwarp(gmask);
  return any_sing != 0;
}

// Everything after candidate staging for one column, PER keys per lane.
// Returns |I_k| (or -1 when the column was queued for the CTA kernel).
template <int PER, typename T, int MODE>
__device__ __forceinline__ int group_column(const SmallArgs& a, WarpSmem<T>& ws, int g, int k, int cs, int nj,
                                            int cand, int lane, unsigned gmask) {
  unsigned key[PER];
#pragma unroll
  for (int s = 0; s < PER; ++s) {
    const int t = lane * PER + s;
    key[s] = (t < cand) ? ws.key[g][t] : kPad;
  }
  group_sort<PER>(key, lane, gmask);

  // distinct rows: flag the first element of each run of equal rows; pre[s]
  // is the inclusive count of firsts in this lane, negated for repeats
  const unsigned prev = __shfl_up_sync(gmask, key[PER - 1], 1, GL);
  int pre[PER];
  int cnt = 0;
#pragma unroll
  for (int s = 0; s < PER; ++s) {
    const bool valid = key[s] != kPad;
    const unsigned before = (s == 0) ? prev : key[s - 1];
    const bool first = valid && ((s == 0 && lane == 0) || (before >> 6) != (key[s] >> 6));
    cnt += first ? 1 : 0;
    pre[s] = first ? cnt : -cnt;
  }
  int inc = cnt;
#pragma unroll
  for (int d = 1; d < GL; d <<= 1) {
    const int t = __shfl_up_sync(gmask, inc, d, GL);
    if (lane >= d) inc += t;
  }
  const int excl = inc - cnt;
  const int m = __shfl_sync(gmask, inc, GL - 1, GL);

  if (m > a.max_ni) {
    if (lane == 0) queue_big(a, k, nj, (long long)cand * (nj + 1));
    return -1;
  }
  const int col = k - a.col_start;
  if (MODE == MODE_COUNT) {
    if (lane == 0) a.icount[col] = m;
    return m;
  }
  if (MODE == MODE_LIST) {
    const long long base = a.iptr[col];
#pragma unroll
    for (int s = 0; s < PER; ++s)
      if (pre[s] > 0) a.ilist[base + excl + pre[s] - 1] = (int)(key[s] >> 6);
    return m;
  }

  // ---- build: gather At = A(I, J) and e_E into shared memory -------------
  int E = -1;
#pragma unroll
  for (int s = 0; s < PER; ++s)
    if (pre[s] > 0 && (int)(key[s] >> 6) == k) E = excl + pre[s] - 1;
#pragma unroll
  for (int d = 1; d < GL; d <<= 1) E = max(E, __shfl_xor_sync(gmask, E, d, GL));
  for (int i = lane; i < SG_COLS * (SG_MMAX + 1); i += GL) (&ws.At[g][0][0])[i] = T(0);
  __syncwarp(gmask);
#pragma unroll
  for (int s = 0; s < PER; ++s) {
    if (key[s] != kPad) {
      const int t = key[s] & 63;
      const int pos = excl + (pre[s] > 0 ? pre[s] : -pre[s]) - 1;
      ws.At[g][ws.jj[g][t]][pos] = (T)__ldg(a.val + ws.src[g][t]);
    }
  }
  if (lane == 0 && E >= 0) ws.At[g][nj][E] = T(1);
  __syncwarp(gmask);
  // row tiles of 16, 26 (a 3D 7-point column has |I| = 25) or 32 rows
  const bool sing = (m < nj) | ((m <= 16) ? group_qr_solve<16, T>(a, ws, g, lane, gmask, k, cs, nj, m)
                                : (m <= 26) ? group_qr_solve<26, T>(a, ws, g, lane, gmask, k, cs, nj, m)
                                            : group_qr_solve<32, T>(a, ws, g, lane, gmask, k, cs, nj, m));
  if (sing && lane == 0) atomicAdd(&a.stats[ST_SINGULAR], 1);
  return m;
}

// Held to 80 registers (12 blocks, 24 warps per SM): the Householder steps are
// latency-bound, and at the unbounded 128 registers only 8 blocks fit (FP64
// build at 128^3: 7.06 -> 5.92 ms, M bit-identical; at 64 registers it spills
// and takes 6.3 ms).
template <typename T, int MODE>
__global__ void __launch_bounds__(SG_BLOCK, 12) k_spai_small(SmallArgs a) {
  __shared__ WarpSmem<T> smem[SG_WARPS];
  const int lane = threadIdx.x & (GL - 1);
  const int g = (threadIdx.x / GL) & (SG_GPW - 1);
  const unsigned gmask = 0xFFFFu << (threadIdx.x & 16);
  WarpSmem<T>& ws = smem[threadIdx.x >> 5];
  const int gid = (blockIdx.x * SG_BLOCK + threadIdx.x) / GL;
  const int ngroups = (gridDim.x * SG_BLOCK) / GL;
  int my_max_ni = 0, my_max_nj = 0, my_cols = 0;

  auto process = [&](int k) {
    const int cs = __ldg(a.ptr + k);
    const int nj = __ldg(a.ptr + k + 1) - cs;
    my_max_nj = max(my_max_nj, nj);
    if (nj == 0) {
      if (lane == 0) {
        if (MODE == MODE_COUNT) a.icount[k - a.col_start] = 0;
        if (MODE == MODE_BUILD && a.colres) a.colres[k - a.col_start] = 1.0;
      }
      ++my_cols;
      return;
    }
    if (nj > SG_NJMAX) {
      // candidate count is only needed as a slab bound: count it here
      long long cand = 0;
      for (int t = lane; t < nj; t += GL) {
        const int j = __ldg(a.idx + cs + t);
        cand += __ldg(a.ptr + j + 1) - __ldg(a.ptr + j);
      }
#pragma unroll
      for (int d = 1; d < GL; d <<= 1) cand += __shfl_xor_sync(gmask, cand, d, GL);
      if (lane == 0) queue_big(a, k, nj, cand * (nj + 1));
      return;
    }
    int bj = 0, lj = 0;
    if (lane < nj) {
      const int j = __ldg(a.idx + cs + lane);
      bj = __ldg(a.ptr + j);
      lj = __ldg(a.ptr + j + 1) - bj;
    }
    int inc = lj;
#pragma unroll
    for (int d = 1; d < GL; d <<= 1) {
      const int t = __shfl_up_sync(gmask, inc, d, GL);
      if (lane >= d) inc += t;
    }
    const int cand = __shfl_sync(gmask, inc, GL - 1, GL);
    const int cb = inc - lj;
    if (cand > SG_CMAX) {
      if (lane == 0) queue_big(a, k, nj, (long long)cand * (nj + 1));
      return;
    }
    for (int j = 0; j < nj; ++j) {
      const int bjj = __shfl_sync(gmask, bj, j, GL);
      const int ljj = __shfl_sync(gmask, lj, j, GL);
      const int cbj = __shfl_sync(gmask, cb, j, GL);
      for (int q = lane; q < ljj; q += GL) {
        const int t = cbj + q;
        const int row = __ldg(a.idx + bjj + q);
        ws.key[g][t] = ((unsigned)row << 6) | (unsigned)t;
        ws.src[g][t] = bjj + q;
        ws.jj[g][t] = (signed char)j;
      }
    }
    __syncwarp(gmask);
    const int m = (cand <= 32) ? group_column<2, T, MODE>(a, ws, g, k, cs, nj, cand, lane, gmask)
                               : group_column<4, T, MODE>(a, ws, g, k, cs, nj, cand, lane, gmask);
    __syncwarp(gmask);
    if (m >= 0) {
      my_max_ni = max(my_max_ni, m);
      ++my_cols;
    }
  };

  if (a.list) {
    // columns handed over by the thread kernel, pulled one at a time
    const int count = a.stats[ST_FB_COUNT];
    for (;;) {
      int q = 0;
      if (lane == 0) q = atomicAdd(&a.stats[ST_FB_HEAD], 1);
      q = __shfl_sync(gmask, q, 0, GL);
      if (q >= count) break;
      process(a.list[q]);
    }
  } else if (a.schedule == DCU_SCHED_BALANCED_COLUMNS) {
    // balanced_columns: the units' contiguous ranges, in order, are the
    // whole column range; the groups sweep it together, group q taking
    // columns q, q + ngroups, ...  Equal column counts per group whatever the
    // unit count, and every group works in one window of the matrix, so a
    // column's J_k neighbours (up to 16384 columns away in a 3D stencil) are
    // still in L2 when the neighbouring columns need them.  (Giving each group
    // its own range spread the groups over the whole matrix: A was read about
    // twice from DRAM, and a small unit count left most groups idle.)
    for (int k = a.col_start + gid; k < a.col_end; k += ngroups) process(k);
  } else {
    // nnz-balanced chunks pulled from the queue
    for (;;) {
      int ch = 0;
      if (lane == 0) ch = atomicAdd(&a.stats[ST_DYN_HEAD], 1);
      ch = __shfl_sync(gmask, ch, 0, GL);
      if (ch >= a.nchunks) break;
      const int s = a.chunks[ch], e = a.chunks[ch + 1];
      for (int k = s; k < e; ++k) process(k);
    }
  }
  if (lane == 0) {
    atomicMax(&a.stats[ST_MAXNI], my_max_ni);
    atomicMax(&a.stats[ST_MAXNJ], my_max_nj);
    atomicAdd(&a.stats[ST_SMALL_COLS], my_cols);
  }
}


// ---------------------------------------------------------------------------
// Thread per column: the batched least-squares path of the mixed forms.
// One thread solves min || A(:,J) m - e_k || for |J_k| <= 8 through the
// normal equations G m = g with G = A(:,J)^T A(:,J) (sparse dot products of
// A's columns) and g = A(k,J)^T, factored G = U^T U by Cholesky in
// registers.  Hundreds of columns per SM are in flight, against tens on the
// group path.  A column whose Cholesky pivots drop below tau * G_jj (the
// normal equations' rounding would exceed the preconditioner's own precision)
// or that exceeds the size limits is handed to the Householder group kernel.
// ---------------------------------------------------------------------------
constexpr int NE_BLOCK = 128;
constexpr int NE_NJ = 8;      // max |J_k| on the thread path
constexpr int NE_CMAX = 52;   // max entries over the J_k columns (a 3D 7-point column has 49)

struct NeArgs {
  int n;
  const int* ptr;
  const int* idx;
  const double* val;
  int col_start, col_end;
  int schedule;
  const int* chunks;
  int nchunks;
  double* mval;
  double* colres;
  int* fb_list;
  int* stats;
  double tau;
};

template <int N>
__host__ __device__ constexpr int tri_n(int a, int b) { return a * N - (a * (a - 1)) / 2 + (b - a); }

template <typename T>
__global__ void __launch_bounds__(NE_BLOCK) k_spai_ne(NeArgs a) {
  extern __shared__ __align__(16) unsigned char ne_raw[];
  int* srow = reinterpret_cast<int*>(ne_raw);                                  // [NE_CMAX][NE_BLOCK]
  T* sval = reinterpret_cast<T*>(ne_raw + sizeof(int) * NE_CMAX * NE_BLOCK);   // [NE_CMAX][NE_BLOCK]
  __shared__ int s_chunk;
  const int tid = threadIdx.x;
  int my_cols = 0, my_max_nj = 0;

  // Column k with |J| <= NJ (NJ: the register tiles' size, a compile-time
  // constant; padding positions hold zeros and the identity, which leave the
  // others' values unchanged bit for bit).
  auto process = [&](auto njc, int k) {
    constexpr int NJ = decltype(njc)::value;
    const int cs = __ldg(a.ptr + k);
    const int nj = __ldg(a.ptr + k + 1) - cs;
    my_max_nj = max(my_max_nj, nj);
    if (nj == 0) {
      if (a.colres) a.colres[k - a.col_start] = 1.0;
      ++my_cols;
      return;
    }
    if (nj > NJ) {
      a.fb_list[atomicAdd(&a.stats[ST_FB_COUNT], 1)] = k;
      return;
    }
    int base[NJ], len[NJ], cb[NJ];
    int cand = 0;
#pragma unroll
    for (int j = 0; j < NJ; ++j) {
      base[j] = 0;
      len[j] = 0;
      if (j < nj) {
        const int col = __ldg(a.idx + cs + j);
        base[j] = __ldg(a.ptr + col);
        len[j] = __ldg(a.ptr + col + 1) - base[j];
      }
      cb[j] = cand;
      cand += len[j];
    }
    if (cand > NE_CMAX) {
      a.fb_list[atomicAdd(&a.stats[ST_FB_COUNT], 1)] = k;
      return;
    }
    bool sorted = true;
#pragma unroll
    for (int j = 0; j < NJ; ++j) {
      int prev = -1;
      for (int q = 0; q < len[j]; ++q) {
        const int r = __ldg(a.idx + base[j] + q);
        sorted = sorted && (r > prev);
        prev = r;
        srow[(cb[j] + q) * NE_BLOCK + tid] = r;
        sval[(cb[j] + q) * NE_BLOCK + tid] = (T)__ldg(a.val + base[j] + q);
      }
    }
    // G (upper triangle) and g = A(k, J)^T
    T G[NJ * (NJ + 1) / 2], g[NJ];
#pragma unroll
    for (int i = 0; i < NJ * (NJ + 1) / 2; ++i) G[i] = T(0);
#pragma unroll
    for (int j = 0; j < NJ; ++j) g[j] = T(0);
    if (sorted) {
      // Rows ascending in every column: one K-way merge over the columns.
      // Each step takes the smallest row r left among the column heads,
      // forms v = A(r, J) (zero where a column lacks r) and adds v v^T to G
      // and v to g when r = k.  Every G entry sums its products in ascending
      // row order, as a pairwise merge would; each entry is read once.  Each
      // step consumes at least one entry, so it runs at most cand times.
      int pos[NJ], head[NJ];
#pragma unroll
      for (int j = 0; j < NJ; ++j) {
        pos[j] = cb[j];
        head[j] = (len[j] > 0) ? srow[cb[j] * NE_BLOCK + tid] : INT_MAX;
      }
      for (int step = 0; step < cand; ++step) {
        int m = head[0];
#pragma unroll
        for (int j = 1; j < NJ; ++j) m = min(m, head[j]);
        if (m == INT_MAX) break;
        T v[NJ];
#pragma unroll
        for (int j = 0; j < NJ; ++j) {
          v[j] = T(0);
          if (head[j] == m) {
            v[j] = sval[pos[j] * NE_BLOCK + tid];
            ++pos[j];
            head[j] = (pos[j] < cb[j] + len[j]) ? srow[pos[j] * NE_BLOCK + tid] : INT_MAX;
          }
        }
        if (m == k) {
#pragma unroll
          for (int j = 0; j < NJ; ++j) g[j] += v[j];
        }
#pragma unroll
        for (int ja = 0; ja < NJ; ++ja) {
#pragma unroll
          for (int jb = ja; jb < NJ; ++jb) G[tri_n<NJ>(ja, jb)] += v[ja] * v[jb];
        }
      }
    } else {
#pragma unroll
      for (int ja = 0; ja < NJ; ++ja) {
        for (int p = cb[ja]; p < cb[ja] + len[ja]; ++p) {
          const int r = srow[p * NE_BLOCK + tid];
          const T v = sval[p * NE_BLOCK + tid];
          if (r == k) g[ja] += v;
          G[tri_n<NJ>(ja, ja)] += v * v;
        }
      }
#pragma unroll
      for (int ja = 0; ja < NJ; ++ja) {
        for (int p = cb[ja]; p < cb[ja] + len[ja]; ++p) {
          const int r = srow[p * NE_BLOCK + tid];
          const T v = sval[p * NE_BLOCK + tid];
#pragma unroll
          for (int jb = ja + 1; jb < NJ; ++jb) {
            T acc = T(0);
            for (int q = cb[jb]; q < cb[jb] + len[jb]; ++q)
              if (srow[q * NE_BLOCK + tid] == r) acc += sval[q * NE_BLOCK + tid];
            G[tri_n<NJ>(ja, jb)] += v * acc;
          }
        }
      }
    }
    // pad to 8 x 8 with the identity, factor G = U^T U in place
#pragma unroll
    for (int j = 0; j < NJ; ++j)
      if (j >= nj) G[tri_n<NJ>(j, j)] = T(1);
    bool ok = true;
#pragma unroll
    for (int j = 0; j < NJ; ++j) {
      const T gjj = G[tri_n<NJ>(j, j)];
      T d = gjj;
#pragma unroll
      for (int p = 0; p < j; ++p) d -= G[tri_n<NJ>(p, j)] * G[tri_n<NJ>(p, j)];
      if (!(d > (T)a.tau * gjj) || !isfinite((double)d)) ok = false;
      const T ujj = sqrt(d > T(0) ? d : T(1));
      const T inv = T(1) / ujj;
      G[tri_n<NJ>(j, j)] = ujj;
#pragma unroll
      for (int i = j + 1; i < NJ; ++i) {
        T t = G[tri_n<NJ>(j, i)];
#pragma unroll
        for (int p = 0; p < j; ++p) t -= G[tri_n<NJ>(p, j)] * G[tri_n<NJ>(p, i)];
        G[tri_n<NJ>(j, i)] = t * inv;
      }
    }
    if (!ok) {
      a.fb_list[atomicAdd(&a.stats[ST_FB_COUNT], 1)] = k;
      return;
    }
    // U^T y = g, U x = y
    T y[NJ];
#pragma unroll
    for (int j = 0; j < NJ; ++j) {
      T t = g[j];
#pragma unroll
      for (int p = 0; p < j; ++p) t -= G[tri_n<NJ>(p, j)] * y[p];
      y[j] = t / G[tri_n<NJ>(j, j)];
    }
#pragma unroll
    for (int j = NJ - 1; j >= 0; --j) {
      T t = y[j];
#pragma unroll
      for (int p = j + 1; p < NJ; ++p) t -= G[tri_n<NJ>(j, p)] * y[p];
      y[j] = t / G[tri_n<NJ>(j, j)];
    }
    double gx = 0.0;
#pragma unroll
    for (int j = 0; j < NJ; ++j)
      if (j < nj) {
        a.mval[cs + j] = (double)y[j];
        gx += (double)g[j] * (double)y[j];
      }
    // || A(:,J) m - e_k ||^2 = 1 - g^T m at the least-squares solution
    if (a.colres) a.colres[k - a.col_start] = sqrt(fmax(0.0, 1.0 - gx));
    ++my_cols;
  };

  // columns with |J| <= 7 (every column of a 2D or 3D stencil) on 7-wide
  // register tiles, the rest on 8-wide ones
  auto column = [&](int k) {
    if (__ldg(a.ptr + k + 1) - __ldg(a.ptr + k) <= 7) process(std::integral_constant<int, 7>{}, k);
    else process(std::integral_constant<int, NE_NJ>{}, k);
  };

  if (a.schedule == DCU_SCHED_BALANCED_COLUMNS) {
    // balanced_columns: one sweep of the whole range by all threads (see
    // k_spai_small)
    for (int k = a.col_start + blockIdx.x * NE_BLOCK + tid; k < a.col_end; k += gridDim.x * NE_BLOCK) column(k);
  } else {
    for (;;) {
      if (tid == 0) s_chunk = atomicAdd(&a.stats[ST_DYN_HEAD], 1);
      __syncthreads();
      const int ch = s_chunk;
      __syncthreads();
      if (ch >= a.nchunks) break;
      for (int k = a.chunks[ch] + tid; k < a.chunks[ch + 1]; k += NE_BLOCK) column(k);
    }
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    my_cols += __shfl_xor_sync(0xffffffffu, my_cols, d);
    my_max_nj = max(my_max_nj, __shfl_xor_sync(0xffffffffu, my_max_nj, d));
  }
  if ((tid & 31) == 0) {
    atomicAdd(&a.stats[ST_NE_COLS], my_cols);
    atomicMax(&a.stats[ST_MAXNJ], my_max_nj);
  }
}

// ---------------------------------------------------------------------------
// CTA per column.
// ---------------------------------------------------------------------------
constexpr int LG_BLOCK = 256;
constexpr int LG_WARPS = LG_BLOCK / 32;
constexpr int LG_NJ_MAX = 2048;      // max |J_k| (J metadata lives in shared memory)
constexpr int LG_WORDS_SMEM = 4096;  // bitmap words kept in shared memory
constexpr int LG_STAGE_NJ = 256;     // J columns staged in shared memory by bulk copies
constexpr int LG_STAGE_BYTES = 48 * 1024;
constexpr long long kStageWaitSpins = 1ll << 22;
constexpr long long kHubPoolMax = 1ll << 28;  // elements of the hub pool (2 GB in FP64)

// A column factored by the hub kernels: its dense block [A(I,J) | e_E]
// (m x (nj+1), column-major) at pool + off, followed by the Householder
// scalars alpha (R's diagonal) and beta of each step, (nj+1) each.
struct HubMeta {
  int k, m, nj, pad;
  long long off;
};

struct LargeArgs {
  int n;
  const int* ptr;
  const int* idx;
  const double* val;
  int col_start;
  double* mval;
  double* colres;
  int* icount;
  const long long* iptr;
  int* ilist;
  const int* big_list;
  int* stats;
  unsigned* gbits;         // per block: 2 * words_per_block words (bits, prefix)
  long long words_per_block;
  void* gA;                // per block: area_per_block elements of T
  long long area_per_block;
  long long smem_area;     // elements of T that fit the shared slab
  int stage_ok;            // idx (and val when building) 16-byte aligned: bulk copies allowed
  long long area_sum;      // ST_AREASUM64 of the queue (host side)
  long long hub_min_area;  // blocks larger than this go to the hub pool
  void* hub_pool;          // build: slabs of columns whose block exceeds shared memory (T)
  long long hub_cap;       // elements of T in hub_pool
  HubMeta* hub_meta;       // one per hub column, in hand-off order
};

// Bulk copies (the TMA engine, no multicast) of global ranges into this CTA's
// shared memory, completing on an mbarrier.  Addresses and sizes are
// multiples of 16 bytes.
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* mbar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%1], %0;" : : "r"(count), "r"(smem_u32(mbar)) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* mbar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%1], %0;" : : "r"(bytes), "r"(smem_u32(mbar))
               : "memory");
}
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* mbar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               :
               : "r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(mbar))
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* mbar, unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}"
      : "=r"(done)
      : "r"(smem_u32(mbar)), "r"(parity)
      : "memory");
  return done != 0;
}
// Bounded wait for the phase with the given parity; false when it gave up.
__device__ __forceinline__ bool mbar_wait(unsigned long long* mbar, unsigned parity) {
  for (long long i = 0; i < kStageWaitSpins; ++i)
    if (mbar_try_wait(mbar, parity)) return true;
  return false;
}

template <typename T>
struct LargeSmem {
  int jbase[LG_NJ_MAX];
  int jlen[LG_NJ_MAX];
  int jcb[LG_NJ_MAX + 1];
  unsigned bits[LG_WORDS_SMEM];
  int wpre[LG_WORDS_SMEM];
  T ys[LG_NJ_MAX];
  T rd[LG_NJ_MAX];
  double red[LG_WARPS];
  int ired[LG_WARPS * 2];
  int jso[LG_STAGE_NJ + 1];  // staged int range of J column j starts at jso[j] ints
  int jvo[LG_STAGE_NJ + 1];  // staged double range of J column j starts at jvo[j] doubles
  unsigned long long mbar;   // completion of the bulk copies
  long long hub_off;
  int col_q;
  int m;
  int E;
  T beta;
};

// Deterministic block sum of one value per thread (fixed tree).
__device__ __forceinline__ double block_sum(double v, double* red) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
#pragma unroll
  for (int w = 0; w < LG_WARPS; ++w) t += red[w];
  return t;
}

// Exclusive scan of `cnt` values (int) produced by f(i), i < count, into out[];
// returns the total.  Chunks of LG_BLOCK with a running carry.
template <typename F>
__device__ int block_scan(int count, F f, int* out, int* ired) {
  int carry = 0;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int base = 0; base < count; base += LG_BLOCK) {
    const int i = base + threadIdx.x;
    const int v = (i < count) ? f(i) : 0;
    int inc = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, inc, d);
      if (lane >= d) inc += t;
    }
    __syncthreads();
    if (lane == 31) ired[wid] = inc;
    __syncthreads();
    int wpre = 0, tot = 0;
#pragma unroll
    for (int w = 0; w < LG_WARPS; ++w) {
      const int x = ired[w];
      if (w < wid) wpre += x;
      tot += x;
    }
    if (i < count) out[i] = carry + wpre + inc - v;
    carry += tot;
  }
  __syncthreads();
  return carry;
}

template <typename T, int MODE>
__global__ void __launch_bounds__(LG_BLOCK, 1) k_spai_large(LargeArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  LargeSmem<T>& S = *reinterpret_cast<LargeSmem<T>*>(smem_raw);
  // [LargeSmem][staging area][dense slab]
  unsigned char* stage = smem_raw + ((sizeof(LargeSmem<T>) + 15) / 16) * 16;
  T* sA = reinterpret_cast<T*>(stage + LG_STAGE_BYTES);
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  if (tid == 0) {
    mbar_init(&S.mbar, 1);
    mbar_fence_init();
  }
  __syncthreads();
  unsigned phase = 0;
  const int nbig = a.stats[ST_BIG_COUNT];
  unsigned* gbits = a.gbits + (long long)blockIdx.x * 2 * a.words_per_block;
  int* gpre = reinterpret_cast<int*>(gbits + a.words_per_block);
  T* gA = reinterpret_cast<T*>(a.gA) + (long long)blockIdx.x * a.area_per_block;

  for (;;) {
    if (tid == 0) S.col_q = atomicAdd(&a.stats[ST_BIG_HEAD], 1);
    __syncthreads();
    const int q = S.col_q;
    __syncthreads();
    if (q >= nbig) break;
    const int k = a.big_list[q];
    const int cs = a.ptr[k];
    const int nj = a.ptr[k + 1] - cs;
    const int col = k - a.col_start;
    if (nj > LG_NJ_MAX) {
      if (tid == 0) atomicAdd(&a.stats[ST_LIMIT], 1);
      continue;
    }
    for (int t = tid; t < nj; t += LG_BLOCK) {
      const int j = a.idx[cs + t];
      S.jbase[t] = a.ptr[j];
      S.jlen[t] = a.ptr[j + 1] - S.jbase[t];
    }
    __syncthreads();
    const int cand = block_scan(nj, [&](int i) { return S.jlen[i]; }, S.jcb, S.ired);
    if (tid == 0) S.jcb[nj] = cand;
    __syncthreads();
    // Stage the J columns' row indices (and, when building, values) in shared
    // memory with one bulk copy per column and array, each range rounded out
    // to 16-byte boundaries, when they fit; the passes below then walk the
    // columns in shared memory instead of locating every candidate in global
    // memory.  The rounding never leaves the 16-byte block that holds an
    // array's last element.
    bool staged = false;
    int* srow = reinterpret_cast<int*>(stage);
    const double* sval = nullptr;
    if (a.stage_ok && cand > 0 && nj <= LG_STAGE_NJ) {
      const int rtot = block_scan(nj, [&](int i) {
        const int b = S.jbase[i];
        return ((b + S.jlen[i] + 3) & ~3) - (b & ~3);
      }, S.jso, S.ired);
      // values only when building (the pattern modes have no value array)
      const int vtot = (MODE == MODE_BUILD) ? block_scan(nj, [&](int i) {
        const int b = S.jbase[i];
        return ((b + S.jlen[i] + 1) & ~1) - (b & ~1);
      }, S.jvo, S.ired) : 0;
      const long long bytes = 4ll * rtot + 8ll * vtot;
      if (bytes > 0 && bytes <= LG_STAGE_BYTES) {
        staged = true;
        sval = reinterpret_cast<const double*>(stage + 4ll * rtot);
        if (tid == 0) mbar_arrive_expect_tx(&S.mbar, (unsigned)bytes);
        fence_async_shared();  // earlier reads of the staging area come first
        __syncthreads();       // the expected bytes are set before any copy lands
        for (int t = tid; t < nj; t += LG_BLOCK) {
          const int b = S.jbase[t], e = b + S.jlen[t];
          const int rb = b & ~3, re = (e + 3) & ~3;
          if (re > rb) bulk_copy_g2s(srow + S.jso[t], a.idx + rb, 4u * (unsigned)(re - rb), &S.mbar);
          if (MODE == MODE_BUILD) {
            const int vb = b & ~1, ve = (e + 1) & ~1;
            if (ve > vb) bulk_copy_g2s((void*)(sval + S.jvo[t]), a.val + vb, 8u * (unsigned)(ve - vb), &S.mbar);
          }
        }
        const bool ok = mbar_wait(&S.mbar, phase);
        phase ^= 1u;
        if (__syncthreads_or(!ok)) {
          // give the copies in flight a second bounded wait, report, stop
          if (tid == 0) {
            mbar_wait(&S.mbar, phase ^ 1u);
            atomicAdd(&a.stats[ST_STAGE_FAIL], 1);
          }
          __syncthreads();
          return;
        }
        if (MODE == MODE_BUILD && tid == 0) atomicAdd(&a.stats[ST_STAGED], 1);
      }
    }
    // row / value of entry q of J column j in the staged copy
    auto srow_at = [&](int j, int q) { return srow[S.jso[j] + (S.jbase[j] & 3) + q]; };
    auto sval_at = [&](int j, int q) { return sval[S.jvo[j] + (S.jbase[j] & 1) + q]; };
    // candidate enumeration: candidate t -> (column slot j, position src)
    auto locate = [&](int t, int& j, int& src) {
      int lo = 0, hi = nj - 1;
      while (lo < hi) {  // last j with jcb[j] <= t
        const int mid = (lo + hi + 1) >> 1;
        if (S.jcb[mid] <= t) lo = mid;
        else hi = mid - 1;
      }
      j = lo;
      src = S.jbase[lo] + (t - S.jcb[lo]);
    };
    int rmin = INT_MAX, rmax = -1;
    if (staged) {
      for (int j = wid; j < nj; j += LG_WARPS)
        for (int q = lane; q < S.jlen[j]; q += 32) {
          const int row = srow_at(j, q);
          rmin = min(rmin, row);
          rmax = max(rmax, row);
        }
    } else {
      for (int t = tid; t < cand; t += LG_BLOCK) {
        int j, src;
        locate(t, j, src);
        const int row = a.idx[src];
        rmin = min(rmin, row);
        rmax = max(rmax, row);
      }
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
      rmin = min(rmin, __shfl_xor_sync(0xffffffffu, rmin, d));
      rmax = max(rmax, __shfl_xor_sync(0xffffffffu, rmax, d));
    }
    __syncthreads();
    if (lane == 0) {
      S.ired[wid] = rmin;
      S.ired[LG_WARPS + wid] = rmax;
    }
    __syncthreads();
    rmin = INT_MAX;
    rmax = -1;
#pragma unroll
    for (int w = 0; w < LG_WARPS; ++w) {
      rmin = min(rmin, S.ired[w]);
      rmax = max(rmax, S.ired[LG_WARPS + w]);
    }
    __syncthreads();
    const int words = (cand > 0) ? ((rmax - rmin) >> 5) + 1 : 0;
    unsigned* bits = (words <= LG_WORDS_SMEM) ? S.bits : gbits;
    int* wpre = (words <= LG_WORDS_SMEM) ? S.wpre : gpre;
    for (int w = tid; w < words; w += LG_BLOCK) bits[w] = 0u;
    __syncthreads();
    if (staged) {
      for (int j = wid; j < nj; j += LG_WARPS)
        for (int q = lane; q < S.jlen[j]; q += 32) {
          const int off = srow_at(j, q) - rmin;
          atomicOr(&bits[off >> 5], 1u << (off & 31));
        }
    } else {
      for (int t = tid; t < cand; t += LG_BLOCK) {
        int j, src;
        locate(t, j, src);
        const int off = a.idx[src] - rmin;
        atomicOr(&bits[off >> 5], 1u << (off & 31));
      }
    }
    __syncthreads();
    const int m = block_scan(words, [&](int w) { return __popc(bits[w]); }, wpre, S.ired);
    auto rank = [&](int row) {
      const int off = row - rmin;
      const unsigned wv = bits[off >> 5];
      return wpre[off >> 5] + __popc(wv & ((1u << (off & 31)) - 1u));
    };
    if (MODE == MODE_COUNT) {
      if (tid == 0) a.icount[col] = m;
      continue;
    }
    if (MODE == MODE_LIST) {
      const long long base = a.iptr[col];
      for (int w = tid; w < words; w += LG_BLOCK) {
        unsigned wv = bits[w];
        int p = wpre[w];
        while (wv) {
          const int b = __ffs(wv) - 1;
          a.ilist[base + p++] = rmin + (w << 5) + b;
          wv &= wv - 1u;
        }
      }
      __syncthreads();
      continue;
    }
    // ---- build ------------------------------------------------------------
    const int W = nj + 1;
    const long long lda = m;
    const long long area = (long long)m * W;
    T* Ad = (area <= a.smem_area) ? sA : gA;
    // A block that does not fit shared memory is gathered into its own slab
    // of the hub pool and factored by the hub kernels (all SMs on all such
    // columns, one launch per Householder step) instead of by this CTA alone.
    bool hub = false;
    if (area > a.hub_min_area && a.hub_pool) {
      if (tid == 0) {
        const long long need = area + 2LL * W;
        const long long off = (long long)atomicAdd(reinterpret_cast<unsigned long long*>(a.stats) + ST_HUBHEAD64,
                                                   (unsigned long long)need);
        S.hub_off = (off + need <= a.hub_cap) ? off : -1;
        if (S.hub_off >= 0) a.hub_meta[atomicAdd(&a.stats[ST_HUB_COUNT], 1)] = HubMeta{k, m, nj, 0, off};
      }
      __syncthreads();
      if (S.hub_off >= 0) {
        Ad = reinterpret_cast<T*>(a.hub_pool) + S.hub_off;
        hub = true;
      }
    }
    if (!hub && area > a.smem_area && area > a.area_per_block) {
      if (tid == 0) atomicAdd(&a.stats[ST_LIMIT], 1);
      continue;
    }
    for (long long e = tid; e < area; e += LG_BLOCK) Ad[e] = T(0);
    if (tid == 0) {
      int E = -1;
      if (cand > 0 && k >= rmin && k <= rmax) {
        const int off = k - rmin;
        if (bits[off >> 5] & (1u << (off & 31))) E = rank(k);
      }
      S.E = E;
    }
    __syncthreads();
    if (staged) {
      for (int j = wid; j < nj; j += LG_WARPS)
        for (int q = lane; q < S.jlen[j]; q += 32) Ad[(long long)j * lda + rank(srow_at(j, q))] = (T)sval_at(j, q);
    } else {
      for (int t = tid; t < cand; t += LG_BLOCK) {
        int j, src;
        locate(t, j, src);
        Ad[(long long)j * lda + rank(a.idx[src])] = (T)a.val[src];
      }
    }
    if (tid == 0 && S.E >= 0) Ad[(long long)nj * lda + S.E] = T(1);
    __syncthreads();
    if (hub) continue;  // factored, solved and scattered by the hub kernels
    bool sing = m < nj;
    const int steps = min(nj, m);
    for (int c = 0; c < steps; ++c) {
      T* vc = Ad + (long long)c * lda;
      double part = 0.0;
      for (int i = c + tid; i < m; i += LG_BLOCK) part += (double)vc[i] * (double)vc[i];
      const double nrm2 = block_sum(part, S.red);
      if (tid == 0) {
        const T x0 = vc[c];
        const T nrm = (T)sqrt(nrm2);
        T alpha = T(0), beta = T(0);
        if (nrm > T(0)) {
          alpha = (x0 > T(0)) ? -nrm : nrm;
          beta = T(1) / (nrm * (nrm + (T)fabs((double)x0)));
          vc[c] = x0 - alpha;
        }
        S.rd[c] = alpha;
        S.beta = beta;
      }
      __syncthreads();
      const T beta = S.beta;
      if (beta != T(0)) {
        for (int j = c + 1 + wid; j <= nj; j += LG_WARPS) {
          T* aj = Ad + (long long)j * lda;
          T w = T(0);
          for (int i = c + lane; i < m; i += 32) w += vc[i] * aj[i];
#pragma unroll
          for (int d = 16; d > 0; d >>= 1) w += __shfl_xor_sync(0xffffffffu, w, d);
          w *= beta;
          for (int i = c + lane; i < m; i += 32) aj[i] -= w * vc[i];
        }
      }
      __syncthreads();
    }
    // back substitution: y = column nj, R(i, j) = Ad[j*lda + i] for i < j, R(i,i) = rd[i]
    T* y = Ad + (long long)nj * lda;
    for (int t = tid; t < nj; t += LG_BLOCK) S.ys[t] = (t < m) ? y[t] : T(0);
    double part = 0.0;
    for (int i = nj + tid; i < m; i += LG_BLOCK) part += (double)y[i] * (double)y[i];
    const double res2 = block_sum(part, S.red);
    __syncthreads();
    for (int i = nj - 1; i >= 0; --i) {
      if (tid == 0) {
        const T rii = (i < m) ? S.rd[i] : T(0);
        if (!(rii != T(0)) || !isfinite((double)rii)) sing = true;
        S.ys[i] = S.ys[i] / rii;
      }
      __syncthreads();
      const T xi = S.ys[i];
      // R has min(m, nj) rows: column i holds R(t, i) for t < min(i, m)
      for (int t = tid; t < min(i, m); t += LG_BLOCK) S.ys[t] -= Ad[(long long)i * lda + t] * xi;
      __syncthreads();
    }
    for (int t = tid; t < nj; t += LG_BLOCK) a.mval[cs + t] = (double)S.ys[t];
    if (tid == 0) {
      if (a.colres) a.colres[col] = sqrt(res2);
      if (sing) atomicAdd(&a.stats[ST_SINGULAR], 1);
      atomicMax(&a.stats[ST_MAXNI], m);
      atomicAdd(&a.stats[ST_BIG_DONE], 1);
    }
    __syncthreads();
  }
}

// ---- hub kernels: columns whose dense block exceeds shared memory ---------
// One launch per Householder step c, over every hub column at once: a block
// of HUB_THREADS per trailing column j > c applies reflector c (dot product
// and update, threads striding the rows), and the block of column c + 1 then
// forms reflector c + 1 from its updated column.  Launch c = -1 forms
// reflector 0.  The hubs are sorted by |J| descending, so the hubs still
// active at step c (|J| > c) are a prefix and block b finds its column by a
// binary search on S(h) - c h, S = prefix sum of |J|.  Each hub's block
// streams through L2 on all SMs instead of through one SM; the steps are
// chained by programmatic dependent launch.  k_hub_solve then
// back-substitutes, one CTA per column.
constexpr int HUB_THREADS = 128;
constexpr int HUB_WARPS = HUB_THREADS / 32;

struct HubArgs {
  const HubMeta* meta;  // sorted by nj descending
  const int* spre;      // spre[h] = sum of nj over hubs before h (nh + 1 entries)
  int nh;
  void* pool;
};

// Sum of one double per thread of a HUB_THREADS block, in a fixed order.
__device__ __forceinline__ double hub_sum(double v, double* red) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
#pragma unroll
  for (int w = 0; w < HUB_WARPS; ++w) t += red[w];
  return t;
}

// Step c: `active` = hubs with nj > c (a prefix of the sorted list); the grid
// has sum over them of (nj - c) blocks.
template <typename T>
__global__ void __launch_bounds__(HUB_THREADS) k_hub_step(HubArgs h, int c, int active) {
  __shared__ double red[HUB_WARPS];
  const int tid = threadIdx.x;
  const int b = blockIdx.x;
  // largest hub index g < active with spre[g] - c g <= b
  int lo = 0, hi = active - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if ((long long)h.spre[mid] - (long long)c * mid <= b) lo = mid;
    else hi = mid - 1;
  }
  const HubMeta hm = h.meta[lo];
  const int j = c + 1 + (b - (int)((long long)h.spre[lo] - (long long)c * lo));
  const int m = hm.m, W = hm.nj + 1;
  const int steps = min(hm.nj, m);
  T* Ad = reinterpret_cast<T*>(h.pool) + hm.off;
  T* rd = Ad + (long long)m * W;
  T* bt = rd + W;
  T* aj = Ad + (long long)j * m;
  cudaGridDependencySynchronize();  // step c - 1 has finished: reflector c and column j are current
  if (c >= 0 && c < steps) {
    const T beta = bt[c];
    if (beta != T(0)) {
      const T* vc = Ad + (long long)c * m;
      double part = 0.0;
      for (int i = c + tid; i < m; i += HUB_THREADS) part += (double)(vc[i] * aj[i]);
      const T w = (T)hub_sum(part, red) * beta;
      for (int i = c + tid; i < m; i += HUB_THREADS) aj[i] -= w * vc[i];
    }
  }
  if (j == c + 1 && j < steps) {
    __syncthreads();  // the update above wrote these rows from other threads
    double part = 0.0;
    for (int i = j + tid; i < m; i += HUB_THREADS) part += (double)aj[i] * (double)aj[i];
    const double nrm2 = hub_sum(part, red);
    if (tid == 0) {
      const T x0 = aj[j];
      const T nrm = (T)sqrt(nrm2);
      T alpha = T(0), beta = T(0);
      if (nrm > T(0)) {
        alpha = (x0 > T(0)) ? -nrm : nrm;
        beta = T(1) / (nrm * (nrm + (T)fabs((double)x0)));
        aj[j] = x0 - alpha;
      }
      rd[j] = alpha;
      bt[j] = beta;
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(LG_BLOCK) k_hub_solve(HubArgs h, LargeArgs a) {
  __shared__ T ys[LG_NJ_MAX];
  __shared__ T xs[LG_NJ_MAX];
  __shared__ double red[LG_WARPS];
  const HubMeta hm = h.meta[blockIdx.x];
  const int tid = threadIdx.x;
  const int m = hm.m, nj = hm.nj, W = nj + 1;
  const T* Ad = reinterpret_cast<const T*>(h.pool) + hm.off;
  const T* rd = Ad + (long long)m * W;
  const T* y = Ad + (long long)nj * m;
  for (int t = tid; t < nj; t += LG_BLOCK) ys[t] = (t < m) ? y[t] : T(0);
  double part = 0.0;
  for (int i = nj + tid; i < m; i += LG_BLOCK) part += (double)y[i] * (double)y[i];
  const double res2 = block_sum(part, red);
  __syncthreads();
  // One barrier per row: every thread forms x_i = ys_i / R_ii itself (ys_i
  // is final once row i + 1 is done), thread 0 records it, and the rows above
  // are updated; ys_i itself is never written again.  R_ii and this thread's
  // entries of column i are loaded during row i + 1, so no global load sits
  // on the per-row chain.
  constexpr int PT = LG_NJ_MAX / LG_BLOCK;  // rows of R per thread
  auto load_col = [&](int i, T (&v)[PT], T& r) {
    r = (i < m) ? rd[i] : T(0);
#pragma unroll
    for (int q = 0; q < PT; ++q) {
      const int t = tid + q * LG_BLOCK;
      v[q] = (t < min(i, m)) ? Ad[(long long)i * m + t] : T(0);
    }
  };
  bool sing = m < nj;
  T cur[PT], nxt[PT], rii = T(0), rnx = T(0);
  if (nj > 0) load_col(nj - 1, cur, rii);
  for (int i = nj - 1; i >= 0; --i) {
    const T xi = ys[i] / rii;
    if (tid == 0) {
      if (!(rii != T(0)) || !isfinite((double)rii)) sing = true;
      xs[i] = xi;
    }
    if (i > 0) load_col(i - 1, nxt, rnx);
#pragma unroll
    for (int q = 0; q < PT; ++q) {
      const int t = tid + q * LG_BLOCK;
      if (t < min(i, m)) ys[t] -= cur[q] * xi;
    }
#pragma unroll
    for (int q = 0; q < PT; ++q) cur[q] = nxt[q];
    rii = rnx;
    __syncthreads();
  }
  const int cs = a.ptr[hm.k];
  for (int t = tid; t < nj; t += LG_BLOCK) a.mval[cs + t] = (double)xs[t];
  if (tid == 0) {
    if (a.colres) a.colres[hm.k - a.col_start] = sqrt(res2);
    if (sing) atomicAdd(&a.stats[ST_SINGULAR], 1);
    atomicMax(&a.stats[ST_MAXNI], m);
    atomicAdd(&a.stats[ST_BIG_DONE], 1);
  }
}

// nnz-balanced chunk bounds for the dynamic schedule: chunk c starts at the
// first column whose nnz prefix reaches c/nchunks of the range's nnz.
__global__ void k_nnz_chunks(const int* __restrict__ ptr, int col_start, int col_end, int nchunks,
                             int* __restrict__ bounds) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c > nchunks) return;
  const long long p0 = ptr[col_start], tot = (long long)ptr[col_end] - p0;
  if (c == 0) { bounds[0] = col_start; return; }
  if (c == nchunks) { bounds[c] = col_end; return; }
  const long long target = p0 + (tot * c) / nchunks;
  int lo = col_start, hi = col_end;
  while (lo < hi) {
    const int mid = lo + ((hi - lo) >> 1);
    if ((long long)ptr[mid] < target) lo = mid + 1;
    else hi = mid;
  }
  bounds[c] = lo;
}

template <typename T, int MODE>
int run_small(Ctx* c, SmallArgs a, int) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_spai_small<T, MODE>, SG_BLOCK, 0) != cudaSuccess ||
      per_sm < 1) {
    cudaGetLastError();
    per_sm = 1;
  }
  const int grid = c->sms * per_sm;
  const int ngroups = grid * SG_BLOCK / GL;
  if (a.schedule == DCU_SCHED_BALANCED_NNZ) {
    const int nchunks = ngroups * 4;
    DCU_TRY(ensure(c, B_CHUNKS, sizeof(int) * (size_t)(nchunks + 1)));
    int* bounds = bp<int>(c, B_CHUNKS);
    k_nnz_chunks<<<(nchunks + 256) / 256, 256, 0, c->stream>>>(a.ptr, a.col_start, a.col_end, nchunks, bounds);
    DCU_LAUNCHED(c, "k_nnz_chunks");
    a.chunks = bounds;
    a.nchunks = nchunks;
  }
  k_spai_small<T, MODE><<<grid, SG_BLOCK, 0, c->stream>>>(a);
  DCU_LAUNCHED(c, "k_spai_small");
  return DCU_OK;
}

template <typename T, int MODE>
int run_large(Ctx* c, LargeArgs& a, int nbig, int cta_max_area = 0) {
  const size_t fixed = ((sizeof(LargeSmem<T>) + 15) / 16) * 16 + LG_STAGE_BYTES;
  size_t cap = c->smem_optin > fixed + 1024 ? c->smem_optin - 1024 : fixed;
  // bulk copies read idx (every mode) and val (build only) in 16-byte units
  a.stage_ok = (a.idx && reinterpret_cast<uintptr_t>(a.idx) % 16 == 0 &&
                (MODE != MODE_BUILD || (a.val && reinterpret_cast<uintptr_t>(a.val) % 16 == 0))) ? 1 : 0;
  a.smem_area = (MODE == MODE_BUILD) ? (long long)((cap - fixed) / sizeof(T)) : 0;
  const size_t smem = fixed + (size_t)a.smem_area * sizeof(T);
  DCU_CUDA(c, cudaFuncSetAttribute(k_spai_large<T, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int grid = nbig < c->sms ? nbig : c->sms;
  // global slabs for columns whose bitmap / dense block exceed shared memory
  a.words_per_block = ((long long)a.n >> 5) + 2;
  const long long area_cap = a.area_per_block;
  a.area_per_block = (MODE == MODE_BUILD && area_cap > a.smem_area) ? area_cap : 0;
  // Blocks that exceed shared memory go to the hub pool, sized by the queue's
  // bound; the per-CTA slabs remain only for what a capped pool cannot hold.
  a.hub_pool = nullptr;
  a.hub_cap = 0;
  a.hub_meta = nullptr;
  a.hub_min_area = a.smem_area > cta_max_area ? a.smem_area : cta_max_area;
  if (MODE == MODE_BUILD && a.area_per_block > a.hub_min_area && cta_max_area >= 0) {
    a.hub_cap = a.area_sum < kHubPoolMax ? a.area_sum : kHubPoolMax;
    // without room for the pool every block stays on one CTA (per-CTA slabs)
    const std::string err = c->err;
    if (ensure(c, B_HUBPOOL, sizeof(T) * (size_t)a.hub_cap) == DCU_OK &&
        ensure(c, B_HUBMETA, sizeof(HubMeta) * (size_t)nbig) == DCU_OK) {
      a.hub_pool = c->buf[B_HUBPOOL].p;
      a.hub_meta = bp<HubMeta>(c, B_HUBMETA);
      // the pool holds every block above shared memory: no per-CTA slabs
      if (a.hub_cap == a.area_sum && a.hub_min_area == a.smem_area) a.area_per_block = 0;
    } else {
      c->err = err;
      a.hub_cap = 0;
    }
  }
  DCU_TRY(ensure(c, B_SLAB_BITS, sizeof(unsigned) * 2 * (size_t)a.words_per_block * grid));
  a.gbits = bp<unsigned>(c, B_SLAB_BITS);
  if (a.area_per_block > 0) DCU_TRY(ensure(c, B_SLAB_A, sizeof(T) * (size_t)a.area_per_block * grid));
  a.gA = a.area_per_block > 0 ? c->buf[B_SLAB_A].p : nullptr;
  k_spai_large<T, MODE><<<grid, LG_BLOCK, smem, c->stream>>>(a);
  DCU_LAUNCHED(c, "k_spai_large");
  if (!a.hub_pool) return DCU_OK;
  // hub columns: read their descriptors, sort them by |J| descending, one
  // step launch per Householder step over the hubs still active, then the
  // solves
  int* st = bp<int>(c, B_STATS);
  DCU_CUDA(c, cudaMemcpyAsync(c->pinned, st + ST_HUB_COUNT, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  DCU_CUDA(c, cudaStreamSynchronize(c->stream));
  const int nh = *reinterpret_cast<int*>(c->pinned);
  if (nh <= 0) return DCU_OK;
  std::vector<HubMeta> hm((size_t)nh);
  DCU_CUDA(c, cudaMemcpyAsync(hm.data(), a.hub_meta, sizeof(HubMeta) * (size_t)nh, cudaMemcpyDeviceToHost,
                              c->stream));
  DCU_CUDA(c, cudaStreamSynchronize(c->stream));
  std::stable_sort(hm.begin(), hm.end(), [](const HubMeta& x, const HubMeta& y) { return x.nj > y.nj; });
  std::vector<int> spre((size_t)nh + 1, 0);
  int steps = 0;
  for (int g = 0; g < nh; ++g) {
    spre[g + 1] = spre[g] + hm[g].nj;
    steps = std::max(steps, std::min(hm[g].nj, hm[g].m));
  }
  DCU_TRY(ensure(c, B_HUBWPRE, sizeof(int) * spre.size()));
  DCU_CUDA(c, cudaMemcpyAsync(a.hub_meta, hm.data(), sizeof(HubMeta) * (size_t)nh, cudaMemcpyHostToDevice,
                              c->stream));
  DCU_CUDA(c, cudaMemcpyAsync(c->buf[B_HUBWPRE].p, spre.data(), sizeof(int) * spre.size(), cudaMemcpyHostToDevice,
                              c->stream));
  HubArgs h{a.hub_meta, bp<int>(c, B_HUBWPRE), nh, a.hub_pool};
  int active = nh;
  for (int cst = -1; cst < steps; ++cst) {
    while (active > 0 && hm[active - 1].nj <= cst) --active;  // hubs with nj > cst
    const long long blocks = (long long)spre[active] - (long long)cst * active;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)blocks);
    cfg.blockDim = dim3(HUB_THREADS);
    cfg.stream = c->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = cst >= 0 ? 1 : 0;  // the first step follows copies, not a step
    DCU_CUDA(c, cudaLaunchKernelEx(&cfg, k_hub_step<T>, h, cst, active));
    c->launches++;
  }
  k_hub_solve<T><<<nh, LG_BLOCK, 0, c->stream>>>(h, a);
  DCU_LAUNCHED(c, "k_hub_solve");
  return DCU_OK;
}

template <typename T>
int run_ne(Ctx* c, NeArgs a) {
  const size_t smem = (sizeof(int) + sizeof(T)) * NE_CMAX * NE_BLOCK;
  DCU_CUDA(c, cudaFuncSetAttribute(k_spai_ne<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_spai_ne<T>, NE_BLOCK, smem) != cudaSuccess ||
      per_sm < 1) {
    cudaGetLastError();
    per_sm = 1;
  }
  const int grid = c->sms * per_sm;
  if (a.schedule == DCU_SCHED_BALANCED_NNZ) {
    const int nchunks = grid * 8;
    DCU_TRY(ensure(c, B_CHUNKS, sizeof(int) * (size_t)(nchunks + 1)));
    int* bounds = bp<int>(c, B_CHUNKS);
    k_nnz_chunks<<<(nchunks + 256) / 256, 256, 0, c->stream>>>(a.ptr, a.col_start, a.col_end, nchunks, bounds);
    DCU_LAUNCHED(c, "k_nnz_chunks");
    a.chunks = bounds;
    a.nchunks = nchunks;
  }
  k_spai_ne<T><<<grid, NE_BLOCK, smem, c->stream>>>(a);
  DCU_LAUNCHED(c, "k_spai_ne");
  return DCU_OK;
}

struct Prepared {
  SmallArgs sa;
  int grid = 0;
  int* stats = nullptr;
};

}  // namespace

struct BuildJobImpl {
  Prepared P;
};

namespace {

int prepare(Ctx* c, int n, const int* ptr, const int* idx, const double* val, int col_start, int col_end,
            int schedule, Prepared* P) {
  const int ncols = col_end - col_start;
  DCU_TRY(ensure(c, B_STATS, sizeof(int) * ST_INTS));
  DCU_TRY(ensure(c, B_BIGLIST, sizeof(int) * (size_t)(ncols > 0 ? ncols : 1)));
  int* stats = bp<int>(c, B_STATS);
  DCU_CUDA(c, cudaMemsetAsync(stats, 0, sizeof(int) * ST_INTS, c->stream));
  P->grid = 0;
  SmallArgs& a = P->sa;
  a = SmallArgs{};
  a.n = n;
  a.ptr = ptr;
  a.idx = idx;
  a.val = val;
  a.col_start = col_start;
  a.col_end = col_end;
  a.schedule = schedule;
  a.big_list = bp<int>(c, B_BIGLIST);
  a.stats = stats;
  a.max_ni = SG_MMAX;
  P->stats = stats;
  return DCU_OK;
}

int read_stats(Ctx* c, int* host) {
  DCU_CUDA(c, cudaMemcpyAsync(c->pinned, bp<int>(c, B_STATS), sizeof(int) * ST_INTS, cudaMemcpyDeviceToHost,
                              c->stream));
  DCU_CUDA(c, cudaStreamSynchronize(c->stream));
  memcpy(host, c->pinned, sizeof(int) * ST_INTS);
  return DCU_OK;
}

// A build in two halves: the launch enqueues the first column kernel and
// returns without waiting; the finish reads its statistics (a host round
// trip), runs the hand-offs, the CTA kernel and the hub kernels, and fills
// info.  Between the two the caller may enqueue independent work on other
// streams (the solver's SELL plan), which then overlaps the first kernel.
template <typename T>
int build_launch(Ctx* c, int n, const int* ptr, const int* idx, const double* val, int col_start, int col_end,
                 int schedule, bool thread_path, int max_ni, double* mval, double* colres, BuildJob* J) {
  Prepared& P = J->impl->P;
  DCU_TRY(prepare(c, n, ptr, idx, val, col_start, col_end, schedule, &P));
  if (max_ni > 0 && max_ni < SG_MMAX) P.sa.max_ni = max_ni;
  P.sa.mval = mval;
  P.sa.colres = colres;
  J->thread_path = thread_path;
  if (thread_path) {
    // thread per column first; its hand-offs go to the group kernel
    DCU_TRY(ensure(c, B_FBLIST, sizeof(int) * (size_t)(col_end - col_start)));
    NeArgs na{};
    na.n = n;
    na.ptr = ptr;
    na.idx = idx;
    na.val = val;
    na.col_start = col_start;
    na.col_end = col_end;
    na.schedule = schedule;
    na.mval = mval;
    na.colres = colres;
    na.fb_list = bp<int>(c, B_FBLIST);
    na.stats = P.stats;
    na.tau = sizeof(T) == sizeof(float) ? 1e-3 : 1e-8;
    J->fb_list = na.fb_list;
    DCU_TRY(run_ne<T>(c, na));
  } else {
    DCU_TRY((run_small<T, MODE_BUILD>(c, P.sa, P.grid)));
  }
  return DCU_OK;
}

template <typename T>
int build_finish(Ctx* c, int n, const int* ptr, const int* idx, const double* val, int col_start, int col_end,
                 int cta_max_area, double* mval, double* colres, BuildJob* J, dcu_build_info* info) {
  Prepared& P = J->impl->P;
  int st[ST_INTS];
  if (J->thread_path) {
    DCU_TRY(read_stats(c, st));
    if (st[ST_FB_COUNT] > 0) {
      P.sa.list = J->fb_list;
      J->finish_launched = true;
      DCU_TRY((run_small<T, MODE_BUILD>(c, P.sa, P.grid)));
    }
  }
  DCU_TRY(read_stats(c, st));
  const int nbig = st[ST_BIG_COUNT];
  if (nbig > 0) {
    if (st[ST_BIG_MAXNJ] > LG_NJ_MAX)
      return fail(c, DCU_ERR_LIMIT, "column with |J| = %d exceeds the supported %d", st[ST_BIG_MAXNJ], LG_NJ_MAX);
    LargeArgs la{};
    la.n = n;
    la.ptr = ptr;
    la.idx = idx;
    la.val = val;
    la.col_start = col_start;
    la.mval = mval;
    la.colres = colres;
    la.big_list = P.sa.big_list;
    la.stats = P.stats;
    long long area = 0;
    memcpy(&area, reinterpret_cast<long long*>(st) + ST_AREA64, sizeof area);
    la.area_per_block = area;
    memcpy(&la.area_sum, reinterpret_cast<long long*>(st) + ST_AREASUM64, sizeof la.area_sum);
    J->finish_launched = true;
    DCU_TRY((run_large<T, MODE_BUILD>(c, la, nbig, cta_max_area)));
    DCU_TRY(read_stats(c, st));
    if (st[ST_LIMIT] > 0) return fail(c, DCU_ERR_LIMIT, "%d columns exceeded the CTA kernel's limits", st[ST_LIMIT]);
    if (st[ST_STAGE_FAIL] > 0) return fail(c, DCU_ERR_CUDA, "a bulk copy into shared memory did not complete");
  }
  if (info) {
    info->cols_total = col_end - col_start;
    info->cols_small = st[ST_SMALL_COLS] + st[ST_NE_COLS];
    info->cols_large = st[ST_BIG_DONE];
    info->cols_singular = st[ST_SINGULAR];
    info->max_nj = st[ST_MAXNJ] > st[ST_BIG_MAXNJ] ? st[ST_MAXNJ] : st[ST_BIG_MAXNJ];
    info->max_ni = st[ST_MAXNI];
    info->cols_staged = st[ST_STAGED];
    info->cols_hub = st[ST_HUB_COUNT];
  }
  return DCU_OK;
}

}  // namespace

int spai_default_units(Ctx* c) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_spai_small<double, MODE_BUILD>, SG_BLOCK, 0) !=
          cudaSuccess ||
      per_sm < 1) {
    cudaGetLastError();
    per_sm = 1;
  }
  return c->sms * per_sm * (SG_BLOCK / GL);
}

BuildJob::BuildJob() : impl(new BuildJobImpl) {}
BuildJob::~BuildJob() { delete impl; }

int spai_build_launch(Ctx* c, int n, int nnz, const int* ptr, const int* idx, const double* val,
                      const dcu_options* opt, double* mval, double* colres, BuildJob* J) {
  const int col_start = opt->col_start;
  const int col_end = opt->col_end;
  J->opt = *opt;
  J->n = n;
  J->ptr = ptr;
  J->idx = idx;
  J->val = val;
  J->mval = mval;
  J->colres = colres;
  J->empty = false;
  if (col_start != 0 || col_end != n)
    DCU_CUDA(c, cudaMemsetAsync(mval, 0, sizeof(double) * (size_t)(nnz > 0 ? nnz : 1), c->stream));
  if (col_end <= col_start) {
    J->empty = true;
    return DCU_OK;
  }
  const int p = opt->precision;
  const bool tuned = p >= 0 && p < 5 && c->tune_set[p];
  J->max_ni = tuned ? c->tune[p].group_max_ni : 0;
  J->cta_max_area = tuned ? c->tune[p].cta_max_area : 0;
  // FP64 (the plain form): Householder on every column unless the normal
  // equations are asked for.  Mixed forms: the thread-per-column path first,
  // Householder for the columns it hands over, unless Householder is asked for.
  if (opt->precision == DCU_PREC_FP64)
    return build_launch<double>(c, n, ptr, idx, val, col_start, col_end, opt->schedule,
                                opt->ls_method == DCU_LS_NORMAL_EQ, J->max_ni, mval, colres, J);
  return build_launch<float>(c, n, ptr, idx, val, col_start, col_end, opt->schedule,
                             opt->ls_method != DCU_LS_HOUSEHOLDER, J->max_ni, mval, colres, J);
}

int spai_build_finish(Ctx* c, BuildJob* J, dcu_build_info* info) {
  if (J->empty) return DCU_OK;
  const dcu_options& o = J->opt;
  if (o.precision == DCU_PREC_FP64)
    return build_finish<double>(c, J->n, J->ptr, J->idx, J->val, o.col_start, o.col_end, J->cta_max_area,
                                J->mval, J->colres, J, info);
  return build_finish<float>(c, J->n, J->ptr, J->idx, J->val, o.col_start, o.col_end, J->cta_max_area, J->mval,
                             J->colres, J, info);
}

int spai_build(Ctx* c, int n, int nnz, const int* ptr, const int* idx, const double* val, const dcu_options* opt,
               double* mval, double* colres, dcu_build_info* info) {
  BuildJob J;
  DCU_TRY(spai_build_launch(c, n, nnz, ptr, idx, val, opt, mval, colres, &J));
  return spai_build_finish(c, &J, info);
}

int spai_pattern(Ctx* c, int n, const int* ptr, const int* idx, int col_start, int col_end, int* icount,
                 long long* iptr, int* ilist, long long cap, long long* total) {
  const int ncols = col_end - col_start;
  if (ncols <= 0) {
    if (total) *total = 0;
    return DCU_OK;
  }
  for (int pass = 0; pass < 2; ++pass) {
    if (pass == 1 && !ilist) break;
    Prepared P;
    DCU_TRY(prepare(c, n, ptr, idx, nullptr, col_start, col_end, DCU_SCHED_BALANCED_COLUMNS, &P));
    P.sa.icount = icount;
    P.sa.iptr = iptr;
    P.sa.ilist = ilist;
    if (pass == 0) DCU_TRY((run_small<double, MODE_COUNT>(c, P.sa, P.grid)));
    else DCU_TRY((run_small<double, MODE_LIST>(c, P.sa, P.grid)));
    int st[ST_INTS];
    DCU_TRY(read_stats(c, st));
    if (st[ST_BIG_COUNT] > 0) {
      if (st[ST_BIG_MAXNJ] > LG_NJ_MAX)
        return fail(c, DCU_ERR_LIMIT, "column with |J| = %d exceeds the supported %d", st[ST_BIG_MAXNJ], LG_NJ_MAX);
      LargeArgs la{};
      la.n = n;
      la.ptr = ptr;
      la.idx = idx;
      la.col_start = col_start;
      la.icount = icount;
      la.iptr = iptr;
      la.ilist = ilist;
      la.big_list = P.sa.big_list;
      la.stats = P.stats;
      if (pass == 0) DCU_TRY((run_large<double, MODE_COUNT>(c, la, st[ST_BIG_COUNT])));
      else DCU_TRY((run_large<double, MODE_LIST>(c, la, st[ST_BIG_COUNT])));
      DCU_TRY(read_stats(c, st));
      if (st[ST_STAGE_FAIL] > 0) return fail(c, DCU_ERR_CUDA, "a bulk copy into shared memory did not complete");
    }
    if (pass == 0) {
      DCU_TRY(scan_exclusive_i64(c, icount, iptr, ncols));
      DCU_CUDA(c, cudaMemcpyAsync(c->pinned, iptr + ncols, sizeof(long long), cudaMemcpyDeviceToHost, c->stream));
      DCU_CUDA(c, cudaStreamSynchronize(c->stream));
      const long long t = *(long long*)c->pinned;
      if (total) *total = t;
      if (ilist && t > cap) return fail(c, DCU_ERR_ARG, "ilist capacity %lld < %lld", cap, t);
    }
  }
  DCU_CUDA(c, cudaStreamSynchronize(c->stream));
  return DCU_OK;
}

}  // namespace dcu
