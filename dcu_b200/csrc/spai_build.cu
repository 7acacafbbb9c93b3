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
//   k_spai_small  one 8-lane group per column, |J_k| <= 7, <= 64 candidate
//                 rows, |I_k| <= 32: candidates sorted in registers (bitonic
//                 network across the group), At staged in shared memory, one
//                 lane per column of [At | e_E] holding it in registers.
//   k_spai_large  one CTA per column for everything else: I_k by a bitmap
//                 over the candidate row range, At in shared memory or a
//                 global slab, Householder with warp-per-trailing-column
//                 updates, column-oriented back substitution.
// Columns that do not fit the small kernel are appended to a list the large
// kernel drains with an atomic counter.  Each column's arithmetic is fixed by
// its own data (fixed reduction trees, no float atomics), so M is identical
// for every schedule and grid size.
#include <climits>

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
  ST_INTS = 16,
  ST_AREA64 = 7       // long long index (ints 14-15): max candidates * (|J|+1) over queued columns
};

constexpr int GL = 8;          // lanes per column group
constexpr int SM_MMAX = 32;    // max |I_k| on the small path
constexpr int SM_CMAX = 64;    // max candidate rows on the small path
constexpr int SM_NJMAX = 7;    // max |J_k| on the small path ([At | e] fits 8 lanes)
constexpr int SM_BLOCK = 128;   // 16 groups: the FP64 group state stays under 48 KB
constexpr int SM_GROUPS = SM_BLOCK / GL;
constexpr unsigned kPad = 0xFFFFFFFFu;

struct SmallArgs {
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
  int* icount;
  const long long* iptr;
  int* ilist;
  int* big_list;
  int* stats;
};

template <typename T>
struct SmallGroup {
  T At[GL][SM_MMAX];     // column j of [A(I,J) | e_E]; later R and x
  T v[SM_MMAX];          // Householder vector, then y = Q^T e_E, then x
  unsigned key[SM_CMAX]; // candidate keys (row << 6 | candidate)
  int src[SM_CMAX];      // candidate -> position in A's arrays
  signed char jj[SM_CMAX];
  T beta;
};

__device__ __forceinline__ void queue_big(const SmallArgs& a, int k, int nj, long long area) {
  int q = atomicAdd(&a.stats[ST_BIG_COUNT], 1);
  a.big_list[q] = k;
  atomicMax(&a.stats[ST_BIG_MAXNJ], nj);
  atomicMax(reinterpret_cast<unsigned long long*>(a.stats) + ST_AREA64, (unsigned long long)area);
}

// Bitonic sort of 8*PER keys held PER per lane (element e = lane*PER + s),
// ascending, across the 8 lanes of a group.
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
          unsigned other = __shfl_xor_sync(gmask, key[s], lx, GL);
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
            const bool swap = up ? (x > y) : (x < y);
            key[s] = swap ? y : x;
            key[p] = swap ? x : y;
          }
        }
      }
    }
  }
}

// Everything after candidate staging for one column, PER keys per lane.
// Returns |I_k| (or -1 when the column was queued for the CTA kernel).
template <int PER, typename T, int MODE>
__device__ __forceinline__ int small_column(const SmallArgs& a, SmallGroup<T>& sg, int k, int cs, int nj, int cand,
                                            int lane, unsigned gmask) {
  unsigned key[PER];
#pragma unroll
  for (int s = 0; s < PER; ++s) {
    const int t = lane * PER + s;
    key[s] = (t < cand) ? sg.key[t] : kPad;
  }
  group_sort<PER>(key, lane, gmask);

  // distinct rows: flag the first element of each run of equal rows
  const unsigned prev = __shfl_up_sync(gmask, key[PER - 1], 1, GL);
  int pre[PER];
  int cnt = 0;
#pragma unroll
  for (int s = 0; s < PER; ++s) {
    const bool valid = key[s] != kPad;
    const unsigned before = (s == 0) ? prev : key[s - 1];
    const bool first = valid && ((s == 0 && lane == 0) || (before >> 6) != (key[s] >> 6));
    cnt += first ? 1 : 0;
    pre[s] = first ? cnt : -cnt;  // sign marks "first", magnitude = inclusive count
  }
  int inc = cnt;
#pragma unroll
  for (int d = 1; d < GL; d <<= 1) {
    const int t = __shfl_up_sync(gmask, inc, d, GL);
    if (lane >= d) inc += t;
  }
  const int excl = inc - cnt;
  const int m = __shfl_sync(gmask, inc, GL - 1, GL);

  if (m > SM_MMAX) {
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
#pragma unroll
  for (int i = 0; i < SM_MMAX; ++i) sg.At[lane][i] = T(0);
  __syncwarp(gmask);
#pragma unroll
  for (int s = 0; s < PER; ++s) {
    if (key[s] != kPad) {
      const int t = key[s] & 63;
      const int pos = excl + (pre[s] > 0 ? pre[s] : -pre[s]) - 1;
      sg.At[sg.jj[t]][pos] = (T)__ldg(a.val + sg.src[t]);
    }
  }
  if (lane == 0 && E >= 0) sg.At[nj][E] = T(1);
  __syncwarp(gmask);

  // ---- Householder QR of [At | e_E]: lane j owns column j ---------------
  T r[SM_MMAX];
#pragma unroll
  for (int i = 0; i < SM_MMAX; ++i) r[i] = sg.At[lane][i];
  bool sing = m < nj;
  const int steps = min(nj, m);
  for (int c = 0; c < steps; ++c) {
    if (lane == c) {
      T nrm2 = T(0), x0 = T(0);
#pragma unroll
      for (int i = 0; i < SM_MMAX; ++i) {
        if (i >= c) {
          nrm2 += r[i] * r[i];
          sg.v[i] = r[i];
        }
        if (i == c) x0 = r[i];
      }
      const T nrm = sqrt(nrm2);
      T alpha = T(0), beta = T(0);
      if (nrm > T(0)) {
        alpha = (x0 > T(0)) ? -nrm : nrm;
        beta = T(1) / (nrm * (nrm + fabs(x0)));  // 2 / (v^T v)
        sg.v[c] = x0 - alpha;
      } else {
        sing = true;
      }
      sg.beta = beta;
#pragma unroll
      for (int i = 0; i < SM_MMAX; ++i) {
        if (i == c) r[i] = alpha;
        else if (i > c) r[i] = T(0);
      }
    }
    __syncwarp(gmask);
    if (lane > c && lane <= nj) {
      const T beta = sg.beta;
      T w = T(0);
#pragma unroll
      for (int i = 0; i < SM_MMAX; ++i)
        if (i >= c) w += sg.v[i] * r[i];
      w *= beta;
#pragma unroll
      for (int i = 0; i < SM_MMAX; ++i)
        if (i >= c) r[i] -= w * sg.v[i];
    }
    __syncwarp(gmask);
  }
  // ---- back substitution R x = (Q^T e_E)[0:nj] ---------------------------
  T res2 = T(0);
  if (lane < nj) {
#pragma unroll
    for (int i = 0; i <= SM_NJMAX; ++i)
      if (i <= lane) sg.At[lane][i] = r[i];
  } else if (lane == nj) {
#pragma unroll
    for (int i = 0; i < SM_MMAX; ++i) {
      if (i < nj) sg.v[i] = r[i];
      else res2 += r[i] * r[i];
    }
  }
  __syncwarp(gmask);
  if (lane == 0) {
    for (int i = nj - 1; i >= 0; --i) {
      T xi = sg.v[i];
      for (int j = i + 1; j < nj; ++j) xi -= sg.At[j][i] * sg.v[j];
      const T rii = sg.At[i][i];
      if (!(rii != T(0)) || !isfinite((double)rii)) sing = true;
      sg.v[i] = xi / rii;
    }
    if (sing) atomicAdd(&a.stats[ST_SINGULAR], 1);
  }
  __syncwarp(gmask);
  if (lane < nj) a.mval[cs + lane] = (double)sg.v[lane];
  if (lane == nj && a.colres) a.colres[col] = sqrt((double)res2);
  __syncwarp(gmask);
  return m;
}

template <typename T, int MODE>
__global__ void __launch_bounds__(SM_BLOCK, 4) k_spai_small(SmallArgs a) {
  __shared__ SmallGroup<T> groups[SM_GROUPS];
  const int lane = threadIdx.x & (GL - 1);
  const unsigned gmask = 0xFFu << (threadIdx.x & 24);
  SmallGroup<T>& sg = groups[threadIdx.x / GL];
  const int gid = (blockIdx.x * SM_BLOCK + threadIdx.x) / GL;
  const int ngroups = (gridDim.x * SM_BLOCK) / GL;
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
    if (nj > SM_NJMAX) {
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
    if (cand > SM_CMAX) {
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
        sg.key[t] = ((unsigned)row << 6) | (unsigned)t;
        sg.src[t] = bjj + q;
        sg.jj[t] = (signed char)j;
      }
    }
    __syncwarp(gmask);
    const int m = (cand <= 32) ? small_column<4, T, MODE>(a, sg, k, cs, nj, cand, lane, gmask)
                               : small_column<8, T, MODE>(a, sg, k, cs, nj, cand, lane, gmask);
    if (m >= 0) {
      my_max_ni = max(my_max_ni, m);
      ++my_cols;
    }
  };

  if (a.schedule == DCU_SCHED_BALANCED_COLUMNS) {
    // unit gid owns a contiguous balanced_columns range
    const int total = a.col_end - a.col_start;
    const int base = total / ngroups, rem = total % ngroups;
    const int start = a.col_start + gid * base + min(gid, rem);
    const int end = start + base + (gid < rem ? 1 : 0);
    for (int k = start; k < end; ++k) process(k);
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
// CTA per column.
// ---------------------------------------------------------------------------
constexpr int LG_BLOCK = 256;
constexpr int LG_WARPS = LG_BLOCK / 32;
constexpr int LG_NJ_MAX = 2048;      // max |J_k| (J metadata lives in shared memory)
constexpr int LG_WORDS_SMEM = 4096;  // bitmap words kept in shared memory

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
};

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
  T* sA = reinterpret_cast<T*>(smem_raw + ((sizeof(LargeSmem<T>) + 15) / 16) * 16);
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
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
    for (int t = tid; t < cand; t += LG_BLOCK) {
      int j, src;
      locate(t, j, src);
      const int row = a.idx[src];
      rmin = min(rmin, row);
      rmax = max(rmax, row);
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
    for (int t = tid; t < cand; t += LG_BLOCK) {
      int j, src;
      locate(t, j, src);
      const int off = a.idx[src] - rmin;
      atomicOr(&bits[off >> 5], 1u << (off & 31));
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
    if (area > a.smem_area && area > a.area_per_block) {
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
    for (int t = tid; t < cand; t += LG_BLOCK) {
      int j, src;
      locate(t, j, src);
      Ad[(long long)j * lda + rank(a.idx[src])] = (T)a.val[src];
    }
    if (tid == 0 && S.E >= 0) Ad[(long long)nj * lda + S.E] = T(1);
    __syncthreads();
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
      for (int t = tid; t < i; t += LG_BLOCK) S.ys[t] -= Ad[(long long)i * lda + t] * xi;
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
int run_small(Ctx* c, const SmallArgs& a, int grid) {
  k_spai_small<T, MODE><<<grid, SM_BLOCK, 0, c->stream>>>(a);
  DCU_LAUNCHED(c, "k_spai_small");
  return DCU_OK;
}

template <typename T, int MODE>
int run_large(Ctx* c, LargeArgs& a, int nbig) {
  const size_t fixed = ((sizeof(LargeSmem<T>) + 15) / 16) * 16;
  size_t cap = c->smem_optin > fixed + 1024 ? c->smem_optin - 1024 : fixed;
  a.smem_area = (MODE == MODE_BUILD) ? (long long)((cap - fixed) / sizeof(T)) : 0;
  const size_t smem = fixed + (size_t)a.smem_area * sizeof(T);
  DCU_CUDA(c, cudaFuncSetAttribute(k_spai_large<T, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int grid = nbig < c->sms ? nbig : c->sms;
  // global slabs for columns whose bitmap / dense block exceed shared memory
  a.words_per_block = ((long long)a.n >> 5) + 2;
  const long long area_cap = a.area_per_block;
  a.area_per_block = (MODE == MODE_BUILD && area_cap > a.smem_area) ? area_cap : 0;
  DCU_TRY(ensure(c, B_SLAB_BITS, sizeof(unsigned) * 2 * (size_t)a.words_per_block * grid));
  a.gbits = bp<unsigned>(c, B_SLAB_BITS);
  if (a.area_per_block > 0) DCU_TRY(ensure(c, B_SLAB_A, sizeof(T) * (size_t)a.area_per_block * grid));
  a.gA = a.area_per_block > 0 ? c->buf[B_SLAB_A].p : nullptr;
  k_spai_large<T, MODE><<<grid, LG_BLOCK, smem, c->stream>>>(a);
  DCU_LAUNCHED(c, "k_spai_large");
  return DCU_OK;
}

struct Prepared {
  SmallArgs sa;
  int grid = 0;
  int* stats = nullptr;
};

int prepare(Ctx* c, int n, const int* ptr, const int* idx, const double* val, int col_start, int col_end,
            int schedule, Prepared* P) {
  const int ncols = col_end - col_start;
  DCU_TRY(ensure(c, B_STATS, sizeof(int) * ST_INTS));
  DCU_TRY(ensure(c, B_BIGLIST, sizeof(int) * (size_t)(ncols > 0 ? ncols : 1)));
  int* stats = bp<int>(c, B_STATS);
  DCU_CUDA(c, cudaMemsetAsync(stats, 0, sizeof(int) * ST_INTS, c->stream));
  P->grid = c->sms * 4;
  const int ngroups = P->grid * SM_GROUPS;
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
  if (schedule == DCU_SCHED_BALANCED_NNZ) {
    const int nchunks = ngroups * 4;
    DCU_TRY(ensure(c, B_CHUNKS, sizeof(int) * (size_t)(nchunks + 1)));
    int* bounds = bp<int>(c, B_CHUNKS);
    k_nnz_chunks<<<(nchunks + 256) / 256, 256, 0, c->stream>>>(ptr, col_start, col_end, nchunks, bounds);
    DCU_LAUNCHED(c, "k_nnz_chunks");
    a.chunks = bounds;
    a.nchunks = nchunks;
  }
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

template <typename T>
int build_typed(Ctx* c, int n, const int* ptr, const int* idx, const double* val, int col_start, int col_end,
                int schedule, double* mval, double* colres, dcu_build_info* info) {
  Prepared P;
  DCU_TRY(prepare(c, n, ptr, idx, val, col_start, col_end, schedule, &P));
  P.sa.mval = mval;
  P.sa.colres = colres;
  DCU_TRY((run_small<T, MODE_BUILD>(c, P.sa, P.grid)));
  int st[ST_INTS];
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
    DCU_TRY((run_large<T, MODE_BUILD>(c, la, nbig)));
    DCU_TRY(read_stats(c, st));
    if (st[ST_LIMIT] > 0) return fail(c, DCU_ERR_LIMIT, "%d columns exceeded the CTA kernel's limits", st[ST_LIMIT]);
  }
  if (info) {
    info->cols_total = col_end - col_start;
    info->cols_small = st[ST_SMALL_COLS];
    info->cols_large = st[ST_BIG_DONE];
    info->cols_singular = st[ST_SINGULAR];
    info->max_nj = st[ST_MAXNJ] > st[ST_BIG_MAXNJ] ? st[ST_MAXNJ] : st[ST_BIG_MAXNJ];
    info->max_ni = st[ST_MAXNI];
  }
  return DCU_OK;
}

}  // namespace

int spai_build(Ctx* c, int n, int nnz, const int* ptr, const int* idx, const double* val, const dcu_options* opt,
               double* mval, double* colres, dcu_build_info* info) {
  const int col_start = opt->col_start;
  const int col_end = opt->col_end;
  if (col_start != 0 || col_end != n)
    DCU_CUDA(c, cudaMemsetAsync(mval, 0, sizeof(double) * (size_t)(nnz > 0 ? nnz : 1), c->stream));
  if (col_end <= col_start) return DCU_OK;
  if (opt->precision == DCU_PREC_FP64)
    return build_typed<double>(c, n, ptr, idx, val, col_start, col_end, opt->schedule, mval, colres, info);
  return build_typed<float>(c, n, ptr, idx, val, col_start, col_end, opt->schedule, mval, colres, info);
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
