// Pattern conversions on the device: CSC -> CSR (the reference's cuCSC2CSR,
// include/common/cuFormatConversion.h:453-589: per-row counts, a scan, a
// scatter into row slots, then ascending column order inside each row) and
// the SELL-32 layout the SpMV kernels read.
//
// Layout in HBM (n rows, nnz entries):
//   CSR    rptr int32[n+1], rcol int32[nnz], rperm int32[nnz] (CSR slot -> CSC slot)
//   SELL   slice s = rows [32 s, 32 s + 32); width[s] = longest row in the slice;
//          slot of (row r, k-th entry) = off[s] + 32 k + (r mod 32), so one warp
//          reads 32 consecutive slots per k (128-byte lines for FP32/int32,
//          256 bytes for FP64).  Padding slots carry column = r and perm = -1.
//          del int16 holds col - r when every |col - r| < 32768.
#include <climits>

#include "internal.cuh"

namespace dcu {
namespace {

__global__ void k_row_count(const int* __restrict__ idx, int nnz, int* __restrict__ cnt) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += gridDim.x * blockDim.x)
    atomicAdd(&cnt[idx[e]], 1);
}

// One thread per column: scatter the column's entries into their rows' slots.
__global__ void k_row_scatter(const int* __restrict__ ptr, const int* __restrict__ idx, int n,
                              const int* __restrict__ rptr, int* __restrict__ fill,
                              int* __restrict__ rcol, int* __restrict__ rperm) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    for (int e = ptr[c]; e < ptr[c + 1]; ++e) {
      int r = idx[e];
      int pos = rptr[r] + atomicAdd(&fill[r], 1);
      rcol[pos] = c;
      rperm[pos] = e;
    }
  }
}

// Structurally symmetric patterns (every PDE stencil): row c of A lists the
// same indices as column c, so with ascending row indices in every column the
// CSR index arrays are the CSC ones, and only the CSR slot -> CSC slot map
// needs work: entry (row c, column r) sits in column r where idx == c, found
// by binary search.  One thread per column; flag bit 1 = a column is not
// strictly ascending, bit 2 = some (r, c) has no (c, r).  Any flag sends the
// conversion to the general count / scatter / sort path, which rewrites all
// three outputs.  With copies = 0 only rperm is written (the caller reads
// ptr and idx as the CSR arrays).
__global__ void k_csr_symmetric(const int* __restrict__ ptr, const int* __restrict__ idx, int n,
                                int* __restrict__ rptr, int* __restrict__ rcol, int* __restrict__ rperm,
                                int* __restrict__ flag, int copies) {
  constexpr int kShort = 8;  // columns up to this long search their partners side by side
  int bad = 0;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    const int s = ptr[c], e = ptr[c + 1];
    if (copies) {
      rptr[c] = s;
      if (c == n - 1) rptr[n] = e;
    }
    if (e - s <= kShort) {
      // the entries' rows, their columns' ranges, then the binary searches
      // one step at a time for all entries: a few dependent loads per column
      // instead of a few per entry
      const int len = e - s;
      int r[kShort], lo[kShort], hi[kShort], q[kShort];
#pragma unroll
      for (int t = 0; t < kShort; ++t) r[t] = (t < len) ? idx[s + t] : 0;
      int prev = -1;
#pragma unroll
      for (int t = 0; t < kShort; ++t) {
        if (t < len) {
          if (copies) rcol[s + t] = r[t];
          if (r[t] <= prev) bad |= 1;
          prev = r[t];
          lo[t] = ptr[r[t]];
          hi[t] = ptr[r[t] + 1] - 1;
        } else {
          lo[t] = 0;
          hi[t] = -1;
        }
        q[t] = -1;
      }
      for (;;) {
        bool active = false;
#pragma unroll
        for (int t = 0; t < kShort; ++t) {
          if (q[t] < 0 && lo[t] <= hi[t]) {
            active = true;
            const int mid = (lo[t] + hi[t]) >> 1;
            const int v = idx[mid];
            if (v == c) q[t] = mid;
            else if (v < c) lo[t] = mid + 1;
            else hi[t] = mid - 1;
          }
        }
        if (!active) break;
      }
#pragma unroll
      for (int t = 0; t < kShort; ++t)
        if (t < len) {
          if (q[t] < 0) bad |= 2;
          rperm[s + t] = q[t];
        }
      continue;
    }
    int prev = -1;
    for (int k = s; k < e; ++k) {
      const int r = idx[k];
      if (copies) rcol[k] = r;
      if (r <= prev) bad |= 1;
      prev = r;
      int lo = ptr[r], hi = ptr[r + 1] - 1, q = -1;
      while (lo <= hi) {
        const int mid = (lo + hi) >> 1;
        const int v = idx[mid];
        if (v == c) {
          q = mid;
          break;
        }
        if (v < c) lo = mid + 1;
        else hi = mid - 1;
      }
      if (q < 0) bad |= 2;
      rperm[k] = q;
    }
  }
  if (__any_sync(0xffffffffu, bad != 0) && bad) atomicOr(flag, bad);
}

constexpr int kRegSortMax = 16;     // rows sorted in registers by one thread
constexpr int kThreadSortMax = 64;  // rows sorted in place by one thread

// Rows up to kRegSortMax entries: loaded into registers as (col << 32 | slot)
// keys, sorted with a static insertion network, written back only when out
// of order.  Rows up to kThreadSortMax: insertion sort in place.  Longer rows
// are queued for the block sort.  Column indices inside a row are distinct
// (a CSC column lists each row once), so the order is unique.
__global__ void k_row_sort_short(const int* __restrict__ rptr, int n, int* __restrict__ rcol,
                                 int* __restrict__ rperm, int* __restrict__ long_rows,
                                 int* __restrict__ long_count) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const int s = rptr[r], e = rptr[r + 1];
    const int len = e - s;
    if (len <= kRegSortMax) {
      unsigned long long key[kRegSortMax];
      bool sorted = true;
      int prev = -1;
#pragma unroll
      for (int i = 0; i < kRegSortMax; ++i) {
        if (i < len) {
          const int cc = rcol[s + i];
          sorted = sorted && (cc > prev);
          prev = cc;
          key[i] = ((unsigned long long)(unsigned)cc << 32) | (unsigned)rperm[s + i];
        } else {
          key[i] = ~0ull;
        }
      }
      if (sorted) continue;
#pragma unroll
      for (int i = 1; i < kRegSortMax; ++i) {
#pragma unroll
        for (int q = i; q > 0; --q) {
          const unsigned long long lo = min(key[q - 1], key[q]), hi = max(key[q - 1], key[q]);
          key[q - 1] = lo;
          key[q] = hi;
        }
      }
#pragma unroll
      for (int i = 0; i < kRegSortMax; ++i) {
        if (i < len) {
          rcol[s + i] = (int)(key[i] >> 32);
          rperm[s + i] = (int)(key[i] & 0xffffffffu);
        }
      }
      continue;
    }
    if (len > kThreadSortMax) {
      long_rows[atomicAdd(long_count, 1)] = r;
      atomicMax(long_count + 1, len);
      continue;
    }
    for (int i = s + 1; i < e; ++i) {
      int kc = rcol[i], kp = rperm[i];
      int j = i - 1;
      while (j >= s && rcol[j] > kc) {
        rcol[j + 1] = rcol[j];
        rperm[j + 1] = rperm[j];
        --j;
      }
      rcol[j + 1] = kc;
      rperm[j + 1] = kp;
    }
  }
}

// One block per long row: bitonic sort of (col << 32 | perm) keys in shared
// memory (rows up to kSmemSortMax) or in a global scratch slab.
constexpr int kSmemSortMax = 8192;

__device__ __forceinline__ void bitonic_block(unsigned long long* key, int npow2) {
  for (int k = 2; k <= npow2; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < npow2; i += blockDim.x) {
        int l = i ^ j;
        if (l > i) {
          unsigned long long a = key[i], b = key[l];
          bool up = (i & k) == 0;
          if ((a > b) == up) {
            key[i] = b;
            key[l] = a;
          }
        }
      }
      __syncthreads();
    }
  }
}

__global__ void __launch_bounds__(512) k_row_sort_long(const int* __restrict__ rptr, const int* __restrict__ rows,
                                                       const int* __restrict__ count, int* __restrict__ rcol,
                                                       int* __restrict__ rperm, unsigned long long* __restrict__ gscratch,
                                                       long long gscratch_per_block) {
  extern __shared__ unsigned long long skey[];
  int nrows = *count;
  for (int q = blockIdx.x; q < nrows; q += gridDim.x) {
    int r = rows[q];
    int s = rptr[r], len = rptr[r + 1] - s;
    int np2 = 1;
    while (np2 < len) np2 <<= 1;
    unsigned long long* key = (np2 <= kSmemSortMax) ? skey : gscratch + (long long)blockIdx.x * gscratch_per_block;
    for (int i = threadIdx.x; i < np2; i += blockDim.x)
      key[i] = (i < len) ? ((unsigned long long)(unsigned)rcol[s + i] << 32 | (unsigned)rperm[s + i]) : ~0ull;
    __syncthreads();
    bitonic_block(key, np2);
    for (int i = threadIdx.x; i < len; i += blockDim.x) {
      rcol[s + i] = (int)(key[i] >> 32);
      rperm[s + i] = (int)(key[i] & 0xffffffffu);
    }
    __syncthreads();
  }
}

__global__ void k_gather_f64(const int* __restrict__ perm, const double* __restrict__ src, int nnz,
                             double* __restrict__ dst) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += gridDim.x * blockDim.x) dst[e] = src[perm[e]];
}

// SELL: slice widths (max row length of each 32-row slice), one warp per slice.
__global__ void k_sell_width(const int* __restrict__ rptr, int n, int nslices, int* __restrict__ width) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  int nw = (gridDim.x * blockDim.x) >> 5;
  for (int s = warp; s < nslices; s += nw) {
    int r = s * 32 + lane;
    int len = (r < n) ? rptr[r + 1] - rptr[r] : 0;
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) len = max(len, __shfl_xor_sync(0xffffffffu, len, d));
    if (lane == 0) width[s] = len * 32;  // slots in the slice (scanned into offsets)
  }
}

// One warp per slice (rows 32 s .. 32 s + 31 on the lanes).  First try the
// offset-aligned layout: slot k of every row holds the entry at the k-th
// smallest column offset (column - row) found in the slice, or a zero-valued
// padding slot at that offset.  It fits when the slice has no more distinct
// offsets than its longest row has entries (every stencil slice away from the
// domain's first row), and then every k has one offset for the whole slice.
// Otherwise the compact layout: row entries in order, padding at the end.
// Rows keep their column order either way; padding slots have perm = -1 and,
// in the compact layout or where row + offset leaves [0, n), column = row.
//
// The same pass describes each slot it writes, from the column in hand:
//   del[q] = column - row as int16 (read only when maxdelta < 32768);
//   kd[off[s] / 32 + k] = (d << 1) | 1 when every row of the slice below n
//     has its k-th slot at one offset d, else 0;
//   su[s] bit 0 when every k has one offset (the SpMV then reads no index),
//     bit 1 (narrow) when in addition the slice is at most kNarrow wide, with
//     its width in bits 3-6 and kd8[kNarrow s + k] = d (kd8h as int16), bit 2
//     (wide) for a full slice wider than kWideSlice made so by at most
//     kWideRows long rows, listed in wide (wide[0] counts);
//   *uslots += the slots of the uniform slices (one atomic per block).
__global__ void k_sell_layout(const int* __restrict__ rptr, const int* __restrict__ rcol,
                              const int* __restrict__ rperm, int n, int nslices, const long long* __restrict__ off,
                              int* __restrict__ sidx, int* __restrict__ sperm, int* __restrict__ maxdelta,
                              int16_t* __restrict__ del, int* __restrict__ kd, int* __restrict__ su,
                              unsigned long long* __restrict__ uslots, int* __restrict__ wide, int allow_wide,
                              int* __restrict__ kd8, int16_t* __restrict__ kd8h) {
  __shared__ unsigned long long blk_uslots;
  if (threadIdx.x == 0) blk_uslots = 0ull;
  __syncthreads();
  unsigned long long my_uslots = 0ull;  // lane 0 of each warp: uniform slots of its slices
  const int rows_total = nslices * 32;
  int local_max = 0;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows_total; r += gridDim.x * blockDim.x) {
    const int s = r >> 5, lane = r & 31;
    const long long o0 = off[s];
    const long long base = o0 + lane;
    const int w = (int)((off[s + 1] - o0) >> 5);
    int rs = 0, len = 0;
    if (r < n) {
      rs = rptr[r];
      len = rptr[r + 1] - rs;
    }
    const int self = (r < n) ? r : 0;
    for (int j = 0; j < len; ++j) local_max = max(local_max, abs(rcol[rs + j] - self));
    bool all = true;
    int my_d = 0;  // lane k < kNarrow: offset of entry position k
    // slot k of this row holds column col: its delta and the slice's offset check
    auto note = [&](int k, long long q, int col) {
      del[q] = (int16_t)(col - self);
      const int d = col - r;
      const int d0 = __shfl_sync(0xffffffffu, d, 0);  // row 32 s < n always
      const bool same = __all_sync(0xffffffffu, r >= n || d == d0);
      all = all && same;
      if (lane == 0) kd[(o0 >> 5) + k] = same ? (int)(((unsigned)d0 << 1) | 1u) : 0;
      if (lane == k) my_d = d0;
    };
    int i = 0;
    for (int k = 0; k < w; ++k) {
      const int cand = (i < len) ? rcol[rs + i] - r : INT_MAX;
      const int m = __reduce_min_sync(0xffffffffu, cand);
      const long long q = base + 32ll * k;
      int col;
      if (i < len && cand == m) {
        col = rcol[rs + i];
        sperm[q] = rperm[rs + i];
        ++i;
      } else {
        col = self;
        if (r < n && m != INT_MAX && (long long)r + m >= 0 && (long long)r + m < n) col = r + m;
        sperm[q] = -1;
      }
      sidx[q] = col;
      note(k, q, col);
    }
    if (!__all_sync(0xffffffffu, i == len)) {
      all = true;
      my_d = 0;
      for (int k = 0; k < w; ++k) {
        const long long q = base + 32ll * k;
        int col;
        if (k < len) {
          col = rcol[rs + k];
          sperm[q] = rperm[rs + k];
        } else {
          col = self;
          sperm[q] = -1;
        }
        sidx[q] = col;
        note(k, q, col);
      }
    }
    const bool narrow = all && w > 0 && w <= kNarrow;
    if (lane < kNarrow) {
      const int d = (narrow && lane < w) ? my_d : 0;
      kd8[(long long)s * kNarrow + lane] = d;
      kd8h[(long long)s * kNarrow + lane] = (int16_t)d;  // read only when every |d| < 32768
    }
    // rows of the slice longer than kWideSlice
    const int nlong = __popc(__ballot_sync(0xffffffffu, len > kWideSlice));
    if (lane == 0) {
      int f = all ? 1 : 0;
      if (narrow) f |= 2 | (w << 3);
      // a full slice made wide by a few long rows: listed for the solver's
      // pre-pass (wide[0] counts, wide[1 + i] = slice)
      if (allow_wide && w > kWideSlice && nlong <= kWideRows && 32 * s + 32 <= n) {
        const int wi = atomicAdd(wide, 1);
        wide[1 + wi] = s;
        f |= 4 | (wi << 3);
      }
      su[s] = f;
      if (all && w > 0) my_uslots += 32ull * (unsigned long long)w;
    }
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) local_max = max(local_max, __shfl_xor_sync(0xffffffffu, local_max, d));
  if ((threadIdx.x & 31) == 0) atomicMax(maxdelta, local_max);
  // one atomic per block (the warps' loop trip counts differ: no barrier
  // inside the loop; lane 0 of each warp adds its total here)
  if ((threadIdx.x & 31) == 0 && my_uslots) atomicAdd(&blk_uslots, my_uslots);
  __syncthreads();
  if (threadIdx.x == 0 && blk_uslots) atomicAdd(uslots, blk_uslots);
}

template <typename T>
__device__ __forceinline__ T cvt_from_double(double v);
template <>
__device__ __forceinline__ double cvt_from_double<double>(double v) { return v; }
template <>
__device__ __forceinline__ float cvt_from_double<float>(double v) { return (float)v; }
template <>
__device__ __forceinline__ __nv_bfloat16 cvt_from_double<__nv_bfloat16>(double v) { return __double2bfloat16(v); }

template <typename T>
__global__ void k_sell_gather(const int* __restrict__ sperm, long long slots, const double* __restrict__ src,
                              T* __restrict__ dst) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < slots;
       q += (long long)gridDim.x * blockDim.x) {
    int p = sperm[q];
    dst[q] = cvt_from_double<T>(p >= 0 ? src[p] : 0.0);
  }
}

// A's values: an FP32 SELL copy, and a flag raised (one atomic per warp)
// when a value does not survive the round trip through FP32 bit for bit (a
// rounded value, an FP64 subnormal, a value beyond FP32's range, a NaN
// payload).
__global__ void k_sell_gather_a(const int* __restrict__ sperm, long long slots, const double* __restrict__ src,
                                float* __restrict__ dst32, int* __restrict__ inexact) {
  bool off = false;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < slots;
       q += (long long)gridDim.x * blockDim.x) {
    const int p = sperm[q];
    const double v = p >= 0 ? src[p] : 0.0;
    const float f = __double2float_rn(v);
    dst32[q] = f;
    off |= __double_as_longlong((double)f) != __double_as_longlong(v);
  }
  if (__any_sync(0xffffffffu, off) && (threadIdx.x & 31) == 0) atomicOr(inexact, 1);
}

// The FP64 SELL copy of A's values, needed only when some value is not exact
// in FP32 or when `force` (the wide-slice pre-pass reads FP64 values): with
// the flag clear and no force every block returns at once.
__global__ void k_sell_gather_a64(const int* __restrict__ sperm, long long slots, const double* __restrict__ src,
                                  double* __restrict__ dst, const int* __restrict__ inexact, int force) {
  if (!force && *inexact == 0) return;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < slots;
       q += (long long)gridDim.x * blockDim.x) {
    const int p = sperm[q];
    dst[q] = p >= 0 ? src[p] : 0.0;
  }
}

template <typename T>
int sell_gather(Ctx* c, const SellPlan& p, const double* src, T* dst) {
  int grid = waves_grid(c, p.slots, 256, 8);
  k_sell_gather<T><<<grid, 256, 0, c->stream>>>(p.perm, p.slots, src, dst);
  DCU_LAUNCHED(c, "k_sell_gather");
  return DCU_OK;
}

// Structural check of a CSC matrix before any kernel chases its indices:
// ptr[0] == 0, ptr non-decreasing, ptr[n] == nnz, 0 <= idx < n.  One thread
// per column walks that column's entries (only once its own bounds are known
// to lie in [0, nnz]): a valid ptr partitions [0, nnz) into the columns, so
// every entry is range-checked, and an invalid ptr is itself an error.  The
// walk also compares neighbours: a repeated row in an ascending run is a
// duplicate (32), a descent marks the matrix as having an unsorted column
// (16), whose duplicates k_csc_duplicates then looks for.
__global__ void k_validate_csc(const int* __restrict__ ptr, const int* __restrict__ idx, int n, int nnz,
                               int* __restrict__ bad) {
  const int stride = gridDim.x * blockDim.x;
  int b = 0;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c <= n; c += stride) {
    const int p = ptr[c];
    if (c == 0 && p != 0) b |= 1;
    if (c == n && p != nnz) b |= 2;
    if (c < n) {
      const int q = ptr[c + 1];
      if (q < p) {
        b |= 4;
      } else if (p >= 0 && q <= nnz) {
        int prev = -1;
        for (int e = p; e < q; ++e) {
          const int r = __ldg(idx + e);
          if (r < 0 || r >= n) b |= 8;
          if (e > p) b |= r == prev ? 32 : (r < prev ? 16 : 0);
          prev = r;
        }
      }
    }
  }
  if (b) atomicOr(bad, b);
}

// Duplicate rows inside unsorted columns (run only when k_validate_csc found
// one, after it passed): one warp per column compares every pair of entries,
// 32 x 32 per step through shuffles, so a column of L entries costs L^2 / 32
// comparisons per lane.  Sorted columns are skipped by a neighbour check.
__global__ void k_csc_duplicates(const int* __restrict__ ptr, const int* __restrict__ idx, int n,
                                 int* __restrict__ bad) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < n; c += warps) {
    const int p = ptr[c], len = ptr[c + 1] - p;
    if (len < 2) continue;
    bool desc = false;
    for (int e = lane + 1; e < len; e += 32) desc |= idx[p + e] < idx[p + e - 1];
    if (!__any_sync(0xffffffffu, desc)) continue;
    bool dup = false;
    for (int a = 0; a < len; a += 32) {
      const int v = a + lane < len ? idx[p + a + lane] : -1;
      for (int bb = a; bb < len; bb += 32) {
        const int w = bb + lane < len ? idx[p + bb + lane] : -2;
        const int lim = min(32, len - bb);
        for (int s = 0; s < lim; ++s) {
          const int ws = __shfl_sync(0xffffffffu, w, s);
          dup |= v >= 0 && (bb > a || s > lane) && v == ws;
        }
      }
    }
    if (__any_sync(0xffffffffu, dup) && lane == 0) atomicOr(bad, 32);
  }
}

__global__ void k_iota(int* __restrict__ out, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = i;
}

// out[e] = alpha * u[idx[e]] * v[j] for every entry e = (idx[e], j) of a CSC
// pattern: the outer product u v^T sampled on the pattern (one warp per
// column, lanes over the column's entries).
__global__ void k_sampled_outer(const int* __restrict__ ptr, const int* __restrict__ idx, int n,
                                const double* __restrict__ u, const double* __restrict__ v, double alpha,
                                double* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < n; j += warps) {
    const double vj = alpha * v[j];
    for (int e = ptr[j] + lane; e < ptr[j + 1]; e += 32) out[e] = u[idx[e]] * vj;
  }
}

}  // namespace

int sampled_outer(Ctx* c, int n, const int* ptr, const int* idx, const double* u, const double* v, double alpha,
                  double* out) {
  k_sampled_outer<<<waves_grid(c, (long long)n * 32, 256, 8), 256, 0, c->stream>>>(ptr, idx, n, u, v, alpha, out);
  DCU_LAUNCHED(c, "k_sampled_outer");
  return DCU_OK;
}

int validate_csc(Ctx* c, int n, int nnz, const int* ptr, const int* idx, bool unique_rows) {
  DCU_TRY(ensure(c, B_ROWCNT, sizeof(int) * (size_t)(n + 1)));
  int* bad = bp<int>(c, B_ROWCNT);
  DCU_CUDA(c, cudaMemsetAsync(bad, 0, sizeof(int), c->stream));
  k_validate_csc<<<waves_grid(c, (long long)n + 1, 256, 8), 256, 0, c->stream>>>(ptr, idx, n, nnz, bad);
  DCU_LAUNCHED(c, "k_validate_csc");
  DCU_CUDA(c, cudaMemcpyAsync(c->pinned, bad, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  DCU_CUDA(c, cudaStreamSynchronize(c->stream));
  int b = *(int*)c->pinned;
  if (b & 15) {
    return fail(c, DCU_ERR_ARG, "malformed CSC matrix:%s%s%s%s", (b & 1) ? " ptr[0] != 0;" : "",
                (b & 2) ? " ptr[n] != nnz;" : "", (b & 4) ? " ptr decreases;" : "",
                (b & 8) ? " row index out of [0, n);" : "");
  }
  if (!unique_rows) return DCU_OK;
  if ((b & 16) && !(b & 32)) {
    k_csc_duplicates<<<waves_grid(c, (long long)n * 32, 256, 8), 256, 0, c->stream>>>(ptr, idx, n, bad);
    DCU_LAUNCHED(c, "k_csc_duplicates");
    DCU_CUDA(c, cudaMemcpyAsync(c->pinned, bad, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    DCU_CUDA(c, cudaStreamSynchronize(c->stream));
    b = *(int*)c->pinned;
  }
  if (b & 32)
    return fail(c, DCU_ERR_ARG, "malformed CSC matrix: a column holds the same row index twice (duplicate entries "
                                "are not accepted; sum them first)");
  return DCU_OK;
}

namespace {

// k_csr_symmetric into (rptr, rcol, rperm) without waiting: *flag (device) is
// 0 when the pattern was symmetric with ascending columns and the result
// stands, else the general path must run.
int csr_try_symmetric(Ctx* c, int n, const int* ptr, const int* idx, int* rptr, int* rcol, int* rperm,
                      int** flag, bool copies) {
  DCU_TRY(ensure(c, B_LONGROWS, sizeof(int) * (size_t)(n + 2)));
  int* longcount = bp<int>(c, B_LONGROWS) + n;
  DCU_CUDA(c, cudaMemsetAsync(longcount, 0, 2 * sizeof(int), c->stream));
  k_csr_symmetric<<<waves_grid(c, n, 256, 8), 256, 0, c->stream>>>(ptr, idx, n, rptr, rcol, rperm, longcount,
                                                                     copies ? 1 : 0);
  DCU_LAUNCHED(c, "k_csr_symmetric");
  *flag = longcount;
  return DCU_OK;
}

// The general CSC -> CSR: counts, scan, scatter, per-row sort.
int csr_general(Ctx* c, int n, int nnz, const int* ptr, const int* idx, int* rptr, int* rcol, int* rperm) {
  DCU_TRY(ensure(c, B_ROWCNT, sizeof(int) * (size_t)(n + 1)));
  DCU_TRY(ensure(c, B_LONGROWS, sizeof(int) * (size_t)(n + 2)));
  int* cnt = bp<int>(c, B_ROWCNT);
  int* longrows = bp<int>(c, B_LONGROWS);
  int* longcount = longrows + n;  // [0] = count, [1] = longest length
  DCU_CUDA(c, cudaMemsetAsync(longcount, 0, 2 * sizeof(int), c->stream));
  DCU_CUDA(c, cudaMemsetAsync(cnt, 0, sizeof(int) * (size_t)(n + 1), c->stream));
  if (nnz > 0) {
    k_row_count<<<waves_grid(c, nnz, 256, 8), 256, 0, c->stream>>>(idx, nnz, cnt);
    DCU_LAUNCHED(c, "k_row_count");
  }
  DCU_TRY(scan_exclusive_i32(c, cnt, rptr, n));
  DCU_CUDA(c, cudaMemsetAsync(cnt, 0, sizeof(int) * (size_t)(n + 1), c->stream));
  k_row_scatter<<<waves_grid(c, n, 256, 8), 256, 0, c->stream>>>(ptr, idx, n, rptr, cnt, rcol, rperm);
  DCU_LAUNCHED(c, "k_row_scatter");
  k_row_sort_short<<<waves_grid(c, n, 256, 8), 256, 0, c->stream>>>(rptr, n, rcol, rperm, longrows, longcount);
  DCU_LAUNCHED(c, "k_row_sort_short");
  // Long rows: the block sort needs the longest row for its global slab.
  DCU_CUDA(c, cudaMemcpyAsync(c->pinned, longcount, 2 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  DCU_CUDA(c, cudaStreamSynchronize(c->stream));
  int nlong = ((int*)c->pinned)[0];
  int maxlen = ((int*)c->pinned)[1];
  if (nlong > 0) {
    long long np2 = 1;
    while (np2 < maxlen) np2 <<= 1;
    int blocks = nlong < c->sms ? nlong : c->sms;
    long long per_block = (np2 > kSmemSortMax) ? np2 : 0;
    if (per_block > 0) DCU_TRY(ensure(c, B_SORTTMP, sizeof(unsigned long long) * (size_t)per_block * blocks));
    unsigned long long* g = per_block > 0 ? bp<unsigned long long>(c, B_SORTTMP) : nullptr;
    size_t smem = sizeof(unsigned long long) * kSmemSortMax;
    DCU_CUDA(c, cudaFuncSetAttribute(k_row_sort_long, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_row_sort_long<<<blocks, 512, smem, c->stream>>>(rptr, longrows, longcount, rcol, rperm, g, per_block);
    DCU_LAUNCHED(c, "k_row_sort_long");
  }
  return DCU_OK;
}

}  // namespace

int csr_from_csc(Ctx* c, int n, int nnz, const int* ptr, const int* idx, int* rptr, int* rcol, int* rperm) {
  if (n > 0 && nnz > 0) {
    int* flag = nullptr;
    DCU_TRY(csr_try_symmetric(c, n, ptr, idx, rptr, rcol, rperm, &flag, true));
    DCU_CUDA(c, cudaMemcpyAsync(c->pinned, flag, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    DCU_CUDA(c, cudaStreamSynchronize(c->stream));
    if (*(int*)c->pinned == 0) return DCU_OK;
  }
  return csr_general(c, n, nnz, ptr, idx, rptr, rcol, rperm);
}

int sell_plan(Ctx* c, int n, int nnz, const int* ptr, const int* idx, SellPlan* plan) {
  DCU_TRY(ensure(c, B_RPTR, sizeof(int) * (size_t)(n + 1)));
  DCU_TRY(ensure(c, B_RCOL, sizeof(int) * (size_t)(nnz > 0 ? nnz : 1)));
  DCU_TRY(ensure(c, B_RPERM, sizeof(int) * (size_t)(nnz > 0 ? nnz : 1)));
  int* rptr = bp<int>(c, B_RPTR);
  int* rcol = bp<int>(c, B_RCOL);
  int* rperm = bp<int>(c, B_RPERM);
  if (n > 0 && nnz > 0) {
    // the layout is built from the symmetric conversion without waiting for
    // its verdict, which comes back with the layout's last round trip; a
    // pattern that is not symmetric (the speculative layout stays in bounds:
    // its row pointers, columns and slots are A's own) is laid out again
    // from the general conversion.  A symmetric pattern's CSR row pointers
    // and columns are A's CSC arrays themselves: the layout reads those.
    int* flag = nullptr;
    DCU_TRY(csr_try_symmetric(c, n, ptr, idx, rptr, rcol, rperm, &flag, false));
    int bad = 0;
    DCU_TRY(sell_fill_from_csr(c, n, nnz, ptr, idx, rperm, plan, flag, &bad));
    if (bad == 0) return DCU_OK;
  }
  DCU_TRY(csr_general(c, n, nnz, ptr, idx, rptr, rcol, rperm));
  return sell_fill_from_csr(c, n, nnz, rptr, rcol, rperm, plan);
}

int sell_fill_from_csr(Ctx* c, int n, int nnz, const int* rptr, const int* rcol, const int* rperm, SellPlan* plan,
                       const int* check, int* check_out) {
  int nslices = (n + 31) / 32;
  DCU_TRY(ensure(c, B_SELL_W, sizeof(int) * (size_t)(nslices + 1)));
  DCU_TRY(ensure(c, B_SELL_OFF, sizeof(long long) * (size_t)(nslices + 1)));
  int* width = bp<int>(c, B_SELL_W);
  long long* off = bp<long long>(c, B_SELL_OFF);
  k_sell_width<<<waves_grid(c, (long long)nslices * 32, 256, 8), 256, 0, c->stream>>>(rptr, n, nslices, width);
  DCU_LAUNCHED(c, "k_sell_width");
  DCU_TRY(scan_exclusive_i64(c, width, off, nslices));
  DCU_CUDA(c, cudaMemcpyAsync(c->pinned, off + nslices, sizeof(long long), cudaMemcpyDeviceToHost, c->stream));
  DCU_CUDA(c, cudaStreamSynchronize(c->stream));
  long long slots = *(long long*)c->pinned;
  DCU_TRY(ensure(c, B_SELL_IDX, sizeof(int) * (size_t)(slots > 0 ? slots : 1)));
  DCU_TRY(ensure(c, B_SELL_PERM, sizeof(int) * (size_t)(slots > 0 ? slots : 1)));
  int* sidx = bp<int>(c, B_SELL_IDX);
  int* sperm = bp<int>(c, B_SELL_PERM);
  DCU_TRY(ensure(c, B_ROWCNT, sizeof(int) * (size_t)(n + 1)));
  int* maxdelta = bp<int>(c, B_ROWCNT);  // row counts are no longer needed
  DCU_CUDA(c, cudaMemsetAsync(maxdelta, 0, sizeof(int), c->stream));
  // the 16-bit deltas are written always and read only when the maximum
  // |col - row| allows them; the host reads that maximum with the wide-slice
  // count at the end, one round trip for both
  DCU_TRY(ensure(c, B_SELL_DEL, sizeof(int16_t) * (size_t)(slots > 0 ? slots : 1)));
  int16_t* del = bp<int16_t>(c, B_SELL_DEL);
  DCU_TRY(ensure(c, B_SELL_KD, sizeof(int) * ((size_t)nslices + (size_t)(slots / 32) + 1)));
  int* su = bp<int>(c, B_SELL_KD);
  int* kd = su + nslices;
  DCU_TRY(ensure(c, B_PLANSTAT, 2 * sizeof(unsigned long long)));
  unsigned long long* pst = bp<unsigned long long>(c, B_PLANSTAT);
  const unsigned long long hst[2] = {(unsigned long long)slots, 0ull};
  DCU_CUDA(c, cudaMemcpyAsync(pst, hst, sizeof(hst), cudaMemcpyHostToDevice, c->stream));
  DCU_TRY(ensure(c, B_SELL_WIDE, sizeof(int) * ((size_t)nslices + 1)));
  int* wide = bp<int>(c, B_SELL_WIDE);
  DCU_TRY(ensure(c, B_SELL_KD8, (sizeof(int) + sizeof(int16_t)) * kNarrow * (size_t)nslices));
  int* kd8 = bp<int>(c, B_SELL_KD8);
  int16_t* kd8h = reinterpret_cast<int16_t*>(kd8 + kNarrow * (size_t)nslices);
  DCU_CUDA(c, cudaMemsetAsync(wide, 0, sizeof(int), c->stream));
  k_sell_layout<<<waves_grid(c, (long long)nslices * 32, 256, 8), 256, 0, c->stream>>>(
      rptr, rcol, rperm, n, nslices, off, sidx, sperm, maxdelta, del, kd, su, pst + 1, wide, c->wide_prepass ? 1 : 0,
      kd8, kd8h);
  DCU_LAUNCHED(c, "k_sell_layout");
  DCU_CUDA(c, cudaMemcpyAsync(c->pinned, wide, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  DCU_CUDA(c, cudaMemcpyAsync(reinterpret_cast<int*>(c->pinned) + 1, maxdelta, sizeof(int), cudaMemcpyDeviceToHost,
                              c->stream));
  if (check)
    DCU_CUDA(c, cudaMemcpyAsync(reinterpret_cast<int*>(c->pinned) + 2, check, sizeof(int), cudaMemcpyDeviceToHost,
                                c->stream));
  DCU_CUDA(c, cudaStreamSynchronize(c->stream));
  if (check_out) *check_out = check ? reinterpret_cast<int*>(c->pinned)[2] : 0;
  plan->nwide = *reinterpret_cast<int*>(c->pinned);
  plan->delta16 = reinterpret_cast<int*>(c->pinned)[1] < 32768;
  plan->del = plan->delta16 ? del : nullptr;
  if (!plan->delta16) kd8h = nullptr;
  c->plan_wide = plan->nwide;
  plan->wide = wide + 1;
  plan->rptr = rptr;
  plan->kd = kd;
  plan->kd8 = kd8;
  plan->kd8h = kd8h;
  plan->su = su;
  plan->n = n;
  plan->nnz = nnz;
  plan->nslices = nslices;
  plan->slots = slots;
  plan->off = off;
  plan->width = width;
  plan->idx = sidx;
  plan->perm = sperm;
  return DCU_OK;
}

// SELL-32 of the operator whose CSR is (rptr, rcol) as given, slot -> entry
// position identity.  A CSC matrix read as CSR is its transpose, so
// sell_plan_rows(A.ptr, A.idx) lays out A^T (and M^T, same pattern) for the
// adjoint solve without any transpose.
int sell_plan_rows(Ctx* c, int n, int nnz, const int* rptr, const int* rcol, SellPlan* plan) {
  DCU_TRY(ensure(c, B_RPERM, sizeof(int) * (size_t)(nnz > 0 ? nnz : 1)));
  int* rperm = bp<int>(c, B_RPERM);
  if (nnz > 0) {
    k_iota<<<waves_grid(c, nnz, 256, 8), 256, 0, c->stream>>>(rperm, nnz);
    DCU_LAUNCHED(c, "k_iota");
  }
  return sell_fill_from_csr(c, n, nnz, rptr, rcol, rperm, plan);
}

int plan_stats(Ctx* c, long long* slots, long long* uniform_slots, long long* wide_slices) {
  if (!c->buf[B_PLANSTAT].p) return fail(c, DCU_ERR_ARG, "no SELL plan has been built on this context");
  unsigned long long h[2] = {0, 0};
  DCU_CUDA(c, cudaMemcpyAsync(h, c->buf[B_PLANSTAT].p, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  DCU_CUDA(c, cudaStreamSynchronize(c->stream));
  if (slots) *slots = (long long)h[0];
  if (uniform_slots) *uniform_slots = (long long)h[1];
  if (wide_slices) *wide_slices = c->plan_wide;
  return DCU_OK;
}

int sell_gather_f64(Ctx* c, const SellPlan& p, const double* src, double* dst) { return sell_gather<double>(c, p, src, dst); }
int sell_gather_a(Ctx* c, const SellPlan& p, const double* src, double* dst, float* dst32, int* inexact) {
  DCU_CUDA(c, cudaMemsetAsync(inexact, 0, sizeof(int), c->stream));
  int grid = waves_grid(c, p.slots, 256, 8);
  k_sell_gather_a<<<grid, 256, 0, c->stream>>>(p.perm, p.slots, src, dst32, inexact);
  DCU_LAUNCHED(c, "k_sell_gather_a");
  k_sell_gather_a64<<<grid, 256, 0, c->stream>>>(p.perm, p.slots, src, dst, inexact, p.nwide > 0 ? 1 : 0);
  DCU_LAUNCHED(c, "k_sell_gather_a64");
  return DCU_OK;
}
int sell_gather_f32(Ctx* c, const SellPlan& p, const double* src, float* dst) { return sell_gather<float>(c, p, src, dst); }
int sell_gather_bf16(Ctx* c, const SellPlan& p, const double* src, __nv_bfloat16* dst) {
  return sell_gather<__nv_bfloat16>(c, p, src, dst);
}

namespace {

// kNarrow values of one row, stored with one (BF16: 16 bytes) or two (FP32:
// 2 x 16 bytes) vector stores.
__device__ __forceinline__ void store_row8(__nv_bfloat16* p, const double (&v)[kNarrow]) {
  __nv_bfloat162 h[kNarrow / 2];
#pragma unroll
  for (int k = 0; k < kNarrow / 2; ++k) h[k] = __halves2bfloat162(__double2bfloat16(v[2 * k]), __double2bfloat16(v[2 * k + 1]));
  *reinterpret_cast<uint4*>(p) = *reinterpret_cast<const uint4*>(h);
}
__device__ __forceinline__ void store_row8(float* p, const double (&v)[kNarrow]) {
  reinterpret_cast<float4*>(p)[0] = make_float4((float)v[0], (float)v[1], (float)v[2], (float)v[3]);
  reinterpret_cast<float4*>(p)[1] = make_float4((float)v[4], (float)v[5], (float)v[6], (float)v[7]);
}

// One thread per row of the layout: a narrow slice's row goes to dst8 (its
// kNarrow values, zeros past the width), any other row to its SELL slots.
template <typename T>
__global__ void k_sell_gather_m8(const long long* __restrict__ off, const int* __restrict__ su,
                                 const int* __restrict__ sperm, int nslices, const double* __restrict__ src,
                                 T* __restrict__ dst, T* __restrict__ dst8) {
  const int rows_total = nslices * 32;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows_total; r += gridDim.x * blockDim.x) {
    const int s = r >> 5, lane = r & 31;
    const long long o0 = off[s];
    const int w = (int)((off[s + 1] - o0) >> 5);
    const long long base = o0 + lane;
    if (su[s] & 2) {
      double v[kNarrow];
#pragma unroll
      for (int k = 0; k < kNarrow; ++k) {
        const int p = (k < w) ? sperm[base + 32ll * k] : -1;
        v[k] = p >= 0 ? src[p] : 0.0;
      }
      store_row8(dst8 + (long long)r * kNarrow, v);
    } else {
      for (int k = 0; k < w; ++k) {
        const long long q = base + 32ll * k;
        const int p = sperm[q];
        dst[q] = cvt_from_double<T>(p >= 0 ? src[p] : 0.0);
      }
    }
  }
}

template <typename T>
int sell_gather_m8(Ctx* c, const SellPlan& p, const double* src, T* dst, T* dst8) {
  k_sell_gather_m8<T><<<waves_grid(c, (long long)p.nslices * 32, 256, 8), 256, 0, c->stream>>>(
      p.off, p.su, p.perm, p.nslices, src, dst, dst8);
  DCU_LAUNCHED(c, "k_sell_gather_m8");
  return DCU_OK;
}

}  // namespace

int sell_gather_m8_f32(Ctx* c, const SellPlan& p, const double* src, float* dst, float* dst8) {
  return sell_gather_m8<float>(c, p, src, dst, dst8);
}
int sell_gather_m8_bf16(Ctx* c, const SellPlan& p, const double* src, __nv_bfloat16* dst, __nv_bfloat16* dst8) {
  return sell_gather_m8<__nv_bfloat16>(c, p, src, dst, dst8);
}

// CSR with values, for the C ABI (dcu_csc_to_csr_d).
int csr_values(Ctx* c, int nnz, const int* rperm, const double* val, double* rval) {
  if (nnz <= 0 || !rval) return DCU_OK;
  k_gather_f64<<<waves_grid(c, nnz, 256, 8), 256, 0, c->stream>>>(rperm, val, nnz, rval);
  DCU_LAUNCHED(c, "k_gather_f64");
  return DCU_OK;
}

// ---------------------------------------------------------------------------
// CSC -> CSR without any device allocation (dcu_csc_to_csr_noalloc_d).
//
// For callers that must not allocate device memory: code that runs inside a
// framework whose memory pool owns the device (an out-of-band cudaMalloc
// fragments or exceeds its budget), or a latency-critical path that cannot
// afford cudaMalloc/cudaFree and the device synchronisation cudaFree implies.
// The scratch of the conversion lives in one file-scope __device__ array of
// fixed size (every GPU that loads this library holds it until the process
// exits).  Limits: n <= kNoAllocMaxN, nnz <= kNoAllocMaxNnz, no row longer
// than kSmemSortMax entries.  Every call shares the array and finds the last
// call's contents, so the parts that must start at zero are cleared on each
// call; calls that overlap on the GPU (other streams, other host threads on
// the same device) race on it.
// ---------------------------------------------------------------------------
constexpr int kNoAllocMaxN = 131072;
constexpr int kNoAllocMaxNnz = 1048576;
constexpr size_t kNoAllocCnt = 0;                                             // int[n + 1]
constexpr size_t kNoAllocLong = kNoAllocCnt + sizeof(int) * (kNoAllocMaxN + 64);  // int[n + 2]
constexpr size_t kNoAllocPerm = kNoAllocLong + sizeof(int) * (kNoAllocMaxN + 64); // int[nnz]
constexpr size_t kNoAllocFlags = kNoAllocPerm + sizeof(int) * kNoAllocMaxNnz;    // int[8]
constexpr size_t kNoAllocBytes = kNoAllocFlags + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

namespace {

// Exclusive scan of n <= kNoAllocMaxN counts by one block of 1024 threads
// (each thread scans a contiguous chunk, then the chunk totals are scanned).
constexpr int kSmallScanThreads = 1024;
__global__ void __launch_bounds__(kSmallScanThreads) k_scan_small(const int* __restrict__ in, int* __restrict__ out,
                                                                   int n) {
  __shared__ int tot[kSmallScanThreads];
  const int per = (n + kSmallScanThreads - 1) / kSmallScanThreads;
  const int b = threadIdx.x * per, e = min(n, b + per);
  int run = 0;
  for (int i = b; i < e; ++i) run += in[i];
  tot[threadIdx.x] = run;
  __syncthreads();
  for (int d = 1; d < kSmallScanThreads; d <<= 1) {
    const int v = (threadIdx.x >= d) ? tot[threadIdx.x - d] : 0;
    __syncthreads();
    tot[threadIdx.x] += v;
    __syncthreads();
  }
  int acc = tot[threadIdx.x] - run;
  for (int i = b; i < e; ++i) {
    out[i] = acc;
    acc += in[i];
  }
  if (threadIdx.x == kSmallScanThreads - 1) out[n] = tot[kSmallScanThreads - 1];
}

// Long rows (more than kThreadSortMax entries) by one block each, shared
// memory only; a row above kSmemSortMax entries sets flags[1] and is skipped.
__global__ void __launch_bounds__(512) k_row_sort_long_smem(const int* __restrict__ rptr, const int* __restrict__ rows,
                                                            const int* __restrict__ count, int* __restrict__ rcol,
                                                            int* __restrict__ rperm, int* __restrict__ flags) {
  extern __shared__ unsigned long long skey2[];
  const int nrows = *count;
  for (int q = blockIdx.x; q < nrows; q += gridDim.x) {
    const int r = rows[q];
    const int s0 = rptr[r], len = rptr[r + 1] - s0;
    if (len > kSmemSortMax) {
      if (threadIdx.x == 0) atomicOr(&flags[1], 1);
      continue;
    }
    int np2 = 1;
    while (np2 < len) np2 <<= 1;
    for (int i = threadIdx.x; i < np2; i += blockDim.x)
      skey2[i] = (i < len) ? ((unsigned long long)(unsigned)rcol[s0 + i] << 32 | (unsigned)rperm[s0 + i]) : ~0ull;
    __syncthreads();
    bitonic_block(skey2, np2);
    for (int i = threadIdx.x; i < len; i += blockDim.x) {
      rcol[s0 + i] = (int)(skey2[i] >> 32);
      rperm[s0 + i] = (int)(skey2[i] & 0xffffffffu);
    }
    __syncthreads();
  }
}

// Device address of g_noalloc_scratch on the current device, looked up on
// every call: the lookup is a host-side table read, and a cached address
// would go stale if the device's context were reset and the module reloaded.
void* noalloc_scratch_address(cudaError_t* err) {
  void* p = nullptr;
  *err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  return *err == cudaSuccess ? p : nullptr;
}

}  // namespace
}  // namespace dcu

extern "C" int dcu_csc_to_csr_noalloc_d(int n, int nnz, const int* ptr, const int* idx, const double* val, int* rptr,
                                        int* ridx, double* rval, void* stream_ptr) {
  using namespace dcu;
  if (n <= 0 || nnz < 0 || !ptr || !rptr || (nnz > 0 && (!idx || !ridx))) return DCU_ERR_ARG;
  if (n > kNoAllocMaxN || nnz > kNoAllocMaxNnz) return DCU_ERR_LIMIT;
  cudaStream_t st = (cudaStream_t)stream_ptr;
  // The call synchronises the stream and reads flags back to the host, which
  // a stream under capture does not allow: refuse it before touching it.
  cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &capture) != cudaSuccess) {
    cudaGetLastError();
    return DCU_ERR_ARG;
  }
  if (capture != cudaStreamCaptureStatusNone) return DCU_ERR_ARG;
  cudaError_t e = cudaSuccess;
  char* base = static_cast<char*>(noalloc_scratch_address(&e));
  if (!base) {
    cudaGetLastError();
    return e == cudaErrorNoDevice || e == cudaErrorInvalidDevice ? DCU_ERR_NO_DEVICE : DCU_ERR_CUDA;
  }
  int* cnt = reinterpret_cast<int*>(base + kNoAllocCnt);
  int* longrows = reinterpret_cast<int*>(base + kNoAllocLong);
  int* longcount = longrows + n;  // [0] count, [1] longest
  int* perm = reinterpret_cast<int*>(base + kNoAllocPerm);
  int* flags = reinterpret_cast<int*>(base + kNoAllocFlags);  // [0] malformed input, [1] row too long
  const int grid_n = (n + 255) / 256 < 1184 ? (n + 255) / 256 : 1184;
  const int grid_z = (nnz + 255) / 256 < 1184 ? ((nnz + 255) / 256 > 0 ? (nnz + 255) / 256 : 1) : 1184;
  int host_flags[2] = {0, 0};
#define NOALLOC_CHECK(call)                    \
  do {                                         \
    if ((call) != cudaSuccess) {               \
      cudaGetLastError();                      \
      return DCU_ERR_CUDA;                     \
    }                                          \
  } while (0)
  // what must start at zero: the row counts, the long-row counters, the flags
  NOALLOC_CHECK(cudaMemsetAsync(cnt, 0, sizeof(int) * (size_t)(n + 1), st));
  NOALLOC_CHECK(cudaMemsetAsync(longcount, 0, 2 * sizeof(int), st));
  NOALLOC_CHECK(cudaMemsetAsync(flags, 0, 8 * sizeof(int), st));
  k_validate_csc<<<grid_n > grid_z ? grid_n : grid_z, 256, 0, st>>>(ptr, idx, n, nnz, flags);
  NOALLOC_CHECK(cudaGetLastError());
  NOALLOC_CHECK(cudaMemcpyAsync(host_flags, flags, sizeof(int), cudaMemcpyDeviceToHost, st));
  NOALLOC_CHECK(cudaStreamSynchronize(st));
  // bits 1-8: malformed ptr / idx; the conversion accepts unsorted columns
  // and repeated rows (bits 16 and 32 of the shared check)
  if (host_flags[0] & 15) return DCU_ERR_ARG;
  if (nnz > 0) {
    k_row_count<<<grid_z, 256, 0, st>>>(idx, nnz, cnt);
    NOALLOC_CHECK(cudaGetLastError());
  }
  k_scan_small<<<1, kSmallScanThreads, 0, st>>>(cnt, rptr, n);
  NOALLOC_CHECK(cudaGetLastError());
  NOALLOC_CHECK(cudaMemsetAsync(cnt, 0, sizeof(int) * (size_t)(n + 1), st));
  k_row_scatter<<<grid_n, 256, 0, st>>>(ptr, idx, n, rptr, cnt, ridx, perm);
  NOALLOC_CHECK(cudaGetLastError());
  k_row_sort_short<<<grid_n, 256, 0, st>>>(rptr, n, ridx, perm, longrows, longcount);
  NOALLOC_CHECK(cudaGetLastError());
  const size_t smem = sizeof(unsigned long long) * kSmemSortMax;
  NOALLOC_CHECK(cudaFuncSetAttribute(k_row_sort_long_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_row_sort_long_smem<<<148, 512, smem, st>>>(rptr, longrows, longcount, ridx, perm, flags);
  NOALLOC_CHECK(cudaGetLastError());
  if (val && rval && nnz > 0) {
    k_gather_f64<<<grid_z, 256, 0, st>>>(perm, val, nnz, rval);
    NOALLOC_CHECK(cudaGetLastError());
  }
  NOALLOC_CHECK(cudaMemcpyAsync(host_flags, flags, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
  NOALLOC_CHECK(cudaStreamSynchronize(st));
#undef NOALLOC_CHECK
  return host_flags[1] ? DCU_ERR_LIMIT : DCU_OK;
}
