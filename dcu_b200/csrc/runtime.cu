// Context, buffers, error reporting and the device prefix scan.
#include <cstdarg>

#include "internal.cuh"

namespace dcu {

int fail(Ctx* c, int code, const char* fmt, ...) {
  char msg[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(msg, sizeof msg, fmt, ap);
  va_end(ap);
  if (c) c->err = msg;
  return code;
}

int cuda_fail(Ctx* c, cudaError_t e, const char* what, const char* file, int line) {
  const char* base = strrchr(file, '/');
  return fail(c, e == cudaErrorMemoryAllocation ? DCU_ERR_ALLOC : DCU_ERR_CUDA, "%s failed: %s (%s:%d)",
              what, cudaGetErrorString(e), base ? base + 1 : file, line);
}

int ensure(Ctx* c, BufId id, size_t bytes) {
  DevBuf& b = c->buf[id];
  if (bytes == 0) bytes = 16;
  if (b.bytes >= bytes) return DCU_OK;
  if (b.p) {
    cudaError_t e = cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaFree", __FILE__, __LINE__);
  }
  size_t want = bytes + bytes / 8;  // headroom against repeated regrowth
  cudaError_t e = cudaMalloc(&b.p, want);
  if (e != cudaSuccess) {
    cudaGetLastError();
    e = cudaMalloc(&b.p, bytes);
    want = bytes;
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    b.p = nullptr;
    return fail(c, DCU_ERR_ALLOC, "cudaMalloc of %zu bytes failed (buffer %d)", bytes, (int)id);
  }
  b.bytes = want;
  return DCU_OK;
}

// ---------------------------------------------------------------------------
// Exclusive scan.  Each block scans 1024 elements (256 threads x 4), writes
// its total; totals are scanned recursively and added back.  Deterministic.
// ---------------------------------------------------------------------------
namespace {

constexpr int kScanThreads = 256;
constexpr int kScanPer = 4;
constexpr int kScanTile = kScanThreads * kScanPer;

template <typename TI, typename TO>
__global__ void __launch_bounds__(kScanThreads) k_scan_tile(const TI* __restrict__ in, TO* __restrict__ out,
                                                            long long* __restrict__ block_sums, int n) {
  __shared__ long long warp_tot[kScanThreads / 32];
  const int base = blockIdx.x * kScanTile + threadIdx.x * kScanPer;
  long long v[kScanPer];
  long long run = 0;
#pragma unroll
  for (int i = 0; i < kScanPer; ++i) {
    long long x = (base + i < n) ? (long long)in[base + i] : 0;
    v[i] = run;
    run += x;
  }
  // inclusive scan of per-thread totals within the warp
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  long long incl = run;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    long long t = __shfl_up_sync(0xffffffffu, incl, d);
    if (lane >= d) incl += t;
  }
  if (lane == 31) warp_tot[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    long long w = (lane < kScanThreads / 32) ? warp_tot[lane] : 0;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      long long t = __shfl_up_sync(0xffffffffu, w, d);
      if (lane >= d) w += t;
    }
    if (lane < kScanThreads / 32) warp_tot[lane] = w;  // inclusive
  }
  __syncthreads();
  long long excl = incl - run + (wid > 0 ? warp_tot[wid - 1] : 0);
#pragma unroll
  for (int i = 0; i < kScanPer; ++i)
    if (base + i < n) out[base + i] = (TO)(excl + v[i]);
  if (threadIdx.x == kScanThreads - 1 && block_sums) block_sums[blockIdx.x] = excl + run;
}

template <typename TO>
__global__ void k_scan_add(TO* __restrict__ out, const long long* __restrict__ offs, int n) {
  int i = blockIdx.x * kScanTile + threadIdx.x;
  long long o = offs[blockIdx.x];
#pragma unroll
  for (int r = 0; r < kScanPer; ++r, i += kScanThreads)
    if (i < n) out[i] = (TO)((long long)out[i] + o);
}

__global__ void k_write_total(const long long* __restrict__ tot, long long* __restrict__ dst) { *dst = *tot; }

// Scan of long long block sums in place, recursively.  `scratch` holds enough
// space for all levels.
int scan_ll_inplace(Ctx* c, long long* data, int n, long long* scratch, long long* total_out) {
  int nb = (n + kScanTile - 1) / kScanTile;
  if (nb <= 1) {
    k_scan_tile<long long, long long><<<1, kScanThreads, 0, c->stream>>>(data, data, total_out, n);
    DCU_LAUNCHED(c, "k_scan_tile");
    return DCU_OK;
  }
  long long* sums = scratch;
  k_scan_tile<long long, long long><<<nb, kScanThreads, 0, c->stream>>>(data, data, sums, n);
  DCU_LAUNCHED(c, "k_scan_tile");
  DCU_TRY(scan_ll_inplace(c, sums, nb, scratch + nb, total_out));
  k_scan_add<long long><<<nb, kScanThreads, 0, c->stream>>>(data, sums, n);
  DCU_LAUNCHED(c, "k_scan_add");
  return DCU_OK;
}

template <typename TO>
int scan_exclusive(Ctx* c, const int* in, TO* out, int n) {
  // out has n + 1 entries; the callers write out[n] = total
  int nb = (n + kScanTile - 1) / kScanTile;
  if (nb < 1) nb = 1;
  size_t need = sizeof(long long) * (size_t)(2 * nb + 64);
  DCU_TRY(ensure(c, B_SCAN, need));
  long long* sums = bp<long long>(c, B_SCAN);
  long long* total = sums + 2 * nb + 32;
  k_scan_tile<int, TO><<<nb, kScanThreads, 0, c->stream>>>(in, out, sums, n);
  DCU_LAUNCHED(c, "k_scan_tile");
  if (nb > 1) {
    DCU_TRY(scan_ll_inplace(c, sums, nb, sums + nb, total));
    k_scan_add<TO><<<nb, kScanThreads, 0, c->stream>>>(out, sums, n);
    DCU_LAUNCHED(c, "k_scan_add");
  } else {
    k_write_total<<<1, 1, 0, c->stream>>>(sums, total);
    DCU_LAUNCHED(c, "k_write_total");
  }
  return DCU_OK;
}

__global__ void k_ll_to_int(const long long* __restrict__ src, int* __restrict__ dst) { *dst = (int)*src; }

}  // namespace

int scan_exclusive_i64(Ctx* c, const int* in, long long* out, int n) {
  int nb = (n + kScanTile - 1) / kScanTile;
  if (nb < 1) nb = 1;
  DCU_TRY(scan_exclusive<long long>(c, in, out, n));
  long long* total = bp<long long>(c, B_SCAN) + 2 * nb + 32;
  k_write_total<<<1, 1, 0, c->stream>>>(total, out + n);
  DCU_LAUNCHED(c, "k_write_total");
  return DCU_OK;
}

int scan_exclusive_i32(Ctx* c, const int* in, int* out, int n) {
  int nb = (n + kScanTile - 1) / kScanTile;
  if (nb < 1) nb = 1;
  DCU_TRY(scan_exclusive<int>(c, in, out, n));
  long long* total = bp<long long>(c, B_SCAN) + 2 * nb + 32;
  k_ll_to_int<<<1, 1, 0, c->stream>>>(total, out + n);
  DCU_LAUNCHED(c, "k_ll_to_int");
  return DCU_OK;
}

}  // namespace dcu
