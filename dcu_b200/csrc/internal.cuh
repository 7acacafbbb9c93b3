// Internal declarations of libdcu_spai (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <functional>
#include <string>
#include <type_traits>
#include <vector>

#include "dcu_spai.h"

namespace dcu {

// ---------------------------------------------------------------------------
// Device buffer owned by the context; grows on demand, never shrinks.
// ---------------------------------------------------------------------------
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

enum BufId {
  B_STATS = 0,     // int stats of the SPAI build
  B_BIGLIST,       // columns for the CTA kernel
  B_CHUNKS,        // dynamic-schedule chunk bounds
  B_SLAB_A,        // CTA kernel dense least-squares slabs
  B_SLAB_BITS,     // CTA kernel bitmap / prefix slabs
  B_MVAL,          // internal FP64 M when the caller passes none
  B_ROWCNT,        // CSR row counts / fill cursors
  B_RPTR,          // CSR row pointers
  B_RCOL,          // CSR column indices
  B_RPERM,         // CSR -> CSC position
  B_LONGROWS,      // rows too long for the thread sort
  B_SCAN,          // scan block sums
  B_SELL_OFF,      // SELL slice offsets (int64)
  B_SELL_W,        // SELL slice widths
  B_SELL_IDX,      // SELL absolute column indices
  B_SELL_DEL,      // SELL 16-bit column deltas
  B_SELL_PERM,     // SELL slot -> CSC position (-1 padding)
  B_SELL_KD,       // SELL per (slice, k) column-offset descriptors
  B_SELL_AVAL,     // A values in SELL order (FP64)
  B_SELL_MVAL,     // M values in SELL order (FP64 / FP32 / BF16)
  B_VEC,           // solver vectors
  B_PART,          // per-block partial sums
  B_SCAL,          // solver scalars
  B_UPLOAD,        // host-API uploads
  B_SORTTMP,       // global scratch of the long-row sort
  B_FBLIST,        // columns handed from the thread kernel to the group kernel
  B_PLANSTAT,      // slots of the last SELL plan in offset-uniform slices
  B_HUBPOOL,       // slabs of the columns factored by the hub kernels
  B_HUBMETA,       // their descriptors
  B_HUBWPRE,       // prefix of their widths (warp -> column map)
  B_SELL_WIDE,     // SELL: count and list of the slices wider than kWideSlice
  B_WIDEVAL,       // solver: row values of those slices, from the wide pre-pass
  B_SELL_KD8,      // SELL: per narrow slice, its (up to 8) column offsets (int32, then int16)
  B_SELL_MVAL8,    // M values (FP32 / BF16) of the narrow slices, 8 per row, row-major
  B_SELL_AVAL32,   // A values in SELL order, FP32 copy (used when every value is exact in FP32)
  B_SELL_AFLAG,    // int: nonzero when some A value is not exactly an FP32 number
  B_COUNT
};

// An instantiated CUDA graph and the buffers/sizes it was captured with.
// Appends the bytes of a trivially copyable value (zero-filled first, so
// padding compares equal) to a graph-cache key.  Keying a graph on the whole
// argument struct its kernels captured means any changed pointer, size or
// scalar gives a new graph: a reallocated buffer never reaches a stale one.
template <typename T>
void key_append(std::vector<const void*>& key, const T& v) {
  static_assert(std::is_trivially_copyable<T>::value, "graph keys copy bytes");
  uintptr_t w[(sizeof(T) + sizeof(uintptr_t) - 1) / sizeof(uintptr_t)] = {};
  std::memcpy(w, &v, sizeof(T));
  for (uintptr_t u : w) key.push_back(reinterpret_cast<const void*>(u));
}

struct GraphSlot {
  std::vector<const void*> key;
  cudaGraphExec_t exec = nullptr;
  int nodes = 0;
};

struct Ctx {
  int device = 0;
  int sms = 0;
  int units = 0;
  bool units_user = false;  // units given by the caller (else the kernels' own worker counts)
  int max_threads_sm = 2048;
  size_t smem_optin = 0;
  cudaStream_t stream = nullptr;       // the context's own non-blocking stream
  cudaStream_t copy_stream = nullptr;  // host-API uploads that overlap work on `stream`
  cudaStream_t aux_stream = nullptr;   // a whole solve's SELL plan and A gather, beside the build
  cudaStream_t user_stream = nullptr;  // caller's stream to order against (optional)
  cudaEvent_t ev_sync = nullptr;       // ordering between user_stream and stream
  std::string err;
  long long launches = 0;
  DevBuf buf[B_COUNT];
  void* pinned = nullptr;   // small pinned host scratch (flags, stats), kPinnedBytes
  // ev[0..1]: timing of one call's device work; ev[2..3]: the solver's
  // stop-flag polling; ev[4..5]: the build inside a whole solve, read only
  // after the solve's own final synchronisation; ev[6..7]: ordering of the
  // auxiliary stream (start after validation, join before M's gather)
  cudaEvent_t ev[8] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  std::vector<GraphSlot> graphs;  // BiCGSTAB iteration graphs (bounded cache)
  // launch configuration per precision form (dcu_set_tuning / dcu_autotune_d)
  dcu_tuning tune[5];
  bool tune_set[5] = {false, false, false, false, false};
  // launches iteration kernel `kind` (IterKernel) of the last solve on its
  // buffers with grid selector `sel`, the solver's stop flag cleared first
  // (diagnostic timing and the autotuner only)
  std::function<int(int kind, int sel)> profile_launch;
  std::function<int(int kind, int sel)> profile_grid;  // the grid that launch uses
  std::vector<int> profile_order;  // kinds in the last solve's launch order
  std::vector<int> profile_sel;    // and the grid selector each ran with
  bool profile_k1_free = false;    // fused and split first steps compute the same values
  int profile_default_split = 0;   // the form's default first step
  int plan_wide = 0;               // slices of the last SELL plan wider than kWideSlice
  bool wide_prepass = true;        // flag wide slices for the pre-pass (dcu_set_wide_prepass)
  bool exact_a32 = true;           // A read from its FP32 copy when exact (dcu_set_exact_a32)
};

// Iteration kernels of BiCGSTAB, for profiling and the autotuner.
enum IterKernel { IK_P = 0, IK_Y, IK_PY, IK_AY, IK_SZ, IK_AZ, IK_XR, IK_COUNT };

constexpr size_t kPinnedBytes = 4096;

// Error helpers: record the message in the context and return a status.
int fail(Ctx* c, int code, const char* fmt, ...);
int cuda_fail(Ctx* c, cudaError_t e, const char* what, const char* file, int line);

#define DCU_CUDA(ctx, call)                                                   \
  do {                                                                        \
    cudaError_t e_ = (call);                                                  \
    if (e_ != cudaSuccess) return ::dcu::cuda_fail(ctx, e_, #call, __FILE__, __LINE__); \
  } while (0)

#define DCU_LAUNCHED(ctx, name)                                               \
  do {                                                                        \
    (ctx)->launches++;                                                        \
    cudaError_t e_ = cudaGetLastError();                                      \
    if (e_ != cudaSuccess) return ::dcu::cuda_fail(ctx, e_, name, __FILE__, __LINE__); \
  } while (0)

#define DCU_TRY(expr)                                                         \
  do {                                                                        \
    int s_ = (expr);                                                          \
    if (s_ != DCU_OK) return s_;                                              \
  } while (0)

// Ensure buffer `id` holds at least `bytes`; contents are not preserved.
int ensure(Ctx* c, BufId id, size_t bytes);
template <typename T>
inline T* bp(Ctx* c, BufId id) { return reinterpret_cast<T*>(c->buf[id].p); }

// Exclusive scan of int32 counts into int32 (or int64) offsets; out[n] = total.
int scan_exclusive_i32(Ctx* c, const int* in, int* out, int n);
int scan_exclusive_i64(Ctx* c, const int* in, long long* out, int n);

// ---------------------------------------------------------------------------
// Sparse pattern analysis of A (CSC): CSR transpose and SELL-32 layout.
// ---------------------------------------------------------------------------
// A full slice wider than kWideSlice slots because of at most kWideRows long
// rows (a long row sharing its slice with short ones) is summed by a warp-
// cooperative pre-pass in the solver.  Slices where more rows are that long
// keep the per-lane loop, which serves them better.
constexpr int kWideSlice = 16;
constexpr int kWideRows = 4;
// Offset-uniform slices at most this wide are "narrow" (every slice of a 5-
// or 7-point stencil): their offsets are kept per slice (SellPlan::kd8) and,
// for an FP32 / BF16 M, their values row-major, kNarrow per row, so one
// vector load brings a row's values.
constexpr int kNarrow = 8;

struct SellPlan {
  int n = 0, nnz = 0;
  int nslices = 0;
  long long slots = 0;
  bool delta16 = false;   // every |col - row| < 32768
  const long long* off = nullptr;
  const int* width = nullptr;
  const int* idx = nullptr;
  const int16_t* del = nullptr;
  const int* perm = nullptr;
  // One int per (slice, k), at kd[off[s] / 32 + k]: (d << 1) | 1 when every
  // row of the slice has its k-th entry at column row + d, else 0.  A warp
  // then forms the column from the row and skips the per-slot index load.
  const int* kd = nullptr;
  // Per slice: bit 0 when every kd of the slice is uniform; bit 1 when, in
  // addition, the slice is at most kNarrow slots wide ("narrow"), with its
  // width in bits 3-6; bit 2 when the slice is full, wider than kWideSlice and
  // has at most kWideRows rows longer than that, with its index in `wide` in
  // the bits above bit 2.
  const int* su = nullptr;
  // kNarrow ints per slice: kd8[kNarrow s + k] = the column offset of entry
  // position k of a narrow slice (0 past its width).  Indexed by the slice
  // alone, so a row's offsets load together with its slice's flags instead
  // of after its slot offset.
  const int* kd8 = nullptr;
  // the same offsets as int16 (one 16-byte load per slice) when delta16
  const int16_t* kd8h = nullptr;
  const int* rptr = nullptr;  // CSR row pointers of the laid-out operator (row lengths)
  const int* wide = nullptr;  // the slices flagged wide (device)
  int nwide = 0;
};

// Slot counts of the last SELL plan built on a context (diagnostics).
int plan_stats(Ctx* c, long long* slots, long long* uniform_slots, long long* wide_slices);

// Fails with DCU_ERR_ARG unless ptr[0] = 0, ptr is non-decreasing,
// ptr[n] = nnz and every row index lies in [0, n).  Every entry point runs it
// before the first kernel that follows the indices.
// Structural check of a CSC matrix (status DCU_ERR_ARG with a message when it
// fails).  unique_rows also refuses a row index repeated inside one column:
// every SPAI and solver entry point needs distinct (row, column) pairs.
int validate_csc(Ctx* c, int n, int nnz, const int* ptr, const int* idx, bool unique_rows = true);
int csr_from_csc(Ctx* c, int n, int nnz, const int* ptr, const int* idx, int* rptr, int* rcol,
                 int* rperm);
int csr_values(Ctx* c, int nnz, const int* rperm, const double* val, double* rval);
int sell_plan(Ctx* c, int n, int nnz, const int* ptr, const int* idx, SellPlan* plan);
// SELL-32 layout of the operator whose CSR is (rptr, rcol, rperm).  With
// `check` (a device int), its value is read back with the layout's last
// round trip into *check_out.
int sell_fill_from_csr(Ctx* c, int n, int nnz, const int* rptr, const int* rcol, const int* rperm, SellPlan* plan,
                       const int* check = nullptr, int* check_out = nullptr);
int sell_plan_rows(Ctx* c, int n, int nnz, const int* rptr, const int* rcol, SellPlan* plan);
// out[e] = alpha * u[idx[e]] * v[col(e)] on a CSC pattern
int sampled_outer(Ctx* c, int n, const int* ptr, const int* idx, const double* u, const double* v, double alpha,
                  double* out);
// dst[slot] = (perm[slot] >= 0) ? src[perm[slot]] : 0, converted to the element type.
int sell_gather_f64(Ctx* c, const SellPlan& p, const double* src, double* dst);
// A's values in SELL order as an FP32 copy (dst32); *inexact (zeroed here)
// becomes nonzero when some value is not exactly an FP32 number, and only
// then, or when the plan has wide slices, is the FP64 copy (dst) written.
int sell_gather_a(Ctx* c, const SellPlan& p, const double* src, double* dst, float* dst32, int* inexact);
int sell_gather_f32(Ctx* c, const SellPlan& p, const double* src, float* dst);
int sell_gather_bf16(Ctx* c, const SellPlan& p, const double* src, __nv_bfloat16* dst);
// An FP32 / BF16 M for the solver: the values of the narrow slices row-major,
// kNarrow per row (dst8, nslices * 32 * kNarrow), the other slices' values in
// SELL order (dst, slots).
int sell_gather_m8_f32(Ctx* c, const SellPlan& p, const double* src, float* dst, float* dst8);
int sell_gather_m8_bf16(Ctx* c, const SellPlan& p, const double* src, __nv_bfloat16* dst, __nv_bfloat16* dst8);

// ---------------------------------------------------------------------------
// SPAI build and pattern.
// ---------------------------------------------------------------------------
// A SPAI build split in two (spai_build = launch + finish): the launch
// enqueues the first column kernel on c->stream and returns without waiting;
// the finish completes the build (host round trips, further kernels) and
// fills info.  Work on other streams may run between the two.
struct BuildJobImpl;  // the prepared launch arguments (spai_build.cu)
struct BuildJob {
  dcu_options opt{};
  int n = 0;
  const int* ptr = nullptr;
  const int* idx = nullptr;
  const double* val = nullptr;
  double* mval = nullptr;
  double* colres = nullptr;
  bool empty = false;
  bool thread_path = false;
  int max_ni = 0, cta_max_area = 0;
  int* fb_list = nullptr;
  bool finish_launched = false;  // the finish enqueued kernels of its own
  BuildJobImpl* impl;
  BuildJob();
  ~BuildJob();
  BuildJob(const BuildJob&) = delete;
  BuildJob& operator=(const BuildJob&) = delete;
};
int spai_build_launch(Ctx* c, int n, int nnz, const int* ptr, const int* idx, const double* val,
                      const dcu_options* opt, double* mval, double* colres, BuildJob* job);
int spai_build_finish(Ctx* c, BuildJob* job, dcu_build_info* info);
int spai_build(Ctx* c, int n, int nnz, const int* ptr, const int* idx, const double* val,
               const dcu_options* opt, double* mval, double* colres, dcu_build_info* info);
// Work units of the static schedule when the caller names none: one per
// resident warp of the column kernel.
int spai_default_units(Ctx* c);
int spai_pattern(Ctx* c, int n, const int* ptr, const int* idx, int col_start, int col_end,
                 int* icount, long long* iptr, int* ilist, long long cap, long long* total);

// ---------------------------------------------------------------------------
// BiCGSTAB on the SELL plan.
// ---------------------------------------------------------------------------
// A's values in SELL order: FP64 (v64), and an FP32 copy (v32, or NULL) that
// the A products read instead when the device flag *inexact is zero.  The
// FP32 copy then holds the same numbers, so the iterates are bit-identical;
// v64 is then written only for a plan with wide slices (whose pre-pass reads
// it).
struct SellA {
  const double* v64 = nullptr;
  const float* v32 = nullptr;
  const int* inexact = nullptr;
};
// mval8_sell: an FP32 / BF16 M's narrow-slice values (sell_gather_m8_*), or
// NULL (every slice then read from mval_sell).
int bicgstab_solve(Ctx* c, const SellPlan& plan, const SellA& aval_sell, const void* mval_sell,
                   const double* b, double* x, const dcu_options* opt, dcu_solve_info* info,
                   const void* mval8_sell = nullptr);
void release_graphs(Ctx* c);

// Batched systems (diagonal blocks [sys_off[s], sys_off[s+1]) of one matrix).
int check_blocks(Ctx* c, int n, const int* ptr, const int* idx, int nsys, const int* sys_off);
int batch_solve(Ctx* c, int nsys, const int* sys_off, const SellPlan& plan, const double* aval, const double* mval,
                int nrhs, const double* B, double* X, const dcu_options* opt, int* iters, int* status,
                dcu_solve_info* info);
int profile_iteration(Ctx* c, int reps, float* ms, int cap, int* count);
// Times the grid selectors of the kernels without a reduction (and the fused
// against the split first step where both compute the same values) on the
// last solve's buffers; writes the fastest into t's iteration fields and the
// report's iteration times.
int tune_iteration(Ctx* c, int reps, dcu_tuning* t, int* timed);

// grid size for grid-stride kernels: whole waves of `per_sm` blocks
inline int waves_grid(const Ctx* c, long long work_items, int block, int per_sm) {
  long long need = (work_items + block - 1) / block;
  long long cap = (long long)c->sms * per_sm;
  if (need < 1) need = 1;
  return (int)(need < cap ? need : cap);
}

}  // namespace dcu

struct dcu_spai_ctx : public dcu::Ctx {};
