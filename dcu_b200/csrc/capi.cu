// The extern "C" entry points declared in include/dcu_spai.h.
#include <new>

#include "internal.cuh"

using dcu::Ctx;

namespace {

// Order the context's stream after the caller's stream (entry) and the
// caller's stream after the context's (exit).
struct StreamScope {
  Ctx* c;
  explicit StreamScope(Ctx* ctx) : c(ctx) {
    cudaSetDevice(c->device);
    if (c->user_stream) {
      cudaEventRecord(c->ev_sync, c->user_stream);
      cudaStreamWaitEvent(c->stream, c->ev_sync, 0);
    }
  }
  ~StreamScope() {
    if (c->user_stream) {
      cudaEventRecord(c->ev_sync, c->stream);
      cudaStreamWaitEvent(c->user_stream, c->ev_sync, 0);
    }
  }
};

constexpr int kMaxN = (1 << 26) - 2;  // row indices must fit the 26-bit sort keys

int check_matrix(Ctx* c, int n, int nnz, const void* ptr, const void* idx, const void* val) {
  if (!c) return DCU_ERR_ARG;
  if (n <= 0) return dcu::fail(c, DCU_ERR_ARG, "n must be positive (got %d)", n);
  if (n > kMaxN) return dcu::fail(c, DCU_ERR_LIMIT, "n = %d exceeds the supported %d", n, kMaxN);
  if (nnz < 0) return dcu::fail(c, DCU_ERR_ARG, "nnz must be >= 0 (got %d)", nnz);
  if (!ptr || (nnz > 0 && (!idx || !val))) return dcu::fail(c, DCU_ERR_ARG, "null matrix pointer");
  return DCU_OK;
}

int resolve_range(Ctx* c, int n, const dcu_options* in, dcu_options* out) {
  dcu_options_default(out);
  if (in) *out = *in;
  if (out->col_end <= 0) out->col_end = n;
  if (out->col_start < 0 || out->col_end > n || out->col_start > out->col_end)
    return dcu::fail(c, DCU_ERR_ARG, "invalid column range [%d, %d) for n = %d", out->col_start, out->col_end, n);
  if (out->schedule != DCU_SCHED_BALANCED_COLUMNS && out->schedule != DCU_SCHED_BALANCED_NNZ)
    return dcu::fail(c, DCU_ERR_ARG, "unknown schedule %d", out->schedule);
  if (out->precision < DCU_PREC_FP64 || out->precision > DCU_PREC_M_BF16)
    return dcu::fail(c, DCU_ERR_ARG, "unknown precision %d", out->precision);
  if (out->tol_mode != DCU_TOL_ABS && out->tol_mode != DCU_TOL_REL)
    return dcu::fail(c, DCU_ERR_ARG, "unknown tolerance mode %d", out->tol_mode);
  if (!(out->tol >= 0.0)) return dcu::fail(c, DCU_ERR_ARG, "tol must be >= 0");
  if (out->ls_method < DCU_LS_AUTO || out->ls_method > DCU_LS_NORMAL_EQ)
    return dcu::fail(c, DCU_ERR_ARG, "unknown least-squares method %d", out->ls_method);
  return DCU_OK;
}

// A's values (FP64) and M's (by form) in SELL order.
int gather_values(Ctx* c, const dcu::SellPlan& pl, const double* val, const double* mval, int precision,
                  const void** msell) {
  const dcu::SellPlan* plan = &pl;
  const size_t slots = (size_t)(plan->slots > 0 ? plan->slots : 1);
  DCU_TRY(dcu::ensure(c, dcu::B_SELL_AVAL, sizeof(double) * slots));
  DCU_TRY(dcu::sell_gather_f64(c, *plan, val, dcu::bp<double>(c, dcu::B_SELL_AVAL)));
  if (precision == DCU_PREC_FP64) {
    DCU_TRY(dcu::ensure(c, dcu::B_SELL_MVAL, sizeof(double) * slots));
    DCU_TRY(dcu::sell_gather_f64(c, *plan, mval, dcu::bp<double>(c, dcu::B_SELL_MVAL)));
  } else if (precision == DCU_PREC_MIXED_FP32 || precision == DCU_PREC_M_FP32) {
    DCU_TRY(dcu::ensure(c, dcu::B_SELL_MVAL, sizeof(float) * slots));
    DCU_TRY(dcu::sell_gather_f32(c, *plan, mval, dcu::bp<float>(c, dcu::B_SELL_MVAL)));
  } else {
    DCU_TRY(dcu::ensure(c, dcu::B_SELL_MVAL, sizeof(__nv_bfloat16) * slots));
    DCU_TRY(dcu::sell_gather_bf16(c, *plan, mval, dcu::bp<__nv_bfloat16>(c, dcu::B_SELL_MVAL)));
  }
  *msell = c->buf[dcu::B_SELL_MVAL].p;
  return DCU_OK;
}

// Solver-side layout of A and M: SELL plan + values.
int prepare_solve(Ctx* c, int n, int nnz, const int* ptr, const int* idx, const double* val, const double* mval,
                  int precision, dcu::SellPlan* plan, const void** msell) {
  DCU_TRY(dcu::sell_plan(c, n, nnz, ptr, idx, plan));
  return gather_values(c, *plan, val, mval, precision, msell);
}

// The whole path on device arrays: validation, the SELL plan (pattern only),
// the SPAI build, A and M in SELL order, BiCGSTAB.  When the values or the
// vectors are still being copied in on the copy stream, val_ready / bx_ready
// (optional) are the events that mark their arrival: the plan is built while
// the values are in flight, and the build while b and x0 are.
int solve_pipeline(Ctx* c, int n, int nnz, const int* ptr, const int* idx, const double* val, const double* b,
                   double* x, const dcu_options& o, double* mval, dcu_build_info* binfo, dcu_solve_info* sinfo,
                   cudaEvent_t val_ready, cudaEvent_t bx_ready) {
  double* m = mval;
  if (!m) {
    DCU_TRY(dcu::ensure(c, dcu::B_MVAL, sizeof(double) * (size_t)(nnz > 0 ? nnz : 1)));
    m = dcu::bp<double>(c, dcu::B_MVAL);
  }
  DCU_TRY(dcu::validate_csc(c, n, nnz, ptr, idx));
  dcu::SellPlan plan;
  DCU_TRY(dcu::sell_plan(c, n, nnz, ptr, idx, &plan));
  if (val_ready) DCU_CUDA(c, cudaStreamWaitEvent(c->stream, val_ready, 0));
  dcu_build_info bl{};
  DCU_CUDA(c, cudaEventRecord(c->ev[0], c->stream));
  DCU_TRY(dcu::spai_build(c, n, nnz, ptr, idx, val, &o, m, nullptr, &bl));
  DCU_CUDA(c, cudaEventRecord(c->ev[1], c->stream));
  DCU_CUDA(c, cudaEventSynchronize(c->ev[1]));
  cudaEventElapsedTime(&bl.ms, c->ev[0], c->ev[1]);
  if (binfo) *binfo = bl;
  const void* msell = nullptr;
  DCU_TRY(gather_values(c, plan, val, m, o.precision, &msell));
  if (bx_ready) DCU_CUDA(c, cudaStreamWaitEvent(c->stream, bx_ready, 0));
  return dcu::bicgstab_solve(c, plan, dcu::bp<double>(c, dcu::B_SELL_AVAL), msell, b, x, &o, sinfo);
}

// Host uploads share one buffer: ptr | idx | val | b | x | mval.
struct Uploads {
  int* ptr;
  int* idx;
  double* val;
  double* b;
  double* x;
  double* mval;
};

int upload(Ctx* c, int n, int nnz, const int* ptr, const int* idx, const double* val, const double* b,
           const double* x, bool want_mval, Uploads* u) {
  auto al = [](size_t v) { return (v + 255) & ~(size_t)255; };
  const size_t sp = al(sizeof(int) * (size_t)(n + 1)), si = al(sizeof(int) * (size_t)(nnz > 0 ? nnz : 1));
  const size_t sv = al(sizeof(double) * (size_t)(nnz > 0 ? nnz : 1)), sn = al(sizeof(double) * (size_t)n);
  DCU_TRY(dcu::ensure(c, dcu::B_UPLOAD, sp + si + 2 * sv + 2 * sn));
  char* base = dcu::bp<char>(c, dcu::B_UPLOAD);
  u->ptr = (int*)base;
  u->idx = (int*)(base + sp);
  u->val = (double*)(base + sp + si);
  u->b = (double*)(base + sp + si + sv);
  u->x = (double*)(base + sp + si + sv + sn);
  u->mval = want_mval ? (double*)(base + sp + si + sv + 2 * sn) : nullptr;
  DCU_CUDA(c, cudaMemcpyAsync(u->ptr, ptr, sizeof(int) * (size_t)(n + 1), cudaMemcpyHostToDevice, c->stream));
  if (nnz > 0) {
    DCU_CUDA(c, cudaMemcpyAsync(u->idx, idx, sizeof(int) * (size_t)nnz, cudaMemcpyHostToDevice, c->stream));
    DCU_CUDA(c, cudaMemcpyAsync(u->val, val, sizeof(double) * (size_t)nnz, cudaMemcpyHostToDevice, c->stream));
  }
  if (b) DCU_CUDA(c, cudaMemcpyAsync(u->b, b, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice, c->stream));
  if (x) DCU_CUDA(c, cudaMemcpyAsync(u->x, x, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice, c->stream));
  return DCU_OK;
}

}  // namespace

extern "C" {

void dcu_options_default(dcu_options* o) {
  if (!o) return;
  o->schedule = DCU_SCHED_BALANCED_COLUMNS;
  o->precision = DCU_PREC_FP64;
  o->tol_mode = DCU_TOL_REL;
  o->maxiter = 1000;
  o->tol = 1e-8;
  o->verify = 1;
  o->col_start = 0;
  o->col_end = 0;
  o->ls_method = DCU_LS_AUTO;
}

int dcu_spai_create(dcu_spai_ctx** out, int device, int units) {
  if (!out) return DCU_ERR_ARG;
  *out = nullptr;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count <= 0) {
    cudaGetLastError();
    return DCU_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= count) return DCU_ERR_NO_DEVICE;
  dcu_spai_ctx* c = new (std::nothrow) dcu_spai_ctx();
  if (!c) return DCU_ERR_ALLOC;
  c->device = device;
  int rc = DCU_OK;
  do {
    if ((e = cudaSetDevice(device)) != cudaSuccess) { rc = dcu::cuda_fail(c, e, "cudaSetDevice", __FILE__, __LINE__); break; }
    cudaDeviceProp prop;
    if ((e = cudaGetDeviceProperties(&prop, device)) != cudaSuccess) { rc = dcu::cuda_fail(c, e, "props", __FILE__, __LINE__); break; }
    c->sms = prop.multiProcessorCount;
    c->max_threads_sm = prop.maxThreadsPerMultiProcessor;
    c->smem_optin = prop.sharedMemPerBlockOptin;
    if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess) { rc = dcu::cuda_fail(c, e, "stream", __FILE__, __LINE__); break; }
    if ((e = cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking)) != cudaSuccess) { rc = dcu::cuda_fail(c, e, "copy stream", __FILE__, __LINE__); break; }
    if ((e = cudaMallocHost(&c->pinned, dcu::kPinnedBytes)) != cudaSuccess) { rc = dcu::cuda_fail(c, e, "cudaMallocHost", __FILE__, __LINE__); break; }
    for (int i = 0; i < 4 && e == cudaSuccess; ++i)
      e = cudaEventCreateWithFlags(&c->ev[i], i < 2 ? cudaEventDefault : cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_sync, cudaEventDisableTiming);
    if (e != cudaSuccess) { rc = dcu::cuda_fail(c, e, "events", __FILE__, __LINE__); break; }
  } while (0);
  if (rc != DCU_OK) {
    dcu_spai_destroy(c);
    return rc;
  }
  // the static schedule splits columns over `units` ranges; by default one
  // per resident warp of the column kernel
  c->units = units > 0 ? units : dcu::spai_default_units(c);
  c->units_user = units > 0;
  *out = c;
  return DCU_OK;
}

void dcu_spai_destroy(dcu_spai_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
  dcu::release_graphs(c);
  for (auto& b : c->buf)
    if (b.p) cudaFree(b.p);
  for (auto& e : c->ev)
    if (e) cudaEventDestroy(e);
  if (c->ev_sync) cudaEventDestroy(c->ev_sync);
  if (c->pinned) cudaFreeHost(c->pinned);
  if (c->stream) cudaStreamDestroy(c->stream);
  if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
  delete c;
}

const char* dcu_spai_last_error(const dcu_spai_ctx* c) { return c ? c->err.c_str() : "null context"; }

int dcu_spai_set_stream(dcu_spai_ctx* c, void* stream) {
  if (!c) return DCU_ERR_ARG;
  c->user_stream = (cudaStream_t)stream;
  return DCU_OK;
}

int dcu_spai_units(const dcu_spai_ctx* c) { return c ? c->units : 0; }

long long dcu_spai_launch_count(const dcu_spai_ctx* c) { return c ? c->launches : 0; }

int dcu_spai_distribute_columns(const int* ptr, int col_start, int col_end, int units, int schedule, int* starts,
                                int* ends) {
  // distributeColumns, src/spai_multi_dcu.cpp:1356-1449
  const int total = col_end - col_start;
  if (!ptr || !starts || !ends || units <= 0 || total <= 0) return DCU_ERR_ARG;
  if (schedule == DCU_SCHED_BALANCED_NNZ && ptr[col_end] - ptr[col_start] > 0) {
    const int target = (ptr[col_end] - ptr[col_start]) / units;
    int cur = 0;
    for (int u = 0; u < units; ++u) {
      starts[u] = col_start + cur;
      const int first = cur;
      int acc = 0;
      if (u == units - 1) {
        cur = total;
      } else {
        while (cur < total) {
          const int g = col_start + cur;
          const int cn = ptr[g + 1] - ptr[g];
          if (acc + cn > target && cur > first) break;
          acc += cn;
          ++cur;
        }
      }
      if (cur <= first) cur = (first + 1 <= total) ? first + 1 : total;
      ends[u] = col_start + cur;
    }
  } else {
    const int base = total / units, rem = total % units;
    int cur = 0;
    for (int u = 0; u < units; ++u) {
      starts[u] = col_start + cur;
      const int cnt = base + (u < rem ? 1 : 0);
      ends[u] = col_start + cur + cnt;
      cur += cnt;
    }
  }
  return DCU_OK;
}

int dcu_spai_pattern_d(dcu_spai_ctx* c, int n, const int* ptr, const int* idx, int col_start, int col_end,
                       int* icount, long long* iptr, int* ilist, long long cap, long long* total) {
  int rc = check_matrix(c, n, 1, ptr, idx, idx);
  if (rc) return rc;
  if (col_end <= 0) col_end = n;
  if (col_start < 0 || col_end > n || col_start > col_end || !icount || !iptr)
    return dcu::fail(c, DCU_ERR_ARG, "invalid pattern arguments");
  try {
    StreamScope scope(c);
    long long nnz = 0;
    DCU_CUDA(c, cudaMemcpy(&nnz, ptr + n, sizeof(int), cudaMemcpyDeviceToHost));
    DCU_TRY(dcu::validate_csc(c, n, (int)nnz, ptr, idx));
    return dcu::spai_pattern(c, n, ptr, idx, col_start, col_end, icount, iptr, ilist, cap, total);
  } catch (const std::bad_alloc&) {
    return dcu::fail(c, DCU_ERR_ALLOC, "host allocation failed");
  }
}

int dcu_spai_build_d(dcu_spai_ctx* c, int n, int nnz, const int* ptr, const int* idx, const double* val,
                     const dcu_options* opt, double* mval, double* colres, dcu_build_info* info) {
  int rc = check_matrix(c, n, nnz, ptr, idx, val);
  if (rc) return rc;
  if (!mval && nnz > 0) return dcu::fail(c, DCU_ERR_ARG, "mval is null");
  dcu_options o;
  if ((rc = resolve_range(c, n, opt, &o))) return rc;
  try {
    StreamScope scope(c);
    dcu_build_info local{};
    DCU_TRY(dcu::validate_csc(c, n, nnz, ptr, idx));
    DCU_CUDA(c, cudaEventRecord(c->ev[0], c->stream));
    DCU_TRY(dcu::spai_build(c, n, nnz, ptr, idx, val, &o, mval, colres, &local));
    DCU_CUDA(c, cudaEventRecord(c->ev[1], c->stream));
    DCU_CUDA(c, cudaEventSynchronize(c->ev[1]));
    cudaEventElapsedTime(&local.ms, c->ev[0], c->ev[1]);
    if (info) *info = local;
    return DCU_OK;
  } catch (const std::bad_alloc&) {
    return dcu::fail(c, DCU_ERR_ALLOC, "host allocation failed");
  }
}

int dcu_spai_build_h(dcu_spai_ctx* c, int n, int nnz, const int* ptr, const int* idx, const double* val,
                     const dcu_options* opt, double* mval, double* colres, dcu_build_info* info) {
  int rc = check_matrix(c, n, nnz, ptr, idx, val);
  if (rc) return rc;
  if (!mval && nnz > 0) return dcu::fail(c, DCU_ERR_ARG, "mval is null");
  dcu_options o;
  if ((rc = resolve_range(c, n, opt, &o))) return rc;
  StreamScope scope(c);
  Uploads u;
  DCU_TRY(upload(c, n, nnz, ptr, idx, val, nullptr, nullptr, true, &u));
  double* dres = nullptr;
  if (colres) dres = u.b;  // n doubles, unused by the build
  rc = dcu_spai_build_d(c, n, nnz, u.ptr, u.idx, u.val, &o, u.mval, dres, info);
  if (rc) return rc;
  if (nnz > 0)
    DCU_CUDA(c, cudaMemcpyAsync(mval, u.mval, sizeof(double) * (size_t)nnz, cudaMemcpyDeviceToHost, c->stream));
  if (colres)
    DCU_CUDA(c, cudaMemcpyAsync(colres, dres, sizeof(double) * (size_t)(o.col_end - o.col_start),
                                cudaMemcpyDeviceToHost, c->stream));
  DCU_CUDA(c, cudaStreamSynchronize(c->stream));
  return DCU_OK;
}

int dcu_csc_to_csr_d(dcu_spai_ctx* c, int n, int nnz, const int* ptr, const int* idx, const double* val, int* rptr,
                     int* ridx, double* rval) {
  int rc = check_matrix(c, n, nnz, ptr, idx, val ? (const void*)val : (const void*)idx);
  if (rc) return rc;
  if (!rptr || (nnz > 0 && !ridx)) return dcu::fail(c, DCU_ERR_ARG, "null CSR output");
  StreamScope scope(c);
  DCU_TRY(dcu::validate_csc(c, n, nnz, ptr, idx));
  DCU_TRY(dcu::ensure(c, dcu::B_RPERM, sizeof(int) * (size_t)(nnz > 0 ? nnz : 1)));
  int* perm = dcu::bp<int>(c, dcu::B_RPERM);
  DCU_TRY(dcu::csr_from_csc(c, n, nnz, ptr, idx, rptr, ridx, perm));
  if (val && rval) DCU_TRY(dcu::csr_values(c, nnz, perm, val, rval));
  DCU_CUDA(c, cudaStreamSynchronize(c->stream));
  return DCU_OK;
}

int dcu_bicgstab_d(dcu_spai_ctx* c, int n, int nnz, const int* ptr, const int* idx, const double* val,
                   const double* mval, const double* b, double* x, const dcu_options* opt, dcu_solve_info* info) {
  int rc = check_matrix(c, n, nnz, ptr, idx, val);
  if (rc) return rc;
  if (!b || !x || (nnz > 0 && !mval)) return dcu::fail(c, DCU_ERR_ARG, "null vector or preconditioner");
  dcu_options o;
  if ((rc = resolve_range(c, n, opt, &o))) return rc;
  try {
    StreamScope scope(c);
    dcu::SellPlan plan;
    const void* msell = nullptr;
    DCU_TRY(dcu::validate_csc(c, n, nnz, ptr, idx));
    DCU_TRY(prepare_solve(c, n, nnz, ptr, idx, val, mval, o.precision, &plan, &msell));
    return dcu::bicgstab_solve(c, plan, dcu::bp<double>(c, dcu::B_SELL_AVAL), msell, b, x, &o, info);
  } catch (const std::bad_alloc&) {
    return dcu::fail(c, DCU_ERR_ALLOC, "host allocation failed");
  }
}

int dcu_bicgstab_h(dcu_spai_ctx* c, int n, int nnz, const int* ptr, const int* idx, const double* val,
                   const double* mval, const double* b, double* x, const dcu_options* opt, dcu_solve_info* info) {
  int rc = check_matrix(c, n, nnz, ptr, idx, val);
  if (rc) return rc;
  if (!b || !x || (nnz > 0 && !mval)) return dcu::fail(c, DCU_ERR_ARG, "null vector or preconditioner");
  StreamScope scope(c);
  Uploads u;
  DCU_TRY(upload(c, n, nnz, ptr, idx, val, b, x, true, &u));
  if (nnz > 0)
    DCU_CUDA(c, cudaMemcpyAsync(u.mval, mval, sizeof(double) * (size_t)nnz, cudaMemcpyHostToDevice, c->stream));
  rc = dcu_bicgstab_d(c, n, nnz, u.ptr, u.idx, u.val, u.mval, u.b, u.x, opt, info);
  if (rc) return rc;
  DCU_CUDA(c, cudaMemcpyAsync(x, u.x, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, c->stream));
  DCU_CUDA(c, cudaStreamSynchronize(c->stream));
  return DCU_OK;
}

int dcu_spai_solve_d(dcu_spai_ctx* c, int n, int nnz, const int* ptr, const int* idx, const double* val,
                     const double* b, double* x, const dcu_options* opt, double* mval, dcu_build_info* binfo,
                     dcu_solve_info* sinfo) {
  int rc = check_matrix(c, n, nnz, ptr, idx, val);
  if (rc) return rc;
  if (!b || !x) return dcu::fail(c, DCU_ERR_ARG, "null vector");
  dcu_options o;
  if ((rc = resolve_range(c, n, opt, &o))) return rc;
  try {
    StreamScope scope(c);
    return solve_pipeline(c, n, nnz, ptr, idx, val, b, x, o, mval, binfo, sinfo, nullptr, nullptr);
  } catch (const std::bad_alloc&) {
    return dcu::fail(c, DCU_ERR_ALLOC, "host allocation failed");
  }
}

int dcu_bicgstab_transpose_d(dcu_spai_ctx* c, int n, int nnz, const int* ptr, const int* idx, const double* val,
                             const double* mval, const double* b, double* x, const dcu_options* opt,
                             dcu_solve_info* info) {
  int rc = check_matrix(c, n, nnz, ptr, idx, val);
  if (rc) return rc;
  if (!b || !x || (nnz > 0 && !mval)) return dcu::fail(c, DCU_ERR_ARG, "null vector or preconditioner");
  dcu_options o;
  if ((rc = resolve_range(c, n, opt, &o))) return rc;
  try {
    StreamScope scope(c);
    DCU_TRY(dcu::validate_csc(c, n, nnz, ptr, idx));
    // A's CSC arrays are the CSR arrays of A^T (and of M^T: same pattern)
    dcu::SellPlan plan;
    DCU_TRY(dcu::sell_plan_rows(c, n, nnz, ptr, idx, &plan));
    const void* msell = nullptr;
    DCU_TRY(gather_values(c, plan, val, mval, o.precision, &msell));
    return dcu::bicgstab_solve(c, plan, dcu::bp<double>(c, dcu::B_SELL_AVAL), msell, b, x, &o, info);
  } catch (const std::bad_alloc&) {
    return dcu::fail(c, DCU_ERR_ALLOC, "host allocation failed");
  }
}

int dcu_sampled_outer_d(dcu_spai_ctx* c, int n, int nnz, const int* ptr, const int* idx, const double* u,
                        const double* v, double alpha, double* out) {
  int rc = check_matrix(c, n, nnz, ptr, idx, idx);
  if (rc) return rc;
  if (!u || !v || (nnz > 0 && !out)) return dcu::fail(c, DCU_ERR_ARG, "null vector");
  StreamScope scope(c);
  DCU_TRY(dcu::validate_csc(c, n, nnz, ptr, idx));
  DCU_TRY(dcu::sampled_outer(c, n, ptr, idx, u, v, alpha, out));
  DCU_CUDA(c, cudaStreamSynchronize(c->stream));
  return DCU_OK;
}

int dcu_batch_solve_d(dcu_spai_ctx* c, int nsys, const int* sys_off, int n, int nnz, const int* ptr, const int* idx,
                      const double* val, int nrhs, const double* B, double* X, const dcu_options* opt, double* mval,
                      int* iters, int* status, dcu_build_info* binfo, dcu_solve_info* sinfo) {
  int rc = check_matrix(c, n, nnz, ptr, idx, val);
  if (rc) return rc;
  if (nsys <= 0 || !sys_off || !B || !X || !iters || !status)
    return dcu::fail(c, DCU_ERR_ARG, "invalid batch arguments");
  dcu_options o;
  if ((rc = resolve_range(c, n, opt, &o))) return rc;
  if (o.col_start != 0 || o.col_end != n) return dcu::fail(c, DCU_ERR_ARG, "a batch builds every column");
  if (o.precision != DCU_PREC_FP64) return dcu::fail(c, DCU_ERR_ARG, "the batched solver runs the FP64 form");
  try {
    StreamScope scope(c);
    DCU_TRY(dcu::validate_csc(c, n, nnz, ptr, idx));
    DCU_TRY(dcu::check_blocks(c, n, ptr, idx, nsys, sys_off));
    double* m = mval;
    if (!m) {
      DCU_TRY(dcu::ensure(c, dcu::B_MVAL, sizeof(double) * (size_t)(nnz > 0 ? nnz : 1)));
      m = dcu::bp<double>(c, dcu::B_MVAL);
    }
    // one build over all columns: M of a block-diagonal A is block diagonal
    dcu_build_info bl{};
    DCU_CUDA(c, cudaEventRecord(c->ev[0], c->stream));
    DCU_TRY(dcu::spai_build(c, n, nnz, ptr, idx, val, &o, m, nullptr, &bl));
    DCU_CUDA(c, cudaEventRecord(c->ev[1], c->stream));
    DCU_CUDA(c, cudaEventSynchronize(c->ev[1]));
    cudaEventElapsedTime(&bl.ms, c->ev[0], c->ev[1]);
    if (binfo) *binfo = bl;
    dcu::SellPlan plan;
    const void* msell = nullptr;
    DCU_TRY(prepare_solve(c, n, nnz, ptr, idx, val, m, DCU_PREC_FP64, &plan, &msell));
    return dcu::batch_solve(c, nsys, sys_off, plan, dcu::bp<double>(c, dcu::B_SELL_AVAL), (const double*)msell,
                            nrhs, B, X, &o, iters, status, sinfo);
  } catch (const std::bad_alloc&) {
    return dcu::fail(c, DCU_ERR_ALLOC, "host allocation failed");
  }
}

int dcu_sell_plan_stats(dcu_spai_ctx* c, long long* slots, long long* uniform_slots) {
  if (!c) return DCU_ERR_ARG;
  StreamScope scope(c);
  return dcu::plan_stats(c, slots, uniform_slots);
}

int dcu_profile_iteration_kernels(dcu_spai_ctx* c, int reps, float* ms_out, int cap, int* count) {
  if (!c || !ms_out) return DCU_ERR_ARG;
  StreamScope scope(c);
  return dcu::profile_iteration(c, reps, ms_out, cap, count);
}

int dcu_spai_solve_h(dcu_spai_ctx* c, int n, int nnz, const int* ptr, const int* idx, const double* val,
                     const double* b, double* x, const dcu_options* opt, double* mval, dcu_build_info* binfo,
                     dcu_solve_info* sinfo) {
  int rc = check_matrix(c, n, nnz, ptr, idx, val);
  if (rc) return rc;
  if (!b || !x) return dcu::fail(c, DCU_ERR_ARG, "null vector");
  dcu_options o;
  if ((rc = resolve_range(c, n, opt, &o))) return rc;
  StreamScope scope(c);
  // ptr and idx first on the context stream (the analysis needs only them);
  // values, then b and x0, on the copy stream while the analysis and the
  // build run.  With pinned host buffers the copies overlap that work.
  auto al = [](size_t v) { return (v + 255) & ~(size_t)255; };
  const size_t sp = al(sizeof(int) * (size_t)(n + 1)), si = al(sizeof(int) * (size_t)(nnz > 0 ? nnz : 1));
  const size_t sv = al(sizeof(double) * (size_t)(nnz > 0 ? nnz : 1)), sn = al(sizeof(double) * (size_t)n);
  DCU_TRY(dcu::ensure(c, dcu::B_UPLOAD, sp + si + 2 * sv + 2 * sn));
  char* base = dcu::bp<char>(c, dcu::B_UPLOAD);
  Uploads u{(int*)base, (int*)(base + sp), (double*)(base + sp + si), (double*)(base + sp + si + sv),
            (double*)(base + sp + si + sv + sn), (double*)(base + sp + si + sv + 2 * sn)};
  // On every return, including early ones, no copy may still be reading the
  // caller's host buffers.
  struct CopyDrain {
    Ctx* c;
    ~CopyDrain() { cudaStreamSynchronize(c->copy_stream); }
  } drain{c};
  // the copy stream starts after everything already queued on the context
  // stream (earlier users of the upload buffer)
  DCU_CUDA(c, cudaEventRecord(c->ev[2], c->stream));
  DCU_CUDA(c, cudaStreamWaitEvent(c->copy_stream, c->ev[2], 0));
  DCU_CUDA(c, cudaMemcpyAsync(u.ptr, ptr, sizeof(int) * (size_t)(n + 1), cudaMemcpyHostToDevice, c->stream));
  if (nnz > 0) {
    DCU_CUDA(c, cudaMemcpyAsync(u.idx, idx, sizeof(int) * (size_t)nnz, cudaMemcpyHostToDevice, c->stream));
    DCU_CUDA(c, cudaMemcpyAsync(u.val, val, sizeof(double) * (size_t)nnz, cudaMemcpyHostToDevice, c->copy_stream));
  }
  DCU_CUDA(c, cudaEventRecord(c->ev[2], c->copy_stream));
  DCU_CUDA(c, cudaMemcpyAsync(u.b, b, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice, c->copy_stream));
  DCU_CUDA(c, cudaMemcpyAsync(u.x, x, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice, c->copy_stream));
  DCU_CUDA(c, cudaEventRecord(c->ev[3], c->copy_stream));
  try {
    rc = solve_pipeline(c, n, nnz, u.ptr, u.idx, u.val, u.b, u.x, o, u.mval, binfo, sinfo, c->ev[2], c->ev[3]);
  } catch (const std::bad_alloc&) {
    rc = dcu::fail(c, DCU_ERR_ALLOC, "host allocation failed");
  }
  if (rc) return rc;
  DCU_CUDA(c, cudaMemcpyAsync(x, u.x, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, c->stream));
  if (mval && nnz > 0)
    DCU_CUDA(c, cudaMemcpyAsync(mval, u.mval, sizeof(double) * (size_t)nnz, cudaMemcpyDeviceToHost, c->stream));
  DCU_CUDA(c, cudaStreamSynchronize(c->stream));
  return DCU_OK;
}

}  // extern "C"
