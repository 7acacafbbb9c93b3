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

// A's values (FP64) in SELL order, and for the forms other than plain FP64
// (which reads FP64 values, as it reads int32 indices), unless
// dcu_set_exact_a32 turned it off, the FP32 copy with its exactness flag.
int gather_a(Ctx* c, const dcu::SellPlan& plan, const double* val, int precision, dcu::SellA* a) {
  const size_t slots = (size_t)(plan.slots > 0 ? plan.slots : 1);
  DCU_TRY(dcu::ensure(c, dcu::B_SELL_AVAL, sizeof(double) * slots));
  *a = dcu::SellA{};
  a->v64 = dcu::bp<double>(c, dcu::B_SELL_AVAL);
  if (!c->exact_a32 || precision == DCU_PREC_FP64)
    return dcu::sell_gather_f64(c, plan, val, dcu::bp<double>(c, dcu::B_SELL_AVAL));
  DCU_TRY(dcu::ensure(c, dcu::B_SELL_AVAL32, sizeof(float) * slots));
  DCU_TRY(dcu::ensure(c, dcu::B_SELL_AFLAG, sizeof(int)));
  a->v32 = dcu::bp<float>(c, dcu::B_SELL_AVAL32);
  a->inexact = dcu::bp<int>(c, dcu::B_SELL_AFLAG);
  return dcu::sell_gather_a(c, plan, val, dcu::bp<double>(c, dcu::B_SELL_AVAL), dcu::bp<float>(c, dcu::B_SELL_AVAL32),
                            dcu::bp<int>(c, dcu::B_SELL_AFLAG));
}

// M's values (by form) in SELL order; an FP32 / BF16 M's narrow slices
// row-major in *msell8 (NULL for an FP64 M).
int gather_m(Ctx* c, const dcu::SellPlan& pl, const double* mval, int precision, const void** msell,
             const void** msell8) {
  const dcu::SellPlan* plan = &pl;
  const size_t slots = (size_t)(plan->slots > 0 ? plan->slots : 1);
  const size_t rows8 = (size_t)plan->nslices * 32 * dcu::kNarrow;
  if (precision == DCU_PREC_FP64) {
    DCU_TRY(dcu::ensure(c, dcu::B_SELL_MVAL, sizeof(double) * slots));
    DCU_TRY(dcu::sell_gather_f64(c, *plan, mval, dcu::bp<double>(c, dcu::B_SELL_MVAL)));
  } else if (precision == DCU_PREC_MIXED_FP32 || precision == DCU_PREC_M_FP32) {
    DCU_TRY(dcu::ensure(c, dcu::B_SELL_MVAL, sizeof(float) * slots));
    DCU_TRY(dcu::ensure(c, dcu::B_SELL_MVAL8, sizeof(float) * rows8));
    DCU_TRY(dcu::sell_gather_m8_f32(c, *plan, mval, dcu::bp<float>(c, dcu::B_SELL_MVAL),
                                    dcu::bp<float>(c, dcu::B_SELL_MVAL8)));
  } else {
    DCU_TRY(dcu::ensure(c, dcu::B_SELL_MVAL, sizeof(__nv_bfloat16) * slots));
    DCU_TRY(dcu::ensure(c, dcu::B_SELL_MVAL8, sizeof(__nv_bfloat16) * rows8));
    DCU_TRY(dcu::sell_gather_m8_bf16(c, *plan, mval, dcu::bp<__nv_bfloat16>(c, dcu::B_SELL_MVAL),
                                     dcu::bp<__nv_bfloat16>(c, dcu::B_SELL_MVAL8)));
  }
  *msell = c->buf[dcu::B_SELL_MVAL].p;
  *msell8 = precision == DCU_PREC_FP64 ? nullptr : c->buf[dcu::B_SELL_MVAL8].p;
  return DCU_OK;
}

// A's values and M's (by form) in SELL order.
int gather_values(Ctx* c, const dcu::SellPlan& plan, const double* val, const double* mval, int precision,
                  dcu::SellA* asell, const void** msell, const void** msell8) {
  DCU_TRY(gather_a(c, plan, val, precision, asell));
  return gather_m(c, plan, mval, precision, msell, msell8);
}

// Points the context's stream at `s` for a scope (the plan and gather
// helpers enqueue on c->stream and synchronise it).
struct OnStream {
  Ctx* c;
  cudaStream_t saved;
  OnStream(Ctx* ctx, cudaStream_t s) : c(ctx), saved(ctx->stream) { c->stream = s; }
  ~OnStream() { c->stream = saved; }
};

// Solver-side layout of A and M: SELL plan + values.
int prepare_solve(Ctx* c, int n, int nnz, const int* ptr, const int* idx, const double* val, const double* mval,
                  int precision, dcu::SellPlan* plan, dcu::SellA* asell, const void** msell, const void** msell8) {
  DCU_TRY(dcu::sell_plan(c, n, nnz, ptr, idx, plan));
  return gather_values(c, *plan, val, mval, precision, asell, msell, msell8);
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
  DCU_CUDA(c, cudaEventRecord(c->ev[6], c->stream));
  if (val_ready) DCU_CUDA(c, cudaStreamWaitEvent(c->stream, val_ready, 0));
  dcu_build_info bl{};
  // the build's time is read after the solve's final synchronisation: no
  // host round trip between the build and the solver's first launches
  DCU_CUDA(c, cudaEventRecord(c->ev[4], c->stream));
  dcu::BuildJob job;
  DCU_TRY(dcu::spai_build_launch(c, n, nnz, ptr, idx, val, &o, m, nullptr, &job));
  // the build's end: after its first kernel, unless the finish adds kernels
  DCU_CUDA(c, cudaEventRecord(c->ev[5], c->stream));
  // While the build's first kernel runs: the SELL plan (pattern only) and A's
  // values in SELL order on the auxiliary stream, whose host round trips wait
  // for that stream alone.
  dcu::SellPlan plan;
  dcu::SellA asell;
  {
    OnStream aux(c, c->aux_stream);
    DCU_CUDA(c, cudaStreamWaitEvent(c->stream, c->ev[6], 0));
    DCU_TRY(dcu::sell_plan(c, n, nnz, ptr, idx, &plan));
    if (val_ready) DCU_CUDA(c, cudaStreamWaitEvent(c->stream, val_ready, 0));
    DCU_TRY(gather_a(c, plan, val, o.precision, &asell));
    DCU_CUDA(c, cudaEventRecord(c->ev[7], c->stream));
  }
  DCU_TRY(dcu::spai_build_finish(c, &job, &bl));
  if (job.finish_launched) DCU_CUDA(c, cudaEventRecord(c->ev[5], c->stream));
  DCU_CUDA(c, cudaStreamWaitEvent(c->stream, c->ev[7], 0));
  const void *msell = nullptr, *msell8 = nullptr;
  DCU_TRY(gather_m(c, plan, m, o.precision, &msell, &msell8));
  if (bx_ready) DCU_CUDA(c, cudaStreamWaitEvent(c->stream, bx_ready, 0));
  DCU_TRY(dcu::bicgstab_solve(c, plan, asell, msell, b, x, &o, sinfo, msell8));
  DCU_CUDA(c, cudaEventSynchronize(c->ev[5]));
  cudaEventElapsedTime(&bl.ms, c->ev[4], c->ev[5]);
  if (binfo) *binfo = bl;
  return DCU_OK;
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

// Device time (ms) of one SPAI build under the context's current tuning.
int timed_build(Ctx* c, int n, int nnz, const int* ptr, const int* idx, const double* val, const dcu_options& o,
                double* m, dcu_build_info* bi, float* ms) {
  DCU_CUDA(c, cudaEventRecord(c->ev[0], c->stream));
  DCU_TRY(dcu::spai_build(c, n, nnz, ptr, idx, val, &o, m, nullptr, bi));
  DCU_CUDA(c, cudaEventRecord(c->ev[1], c->stream));
  DCU_CUDA(c, cudaEventSynchronize(c->ev[1]));
  cudaEventElapsedTime(ms, c->ev[0], c->ev[1]);
  return DCU_OK;
}

// Scratch of the autotuner, released by the caller.
struct TuneScratch {
  double* x = nullptr;
  int* icount = nullptr;
  long long* iptr = nullptr;
};

// The autotuner's steps (dcu_autotune_d): warp-group |I| limit, then the
// iteration's launch configuration on the buffers of one solve.  The
// context's tuning of o.precision is what each timed run uses.
int autotune(Ctx* c, int n, int nnz, const int* ptr, const int* idx, const double* val, const double* b,
             const dcu_options& o, int reps, dcu_tuning* t, TuneScratch* tmp) {
  const int p = o.precision;
  dcu_tuning_default(t);
  c->tune[p] = *t;
  c->tune_set[p] = true;
  DCU_TRY(dcu::validate_csc(c, n, nnz, ptr, idx));
  DCU_TRY(dcu::ensure(c, dcu::B_MVAL, sizeof(double) * (size_t)(nnz > 0 ? nnz : 1)));
  double* m = dcu::bp<double>(c, dcu::B_MVAL);
  dcu_build_info bi{};
  int timed = 0;
  // each build twice, the faster counts (the first may grow buffers)
  auto build2 = [&](float* best) -> int {
    float ms = 0.f;
    for (int r = 0; r < 2; ++r) {
      DCU_TRY(timed_build(c, n, nnz, ptr, idx, val, o, m, &bi, &ms));
      *best = (r == 0 || ms < *best) ? ms : *best;
    }
    ++timed;
    return DCU_OK;
  };
  DCU_TRY(build2(&t->build_ms_default));
  t->build_ms_tuned = t->build_ms_default;
  const int ncols = o.col_end - o.col_start;
  if (bi.max_ni > 16 && ncols > 0) {
    // |I_k| of every column, to skip limits that would hand more than 1/8 of
    // the columns to the CTA kernel (a CTA per column costs more than a group
    // of a warp by construction)
    DCU_CUDA(c, cudaMalloc(&tmp->icount, sizeof(int) * (size_t)ncols));
    DCU_CUDA(c, cudaMalloc(&tmp->iptr, sizeof(long long) * ((size_t)ncols + 1)));
    long long total = 0;
    DCU_TRY(dcu::spai_pattern(c, n, ptr, idx, o.col_start, o.col_end, tmp->icount, tmp->iptr, nullptr, 0, &total));
    std::vector<int> h((size_t)ncols);
    DCU_CUDA(c, cudaMemcpy(h.data(), tmp->icount, sizeof(int) * (size_t)ncols, cudaMemcpyDeviceToHost));
    for (int v : {24, 16}) {
      long long moved = 0;
      for (int k : h) moved += (k > v && k <= 32) ? 1 : 0;
      if (moved == 0 || moved > ncols / 8) continue;
      c->tune[p].group_max_ni = v;
      float ms = 0.f;
      DCU_TRY(build2(&ms));
      if (ms < 0.99f * t->build_ms_tuned) {
        t->build_ms_tuned = ms;
        t->group_max_ni = v;
      }
    }
    c->tune[p].group_max_ni = t->group_max_ni;
  }
  if (bi.cols_hub > 0) {
    // every block on one CTA (per-CTA slabs) against the hub kernels
    c->tune[p].cta_max_area = -1;
    float ms = 0.f;
    DCU_TRY(build2(&ms));
    if (ms < 0.99f * t->build_ms_tuned) {
      t->build_ms_tuned = ms;
      t->cta_max_area = -1;
    }
    c->tune[p].cta_max_area = t->cta_max_area;
  }
  // one solve from x0 = 0 with the chosen build and the default iteration
  DCU_CUDA(c, cudaMalloc(&tmp->x, sizeof(double) * (size_t)n));
  dcu_build_info b2{};
  dcu_solve_info si{};
  // best device time (ms) of the solve phase over three solves from x0 = 0
  auto solve3 = [&](float* best) -> int {
    for (int r = 0; r < 3; ++r) {
      DCU_CUDA(c, cudaMemsetAsync(tmp->x, 0, sizeof(double) * (size_t)n, c->stream));
      DCU_TRY(solve_pipeline(c, n, nnz, ptr, idx, val, b, tmp->x, o, nullptr, &b2, &si, nullptr, nullptr));
      *best = (r == 0 || si.ms < *best) ? si.ms : *best;
    }
    ++timed;
    return DCU_OK;
  };
  DCU_CUDA(c, cudaMemsetAsync(tmp->x, 0, sizeof(double) * (size_t)n, c->stream));
  DCU_TRY(solve_pipeline(c, n, nnz, ptr, idx, val, b, tmp->x, o, nullptr, &b2, &si, nullptr, nullptr));
  // per kernel: the fastest grid of each kernel without a reduction, single launches
  dcu_tuning k = *t;
  int it_timed = 0;
  DCU_TRY(dcu::tune_iteration(c, reps, &k, &it_timed));
  // Whole solves decide between the default, the per-kernel choice with the
  // split and (where it computes the same values) with the fused first step:
  // in a solve the kernels run inside a graph with programmatic dependent
  // launch, where an extra launch costs less than it does alone.  Every
  // candidate gives the same iterates, so the solve times compare launch
  // configurations only.
  const dcu_tuning base = c->tune[p];
  std::vector<dcu_tuning> cands = {base};
  auto add = [&](int k1) {
    dcu_tuning v = base;
    v.k1_split = k1;
    v.grid_p = k.grid_p;
    v.grid_y = k.grid_y;
    v.grid_py = k.grid_py;
    v.grid_sz = k.grid_sz;
    const int eff = (k1 < 0) ? c->profile_default_split : k1;
    const bool same = eff == c->profile_default_split && v.grid_sz == 0 &&
                      (eff ? v.grid_p == 0 && v.grid_y == 0 : v.grid_py == 0);
    if (!same) cands.push_back(v);
  };
  if (c->profile_k1_free) {
    add(1);
    add(0);
  } else {
    add(-1);
  }
  float def_ms = 0.f, best_ms = 0.f;
  size_t pick = 0;
  for (size_t i = 0; i < cands.size(); ++i) {
    c->tune[p] = cands[i];
    float ms = 0.f;
    DCU_TRY(solve3(&ms));
    if (i == 0) {
      def_ms = best_ms = ms;
    } else if (ms < 0.995f * best_ms) {  // a change must win by more than 0.5%
      best_ms = ms;
      pick = i;
    }
  }
  const int iters = si.iters > 0 ? si.iters : 1;
  t->k1_split = cands[pick].k1_split;
  t->grid_p = cands[pick].grid_p;
  t->grid_y = cands[pick].grid_y;
  t->grid_py = cands[pick].grid_py;
  t->grid_sz = cands[pick].grid_sz;
  t->iter_us_default = 1000.f * def_ms / iters;
  t->iter_us_tuned = 1000.f * best_ms / iters;
  t->candidates = timed + it_timed;
  c->tune[p] = *t;
  return DCU_OK;
}

int check_tuning(Ctx* c, const dcu_tuning* t) {
  if (t->k1_split < -1 || t->k1_split > 1) return dcu::fail(c, DCU_ERR_ARG, "k1_split must be -1, 0 or 1");
  for (int g : {t->grid_p, t->grid_y, t->grid_py, t->grid_sz})
    if (g < -1 || g > 64) return dcu::fail(c, DCU_ERR_ARG, "grid selector %d outside [-1, 64]", g);
  if (t->group_max_ni < 0 || t->group_max_ni > 32)
    return dcu::fail(c, DCU_ERR_ARG, "group_max_ni %d outside [0, 32]", t->group_max_ni);
  if (t->cta_max_area < -1) return dcu::fail(c, DCU_ERR_ARG, "cta_max_area must be >= -1");
  return DCU_OK;
}

}  // namespace

extern "C" {

void dcu_tuning_default(dcu_tuning* t) {
  if (!t) return;
  std::memset(t, 0, sizeof(*t));
  t->k1_split = -1;
}

int dcu_set_tuning(dcu_spai_ctx* c, int precision, const dcu_tuning* t) {
  if (!c) return DCU_ERR_ARG;
  if (precision < DCU_PREC_FP64 || precision > DCU_PREC_M_BF16)
    return dcu::fail(c, DCU_ERR_ARG, "unknown precision %d", precision);
  if (!t) {
    dcu_tuning_default(&c->tune[precision]);
    c->tune_set[precision] = false;
    return DCU_OK;
  }
  DCU_TRY(check_tuning(c, t));
  c->tune[precision] = *t;
  c->tune_set[precision] = true;
  return DCU_OK;
}

int dcu_get_tuning(dcu_spai_ctx* c, int precision, dcu_tuning* t) {
  if (!c || !t) return DCU_ERR_ARG;
  if (precision < DCU_PREC_FP64 || precision > DCU_PREC_M_BF16)
    return dcu::fail(c, DCU_ERR_ARG, "unknown precision %d", precision);
  if (c->tune_set[precision]) *t = c->tune[precision];
  else dcu_tuning_default(t);
  return DCU_OK;
}

int dcu_autotune_d(dcu_spai_ctx* c, int n, int nnz, const int* ptr, const int* idx, const double* val,
                   const double* b, const dcu_options* opt, int reps, dcu_tuning* out) {
  int rc = check_matrix(c, n, nnz, ptr, idx, val);
  if (rc) return rc;
  if (!b) return dcu::fail(c, DCU_ERR_ARG, "null vector");
  dcu_options o;
  if ((rc = resolve_range(c, n, opt, &o))) return rc;
  const int p = o.precision;
  const bool was_set = c->tune_set[p];
  const dcu_tuning was = c->tune[p];
  dcu_tuning t;
  TuneScratch tmp;
  try {
    StreamScope scope(c);
    rc = autotune(c, n, nnz, ptr, idx, val, b, o, reps, &t, &tmp);
    cudaStreamSynchronize(c->stream);
  } catch (const std::bad_alloc&) {
    rc = dcu::fail(c, DCU_ERR_ALLOC, "host allocation failed");
  }
  cudaFree(tmp.x);
  cudaFree(tmp.icount);
  cudaFree(tmp.iptr);
  if (rc) {
    c->tune[p] = was;
    c->tune_set[p] = was_set;
    return rc;
  }
  c->tune[p] = t;
  c->tune_set[p] = true;
  if (out) *out = t;
  return DCU_OK;
}

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
    if ((e = cudaStreamCreateWithFlags(&c->aux_stream, cudaStreamNonBlocking)) != cudaSuccess) { rc = dcu::cuda_fail(c, e, "aux stream", __FILE__, __LINE__); break; }
    for (int i = 0; i < 8 && e == cudaSuccess; ++i)
      e = cudaEventCreateWithFlags(&c->ev[i], (i < 2 || i == 4 || i == 5) ? cudaEventDefault : cudaEventDisableTiming);
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
  if (c->aux_stream) cudaStreamSynchronize(c->aux_stream);
  dcu::release_graphs(c);
  for (auto& b : c->buf)
    if (b.p) cudaFree(b.p);
  for (auto& e : c->ev)
    if (e) cudaEventDestroy(e);
  if (c->ev_sync) cudaEventDestroy(c->ev_sync);
  if (c->pinned) cudaFreeHost(c->pinned);
  if (c->stream) cudaStreamDestroy(c->stream);
  if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
  if (c->aux_stream) cudaStreamDestroy(c->aux_stream);
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
  DCU_TRY(dcu::validate_csc(c, n, nnz, ptr, idx, /*unique_rows=*/false));
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
    dcu::SellA asell;
    const void *msell = nullptr, *msell8 = nullptr;
    DCU_TRY(dcu::validate_csc(c, n, nnz, ptr, idx));
    DCU_TRY(prepare_solve(c, n, nnz, ptr, idx, val, mval, o.precision, &plan, &asell, &msell, &msell8));
    return dcu::bicgstab_solve(c, plan, asell, msell, b, x, &o, info, msell8);
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
    dcu::SellA asell;
    const void *msell = nullptr, *msell8 = nullptr;
    DCU_TRY(gather_values(c, plan, val, mval, o.precision, &asell, &msell, &msell8));
    return dcu::bicgstab_solve(c, plan, asell, msell, b, x, &o, info, msell8);
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
  DCU_TRY(dcu::validate_csc(c, n, nnz, ptr, idx, /*unique_rows=*/false));
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
    dcu::SellA asell;
    const void *msell = nullptr, *msell8 = nullptr;
    DCU_TRY(prepare_solve(c, n, nnz, ptr, idx, val, m, DCU_PREC_FP64, &plan, &asell, &msell, &msell8));
    return dcu::batch_solve(c, nsys, sys_off, plan, asell.v64, (const double*)msell,
                            nrhs, B, X, &o, iters, status, sinfo);
  } catch (const std::bad_alloc&) {
    return dcu::fail(c, DCU_ERR_ALLOC, "host allocation failed");
  }
}

int dcu_sell_plan_stats(dcu_spai_ctx* c, long long* slots, long long* uniform_slots, long long* wide_slices) {
  if (!c) return DCU_ERR_ARG;
  StreamScope scope(c);
  return dcu::plan_stats(c, slots, uniform_slots, wide_slices);
}

int dcu_set_wide_prepass(dcu_spai_ctx* c, int enabled) {
  if (!c) return DCU_ERR_ARG;
  c->wide_prepass = enabled != 0;
  return DCU_OK;
}

int dcu_set_exact_a32(dcu_spai_ctx* c, int enabled) {
  if (!c) return DCU_ERR_ARG;
  c->exact_a32 = enabled != 0;
  return DCU_OK;
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
