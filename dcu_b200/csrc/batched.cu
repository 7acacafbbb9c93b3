// Batched BiCGSTAB: many independent systems (the diagonal blocks of one
// block-diagonal matrix) times R right-hand sides each, solved together.
//
// Every (system, right-hand side) pair runs the recurrences of
// cublas2_pbicgstabv2 (include/bicgstab/bicgstab_solver.h:33-275) with its own
// rho, alpha, omega, beta and stop test; pairs that converge are frozen (x no
// longer changes) while the others continue.  Layout: A and M in SELL-32 over
// all N rows; vectors row-major N x R.  R threads share a row, one per
// right-hand side, so every matrix entry read from HBM serves R products (a
// warp broadcast) and a gathered column is R contiguous doubles read by R
// neighbouring lanes.  Thread blocks are tiles of 256 rows inside one
// system; each dot product leaves one partial per tile and the last tile of a
// system to finish sums that system's partials in tile order (deterministic)
// and updates the system's scalars.
#include <algorithm>

#include "internal.cuh"

namespace dcu {
namespace {

constexpr int BT = 256;           // rows per tile (= threads per block)
constexpr int BT_WARPS = BT / 32;
constexpr int BCHUNK = 8;         // iterations per graph launch

struct BState {                   // per (system, rhs) pair, length S * R
  double* rho;
  double* alpha;
  double* omega;
  double* beta;
  double* res;
  double* thr;
  double* bnorm;
  int* active;                    // 1 while iterating
  int* sys_live;                  // per system: pairs still iterating
  int* conv_it;                   // iteration counter when it stopped
  int* status;                    // dcu_solve_status
};

struct BGlobal {
  int it;                         // the reference's counter, shared by all pairs
  int done;
  int active_count;
  int systems_done;               // systems finished in the current kernel
  int pidx;
  int maxiter;
  int pad[2];
};

template <int R>
struct BArgs {
  int n, nsys, ntiles;
  const int* sys_off;             // [nsys + 1]
  const int* tile_sys;            // [ntiles]
  const int* tile_row0;           // [ntiles]
  const int* tile_off;            // [nsys + 1] first tile of each system
  const long long* off;
  const int* kd;                  // per (slice, k) offset descriptors
  const int* su;                  // per slice: all of its k uniform
  const int* ix;
  const double* aval;
  const double* mval;
  const double* b;
  double* x;
  double* r;
  double* rs;
  double* p0;
  double* p1;
  double* y;
  double* ay;
  double* s;
  double* z;
  double* az;
  double* part;                   // [ntiles][3][R]
  unsigned* cnt;                  // [nsys] tiles finished, per kernel
  BState st;
  BGlobal* g;
};

// out[q] = sum_k val * X[col][q], q < R, X row-major with R columns.
// V right-hand sides per thread: 2 (one 16-byte load per gathered column)
// when R >= 2, else 1.
template <int R>
__host__ __device__ constexpr int vals_per_thread() {
  return R >= 2 ? 2 : 1;
}

template <int V>
__device__ __forceinline__ void ldv(const double* __restrict__ p, double (&o)[V]) {
  if constexpr (V == 2) {
    const double2 t = __ldg(reinterpret_cast<const double2*>(p));
    o[0] = t.x;
    o[1] = t.y;
  } else {
    o[0] = __ldg(p);
  }
}
template <int V>
__device__ __forceinline__ void ldp(const double* p, double (&o)[V]) {  // plain load (data written this launch)
  if constexpr (V == 2) {
    const double2 t = *reinterpret_cast<const double2*>(p);
    o[0] = t.x;
    o[1] = t.y;
  } else {
    o[0] = *p;
  }
}
template <int V>
__device__ __forceinline__ void stv(double* p, const double (&o)[V]) {
  if constexpr (V == 2) *reinterpret_cast<double2*>(p) = make_double2(o[0], o[1]);
  else *p = o[0];
}

// One SELL-32 row for V right-hand sides: acc[e] = sum_k val[q] * xf(col[q])[e].
// A slice whose every k has one column offset (su, kd: SellPlan) forms its
// columns from the row and reads no index.
template <int V, typename F>
__device__ __forceinline__ void sell_row_v(const long long* __restrict__ off, const int* __restrict__ kd,
                                           const int* __restrict__ su, const double* __restrict__ val,
                                           const int* __restrict__ ix, int row, F xf, double (&acc)[V]) {
  const int sl = row >> 5;
  const long long o0 = __ldg(off + sl), o1 = __ldg(off + sl + 1);
  const long long base = o0 + (row & 31);
  const int w = (int)((o1 - o0) >> 5);
#pragma unroll
  for (int e = 0; e < V; ++e) acc[e] = 0.0;
  auto step = [&](const double (&av)[8], const int (&cv)[8], int k0) {
#pragma unroll
    for (int t = 0; t < 8; ++t)
      if (k0 + t < w) {
        double xv[V];
        xf(cv[t], xv);
#pragma unroll
        for (int e = 0; e < V; ++e) acc[e] += av[t] * xv[e];
      }
  };
  if (__ldg(su + sl) & 1) {
    const int* __restrict__ kp = kd + (o0 >> 5);
    for (int k0 = 0; k0 < w; k0 += 8) {
      double av[8];
      int cv[8];
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        av[t] = (k0 + t < w) ? __ldcs(val + base + 32ll * (k0 + t)) : 0.0;
        cv[t] = (k0 + t < w) ? row + (__ldg(kp + k0 + t) >> 1) : row;
      }
      step(av, cv, k0);
    }
    return;
  }
  for (int k0 = 0; k0 < w; k0 += 8) {
    double av[8];
    int cv[8];
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      const long long q = base + 32ll * (k0 + t);
      av[t] = (k0 + t < w) ? __ldcs(val + q) : 0.0;
      cv[t] = (k0 + t < w) ? __ldcs(ix + q) : row;
    }
    step(av, cv, k0);
  }
}

// Thread layout: a block covers one tile of BT rows of one system.  T = R / V
// threads share a row; thread t owns right-hand sides q0 .. q0 + V - 1 with
// q0 = (t % T) * V and takes the tile's rows in T passes of BT / T
// consecutive rows (row = row0 + pass * BT / T + t / T).  A warp reads 32 x V
// consecutive doubles of each row-major N x R vector and gathers 32 / T
// neighbouring rows x R right-hand sides (contiguous) per column offset.
template <int R>
struct TileRows {
  static constexpr int V = vals_per_thread<R>();
  static constexpr int T = R / V;
  int row0, row_end, q0, j;
  __device__ TileRows(const int* tile_row0, const int* sys_off, int tile, int sys) {
    row0 = tile_row0[tile];
    row_end = min(row0 + BT, sys_off[sys + 1]);
    q0 = (threadIdx.x % T) * V;
    j = threadIdx.x / T;
  }
  __device__ int row(int pass) const { return row0 + pass * (BT / T) + j; }
};

// Block sums of ND x V values per thread (value [d][e] belongs to right-hand
// side q0 + e) into part[tile][d * R + q]; the last tile of the system to
// finish gets a pointer to the system totals (summed in tile order, entry
// d * R + q, in shared memory), every other tile nullptr.
template <int ND, int R>
__device__ __forceinline__ const double* system_reduce(double (&v)[ND][vals_per_thread<R>()],
                                                       double* __restrict__ part, unsigned* cnt, int tile, int t0,
                                                       int t1, int sys) {
  constexpr int V = vals_per_thread<R>(), T = R / V;
  __shared__ double red[ND * R][BT_WARPS];
  __shared__ double totals[ND * R];
  __shared__ int amlast;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int d = 0; d < ND; ++d)
#pragma unroll
    for (int e = 0; e < V; ++e) {
      double xs = v[d][e];
      // lanes j * T + qt of a warp share qt: fold over the row bits
#pragma unroll
      for (int o = 16; o >= T; o >>= 1) xs += __shfl_xor_sync(0xffffffffu, xs, o);
      if (lane < T) red[d * R + lane * V + e][wid] = xs;
    }
  __syncthreads();
  if (threadIdx.x < ND * R) {
    double ssum = 0.0;
#pragma unroll
    for (int w = 0; w < BT_WARPS; ++w) ssum += red[threadIdx.x][w];
    part[(size_t)tile * (3 * R) + threadIdx.x] = ssum;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned done = atomicAdd(&cnt[sys], 1u);
    amlast = (done == (unsigned)(t1 - t0 - 1)) ? 1 : 0;
  }
  __syncthreads();
  if (!amlast) return nullptr;
  __threadfence();
  // thread j < ND * R sums slot j over the system's tiles in order
  if (threadIdx.x < ND * R) {
    double ssum = 0.0;
    for (int t = t0; t < t1; ++t) ssum += __ldcg(part + (size_t)t * (3 * R) + threadIdx.x);
    totals[threadIdx.x] = ssum;
  }
  __syncthreads();
  if (threadIdx.x == 0) cnt[sys] = 0u;
  return totals;
}

// Every kernel of the batched iteration starts here: it lets the next kernel
// (programmatic dependent launch) be scheduled once all its blocks have
// passed this point, waits for the previous kernel to complete with its
// memory visible, then reads the batch's stop flag.
__device__ __forceinline__ bool g_finished(const BGlobal* g) {
  cudaTriggerProgrammaticLaunchCompletion();
  cudaGridDependencySynchronize();
  return *(volatile const int*)&g->done != 0;
}

// Launch with programmatic dependent launch (inside the captured graph: a
// programmatic edge from the previous kernel).
template <typename K, typename A>
cudaError_t launch_pdl_b(K kernel, int grid, int block, cudaStream_t st, const A& args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, args);
}

// A system whose every pair stopped is skipped by all its tiles (nothing reads
// its vectors or partials any more).
template <int R>
__device__ __forceinline__ bool system_idle(const BArgs<R>& a, int sys) { return a.st.sys_live[sys] == 0; }

template <int R>
__global__ void __launch_bounds__(BT) kb_init(BArgs<R> a, double tol, int tol_mode) {
  constexpr int V = vals_per_thread<R>(), T = R / V;
  const int tile = blockIdx.x, sys = a.tile_sys[tile];
  const TileRows<R> tr(a.tile_row0, a.sys_off, tile, sys);
  double v[3][V] = {};
#pragma unroll 1
  for (int pass = 0; pass < T; ++pass) {
    const int row = tr.row(pass);
    if (row >= tr.row_end) break;
    double ax[V], bb[V], rr[V], zero[V];
    sell_row_v<V>(a.off, a.kd, a.su, a.aval, a.ix, row,
                  [&](int c, double (&o)[V]) { ldv<V>(a.x + (size_t)c * R + tr.q0, o); }, ax);
    const size_t i = (size_t)row * R + tr.q0;
    ldv<V>(a.b + i, bb);
#pragma unroll
    for (int e = 0; e < V; ++e) {
      rr[e] = bb[e] + (-1.0) * ax[e];
      zero[e] = 0.0;
      v[0][e] += rr[e] * rr[e];   // (r*, r) = (r, r) at the start
      v[1][e] += rr[e] * rr[e];
      v[2][e] += bb[e] * bb[e];
    }
    stv<V>(a.r + i, rr);
    stv<V>(a.rs + i, rr);
    stv<V>(a.p0 + i, zero);
    stv<V>(a.p1 + i, zero);
    stv<V>(a.ay + i, zero);
  }
  const double* tot = system_reduce<3, R>(v, a.part, a.cnt, tile, a.tile_off[sys], a.tile_off[sys + 1], sys);
  if (tot && threadIdx.x == 0) {
    int live = 0;
    for (int qq = 0; qq < R; ++qq) {
      const int i = sys * R + qq;
      a.st.rho[i] = tot[0 * R + qq];
      a.st.res[i] = sqrt(tot[1 * R + qq]);
      a.st.bnorm[i] = sqrt(tot[2 * R + qq]);
      a.st.thr[i] = (tol_mode == DCU_TOL_REL) ? tol * a.st.bnorm[i] : tol;
      a.st.alpha[i] = 0.0;
      a.st.omega[i] = 1.0;
      a.st.beta[i] = 0.0;
      const bool run = a.st.res[i] != 0.0 && a.g->maxiter > 1;
      a.st.active[i] = run ? 1 : 0;
      a.st.conv_it[i] = 1;
      a.st.status[i] = run ? -1 : (a.st.res[i] == 0.0 ? DCU_SOLVE_CONVERGED : DCU_SOLVE_MAXITER);
      live += run ? 1 : 0;
    }
    atomicAdd(&a.g->active_count, live);
    a.st.sys_live[sys] = live;
  }
}

// K1: p = r + beta (p - omega ay) at gathered columns; y = M p
template <int R>
__global__ void __launch_bounds__(BT) kb_py(BArgs<R> a) {
  constexpr int V = vals_per_thread<R>(), T = R / V;
  if (g_finished(a.g)) return;
  const int tile = blockIdx.x, sys = a.tile_sys[tile];
  if (system_idle(a, sys)) return;
  const TileRows<R> tr(a.tile_row0, a.sys_off, tile, sys);
  double beta[V], omega[V];
#pragma unroll
  for (int e = 0; e < V; ++e) {
    beta[e] = a.st.beta[sys * R + tr.q0 + e];
    omega[e] = a.st.omega[sys * R + tr.q0 + e];
  }
  const int pidx = a.g->pidx;
  const double* __restrict__ pold = pidx ? a.p1 : a.p0;
  double* __restrict__ pnew = pidx ? a.p0 : a.p1;
  auto pf = [&](int c, double (&o)[V]) {
    const size_t i = (size_t)c * R + tr.q0;
    double rr[V], pp[V], yy[V];
    ldv<V>(a.r + i, rr);
    ldv<V>(pold + i, pp);
    ldv<V>(a.ay + i, yy);
#pragma unroll
    for (int e = 0; e < V; ++e) o[e] = rr[e] + beta[e] * (pp[e] - omega[e] * yy[e]);
  };
#pragma unroll 1
  for (int pass = 0; pass < T; ++pass) {
    const int row = tr.row(pass);
    if (row >= tr.row_end) break;
    double yv[V], pv[V];
    sell_row_v<V>(a.off, a.kd, a.su, a.mval, a.ix, row, pf, yv);
    pf(row, pv);
    const size_t i = (size_t)row * R + tr.q0;
    stv<V>(pnew + i, pv);
    stv<V>(a.y + i, yv);
  }
}

// K2: ay = A y; alpha = rho / (r*, ay)
template <int R>
__global__ void __launch_bounds__(BT) kb_ay(BArgs<R> a) {
  constexpr int V = vals_per_thread<R>(), T = R / V;
  if (g_finished(a.g)) return;
  const int tile = blockIdx.x, sys = a.tile_sys[tile];
  if (system_idle(a, sys)) return;
  const TileRows<R> tr(a.tile_row0, a.sys_off, tile, sys);
  double v[1][V] = {};
#pragma unroll 1
  for (int pass = 0; pass < T; ++pass) {
    const int row = tr.row(pass);
    if (row >= tr.row_end) break;
    double ayv[V], rsv[V];
    sell_row_v<V>(a.off, a.kd, a.su, a.aval, a.ix, row,
                  [&](int c, double (&o)[V]) { ldv<V>(a.y + (size_t)c * R + tr.q0, o); }, ayv);
    const size_t i = (size_t)row * R + tr.q0;
    ldv<V>(a.rs + i, rsv);
    stv<V>(a.ay + i, ayv);
#pragma unroll
    for (int e = 0; e < V; ++e) v[0][e] += rsv[e] * ayv[e];
  }
  const double* tot = system_reduce<1, R>(v, a.part, a.cnt, tile, a.tile_off[sys], a.tile_off[sys + 1], sys);
  if (tot && threadIdx.x == 0) {
    for (int qq = 0; qq < R; ++qq) {
      const int i = sys * R + qq;
      if (!a.st.active[i]) continue;
      const double alpha = a.st.rho[i] / tot[0 * R + qq];
      a.st.alpha[i] = alpha;
      if (tot[0 * R + qq] == 0.0 || !isfinite(alpha)) {
        a.st.active[i] = 0;
        a.st.status[i] = DCU_SOLVE_BREAKDOWN;
        a.st.alpha[i] = a.st.omega[i] = a.st.beta[i] = 0.0;
        atomicSub(&a.g->active_count, 1);
        a.st.sys_live[sys] -= 1;
      }
    }
  }
}

// K3: s = r - alpha ay (on the fly at gathered columns); z = M s
template <int R>
__global__ void __launch_bounds__(BT) kb_sz(BArgs<R> a) {
  constexpr int V = vals_per_thread<R>(), T = R / V;
  if (g_finished(a.g)) return;
  const int tile = blockIdx.x, sys = a.tile_sys[tile];
  if (system_idle(a, sys)) return;
  const TileRows<R> tr(a.tile_row0, a.sys_off, tile, sys);
  double nalpha[V];
#pragma unroll
  for (int e = 0; e < V; ++e) nalpha[e] = -1.0 * a.st.alpha[sys * R + tr.q0 + e];
  auto sf = [&](int c, double (&o)[V]) {
    const size_t i = (size_t)c * R + tr.q0;
    double rr[V], yy[V];
    ldv<V>(a.r + i, rr);
    ldv<V>(a.ay + i, yy);
#pragma unroll
    for (int e = 0; e < V; ++e) o[e] = rr[e] + nalpha[e] * yy[e];
  };
#pragma unroll 1
  for (int pass = 0; pass < T; ++pass) {
    const int row = tr.row(pass);
    if (row >= tr.row_end) break;
    double zv[V], sv[V];
    sell_row_v<V>(a.off, a.kd, a.su, a.mval, a.ix, row, sf, zv);
    sf(row, sv);
    const size_t i = (size_t)row * R + tr.q0;
    stv<V>(a.s + i, sv);
    stv<V>(a.z + i, zv);
  }
}

// K4: az = A z; omega = (az, s) / (az, az)
template <int R>
__global__ void __launch_bounds__(BT) kb_az(BArgs<R> a) {
  constexpr int V = vals_per_thread<R>(), T = R / V;
  if (g_finished(a.g)) return;
  const int tile = blockIdx.x, sys = a.tile_sys[tile];
  if (system_idle(a, sys)) return;
  const TileRows<R> tr(a.tile_row0, a.sys_off, tile, sys);
  double v[2][V] = {};
#pragma unroll 1
  for (int pass = 0; pass < T; ++pass) {
    const int row = tr.row(pass);
    if (row >= tr.row_end) break;
    double azv[V], sv[V];
    sell_row_v<V>(a.off, a.kd, a.su, a.aval, a.ix, row,
                  [&](int c, double (&o)[V]) { ldv<V>(a.z + (size_t)c * R + tr.q0, o); }, azv);
    const size_t i = (size_t)row * R + tr.q0;
    ldv<V>(a.s + i, sv);
    stv<V>(a.az + i, azv);
#pragma unroll
    for (int e = 0; e < V; ++e) {
      v[0][e] += azv[e] * sv[e];
      v[1][e] += azv[e] * azv[e];
    }
  }
  const double* tot = system_reduce<2, R>(v, a.part, a.cnt, tile, a.tile_off[sys], a.tile_off[sys + 1], sys);
  if (tot && threadIdx.x == 0) {
    for (int qq = 0; qq < R; ++qq) {
      const int i = sys * R + qq;
      if (!a.st.active[i]) continue;
      // Az = 0 (s = 0 when the half step solved the pair): omega = 0
      const double omega = (tot[1 * R + qq] == 0.0) ? 0.0 : tot[0 * R + qq] / tot[1 * R + qq];
      a.st.omega[i] = omega;
      if (!isfinite(omega)) {
        a.st.active[i] = 0;
        a.st.status[i] = DCU_SOLVE_BREAKDOWN;
        a.st.alpha[i] = a.st.omega[i] = a.st.beta[i] = 0.0;
        atomicSub(&a.g->active_count, 1);
        a.st.sys_live[sys] -= 1;
      }
    }
  }
}

// K5: x += alpha y + omega z (active pairs); r = s - omega az; rho, beta, ||r||
template <int R>
__global__ void __launch_bounds__(BT) kb_xr(BArgs<R> a) {
  constexpr int V = vals_per_thread<R>(), T = R / V;
  if (g_finished(a.g)) return;
  const int tile = blockIdx.x, sys = a.tile_sys[tile];
  if (system_idle(a, sys)) return;
  const TileRows<R> tr(a.tile_row0, a.sys_off, tile, sys);
  double alpha[V], omega[V];
  bool active[V];
#pragma unroll
  for (int e = 0; e < V; ++e) {
    const int ip = sys * R + tr.q0 + e;
    alpha[e] = a.st.alpha[ip];
    omega[e] = a.st.omega[ip];
    active[e] = a.st.active[ip] != 0;
  }
  double v[2][V] = {};
#pragma unroll 1
  for (int pass = 0; pass < T; ++pass) {
    const int row = tr.row(pass);
    if (row >= tr.row_end) break;
    const size_t i = (size_t)row * R + tr.q0;
    double xv[V], yv[V], zv[V], sv[V], azv[V], rsv[V], rn[V];
    ldp<V>(a.x + i, xv);
    ldv<V>(a.y + i, yv);
    ldv<V>(a.z + i, zv);
    ldv<V>(a.s + i, sv);
    ldv<V>(a.az + i, azv);
    ldv<V>(a.rs + i, rsv);
#pragma unroll
    for (int e = 0; e < V; ++e) {
      if (active[e]) {
        double t = xv[e] + alpha[e] * yv[e];
        xv[e] = t + omega[e] * zv[e];
      }
      rn[e] = sv[e] + (-1.0 * omega[e]) * azv[e];
      v[0][e] += rsv[e] * rn[e];
      v[1][e] += rn[e] * rn[e];
    }
    stv<V>(a.x + i, xv);
    stv<V>(a.r + i, rn);
  }
  const double* tot = system_reduce<2, R>(v, a.part, a.cnt, tile, a.tile_off[sys], a.tile_off[sys + 1], sys);
  if (tot && threadIdx.x == 0) {
    const int it = a.g->it;
    for (int qq = 0; qq < R; ++qq) {
      const int i = sys * R + qq;
      if (!a.st.active[i]) continue;
      const double rho_new = tot[0 * R + qq];
      const double beta = (rho_new / a.st.rho[i]) * (a.st.alpha[i] / a.st.omega[i]);
      a.st.rho[i] = rho_new;
      a.st.beta[i] = beta;
      a.st.res[i] = sqrt(tot[1 * R + qq]);
      a.st.conv_it[i] = it;
      // the stop test first, as in the reference (it never examines beta)
      if (!isfinite(a.st.res[i])) {
        a.st.active[i] = 0;
        a.st.status[i] = DCU_SOLVE_BREAKDOWN;
      } else if (a.st.res[i] < a.st.thr[i]) {
        a.st.active[i] = 0;
        a.st.status[i] = DCU_SOLVE_CONVERGED;
      } else if (!isfinite(beta) || rho_new == 0.0) {
        a.st.active[i] = 0;
        a.st.status[i] = DCU_SOLVE_BREAKDOWN;
      } else if (it + 1 >= a.g->maxiter) {
        a.st.status[i] = DCU_SOLVE_MAXITER;
        a.st.conv_it[i] = it + 1;
      }
      if (!a.st.active[i]) {
        a.st.alpha[i] = a.st.omega[i] = a.st.beta[i] = 0.0;
        atomicSub(&a.g->active_count, 1);
        a.st.sys_live[sys] -= 1;
      }
    }
  }
}

// K6: one thread advances the shared counter after K5 and decides whether the
// batch is done.
template <int R>
__global__ void kb_step(BArgs<R> a) {
  if (g_finished(a.g)) return;
  BGlobal* g = a.g;
  g->pidx ^= 1;
  if (g->active_count <= 0) {
    g->done = 1;
  } else {
    g->it += 1;
    if (g->it >= g->maxiter) g->done = 1;
  }
}

__global__ void kb_check_blocks(const int* __restrict__ ptr, const int* __restrict__ idx, const int* __restrict__ sys_off,
                                int nsys, int n, int* __restrict__ bad) {
  // every column's rows lie in its own diagonal block
  for (int s = blockIdx.x; s < nsys; s += gridDim.x) {
    const int c0 = sys_off[s], c1 = sys_off[s + 1];
    if (threadIdx.x == 0 && (c1 < c0 || c0 < 0 || c1 > n)) atomicOr(bad, 1);
    for (int c = c0 + threadIdx.x; c < c1 && c0 >= 0 && c1 <= n; c += blockDim.x)
      for (int e = ptr[c]; e < ptr[c + 1]; ++e)
        if (idx[e] < c0 || idx[e] >= c1) atomicOr(bad, 2);
  }
}

template <int R>
int run_batch(Ctx* c, int nsys, const int* sys_off_d, const SellPlan& plan, const double* aval, const double* mval,
              const double* B, double* X, const dcu_options* opt, int* iters_h, int* status_h,
              dcu_solve_info* info) {
  const int n = plan.n;
  // host copy of the system offsets -> tiles
  std::vector<int> so(nsys + 1);
  DCU_CUDA(c, cudaMemcpyAsync(so.data(), sys_off_d, sizeof(int) * (nsys + 1), cudaMemcpyDeviceToHost, c->stream));
  DCU_CUDA(c, cudaStreamSynchronize(c->stream));
  std::vector<int> tsys, trow, toff(nsys + 1, 0);
  for (int s = 0; s < nsys; ++s) {
    toff[s] = (int)tsys.size();
    for (int r0 = so[s]; r0 < so[s + 1]; r0 += BT) {
      tsys.push_back(s);
      trow.push_back(r0);
    }
  }
  toff[nsys] = (int)tsys.size();
  const int ntiles = (int)tsys.size();
  if (ntiles == 0) return fail(c, DCU_ERR_ARG, "empty batch");
  auto al = [](size_t v) { return (v + 255) & ~(size_t)255; };
  const size_t vec = al(sizeof(double) * (size_t)n * R);
  const size_t pairs = (size_t)nsys * R;
  const size_t small = al(sizeof(int) * (2 * (size_t)ntiles + nsys + 1)) + al(sizeof(unsigned) * nsys) +
                       al(sizeof(double) * 3 * R * (size_t)ntiles) + al(sizeof(double) * 7 * pairs) +
                       al(sizeof(int) * 3 * pairs) + al(sizeof(int) * (size_t)nsys) + al(sizeof(BGlobal));
  DCU_TRY(ensure(c, B_VEC, 9 * vec + small));
  char* p = bp<char>(c, B_VEC);
  BArgs<R> a;
  std::memset(&a, 0, sizeof(a));  // padding included: the struct keys the graph cache
  a.n = n;
  a.nsys = nsys;
  a.ntiles = ntiles;
  a.sys_off = sys_off_d;
  a.off = plan.off;
  a.kd = plan.kd;
  a.su = plan.su;
  a.ix = plan.idx;
  a.aval = aval;
  a.mval = mval;
  a.b = B;
  a.x = X;
  double* vecs[9];
  for (int i = 0; i < 9; ++i) vecs[i] = reinterpret_cast<double*>(p + i * vec);
  a.r = vecs[0]; a.rs = vecs[1]; a.p0 = vecs[2]; a.p1 = vecs[3]; a.y = vecs[4];
  a.ay = vecs[5]; a.s = vecs[6]; a.z = vecs[7]; a.az = vecs[8];
  char* q = p + 9 * vec;
  int* tiles = reinterpret_cast<int*>(q);
  a.tile_sys = tiles;
  a.tile_row0 = tiles + ntiles;
  a.tile_off = tiles + 2 * ntiles;
  q += al(sizeof(int) * (2 * (size_t)ntiles + nsys + 1));
  a.cnt = reinterpret_cast<unsigned*>(q);
  q += al(sizeof(unsigned) * nsys);
  a.part = reinterpret_cast<double*>(q);
  q += al(sizeof(double) * 3 * R * (size_t)ntiles);
  double* dst = reinterpret_cast<double*>(q);
  a.st.rho = dst; a.st.alpha = dst + pairs; a.st.omega = dst + 2 * pairs; a.st.beta = dst + 3 * pairs;
  a.st.res = dst + 4 * pairs; a.st.thr = dst + 5 * pairs; a.st.bnorm = dst + 6 * pairs;
  q += al(sizeof(double) * 7 * pairs);
  int* ist = reinterpret_cast<int*>(q);
  a.st.active = ist; a.st.conv_it = ist + pairs; a.st.status = ist + 2 * pairs;
  q += al(sizeof(int) * 3 * pairs);
  a.st.sys_live = reinterpret_cast<int*>(q);
  q += al(sizeof(int) * (size_t)nsys);
  a.g = reinterpret_cast<BGlobal*>(q);
  DCU_CUDA(c, cudaMemcpyAsync(tiles, tsys.data(), sizeof(int) * ntiles, cudaMemcpyHostToDevice, c->stream));
  DCU_CUDA(c, cudaMemcpyAsync(tiles + ntiles, trow.data(), sizeof(int) * ntiles, cudaMemcpyHostToDevice, c->stream));
  DCU_CUDA(c, cudaMemcpyAsync(tiles + 2 * ntiles, toff.data(), sizeof(int) * (nsys + 1), cudaMemcpyHostToDevice,
                              c->stream));
  DCU_CUDA(c, cudaMemsetAsync(a.cnt, 0, sizeof(unsigned) * nsys, c->stream));
  const int maxiter = opt->maxiter > 0 ? opt->maxiter : n;
  BGlobal g0{};
  g0.it = 1;
  g0.maxiter = maxiter;
  DCU_CUDA(c, cudaMemcpyAsync(a.g, &g0, sizeof(BGlobal), cudaMemcpyHostToDevice, c->stream));
  DCU_CUDA(c, cudaEventRecord(c->ev[0], c->stream));
  kb_init<R><<<ntiles, BT, 0, c->stream>>>(a, opt->tol, opt->tol_mode);
  DCU_LAUNCHED(c, "kb_init");
  // the first iteration starts with p = r: beta = 0 and p, ay zero-filled
  std::vector<const void*> key = {(const void*)&kb_py<R>, (const void*)(intptr_t)ntiles};
  key_append(key, a);
  GraphSlot* ge = nullptr;
  for (auto& e : c->graphs)
    if (e.key == key) ge = &e;
  if (!ge) {
    cudaGraph_t gr = nullptr;
    DCU_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t le = cudaSuccess;
    for (int i = 0; i < BCHUNK && le == cudaSuccess; ++i) {
      le = launch_pdl_b(kb_py<R>, ntiles, BT, c->stream, a);
      if (le == cudaSuccess) le = launch_pdl_b(kb_ay<R>, ntiles, BT, c->stream, a);
      if (le == cudaSuccess) le = launch_pdl_b(kb_sz<R>, ntiles, BT, c->stream, a);
      if (le == cudaSuccess) le = launch_pdl_b(kb_az<R>, ntiles, BT, c->stream, a);
      if (le == cudaSuccess) le = launch_pdl_b(kb_xr<R>, ntiles, BT, c->stream, a);
      if (le == cudaSuccess) le = launch_pdl_b(kb_step<R>, 1, 1, c->stream, a);
    }
    cudaError_t e = cudaStreamEndCapture(c->stream, &gr);
    if (le != cudaSuccess) {
      if (gr) cudaGraphDestroy(gr);
      return cuda_fail(c, le, "cudaLaunchKernelEx (capture)", __FILE__, __LINE__);
    }
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaStreamEndCapture", __FILE__, __LINE__);
    GraphSlot ne;
    ne.key = key;
    ne.nodes = 6 * BCHUNK;
    e = cudaGraphInstantiate(&ne.exec, gr, 0);
    cudaGraphDestroy(gr);
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaGraphInstantiate", __FILE__, __LINE__);
    if (c->graphs.size() >= 8) {
      cudaGraphExecDestroy(c->graphs.front().exec);
      c->graphs.erase(c->graphs.begin());
    }
    c->graphs.push_back(ne);
    ge = &c->graphs.back();
  }
  int* flag = reinterpret_cast<int*>(reinterpret_cast<char*>(c->pinned) + 1024);
  const long long max_chunks = (long long)maxiter / BCHUNK + 4;
  for (long long i = 0;; ++i) {
    if (i > max_chunks) return fail(c, DCU_ERR_CUDA, "batched solver did not terminate");
    DCU_CUDA(c, cudaGraphLaunch(ge->exec, c->stream));
    c->launches += ge->nodes;
    DCU_CUDA(c, cudaMemcpyAsync(flag + (i & 1), &a.g->done, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    DCU_CUDA(c, cudaEventRecord(c->ev[2 + (i & 1)], c->stream));
    if (i > 0) {
      DCU_CUDA(c, cudaEventSynchronize(c->ev[2 + ((i - 1) & 1)]));
      if (flag[(i - 1) & 1]) break;
    }
  }
  DCU_CUDA(c, cudaEventRecord(c->ev[1], c->stream));
  DCU_CUDA(c, cudaMemcpyAsync(iters_h, a.st.conv_it, sizeof(int) * pairs, cudaMemcpyDeviceToHost, c->stream));
  DCU_CUDA(c, cudaMemcpyAsync(status_h, a.st.status, sizeof(int) * pairs, cudaMemcpyDeviceToHost, c->stream));
  BGlobal gh;
  DCU_CUDA(c, cudaMemcpyAsync(&gh, a.g, sizeof(BGlobal), cudaMemcpyDeviceToHost, c->stream));
  DCU_CUDA(c, cudaStreamSynchronize(c->stream));
  int worst = DCU_SOLVE_CONVERGED;
  for (size_t i = 0; i < pairs; ++i) {
    if (status_h[i] < 0) {   // still running when the shared counter hit maxiter
      status_h[i] = DCU_SOLVE_MAXITER;
      iters_h[i] = gh.it;
    }
    worst = std::max(worst, status_h[i]);
  }
  if (info) {
    info->iters = gh.it;
    info->status = worst;
    info->replacements = 0;
    info->res = info->true_res = info->bnorm = 0.0;
    info->a_fp32 = 0;  // the batched kernels read A's FP64 values
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
    info->ms = ms;
  }
  return DCU_OK;
}

}  // namespace

int check_blocks(Ctx* c, int n, const int* ptr, const int* idx, int nsys, const int* sys_off) {
  DCU_TRY(ensure(c, B_STATS, sizeof(int) * 16));
  int* bad = bp<int>(c, B_STATS);
  DCU_CUDA(c, cudaMemsetAsync(bad, 0, sizeof(int), c->stream));
  kb_check_blocks<<<std::min(nsys, 4096), 128, 0, c->stream>>>(ptr, idx, sys_off, nsys, n, bad);
  DCU_LAUNCHED(c, "kb_check_blocks");
  int h = 0;
  DCU_CUDA(c, cudaMemcpyAsync(&h, bad, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  DCU_CUDA(c, cudaStreamSynchronize(c->stream));
  if (h) return fail(c, DCU_ERR_ARG, "matrix is not block diagonal with respect to the system offsets (%d)", h);
  return DCU_OK;
}

int batch_solve(Ctx* c, int nsys, const int* sys_off, const SellPlan& plan, const double* aval, const double* mval,
                int nrhs, const double* B, double* X, const dcu_options* opt, int* iters, int* status,
                dcu_solve_info* info) {
  switch (nrhs) {
    case 1: return run_batch<1>(c, nsys, sys_off, plan, aval, mval, B, X, opt, iters, status, info);
    case 2: return run_batch<2>(c, nsys, sys_off, plan, aval, mval, B, X, opt, iters, status, info);
    case 4: return run_batch<4>(c, nsys, sys_off, plan, aval, mval, B, X, opt, iters, status, info);
    case 8: return run_batch<8>(c, nsys, sys_off, plan, aval, mval, B, X, opt, iters, status, info);
    default: return fail(c, DCU_ERR_ARG, "nrhs must be 1, 2, 4 or 8 (got %d)", nrhs);
  }
}

}  // namespace dcu
