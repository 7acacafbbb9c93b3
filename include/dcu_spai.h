/*
 * dcu_spai.h -- C ABI of the B200 SPAI-preconditioned BiCGSTAB library
 * (libdcu_spai.so).  Plain pointers and sizes only; every function returns a
 * dcu_status code and never exits the process.
 *
 * Reference interfaces this layer replaces (SingkiWong/DCU):
 *   dcu_spai_create / dcu_spai_destroy
 *       initMultiDCU / cleanupMultiDCU        src/spai_multi_dcu.cpp:1296-1350, 2335-2380
 *   dcu_spai_distribute_columns
 *       distributeColumns                     src/spai_multi_dcu.cpp:1356-1449
 *   dcu_spai_build_d / dcu_spai_build_h
 *       StaticSPAIv20 (single-pass semantics) src/spai_single_dcu.cpp:1224-2687,
 *       reached through RunStatic/DynamicSPAI_MultiDCU_MPI
 *                                             src/spai_multi_dcu.cpp:1867-1875
 *   dcu_spai_pattern_d
 *       computeJ_SSPAIv10 + computeI*_Symbol_SpMMv1
 *                                             src/spai_multi_dcu.cpp:275-319, 321-834
 *   dcu_csc_to_csr_d
 *       cuCSC2CSR                             include/common/cuFormatConversion.h:453-589
 *   dcu_bicgstab_d / dcu_bicgstab_h
 *       cublas2_pbicgstabv2                   include/bicgstab/bicgstab_solver.h:33-275
 *       (driven as in runBiCGSTABOnRank0      src/spai_multi_dcu.cpp:1878-1951)
 *   dcu_spai_solve_d / dcu_spai_solve_h
 *       the whole path: SPAI build, CSC->CSR, BiCGSTAB
 *
 * Matrices are square, CSC, 0-based: ptr[n+1] (int32), idx[nnz] row indices
 * (int32), val[nnz] (float64) -- the CSC_Matrix layout of
 * include/common/dataType.h:33-41.  The preconditioner M has A's pattern, so
 * it is passed as values only (mval[nnz], aligned with A's idx).  A row index
 * may appear only once per column: the SPAI and solver entry points refuse a
 * repeated (row, column) pair with DCU_ERR_ARG.  (The reference's gather
 * takes the first match, src/spai_multi_dcu.cpp:945-983, and its J_k then
 * holds the column twice: two equal columns of A(I,J), a zero R pivot and a
 * NaN column of M.)  dcu_csc_to_csr_d and dcu_sampled_outer_d accept
 * repeated pairs.  Columns may list their rows in any order.
 * Suffix _d: device pointers (cudaMalloc'ed, on the context's device; the
 * solution vector x must be 16-byte aligned, as cudaMalloc and torch
 * allocations are, else DCU_ERR_ARG);
 * suffix _h: host pointers (copies are made inside the call).
 */
#ifndef DCU_SPAI_H
#define DCU_SPAI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dcu_spai_ctx dcu_spai_ctx;

typedef enum {
  DCU_OK = 0,
  DCU_ERR_ARG = 1,        /* invalid argument (sizes, pointers, ranges)   */
  DCU_ERR_CUDA = 2,       /* a CUDA call failed; see dcu_spai_last_error  */
  DCU_ERR_ALLOC = 3,      /* device or host allocation failed             */
  DCU_ERR_NO_DEVICE = 4,  /* no CUDA device / device index out of range   */
  DCU_ERR_LIMIT = 5       /* a size exceeds a documented limit            */
} dcu_status;

/* Column schedules of the device work queue (the reference's partitions). */
typedef enum {
  DCU_SCHED_BALANCED_COLUMNS = 0, /* static: equal contiguous column counts   */
  DCU_SCHED_BALANCED_NNZ = 1      /* dynamic: nnz-balanced chunks, atomic pull */
} dcu_schedule;

/* Precision forms. */
typedef enum {
  DCU_PREC_FP64 = 0,      /* plain: FP64 least squares, FP64 M, FP64 vectors, int32 indices */
  DCU_PREC_MIXED_FP32 = 1,/* FP32 least squares, M stored FP32, FP32 preconditioned vectors,
                             16-bit index deltas where they fit; FP64 A, residual, dots   */
  DCU_PREC_MIXED_BF16 = 2,/* as MIXED_FP32 with M stored as BF16                           */
  DCU_PREC_M_FP32 = 3,    /* FP32 least squares and M (FP32, 16-bit deltas); every vector FP64 */
  DCU_PREC_M_BF16 = 4     /* as M_FP32 with M stored as BF16                               */
} dcu_precision;

/* Least-squares method of the SPAI build. */
typedef enum {
  DCU_LS_AUTO = 0,        /* FP64 form: Householder; mixed forms: NORMAL_EQ        */
  DCU_LS_HOUSEHOLDER = 1, /* Householder QR for every column                       */
  DCU_LS_NORMAL_EQ = 2    /* columns with |J| <= 8 and <= 52 entries over J: one
                             thread per column, normal equations + Cholesky in the
                             form's precision; a column whose Cholesky pivot falls
                             below tau G_jj (tau 1e-3 FP32, 1e-8 FP64) or that
                             exceeds those sizes goes to Householder QR            */
} dcu_ls_method;

/* Stopping rule. */
typedef enum {
  DCU_TOL_ABS = 0,        /* ||r||_2 < tol (the reference, bicgstab_solver.h:229) */
  DCU_TOL_REL = 1         /* ||r||_2 < tol * ||b||_2                             */
} dcu_tol_mode;

/* Solver outcome codes (dcu_solve_info.status). */
typedef enum {
  DCU_SOLVE_CONVERGED = 0,
  DCU_SOLVE_MAXITER = 1,
  DCU_SOLVE_BREAKDOWN = 2 /* rho or (r*,Ay) zero, a non-finite scalar or residual, or
                             beta undefined (omega = 0) while ||r|| is above the threshold.
                             (Az,Az) = 0 gives omega = 0: when the half step solved the
                             system, r = s meets the threshold and the solve converges. */
} dcu_solve_status;

typedef struct {
  int cols_total;         /* columns built                                        */
  int cols_small;         /* columns solved by the warp-group kernel              */
  int cols_large;         /* columns solved by the CTA kernel                     */
  int cols_singular;      /* columns with a zero / non-finite Householder pivot   */
  int max_nj;             /* max |J_k|                                            */
  int max_ni;             /* max |I_k|                                            */
  float ms;               /* device time of the build (CUDA events)              */
  int cols_staged;        /* CTA-kernel columns whose J columns were brought into
                             shared memory by bulk (TMA) copies                    */
  int cols_hub;           /* CTA-kernel columns whose dense block exceeded shared
                             memory and was factored by the all-SM hub kernels
                             (one launch per Householder step)                     */
} dcu_build_info;

typedef struct {
  int iters;              /* the reference's counter (starts at 1; see dcu_bicgstab_d) */
  int status;             /* dcu_solve_status                                          */
  int replacements;       /* residual replacements performed                          */
  double res;             /* recurrence ||r||_2 at exit                                */
  double true_res;        /* ||b - A x||_2 recomputed in FP64 at exit                  */
  double bnorm;           /* ||b||_2                                                   */
  float ms;               /* device time of the solve (CUDA events)                   */
  int a_fp32;             /* 1 when the A products read A's FP32 copy (a form other than
                             DCU_PREC_FP64, every value of A exact in FP32;
                             dcu_set_exact_a32)                                        */
} dcu_solve_info;

typedef struct {
  int schedule;           /* dcu_schedule                                   */
  int precision;          /* dcu_precision                                  */
  int tol_mode;           /* dcu_tol_mode                                   */
  int maxiter;            /* <= 0 means n, as the reference (:134)           */
  double tol;
  int verify;             /* 1: on recurrence convergence recompute b - A x in
                             FP64 and continue from it unless it also meets
                             the threshold (residual replacement); 0: stop on
                             the recurrence residual exactly as the reference */
  int col_start, col_end; /* SPAI column range; col_end <= 0 means n          */
  int ls_method;          /* dcu_ls_method                                  */
} dcu_options;

/* Fill *opt with the defaults of the benchmark workloads: balanced_columns,
 * FP64, relative tol 1e-8, maxiter 1000, verify on, all columns. */
void dcu_options_default(dcu_options* opt);

/* ---- context ------------------------------------------------------------- */

/* Create a context on CUDA device `device`.  `units` is the schedule's unit
 * count P (the reference's numDCUs; <= 0 picks one per resident warp group of
 * the column kernel): the P contiguous ranges of balanced_columns that
 * dcu_spai_distribute_columns reports and the sharded build uses.  On one
 * device the static schedule takes those ranges in order, which is the whole
 * column range, in one sweep by all resident workers (equal column counts per
 * worker for any P); the dynamic schedule pulls nnz-balanced chunks from an
 * atomic queue.  M does not depend on either.  Replaces initMultiDCU. */
int dcu_spai_create(dcu_spai_ctx** ctx, int device, int units);
/* Frees every device buffer the context owns.  Replaces cleanupMultiDCU. */
void dcu_spai_destroy(dcu_spai_ctx* ctx);
/* Last error message of this context ("" when none). */
const char* dcu_spai_last_error(const dcu_spai_ctx* ctx);
/* Use `stream` (a cudaStream_t) for all work of this context; NULL = the
 * context's own stream. */
int dcu_spai_set_stream(dcu_spai_ctx* ctx, void* stream);
/* Number of work units the schedules split columns over. */
int dcu_spai_units(const dcu_spai_ctx* ctx);
/* Number of kernel launches this context has issued (diagnostic counter). */
long long dcu_spai_launch_count(const dcu_spai_ctx* ctx);

/* Column split of [col_start, col_end) over `units` (host arrays starts/ends
 * of length units), identical to distributeColumns: schedule 0 =
 * balanced_columns, 1 = balanced_nnz.  `ptr` is a host array. */
int dcu_spai_distribute_columns(const int* ptr, int col_start, int col_end, int units,
                                int schedule, int* starts, int* ends);

/* ---- SPAI ------------------------------------------------------------------ */

/* Pattern pass: |I_k| (icount[k - col_start]) and, when ilist != NULL, the
 * sorted rows of I_k at ilist[iptr[k - col_start]] where iptr is the
 * exclusive prefix of icount (written by this call, length ncols + 1,
 * int64).  Call with ilist == NULL first to learn *total.  Device pointers. */
int dcu_spai_pattern_d(dcu_spai_ctx* ctx, int n, const int* ptr, const int* idx, int col_start,
                       int col_end, int* icount, long long* iptr, int* ilist,
                       long long ilist_capacity, long long* total);

/* SPAI build on A's pattern: mval[nnz] (device, FP64) receives M's values in
 * A's CSC order; columns outside [opt->col_start, opt->col_end) are zero.
 * colres (device, optional, length ncols) receives ||A m_k - e_k||_2.
 * Uses opt->schedule and opt->precision (FP32 least squares for the mixed
 * forms; mval is FP64 either way). */
int dcu_spai_build_d(dcu_spai_ctx* ctx, int n, int nnz, const int* ptr, const int* idx,
                     const double* val, const dcu_options* opt, double* mval, double* colres,
                     dcu_build_info* info);
int dcu_spai_build_h(dcu_spai_ctx* ctx, int n, int nnz, const int* ptr, const int* idx,
                     const double* val, const dcu_options* opt, double* mval, double* colres,
                     dcu_build_info* info);

/* CSC -> CSR (ascending columns inside each row, values carried along).
 * Device pointers; rptr[n+1], ridx[nnz], rval[nnz] (rval may be NULL). */
int dcu_csc_to_csr_d(dcu_spai_ctx* ctx, int n, int nnz, const int* ptr, const int* idx,
                     const double* val, int* rptr, int* ridx, double* rval);

/* CSC -> CSR exactly as dcu_csc_to_csr_d, for callers that cannot allocate
 * device memory: code running under a framework's memory pool that owns the
 * device (an out-of-band cudaMalloc fragments or exceeds its budget) or a
 * latency-critical path that cannot take cudaMalloc/cudaFree and the device
 * synchronisation cudaFree implies.  No context, no cudaMalloc/cudaFree, no
 * allocating library call: the scratch is one fixed __device__ array of about
 * 5 MB in this library, which every GPU that loads the library holds until the
 * process exits.  Limits: n <= 131072, nnz <= 1048576 (DCU_ERR_LIMIT beyond),
 * no row longer than 8192 entries (DCU_ERR_LIMIT after the call).  Runs on
 * `stream` (a cudaStream_t, NULL = legacy default) on the current device and
 * returns after it finished there: it synchronises the stream and reads a
 * status back to the host, and returns DCU_ERR_ARG without using a stream
 * that is capturing.  Each call looks up the array's device address on the
 * current device.  Every call reuses the same array (the parts that must
 * start at zero are cleared each time), so calls that overlap on one GPU
 * race.  After a return other than DCU_OK the outputs are undefined (they may
 * be partly written).  Duplicate (row, column) pairs and unsorted columns are
 * accepted, as by dcu_csc_to_csr_d.
 * No counterpart in the reference. */
int dcu_csc_to_csr_noalloc_d(int n, int nnz, const int* ptr, const int* idx, const double* val,
                             int* rptr, int* ridx, double* rval, void* stream);

/* ---- BiCGSTAB --------------------------------------------------------------- */

/* Right-preconditioned BiCGSTAB for A x = b with preconditioner M (values on
 * A's pattern).  x holds x0 on entry and the solution on exit.  The iteration
 * counter follows the reference: it starts at 1, the loop runs while
 * iters < maxiter, and stops when the residual meets the threshold.
 * opt->precision selects how M and the preconditioned vectors are stored. */
int dcu_bicgstab_d(dcu_spai_ctx* ctx, int n, int nnz, const int* ptr, const int* idx,
                   const double* val, const double* mval, const double* b, double* x,
                   const dcu_options* opt, dcu_solve_info* info);
int dcu_bicgstab_h(dcu_spai_ctx* ctx, int n, int nnz, const int* ptr, const int* idx,
                   const double* val, const double* mval, const double* b, double* x,
                   const dcu_options* opt, dcu_solve_info* info);

/* The adjoint solve A^T x = b, right-preconditioned with M^T (same options
 * and counter as dcu_bicgstab_d).  A's CSC arrays are read as the CSR arrays
 * of A^T, so no transpose is formed.  No counterpart in the reference (the
 * differentiation path of this library). */
int dcu_bicgstab_transpose_d(dcu_spai_ctx* ctx, int n, int nnz, const int* ptr, const int* idx,
                             const double* val, const double* mval, const double* b, double* x,
                             const dcu_options* opt, dcu_solve_info* info);

/* out[e] = alpha * u[idx[e]] * v[j] for every entry e of CSC column j: the
 * outer product alpha u v^T sampled on A's pattern.  With u = lambda (adjoint
 * solution), v = x and alpha = -1 this is dL/dA on A's nonzeros.  Device
 * pointers.  No counterpart in the reference. */
int dcu_sampled_outer_d(dcu_spai_ctx* ctx, int n, int nnz, const int* ptr, const int* idx,
                        const double* u, const double* v, double alpha, double* out);

/* The whole path: SPAI build of M on A's pattern, then BiCGSTAB.  mval
 * (optional) receives M (FP64, A's CSC order).  Device pointers. */
int dcu_spai_solve_d(dcu_spai_ctx* ctx, int n, int nnz, const int* ptr, const int* idx,
                     const double* val, const double* b, double* x, const dcu_options* opt,
                     double* mval, dcu_build_info* binfo, dcu_solve_info* sinfo);
/* Same with host buffers: uploads A and b, runs, downloads x (and mval when
 * non-NULL). */
int dcu_spai_solve_h(dcu_spai_ctx* ctx, int n, int nnz, const int* ptr, const int* idx,
                     const double* val, const double* b, double* x, const dcu_options* opt,
                     double* mval, dcu_build_info* binfo, dcu_solve_info* sinfo);

/* Batched solve of independent systems: the diagonal blocks
 * [sys_off[s], sys_off[s+1]) of one block-diagonal CSC matrix (device
 * sys_off, int32, nsys + 1 entries, sys_off[0] = 0, sys_off[nsys] = n), each
 * with nrhs (1, 2, 4 or 8) right-hand sides.  B and X are device, row-major
 * n x nrhs; X holds x0 on entry.  One SPAI build covers every column (M of a
 * block-diagonal A is block diagonal); then one BiCGSTAB iteration stream
 * advances all (system, rhs) pairs, each with its own scalars and stop test,
 * freezing converged pairs.  iters / status (host, nsys * nrhs, pair
 * s * nrhs + q) receive each pair's counter and dcu_solve_status; sinfo->iters
 * is the shared counter at exit.  FP64 form only (opt->precision 0);
 * opt->ls_method applies to the build.  Fails with DCU_ERR_ARG when an entry
 * lies outside its diagonal block. */
int dcu_batch_solve_d(dcu_spai_ctx* ctx, int nsys, const int* sys_off, int n, int nnz, const int* ptr,
                      const int* idx, const double* val, int nrhs, const double* B, double* X,
                      const dcu_options* opt, double* mval, int* iters, int* status,
                      dcu_build_info* binfo, dcu_solve_info* sinfo);

/* Diagnostic timing: re-launch each iteration kernel of the last solve on
 * this context `reps` times on that solve's buffers, each timed launch right
 * after an untimed launch of the kernel that precedes it in the iteration (so
 * the L2 cache holds what it holds in a solve), and write the mean device
 * time per launch (ms) to ms_out[0..count-1], in launch order.  With an FP64
 * preconditioner the iteration runs five fused kernels:
 *   p/y = M p | A y + (r*, Ay) | s/z = M s | A z + dots | x/r update + dots
 * with a narrow (FP32 / BF16) preconditioner six, the first one split in two:
 *   p = r + beta (p - omega Ay) | y = M p | ... (as above)
 * *count (optional) receives the number of kernels; DCU_ERR_ARG when cap is
 * smaller.  The solver vectors and x are left in an unspecified state. */
int dcu_profile_iteration_kernels(dcu_spai_ctx* ctx, int reps, float* ms_out, int cap, int* count);

/* Diagnostics of the last SELL-32 layout built on this context (by any solve
 * that runs BiCGSTAB): *slots = slots including padding, *uniform_slots =
 * slots in slices whose every entry position has one column offset for all
 * 32 rows (those slices read no index array), *wide_slices = full slices
 * wider than 16 slots because of at most 4 longer rows, whose rows a
 * warp-cooperative pre-pass sums before each SpMV.  Any output may be NULL.  No counterpart in the
 * reference. */
int dcu_sell_plan_stats(dcu_spai_ctx* ctx, long long* slots, long long* uniform_slots, long long* wide_slices);

/* Turn the wide-slice pre-pass of this context's later solves on (enabled !=
 * 0, the default) or off (every slice's rows summed by the SpMV kernels'
 * per-lane loop).  Each row is summed in its own order either way, so the
 * two give bit-identical iterates; off exists to show that, and to time the
 * pre-pass.  No counterpart in the reference. */
int dcu_set_wide_prepass(dcu_spai_ctx* ctx, int enabled);

/* Let this context's later solves in the forms other than DCU_PREC_FP64 read
 * A's values from an FP32 copy when every value of A is exactly an FP32
 * number (enabled != 0, the default), or always from the FP64 array (0).
 * The check runs on the device while A is laid out for the solver; the
 * products are formed in FP64 from the same numbers either way, so the
 * iterates are bit-identical, and a matrix with one value that FP32 rounds
 * keeps the FP64 reads.  Integer and dyadic stencil coefficients qualify;
 * values read from decimal text usually do not.  The plain FP64 form always
 * reads FP64 values (as it always reads int32 indices).  No counterpart in
 * the reference. */
int dcu_set_exact_a32(dcu_spai_ctx* ctx, int enabled);

/* ---- autotuner (no counterpart in the reference) ----------------------------- */

/* Launch configuration of one precision form.  Grid selectors: 0 = one wave
 * of as many blocks as fit on the GPU at once (each thread loops over rows),
 * -1 = one block per 256 rows (row pairs for the p pass: no loop), k > 0 =
 * k blocks per SM (capped at what fits).  A row's arithmetic does not depend
 * on the grid, and the two first steps compute the same values, so every
 * field except group_max_ni leaves the solution bit-identical:
 *   k1_split   -1: the form's default (split with an FP32 / BF16 M, fused
 *              with an FP64 M); 0: fused (p formed at every gathered column
 *              inside y = M p); 1: split (a p pass, then y = M p).  Forms with
 *              FP32 vectors keep their default: their fused step multiplies
 *              by the unrounded p, so the two differ in rounding there.
 *   grid_p, grid_y, grid_py, grid_sz   the kernels without a reduction:
 *              p pass, y = M p, fused p/y, s/z = M s.  The kernels that end
 *              in a dot product keep one full wave: their grid fixes the
 *              summation order of the partial sums.
 *   group_max_ni   SPAI build: largest |I_k| the warp-group (warp-per-small)
 *              kernel takes, 1..32 (0 = 32); larger columns go to the
 *              CTA-per-column kernel.  Changes M by rounding only.
 *   cta_max_area   SPAI build: largest dense block |I_k| x (|J_k| + 1) one CTA
 *              factors; a larger block is gathered into its own slab and
 *              factored by the hub kernels, every SM on every such column.
 *              0 = what fits the CTA's shared memory; -1 = no limit (every
 *              block on one CTA, larger ones from a per-CTA global slab).
 *              Changes M by rounding only.
 * The report fields are written by dcu_autotune_d and ignored on input. */
typedef struct {
  int k1_split;
  int grid_p, grid_y, grid_py, grid_sz;
  int group_max_ni;
  int cta_max_area;
  /* report */
  float iter_us_default;  /* solve ms / iterations with the default iteration configuration      */
  float iter_us_tuned;    /* the same with the chosen one                                         */
  float build_ms_default; /* SPAI build with the default build fields                            */
  float build_ms_tuned;   /* SPAI build with the chosen ones                                      */
  int candidates;         /* launch configurations timed                                         */
} dcu_tuning;

/* Defaults: every selector 0, k1_split -1, group_max_ni 0, report zero. */
void dcu_tuning_default(dcu_tuning* t);

/* Use *t for every later build and solve of `precision` on this context
 * (NULL: back to the defaults).  DCU_ERR_ARG on a selector out of range. */
int dcu_set_tuning(dcu_spai_ctx* ctx, int precision, const dcu_tuning* t);
int dcu_get_tuning(dcu_spai_ctx* ctx, int precision, dcu_tuning* t);

/* Time the candidate configurations of opt->precision on this matrix and
 * keep the fastest (as dcu_set_tuning would).  Steps: (1) two builds per
 * group_max_ni candidate (32, 24, 16; a candidate that would hand more than
 * 1/8 of the columns to the CTA kernel is not timed), and with
 * cta_max_area = -1 when the default build used the hub kernels; (2) one solve of
 * A x = b from x0 = 0 with the chosen build, then each kernel without a
 * reduction at grid selectors 0, -1 and half the resident blocks, `reps`
 * single launches each (<= 0: 10), every timed launch right after an untimed
 * launch of its predecessor in the iteration; (3) three whole solves each of
 * the default, the per-kernel choice with the split and (FP64 vectors) with
 * the fused first step: the fastest solve phase wins, a change by more than
 * 0.5%.  Every candidate of (2)-(3) gives the same iterates, so solve times
 * compare launch configurations only.  Device arrays; b is not modified.
 * *out (optional) receives the choice and the report. */
int dcu_autotune_d(dcu_spai_ctx* ctx, int n, int nnz, const int* ptr, const int* idx, const double* val,
                   const double* b, const dcu_options* opt, int reps, dcu_tuning* out);

/* ---- MatrixMarket input (command-line driver) --------------------------------- */

/* Read a MatrixMarket file into host CSC arrays with the semantics of
 * readMatrixToCSC (include/common/read.h:1296-1320): "symmetric" in the first
 * line mirrors off-diagonal entries, explicit zeros are dropped, entries keep
 * file order inside each column, indices become 0-based.  Arrays are
 * malloc'ed; release each with dcu_mtx_free.  Returns 0 on success. */
int dcu_mtx_read(const char* path, int* n, int* nnz, int** ptr, int** idx, double** val);
void dcu_mtx_free(void* p);

#ifdef __cplusplus
}
#endif

#endif /* DCU_SPAI_H */
