// CPU oracle for the SPAI-preconditioned BiCGSTAB path.
//
// TEST INFRASTRUCTURE ONLY.  This file is a plain C++ restatement of the
// reference algorithm (SingkiWong/DCU) used as the checker for the CUDA
// library in dcu_b200/csrc.  Only tests/, __graft_entry__.smoke() and the
// cpu_baseline / --impl reference legs of bench.py load it.  The product path
// never calls it and has no CPU fallback.
//
// Parity status of each part:
//   * CSC->CSR and the |I_k| sizing are pinned against the reference's own
//     CPU code (include/common/assemble.h, init.h) compiled from the
//     reference tree into oracle/_ref by oracle/Makefile (see
//     tests/test_oracle_pinned.py); the library's MatrixMarket reader is
//     pinned the same way against include/common/read.h.
//   * The SPAI kernels and the BiCGSTAB loop exist in the reference only as HIP
//     code on top of hipSPARSE/hipBLAS (ROCm, version not pinned), which cannot
//     be compiled here and ship no golden vectors: that part is
//     "parity unpinned" -- restated from source, cited line by line below.
//
// All functions are extern "C", take plain pointers, and are deterministic
// for any OpenMP thread count (fixed-size chunked reductions).
// Build: g++ -O2 -fopenmp -ffp-contract=off -shared -fPIC (oracle/build.sh).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr long kChunk = 8192;  // fixed reduction chunk -> thread-count independent sums

double chunked_dot(long n, const double* a, const double* b) {
  long nch = (n + kChunk - 1) / kChunk;
  std::vector<double> part(nch > 0 ? nch : 1, 0.0);
#pragma omp parallel for schedule(static)
  for (long c = 0; c < nch; ++c) {
    long s = c * kChunk, e = std::min(n, s + kChunk);
    double acc = 0.0;
    for (long i = s; i < e; ++i) acc += a[i] * b[i];
    part[c] = acc;
  }
  double t = 0.0;
  for (long c = 0; c < nch; ++c) t += part[c];
  return t;
}

// y = A x for CSR A (row order of the column indices as stored).
void csr_spmv(int n, const int* rp, const int* ci, const double* v, const double* x, double* y) {
#pragma omp parallel for schedule(static, 4096)
  for (int r = 0; r < n; ++r) {
    double acc = 0.0;
    for (int e = rp[r]; e < rp[r + 1]; ++e) acc += v[e] * x[ci[e]];
    y[r] = acc;
  }
}

// Sorted, duplicate-free union of the row patterns of A(:,j), j in J_k.
// Restates computeJ_SSPAIv10 (src/spai_multi_dcu.cpp:275-295) and
// computeI_Symbol_SpMMv1 (:738-834): first column copied, the others appended
// when absent, then the odd-even transposition sort (:806-831), whose result is
// the ascending order of the set.
void column_pattern(const int* ptr, const int* idx, int k, std::vector<int>& I) {
  I.clear();
  int cs = ptr[k], ce = ptr[k + 1];
  for (int t = cs; t < ce; ++t) {
    int j = idx[t];
    int js = ptr[j], je = ptr[j + 1];
    size_t before = I.size();  // tN snapshot: elements of earlier columns only
    for (int q = js; q < je; ++q) {
      int r = idx[q];
      bool found = false;
      if (t != cs)
        for (size_t u = 0; u < before; ++u)
          if (I[u] == r) { found = true; break; }
      if (!found) I.push_back(r);
    }
  }
  std::sort(I.begin(), I.end());
}

}  // namespace

extern "C" {

void orc_free(void* p) { free(p); }

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void orc_set_threads(int t) {
#ifdef _OPENMP
  if (t > 0) omp_set_num_threads(t);
#else
  (void)t;
#endif
}

// ---------------------------------------------------------------------------
// Column schedules: restates distributeColumns (src/spai_multi_dcu.cpp:1356-1449).
// use_nnz = 0: balanced_columns (:1420-1440); 1: balanced_nnz (:1380-1419).
// ---------------------------------------------------------------------------
void orc_distribute_columns(const int* ptr, int colStart, int colEnd, int units, int use_nnz,
                            int* starts, int* ends) {
  int total = colEnd - colStart;
  if (units <= 0 || total <= 0) return;
  if (use_nnz && ptr[colEnd] - ptr[colStart] > 0) {
    int totalNnz = ptr[colEnd] - ptr[colStart];
    int target = totalNnz / units;
    int cur = 0;
    for (int u = 0; u < units; ++u) {
      starts[u] = colStart + cur;
      int startCol = cur, acc = 0;
      if (u == units - 1) {
        cur = total;
      } else {
        while (cur < total) {
          int g = colStart + cur;
          int cn = ptr[g + 1] - ptr[g];
          if (acc + cn > target && cur > startCol) break;
          acc += cn;
          ++cur;
        }
      }
      if (cur <= startCol) cur = (startCol + 1 <= total) ? startCol + 1 : total;
      ends[u] = colStart + cur;
    }
  } else {
    int base = total / units, rem = total % units, cur = 0;
    for (int u = 0; u < units; ++u) {
      starts[u] = colStart + cur;
      int c = base + (u < rem ? 1 : 0);
      ends[u] = colStart + cur + c;
      cur += c;
    }
  }
}

// ---------------------------------------------------------------------------
// Pattern pass.  With ilist == NULL only icount is filled (sizing, like
// cuComputeN1withSparityofA_SpMMv1 :122-198); otherwise I_k is written at
// ilist[iptr[k - colStart]].  Returns sum |I_k| over the range.
// ---------------------------------------------------------------------------
long long orc_spai_pattern(int n, const int* ptr, const int* idx, int colStart, int colEnd,
                           int* icount, const long long* iptr, int* ilist) {
  (void)n;
  long long total = 0;
#pragma omp parallel
  {
    std::vector<int> I;
#pragma omp for schedule(dynamic, 256) reduction(+ : total)
    for (int k = colStart; k < colEnd; ++k) {
      column_pattern(ptr, idx, k, I);
      icount[k - colStart] = (int)I.size();
      total += (long long)I.size();
      if (ilist) std::memcpy(ilist + iptr[k - colStart], I.data(), I.size() * sizeof(int));
    }
  }
  return total;
}

// ---------------------------------------------------------------------------
// SPAI build.  For every column k in [colStart, colEnd):
//   J = A(:,k) rows (as stored), I = sorted union, At = A(I,J) (row-major,
//   gather of ComputeTildeACSR_SSPAIv10 :945-983, first match per column),
//   E = position of k in I (ComputeTildeE_SSPAIv10 :985-1004),
//   method 0: modified Gram-Schmidt exactly as QR_RShared_SSPAIv10
//             (:1069-1133) followed by Sol_SSPAIv10 (:1028-1067);
//   method 1: Householder QR of [At | e_E] with back substitution (the FP64
//             accuracy oracle; mathematically the same least-squares solution).
//   mval[ptr[k] + j] = x_j  (modifyData4_SSPAIv10 :1135-1152).
// colres[k - colStart] (optional) = ||A m_k - e_k||_2 = ||At x - e_E||_2.
// Ecol[k - colStart] (optional) = E.
// Returns the number of columns with a zero pivot (r_ii == 0 or non-finite).
// ---------------------------------------------------------------------------
int orc_spai_build(int n, const int* ptr, const int* idx, const double* val, int colStart,
                   int colEnd, int method, double* mval, double* colres, int* Ecol) {
  (void)n;
  int singular = 0;
#pragma omp parallel
  {
    std::vector<int> I;
    std::vector<double> Q, R, X, Rs, b;
#pragma omp for schedule(dynamic, 64) reduction(+ : singular)
    for (int k = colStart; k < colEnd; ++k) {
      column_pattern(ptr, idx, k, I);
      const int cs = ptr[k];
      const int AN = ptr[k + 1] - cs;
      const int AM = (int)I.size();
      Q.assign((size_t)AM * AN, 0.0);
      for (int i = 0; i < AM; ++i) {
        int irow = I[i];
        for (int j = 0; j < AN; ++j) {
          int jc = idx[cs + j];
          double d = 0.0;
          for (int q = ptr[jc]; q < ptr[jc + 1]; ++q)
            if (idx[q] == irow) { d = val[q]; break; }
          Q[(size_t)i * AN + j] = d;
        }
      }
      int E = -1;
      for (int i = 0; i < AM; ++i)
        if (I[i] == k) { E = i; break; }
      if (Ecol) Ecol[k - colStart] = E;
      const std::vector<double> At = Q;  // kept for the residual
      X.assign(AN, 0.0);
      bool sing = false;
      if (method == 0) {
        R.assign((size_t)AN * AN, 0.0);
        Rs.assign(AN, 0.0);
        for (int i = 0; i < AN; ++i) {
          for (int j = i; j < AN; ++j) {
            double tR = 0.0;
            for (int q = 0; q < AM; ++q) tR += Q[(size_t)q * AN + i] * Q[(size_t)q * AN + j];
            Rs[j - i] = tR;
          }
          double rii = std::sqrt(Rs[0]);
          if (!(rii != 0.0) || !std::isfinite(rii)) sing = true;
          for (int q = 0; q < AM; ++q) Q[(size_t)q * AN + i] /= rii;
          for (int j = i; j < AN; ++j) {
            Rs[j - i] /= rii;
            R[(size_t)i * AN + j] = Rs[j - i];
          }
          for (int j = i + 1; j < AN; ++j)
            for (int q = 0; q < AM; ++q) Q[(size_t)q * AN + j] -= Rs[j - i] * Q[(size_t)q * AN + i];
        }
        for (int i = 0; i < AN; ++i) X[i] = (E == -1) ? 0.0 : Q[(size_t)E * AN + i];
        for (int i = AN - 1; i >= 0; --i) {
          X[i] /= R[(size_t)i * AN + i];
          for (int j = 0; j < i; ++j) X[j] -= R[(size_t)j * AN + i] * X[i];
        }
      } else {
        // Householder on the augmented matrix [At | e_E], column-major copy.
        const int W = AN + 1;
        std::vector<double> C((size_t)AM * W, 0.0);
        for (int i = 0; i < AM; ++i)
          for (int j = 0; j < AN; ++j) C[(size_t)j * AM + i] = Q[(size_t)i * AN + j];
        if (E >= 0) C[(size_t)AN * AM + E] = 1.0;
        const int steps = std::min(AN, AM);
        for (int c = 0; c < steps; ++c) {
          double* col = &C[(size_t)c * AM];
          double sigma = 0.0;
          for (int i = c + 1; i < AM; ++i) sigma += col[i] * col[i];
          double x0 = col[c];
          double nrm = std::sqrt(x0 * x0 + sigma);
          if (nrm == 0.0) { sing = true; continue; }
          double alpha = (x0 > 0.0) ? -nrm : nrm;
          double v0 = x0 - alpha;
          double vtv = v0 * v0 + sigma;
          double beta = (vtv > 0.0) ? 2.0 / vtv : 0.0;
          col[c] = v0;  // v stored in place below the diagonal
          for (int j = c + 1; j < W; ++j) {
            double* cj = &C[(size_t)j * AM];
            double w = 0.0;
            for (int i = c; i < AM; ++i) w += col[i] * cj[i];
            w *= beta;
            for (int i = c; i < AM; ++i) cj[i] -= w * col[i];
          }
          col[c] = alpha;
        }
        if (AM < AN) sing = true;
        const double* y = &C[(size_t)AN * AM];
        for (int i = 0; i < AN; ++i) X[i] = (i < AM) ? y[i] : 0.0;
        for (int i = AN - 1; i >= 0; --i) {
          double rii = (i < AM) ? C[(size_t)i * AM + i] : 0.0;
          if (rii == 0.0) sing = true;
          X[i] /= rii;
          for (int j = 0; j < i; ++j) X[j] -= C[(size_t)i * AM + j] * X[i];
        }
      }
      if (sing) ++singular;
      for (int j = 0; j < AN; ++j) mval[cs + j] = X[j];
      if (colres) {
        double s = 0.0;
        for (int i = 0; i < AM; ++i) {
          double t = (i == E) ? -1.0 : 0.0;
          for (int j = 0; j < AN; ++j) t += At[(size_t)i * AN + j] * X[j];
          s += t * t;
        }
        colres[k - colStart] = std::sqrt(s);
      }
    }
  }
  return singular;
}

// ---------------------------------------------------------------------------
// CSC -> CSR with ascending column order inside each row, values carried
// along: the output of cuCSC2CSR (include/common/cuFormatConversion.h:453-589)
// and of the CPU CSC2CSR (include/common/assemble.h:34-67).
// ---------------------------------------------------------------------------
void orc_csc2csr(int n, const int* cptr, const int* cidx, const double* cval, int* rptr,
                 int* ridx, double* rval) {
  std::vector<int> cnt(n + 1, 0);
  int nnz = cptr[n];
  for (int e = 0; e < nnz; ++e) cnt[cidx[e] + 1]++;
  for (int r = 0; r < n; ++r) cnt[r + 1] += cnt[r];
  for (int r = 0; r <= n; ++r) rptr[r] = cnt[r];
  for (int c = 0; c < n; ++c)
    for (int e = cptr[c]; e < cptr[c + 1]; ++e) {
      int r = cidx[e];
      int pos = cnt[r]++;
      ridx[pos] = c;
      if (rval) rval[pos] = cval[e];
    }
}

// ---------------------------------------------------------------------------
// Right-preconditioned BiCGSTAB, the recurrences of cublas2_pbicgstabv2
// (include/bicgstab/bicgstab_solver.h:33-275) in the same order:
//   r = b - A x; r* = p = r; rho = (r*, r); it = 1
//   while it < maxiter:
//     y = M p; ay = A y; alpha = rho / (r*, ay); s = r - alpha ay
//     z = M s; az = A z; w = (az, s) / (az, az)
//     x += alpha y; x += w z; r = s - w az
//     rho' = (r*, r); beta = (rho'/rho)(alpha/w); p = beta p + r - beta w ay
//     err = ||r||; if err < thr: break; it++
// tol_mode 0: thr = tol (absolute, :229); tol_mode 1: thr = tol * ||b||.
// Returns the reference's iteration counter; *status = 0 converged, 1 hit
// maxiter, 2 non-finite scalar seen (the reference keeps iterating on NaN, so
// the counter then runs to maxiter exactly as there).
// hist (optional, length >= maxiter): recurrence ||r|| after each iteration.
// ---------------------------------------------------------------------------
int orc_bicgstab(int n, const int* Arp, const int* Aci, const double* Av, const int* Mrp,
                 const int* Mci, const double* Mv, const double* b, double* x, double tol,
                 int tol_mode, int maxiter, double* final_res, double* true_res, int* status,
                 double* hist) {
  std::vector<double> r(n), rs(n), p(n), y(n), ay(n), s(n), z(n), az(n);
  csr_spmv(n, Arp, Aci, Av, x, r.data());
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) r[i] = b[i] + (-1.0) * r[i];
  rs = r;
  p = r;
  double bnrm = std::sqrt(chunked_dot(n, b, b));
  double thr = (tol_mode == 1) ? tol * bnrm : tol;
  double temp1 = chunked_dot(n, rs.data(), r.data());
  double err = std::sqrt(chunked_dot(n, r.data(), r.data()));
  int it = 1;
  if (maxiter <= 0) maxiter = n;
  bool nonfinite = false;
  bool conv = false;
  while (it < maxiter) {
    csr_spmv(n, Mrp, Mci, Mv, p.data(), y.data());
    double temp = temp1;
    csr_spmv(n, Arp, Aci, Av, y.data(), ay.data());
    double temp2 = chunked_dot(n, rs.data(), ay.data());
    double alpha = temp / temp2;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) s[i] = r[i] + (-1.0 * alpha) * ay[i];
    csr_spmv(n, Mrp, Mci, Mv, s.data(), z.data());
    csr_spmv(n, Arp, Aci, Av, z.data(), az.data());
    temp1 = chunked_dot(n, az.data(), s.data());
    temp2 = chunked_dot(n, az.data(), az.data());
    double w = temp1 / temp2;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
      x[i] = x[i] + alpha * y[i];
      x[i] = x[i] + w * z[i];
      r[i] = s[i] + (-1.0 * w) * az[i];
    }
    temp1 = chunked_dot(n, rs.data(), r.data());
    double beta = (temp1 / temp) * (alpha / w);
    double bw = -1.0 * beta * w;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
      double t = beta * p[i];
      t = t + r[i];
      p[i] = t + bw * ay[i];
    }
    err = std::sqrt(chunked_dot(n, r.data(), r.data()));
    if (hist) hist[it - 1] = err;
    if (!std::isfinite(alpha) || !std::isfinite(w) || !std::isfinite(beta)) nonfinite = true;
    if (err < thr) { conv = true; break; }
    ++it;
  }
  if (final_res) *final_res = err;
  if (true_res) {
    csr_spmv(n, Arp, Aci, Av, x, y.data());
    double acc = 0.0;
    long nch = ((long)n + kChunk - 1) / kChunk;
    std::vector<double> part(nch > 0 ? nch : 1, 0.0);
#pragma omp parallel for schedule(static)
    for (long c = 0; c < nch; ++c) {
      long s0 = c * kChunk, e0 = std::min((long)n, s0 + kChunk);
      double a = 0.0;
      for (long i = s0; i < e0; ++i) { double d = b[i] - y[i]; a += d * d; }
      part[c] = a;
    }
    for (long c = 0; c < nch; ++c) acc += part[c];
    *true_res = std::sqrt(acc);
  }
  if (status) *status = conv ? 0 : (nonfinite ? 2 : 1);
  return it;
}

}  // extern "C"
