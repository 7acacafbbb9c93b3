// MatrixMarket reader of the command-line driver: the semantics of the
// reference's readMatrixToCSC, restated (see the comment on dcu_mtx_read).
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "dcu_spai.h"

extern "C" {

void dcu_mtx_free(void* p) { free(p); }

// ---------------------------------------------------------------------------
// MatrixMarket reader with the semantics of readMatrixToCSC
// (include/common/read.h:1296-1320):
//   * "symmetric" anywhere in the first line -> mirrored read
//     (readCSCBYfilling :1250-1294): every off-diagonal (i,j) is appended to
//     column j then (j,i) to column i, entries read until end of file;
//   * otherwise general (readCSC :935-979): exactly nnz entries;
//   * the value count is the number of whitespace runs on the first data line
//     (computeNumOfValues :28-43): 2 = pattern (value 1.0), 3 = one value,
//     4 = two values (general two-value files produce an empty matrix, as
//     readCSCTwoValues :853-864 reads nothing);
//   * explicit zeros (fabs(v) == 0) are dropped except in pattern files;
//   * entries keep file order inside each column; indices become 0-based.
// Arrays are malloc'ed; free with dcu_mtx_free.  Returns 0 on success.
// ---------------------------------------------------------------------------
static int count_value_runs(const char* s) {
  int spacePos = -1, runs = 0;
  int len = (int)strlen(s);
  for (int i = 0; i < len; ++i)
    if (isspace((unsigned char)s[i]) && i != spacePos && (i - 1) != spacePos) {
      ++runs;
      spacePos = i;
    }
  return runs;
}

int dcu_mtx_read(const char* path, int* n_out, int* nnz_out, int** ptr_out, int** idx_out,
                 double** val_out) {
  FILE* fp = fopen(path, "r");
  if (!fp) return -1;
  char line[1024];
  if (!fgets(line, sizeof line, fp)) { fclose(fp); return -2; }
  bool symmetric = std::string(line).find("symmetric") != std::string::npos;
  // skip comment lines; the first non-comment line is the size line
  bool have = true;
  while (line[0] == '%') {
    if (!fgets(line, sizeof line, fp)) { have = false; break; }
  }
  if (!have) { fclose(fp); return -2; }
  int nr = 0, nc = 0, nz = 0;
  if (sscanf(line, "%d %d %d", &nr, &nc, &nz) != 3) { fclose(fp); return -3; }
  long dataPos = ftell(fp);
  char first[1024] = {0};
  int nvals = 0;
  if (fgets(first, sizeof first, fp)) nvals = count_value_runs(first);
  fseek(fp, dataPos, SEEK_SET);
  std::vector<std::vector<int>> ci(nr > 0 ? nr : 0);
  std::vector<std::vector<double>> cv(nr > 0 ? nr : 0);
  long total = 0;
  auto push = [&](int col, int row, double v) {
    ci[col].push_back(row);
    cv[col].push_back(v);
    ++total;
  };
  if (nvals != 2 && nvals != 3 && nvals != 4) { fclose(fp); return -4; }
  if (!symmetric) {
    if (nvals == 4) {
      // two-value general files: the reference leaves the matrix empty
    } else {
      for (int t = 0; t < nz; ++t) {
        int i1, j1;
        double d = 1.0;
        int rv = (nvals == 2) ? fscanf(fp, "%d %d", &i1, &j1) : fscanf(fp, "%d %d %lf", &i1, &j1, &d);
        if (rv == EOF || rv < 2) { fclose(fp); return -5; }
        if (nvals == 3 && std::fabs(d) == 0) continue;
        push(j1 - 1, i1 - 1, d);
      }
    }
  } else {
    for (;;) {
      int i1, j1;
      double d = 1.0, d2;
      int rv;
      if (nvals == 2) rv = fscanf(fp, "%d %d", &i1, &j1);
      else if (nvals == 3) rv = fscanf(fp, "%d %d %lf", &i1, &j1, &d);
      else rv = fscanf(fp, "%d %d %lf %lf", &i1, &j1, &d, &d2);
      if (rv == EOF) break;
      if (rv < 2) { fclose(fp); return -5; }
      if (nvals != 2 && std::fabs(d) == 0) continue;
      push(j1 - 1, i1 - 1, d);
      if (i1 != j1) push(i1 - 1, j1 - 1, d);
    }
  }
  fclose(fp);
  if (nvals == 4 && !symmetric) {
    *n_out = 0;
    *nnz_out = 0;
    *ptr_out = nullptr;
    *idx_out = nullptr;
    *val_out = nullptr;
    return 0;
  }
  int* P = (int*)malloc(sizeof(int) * (nc + 1));
  int* Ix = (int*)malloc(sizeof(int) * (total > 0 ? total : 1));
  double* V = (double*)malloc(sizeof(double) * (total > 0 ? total : 1));
  P[0] = 0;
  long off = 0;
  for (int c = 0; c < nc; ++c) {
    if (c < nr) {
      for (size_t t = 0; t < ci[c].size(); ++t) {
        Ix[off + t] = ci[c][t];
        V[off + t] = cv[c][t];
      }
      off += (long)ci[c].size();
    }
    P[c + 1] = (int)off;
  }
  *n_out = nc;
  *nnz_out = (int)off;
  *ptr_out = P;
  *idx_out = Ix;
  *val_out = V;
  return 0;
}

}  // extern "C"
