/*
 * Helpers shared by the MEX gateways: MATLAB's CSC index arrays (mwIndex)
 * to the library's 0-based int32 CSR, and the error a gateway raises when
 * the device library reports a failure.
 */
#ifndef BN_MEX_UTIL_H
#define BN_MEX_UTIL_H

#include <limits.h>
#include <stdlib.h>
#include <string.h>

#include "amg_b200.h"
#include "mex.h"

/* int32 copy of an index array (error when an index does not fit) */
static inline int* bn_mex_ints(const mwIndex* a, size_t n, const char* errid) {
  int* out = (int*)mxMalloc((n > 0 ? n : 1) * sizeof(int));
  for (size_t k = 0; k < n; k++) {
    if (a[k] > (mwIndex)INT_MAX) mexErrMsgIdAndTxt(errid, "Index exceeds the int32 range.");
    out[k] = (int)a[k];
  }
  return out;
}

/* CSR arrays of the matrix whose CSC arrays are (jc, ir): rows' column
 * indices come out ascending (columns are visited in order) */
static inline void bn_mex_csc_to_csr(size_t m, size_t n, const mwIndex* jc, const mwIndex* ir,
                              int** ia_out, int** ja_out) {
  const size_t nnz = jc[n];
  int* ia = (int*)mxCalloc(m + 1, sizeof(int));
  int* ja = (int*)mxMalloc((nnz > 0 ? nnz : 1) * sizeof(int));
  int* fill = (int*)mxCalloc(m > 0 ? m : 1, sizeof(int));
  for (size_t k = 0; k < nnz; k++) ia[ir[k] + 1]++;
  for (size_t i = 0; i < m; i++) ia[i + 1] += ia[i];
  for (size_t c = 0; c < n; c++)
    for (mwIndex k = jc[c]; k < jc[c + 1]; k++) {
      const size_t r = ir[k];
      ja[ia[r] + fill[r]++] = (int)c;
    }
  mxFree(fill);
  *ia_out = ia;
  *ja_out = ja;
}

/* a MATLAB sparse m x n from CSR (ia, ja, val): entries of a column in
 * ascending row order */
static inline mxArray* bn_mex_sparse_from_csr(size_t m, size_t n, const int* ia, const int* ja,
                                       const double* val) {
  const size_t nnz = (size_t)ia[m];
  mxArray* out = mxCreateSparse(m, n, nnz > 0 ? nnz : 1, mxREAL);
  mwIndex* jc = mxGetJc(out);
  mwIndex* ir = mxGetIr(out);
  double* pr = mxGetPr(out);
  size_t* fill = (size_t*)mxCalloc(n > 0 ? n : 1, sizeof(size_t));
  memset(jc, 0, (n + 1) * sizeof(mwIndex));
  for (size_t k = 0; k < nnz; k++) jc[ja[k] + 1]++;
  for (size_t c = 0; c < n; c++) jc[c + 1] += jc[c];
  for (size_t r = 0; r < m; r++)
    for (int k = ia[r]; k < ia[r + 1]; k++) {
      const size_t c = (size_t)ja[k];
      const size_t dst = jc[c] + fill[c]++;
      ir[dst] = r;
      pr[dst] = val[k];
    }
  mxFree(fill);
  return out;
}

static inline void bn_mex_check(const char* errid) {
  if (amg_solver_last_status() != AMG_OK)
    mexErrMsgIdAndTxt(errid, "%s", amg_solver_last_error());
}

#endif /* BN_MEX_UTIL_H */
