/*
 * A stand-in for the MATLAB runtime, test infrastructure only: enough of the
 * C matrix / MEX API for the gateways in blood_network_b200/mex to run
 * outside MATLAB.  Linked with one gateway into a shared library that the
 * tests load with ctypes.  mexErrMsgIdAndTxt jumps back to mxfake_run,
 * which reports the error id.
 */
#include <setjmp.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mex.h"

struct mxArray_tag {
  mxClassID cls;
  int sparse;
  size_t m, n, nzmax;
  mwIndex* jc;
  mwIndex* ir;
  double* pr;
  void* data; /* numeric (non-double) payload */
};

static jmp_buf g_jmp;
static char g_id[128];
static char g_msg[512];

bool mxIsSparse(const mxArray* a) { return a->sparse != 0; }
bool mxIsInt32(const mxArray* a) { return a->cls == mxINT32_CLASS; }
size_t mxGetM(const mxArray* a) { return a->m; }
size_t mxGetN(const mxArray* a) { return a->n; }
size_t mxGetNumberOfElements(const mxArray* a) { return a->m * a->n; }
mwIndex* mxGetJc(const mxArray* a) { return a->jc; }
mwIndex* mxGetIr(const mxArray* a) { return a->ir; }
double* mxGetPr(const mxArray* a) { return a->pr; }
void* mxGetData(const mxArray* a) { return a->data ? a->data : (void*)a->pr; }
double mxGetScalar(const mxArray* a) {
  if (a->cls == mxINT32_CLASS) return (double)*(int*)a->data;
  return a->pr ? a->pr[0] : 0.0;
}

mxArray* mxCreateSparse(mwSize m, mwSize n, mwSize nzmax, mxComplexity flag) {
  (void)flag;
  mxArray* a = (mxArray*)calloc(1, sizeof(mxArray));
  a->cls = mxDOUBLE_CLASS;
  a->sparse = 1;
  a->m = m;
  a->n = n;
  a->nzmax = nzmax;
  a->jc = (mwIndex*)calloc(n + 1, sizeof(mwIndex));
  a->ir = (mwIndex*)calloc(nzmax ? nzmax : 1, sizeof(mwIndex));
  a->pr = (double*)calloc(nzmax ? nzmax : 1, sizeof(double));
  return a;
}
mxArray* mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity flag) {
  (void)flag;
  mxArray* a = (mxArray*)calloc(1, sizeof(mxArray));
  a->cls = mxDOUBLE_CLASS;
  a->m = m;
  a->n = n;
  a->pr = (double*)calloc((m * n) > 0 ? (m * n) : 1, sizeof(double));
  return a;
}
mxArray* mxCreateDoubleScalar(double v) {
  mxArray* a = mxCreateDoubleMatrix(1, 1, mxREAL);
  a->pr[0] = v;
  return a;
}
mxArray* mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID cls, mxComplexity flag) {
  (void)flag;
  mxArray* a = (mxArray*)calloc(1, sizeof(mxArray));
  a->cls = cls;
  a->m = m;
  a->n = n;
  a->data = calloc((m * n) > 0 ? (m * n) : 1, 8);
  return a;
}
void* mxMalloc(size_t n) { return malloc(n ? n : 1); }
void* mxCalloc(size_t n, size_t size) { return calloc(n ? n : 1, size ? size : 1); }
void mxFree(void* p) { free(p); }

void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_msg, sizeof g_msg, fmt, ap);
  va_end(ap);
  snprintf(g_id, sizeof g_id, "%s", id);
  longjmp(g_jmp, 1);
}

/* ---- driver side (called from the tests) ---- */
int mxfake_run(int nlhs, mxArray** plhs, int nrhs, const mxArray** prhs) {
  g_id[0] = g_msg[0] = 0;
  if (setjmp(g_jmp)) return 1;
  mexFunction(nlhs, plhs, nrhs, prhs);
  return 0;
}
const char* mxfake_error_id(void) { return g_id; }
const char* mxfake_error_msg(void) { return g_msg; }

mxArray* mxfake_sparse(size_t m, size_t n, size_t nnz, const long long* jc, const long long* ir,
                       const double* pr) {
  mxArray* a = mxCreateSparse(m, n, nnz, mxREAL);
  for (size_t c = 0; c <= n; c++) a->jc[c] = (mwIndex)jc[c];
  for (size_t k = 0; k < nnz; k++) {
    a->ir[k] = (mwIndex)ir[k];
    a->pr[k] = pr[k];
  }
  return a;
}
mxArray* mxfake_double(size_t m, size_t n, const double* v) {
  mxArray* a = mxCreateDoubleMatrix(m, n, mxREAL);
  memcpy(a->pr, v, m * n * sizeof(double));
  return a;
}
mxArray* mxfake_int32(int v) {
  mxArray* a = mxCreateNumericMatrix(1, 1, mxINT32_CLASS, mxREAL);
  *(int*)a->data = v;
  return a;
}
int mxfake_class(const mxArray* a) { return (int)a->cls; }
int mxfake_is_sparse(const mxArray* a) { return a->sparse; }
size_t mxfake_m(const mxArray* a) { return a->m; }
size_t mxfake_n(const mxArray* a) { return a->n; }
size_t mxfake_nnz(const mxArray* a) { return a->sparse ? a->jc[a->n] : a->m * a->n; }
void mxfake_copy_sparse(const mxArray* a, long long* jc, long long* ir, double* pr) {
  for (size_t c = 0; c <= a->n; c++) jc[c] = (long long)a->jc[c];
  for (size_t k = 0; k < a->jc[a->n]; k++) {
    ir[k] = (long long)a->ir[k];
    pr[k] = a->pr[k];
  }
}
void mxfake_copy_double(const mxArray* a, double* out) {
  memcpy(out, a->pr, a->m * a->n * sizeof(double));
}
int mxfake_int32_value(const mxArray* a) { return *(int*)a->data; }
void mxfake_free(mxArray* a) {
  if (!a) return;
  free(a->jc);
  free(a->ir);
  free(a->pr);
  free(a->data);
  free(a);
}
